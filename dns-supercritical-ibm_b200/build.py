"""Build the engine's shared library for sm_100a with nvcc.

    python dns-supercritical-ibm_b200/build.py [--verbose]

Output: dns-supercritical-ibm_b200/libprj_b200.so (in-tree; it travels with the
source tree to the GPU host).  Rebuilds only when a source is newer than the
library unless ``force`` is set.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libprj_b200.so")
SOURCES = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
DEPS = SOURCES + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + sorted(
    glob.glob(os.path.join(HERE, "csrc", "*.h"))) + [os.path.join(REPO, "include", "projection.h")]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS)


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    """Compile every source to an object in parallel (one nvcc per source, up to the host's
    cores), then link the shared library."""
    if not force and not needs_build():
        return LIB
    flags = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(REPO, "include")]
    if verbose:
        flags.insert(0, "-Xptxas=-v")
    if extra:
        flags[0:0] = list(extra)
    if os.environ.get("PRJ_NVCC_FLAGS"):  # experiments: extra -D options
        flags[0:0] = os.environ["PRJ_NVCC_FLAGS"].split()
    with tempfile.TemporaryDirectory(prefix="prj_build_") as tmp:
        objs = [os.path.join(tmp, os.path.basename(src)[:-3] + ".o") for src in SOURCES]
        jobs = list(zip(SOURCES, objs))
        width = max(1, min(len(jobs), os.cpu_count() or 1))
        logs = []
        while jobs:
            batch, jobs = jobs[:width], jobs[width:]
            procs = [(src, subprocess.Popen([nvcc_path(), *flags, "-c", src, "-o", obj], stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT, text=True)) for src, obj in batch]
            for src, p in procs:
                out, _ = p.communicate()
                logs.append(out)
                if p.returncode != 0:
                    sys.stderr.write(out)
                    raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
        res = subprocess.run([nvcc_path(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"],
                             capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("nvcc failed linking libprj_b200.so")
    if verbose:
        sys.stderr.write("".join(logs))
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
