"""Shared test set-up: import paths, the gpu marker, the oracle and fixtures.

Tests marked ``gpu`` run on a B200 and call the engine through its C ABI;
everything else runs on CPU (oracle against golden vectors, host logic, ABI
symbol checks).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dns-supercritical-ibm_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, os.path.join(ROOT, "oracle"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the engine through its C ABI")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    return pyoracle.COracle()


@pytest.fixture(scope="session")
def trials():
    d = np.load(os.path.join(GOLDEN, "trials_seed0.npz"))
    out = []
    for it in range(int(d["n_trials"])):
        p = f"t{it}_"
        out.append(dict(
            shape=tuple(int(v) for v in d[p + "shape"]), divs_zy=tuple(int(v) for v in d[p + "divs_zy"]),
            dx=float(d[p + "dxdz"][0]), dz=float(d[p + "dxdz"][1]), yu=d[p + "yu"],
            A=np.asfortranarray(d[p + "A_input"]), B=np.asfortranarray(d[p + "B_output"]),
            bands=(*d[p + "abc"].T, *d[p + "abc00"].T)))
    return out


@pytest.fixture(scope="session")
def mms():
    return dict(np.load(os.path.join(GOLDEN, "mms.npz")))


@pytest.fixture(scope="session")
def channel_golden():
    return dict(np.load(os.path.join(GOLDEN, "channel_128x96x64.npz")))


def mean_removed_maxabs(a, b):
    """The reference's Poisson check: subtract each field's arithmetic mean, then max |a - b|
    (tests/test_poisson_solver_and_ibm_rand/main_poi_test.f90:224-262)."""
    return float(np.abs((a - a.mean()) - (b - b.mean())).max())


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test collected on a machine without a CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
