"""Golden field file for the reference's field I/O format (src/mod_io.f90:7-149).

Run in a container where the reference project is importable; writes
tests/golden/field_5x3x4.dat with the reference's own Python writer
(misc/reinterp/tester_mk_ini_data_bin.py:54-61, the format cfd_read_arr reads) and
tests/golden/field_5x3x4.npz with the values, then checks the file with the
reference's reader (CFD_Folder.import_array_bin, :174-183).

    python tests/golden/make_golden_io.py [path-to-reference]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "misc", "reinterp"))
    import tester_mk_ini_data_bin as ref  # the reference's binary writer and reader
    A = np.random.default_rng(21).normal(size=(5, 3, 4))
    A[0, 0, 0] = np.pi  # an exactly known first value
    path = os.path.join(HERE, "field_5x3x4.dat")
    ref.writer_bin(path, A, [5, 3, 4])
    np.savez(os.path.join(HERE, "field_5x3x4.npz"), A=A)
    back = ref.CFD_Folder.import_array_bin(path)
    assert np.array_equal(back, A)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
