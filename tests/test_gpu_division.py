"""The reciprocal-and-correction division (div_rn.cuh) equals __ddiv_rn bit for bit over
pseudo-random operand pairs with random and edge-case mantissas (prj_selftest_division)."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_division_matches_ddiv_rn(cuda_device, seed):
    import prj
    L = prj.load_library()
    bad = ctypes.c_longlong(-1)
    fu, fd = ctypes.c_double(), ctypes.c_double()
    prj._check(L.prj_selftest_division(0, 1 << 26, seed, ctypes.byref(bad), ctypes.byref(fu), ctypes.byref(fd)))
    assert bad.value == 0, (bad.value, fu.value, fd.value)
