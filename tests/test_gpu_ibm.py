"""GPU tests of the immersed-boundary forcing of the predictor (prj_rough_force,
prj_ibm_interp) against the oracle's restatement of src/ibm_setup/mod_cfd_ibm.f90:64-116 and
src/diezdecomp_api_ibm.f90:374-424.  Assignments and the two-term interpolation are exact."""
import numpy as np
import pytest

from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu


def rough_indices(solid, ny):
    """Per-column bottom/top indices of a solid mask [x, z, y] (cells 0..bot and top..ny-1 solid)."""
    nx, nz, _ = solid.shape
    bot = np.full((nx, nz), -1, dtype=np.int32)
    top = np.full((nx, nz), ny, dtype=np.int32)
    for i in range(nx):
        for j in range(nz):
            col = solid[i, j]
            k = 0
            while k < ny and col[k]:
                k += 1
            bot[i, j] = k - 1
            k = ny - 1
            while k >= 0 and col[k]:
                k -= 1
            top[i, j] = k + 1
    return bot, top


def dev_inds(inds):
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(v.T)).to("cuda:0") for k, v in inds.items()}


def test_rough_force_matches_oracle(cuda_device):
    import prj
    import pyoracle
    import workloads
    nx, ny, nz = 40, 32, 24
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=2)
    rng = np.random.default_rng(7)
    inds = {}
    for c in "UVW":
        inds[f"{c}_bot"] = rng.integers(-1, 6, size=(nx, nz)).astype(np.int32)
        top = rng.integers(ny - 5, ny + 1, size=(nx, nz)).astype(np.int32)
        if c == "V":
            top = np.minimum(top + 1, ny + 1).astype(np.int32)  # v reaches the top wall face
        inds[f"{c}_top"] = top
    wall = (0.25, -0.5, 0.75, 1.25, 1.5, -1.75)
    U, V, W = (to_dev(a) for a in (Uh, Vh, Wh))
    prj.rough_force(U, V, W, dev_inds(inds), wall)
    Uo, Vo, Wo = pyoracle.rough_force(Uh, Vh, Wh, inds, wall)
    for d, o in ((U, Uo), (V, Vo), (W, Wo)):
        np.testing.assert_array_equal(from_dev(d), o)


def test_rough_force_reproduces_masked_predictor(cuda_device):
    """Forcing the unmasked channel predictor with the indices of the rough-wall mask (wall value 0)
    gives the masked predictor of the rough-wall workload."""
    import prj
    import workloads
    nx, ny, nz = 48, 64, 32
    Uh, Vh, Wh, yu, dx, dz, solid = workloads.rough_projection_inputs(nx, ny, nz)
    U0, V0, W0, _, _, _ = workloads.projection_inputs(nx, ny, nz, seed=6, yu=yu)
    bot, top = rough_indices(solid, ny)
    inds = {f"{c}_{w}": (bot if w == "bot" else top) for c in "UVW" for w in ("bot", "top")}
    U, V, W = (to_dev(a) for a in (U0, V0, W0))
    prj.rough_force(U, V, W, dev_inds(inds))
    for d, want in ((U, Uh), (V, Vh), (W, Wh)):
        np.testing.assert_array_equal(from_dev(d)[1:-1, 1:-1, 1:-1], want[1:-1, 1:-1, 1:-1])


def test_ibm_interp_matches_oracle(cuda_device):
    import prj
    import pyoracle
    import torch
    nx, ny, nz = 20, 12, 16
    rng = np.random.default_rng(11)
    A = np.asfortranarray(rng.normal(size=(nx + 2, nz + 2, ny + 2)))
    size = A.size
    n = 300
    perm = rng.permutation(size)
    pos, src1, src2 = perm[:n], perm[n:2 * n], perm[2 * n:3 * n]
    pos = pos.astype(np.int64); src1 = src1.astype(np.int64); src2 = src2.astype(np.int64)
    c0, c1, c2 = (rng.normal(size=n) for _ in range(3))
    dst, src = perm[3 * n:3 * n + 40].astype(np.int64), pos[:40]
    want = pyoracle.ibm_interp(A, pos, src1, src2, c0, c1, c2, dst, src)
    d = to_dev(A)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")
    # offsets are into the Fortran-ordered storage, which is the tensor's contiguous storage
    prj.ibm_interp(d, T(pos), T(src1), T(src2), T(c0), T(c1), T(c2), T(dst), T(src))
    np.testing.assert_array_equal(from_dev(d), want)


def test_ibm_interp_rejects_outside_offsets(cuda_device):
    import prj
    import torch
    A = torch.zeros((6, 5, 4), dtype=torch.float64, device="cuda:0")
    T = lambda a, dt=torch.int64: torch.tensor(a, dtype=dt, device="cuda:0")
    with pytest.raises(prj.PrjError) as e:
        prj.ibm_interp(A, T([0, 120]), T([1, 2]), T([3, 4]), T([0.0, 0.0], torch.float64), T([1.0, 1.0], torch.float64),
                       T([1.0, 1.0], torch.float64))
    assert e.value.code == prj.PRJ_ERR_ARG
    assert float(A.abs().sum()) == 0.0
