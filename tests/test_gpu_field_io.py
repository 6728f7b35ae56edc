"""Device-side field files: staged through pinned host memory in y-plane chunks."""
import numpy as np
import pytest

from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(5, 3, 4), (256, 192, 400)])
def test_device_round_trip_matches_host(cuda_device, tmp_path, shape):
    """A device write gives the host writer's bytes; a device read restores the field; 256 x 192
    x 400 spans several 64 MB staging chunks."""
    import prj
    import torch
    nx, nz, ny = shape
    A = np.asfortranarray(np.random.default_rng(9).normal(size=shape))
    p_host, p_dev = str(tmp_path / "h.dat"), str(tmp_path / "d.dat")
    prj.write_field(p_host, A)
    prj.write_field(p_dev, to_dev(A))
    assert open(p_host, "rb").read() == open(p_dev, "rb").read()
    t = torch.empty((ny, nz, nx), dtype=torch.float64, device="cuda:0")
    prj.read_field(p_host, t)
    np.testing.assert_array_equal(from_dev(t), A)


def test_device_halo_interior(cuda_device, tmp_path):
    import prj
    import torch
    nx, nz, ny = 33, 17, 300
    H = np.asfortranarray(np.random.default_rng(4).normal(size=(nx + 2, nz + 2, ny + 2)))
    path = str(tmp_path / "h.dat")
    prj.write_field(path, to_dev(H), halo=True)
    np.testing.assert_array_equal(prj.read_field(path), H[1:-1, 1:-1, 1:-1])
    G = torch.full((ny + 2, nz + 2, nx + 2), -3.0, dtype=torch.float64, device="cuda:0")
    prj.read_field(path, G, halo=True)
    g = from_dev(G)
    np.testing.assert_array_equal(g[1:-1, 1:-1, 1:-1], H[1:-1, 1:-1, 1:-1])
    g[1:-1, 1:-1, 1:-1] = -3.0
    assert np.all(g == -3.0)
