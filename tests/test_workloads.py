"""CPU tests of the seeded workload generators (grids, rough-wall height field)."""
import numpy as np


def test_wall_refined_faces():
    import workloads
    yu = workloads.wall_refined_faces(512)
    d = np.diff(yu)
    assert yu[0] == 0.0 and yu[-1] == 2.0 and yu.size == 513
    np.testing.assert_allclose(d, d[::-1], rtol=0, atol=1e-15)  # mirrored about y = 1
    n0 = int((yu[:257] < 0.1).sum())  # uniform cells below y = 0.1
    np.testing.assert_allclose(d[:n0 - 1], d[0], rtol=1e-12)
    ratio = d[n0:256] / d[n0 - 1:255]
    np.testing.assert_allclose(ratio, 1.015, rtol=1e-12)


def test_rough_height_field_peak_rms():
    import workloads
    h = workloads.rough_height_field(192, 96, seed=5)
    assert h.shape == (192, 96)
    assert abs(h.max() - 0.08) < 1e-15 and h.min() >= 0.0
    assert abs(np.sqrt(np.mean(h ** 2)) - 0.02) < 1e-12
    # seeded: the same seed gives the same field
    h2 = workloads.rough_height_field(192, 96, seed=5)
    np.testing.assert_array_equal(h, h2)


def test_rough_inputs_zero_inside_roughness():
    import workloads
    Uh, Vh, Wh, yu, dx, dz, solid = workloads.rough_projection_inputs(48, 64, 32)
    assert solid.any() and not solid.all()
    for f in (Uh, Vh, Wh):
        assert np.all(f[1:-1, 1:-1, 1:-1][solid] == 0.0)
        assert np.any(f[1:-1, 1:-1, 1:-1][~solid] != 0.0)
    assert np.all(Vh[:, :, 1] == 0.0)
    # solid cells sit next to the walls only
    yp = (yu[:-1] + yu[1:]) / 2
    js = np.nonzero(solid.any(axis=(0, 1)))[0]
    assert np.all((yp[js] < 0.08) | (yp[js] > 1.92))
