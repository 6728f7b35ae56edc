"""Seeded synthetic workloads of the channel projection (no dataset is involved).

The reference measures on user cases (``input/yu.txt`` + restart files); these
generators stand in for them with the shapes, grids and value distributions of
the channel configurations the engine is benchmarked on.

Layout: numpy arrays indexed ``[x, z, y]`` in Fortran order (x fastest, the
reference's ``P(i, j, k)``); halo'd fields are ``(nx+2, nz+2, ny+2)``.
"""
from __future__ import annotations

import numpy as np


def tanh_faces(ny: int, beta: float = 2.0) -> np.ndarray:
    """Faces y_j = 1 + tanh(beta (2j/ny - 1)) / tanh(beta), j = 0..ny; walls at y = 0 and 2."""
    j = np.arange(ny + 1, dtype=np.float64)
    return 1.0 + np.tanh(beta * (2.0 * j / ny - 1.0)) / np.tanh(beta)


def wall_refined_faces(ny: int, h_uniform: float = 0.1, growth: float = 0.015) -> np.ndarray:
    """Faces uniform for y < h_uniform, then growing by ``growth`` per cell toward the
    centre, mirrored about y = 1 (walls at 0 and 2).  ny must be even."""
    if ny % 2:
        raise ValueError("ny must be even")
    half = ny // 2
    # find the first spacing d0 such that the half channel closes at y = 1
    def total(d0):
        y, d, out = 0.0, d0, [0.0]
        for _ in range(half):
            y += d
            out.append(y)
            if y >= h_uniform:
                d *= 1.0 + growth
        return y, out
    lo, hi = 1e-9, 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if total(mid)[0] > 1.0:
            hi = mid
        else:
            lo = mid
    _, half_faces = total(0.5 * (lo + hi))
    h = np.array(half_faces) / half_faces[-1]
    return np.concatenate([h, 2.0 - h[-2::-1]])


def channel_spacing(nx: int, nz: int, lx: float = 2 * np.pi, lz: float = np.pi):
    return lx / nx, lz / nz


def poisson_rhs(nx: int, ny: int, nz: int, beta: float = 2.0, seed: int = 0):
    """Poisson case: uniform[-1,1] RHS minus its dy-weighted mean on tanh faces.

    Lx = 2 pi, Lz = pi.  Returns (rhs [x, z, y] F-order, yu, dx, dz)."""
    yu = tanh_faces(ny, beta)
    dx, dz = channel_spacing(nx, nz)
    rng = np.random.default_rng(seed)
    rhs = rng.uniform(-1.0, 1.0, size=(nx, nz, ny))
    w = np.diff(yu)
    rhs -= (rhs.sum(axis=(0, 1)) * w).sum() / (nx * nz * w.sum())
    return np.asfortranarray(rhs), yu, dx, dz


def projection_inputs(nx: int, ny: int, nz: int, beta: float = 2.0, seed: int = 1, sigma: float = 0.1, yu=None):
    """Predictor field of the channel projection: Poiseuille u = 1.5 (1 - (y-1)^2) plus
    N(0, sigma) noise in u, v, w (drawn in that order from default_rng(seed)); v = 0 on
    both walls.  Interior values only (the engine wraps periodic halos itself).

    Returns (Uh, Vh, Wh, yu, dx, dz)."""
    if yu is None:
        yu = tanh_faces(ny, beta)
    yp = (yu[:-1] + yu[1:]) / 2
    dx, dz = channel_spacing(nx, nz)
    rng = np.random.default_rng(seed)
    shape = (nx + 2, nz + 2, ny + 2)
    Uh = np.zeros(shape, order="F")
    Vh = np.zeros(shape, order="F")
    Wh = np.zeros(shape, order="F")
    Uh[1:-1, 1:-1, 1:-1] = 1.5 * (1.0 - (yp[None, None, :] - 1.0) ** 2) + rng.normal(0.0, sigma, size=(nx, nz, ny))
    Vh[1:-1, 1:-1, 1:-1] = rng.normal(0.0, sigma, size=(nx, nz, ny))
    Wh[1:-1, 1:-1, 1:-1] = rng.normal(0.0, sigma, size=(nx, nz, ny))
    Vh[:, :, 1] = 0.0  # V(k = 0) is the bottom wall face
    return Uh, Vh, Wh, yu, dx, dz


def halo_shape(nx, nz, ny):
    return (nx + 2, nz + 2, ny + 2)


def rough_height_field(nx: int, nz: int, lx: float = 2 * np.pi, lz: float = np.pi, seed: int = 5,
                       kmin: float = 2 * np.pi / 0.5, kmax: float = 2 * np.pi / 0.05, peak: float = 0.08,
                       rms: float = 0.02) -> np.ndarray:
    """Rough-wall height h(x, z) >= 0 at the cell centres, shape (nx, nz).

    A Gaussian random field g with isotropic power spectrum |k|^-2 for kmin <= |k| <= kmax
    (zero elsewhere; complex normal Fourier coefficients from default_rng(seed)) is mapped to
    h = max(0, peak - s (max g - g)), with s found by bisection so that sqrt(mean h^2) = rms.
    The map fixes both the peak height and the RMS height, and h = 0 marks smooth wall."""
    rng = np.random.default_rng(seed)
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=lx / nx)
    kz = 2 * np.pi * np.fft.rfftfreq(nz, d=lz / nz)
    k = np.hypot(kx[:, None], kz[None, :])
    amp = np.zeros_like(k)
    band = (k >= kmin) & (k <= kmax)
    amp[band] = 1.0 / k[band]
    coef = amp * (rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape))
    g = np.fft.irfft2(coef, s=(nx, nz))
    g = (g - g.mean()) / g.std()
    gap = g.max() - g

    def rms_of(s):
        return np.sqrt(np.mean(np.maximum(0.0, peak - s * gap) ** 2))

    lo, hi = 0.0, 1.0
    while rms_of(hi) > rms:
        hi *= 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if rms_of(mid) > rms:
            lo = mid
        else:
            hi = mid
    return np.maximum(0.0, peak - 0.5 * (lo + hi) * gap)


def solid_cells(h: np.ndarray, yu: np.ndarray) -> np.ndarray:
    """Cells (i, k, j) inside the roughness, shape (nx, nz, ny): cell centre y_p below h on the
    bottom wall or above 2 - h on the top wall (the same height field on both walls)."""
    yp = (yu[:-1] + yu[1:]) / 2
    return (yp[None, None, :] < h[:, :, None]) | (yp[None, None, :] > 2.0 - h[:, :, None])


def rough_projection_inputs(nx: int, ny: int, nz: int, seed: int = 5, sigma: float = 0.1):
    """Projection inputs of the rough-wall channel: wall-refined faces (uniform below
    y = 0.1, 1.5% growth toward the centre), the channel predictor of projection_inputs
    (noise from default_rng(seed + 1)), and every velocity component whose cell lies in the
    roughness (height field from default_rng(seed)) set to zero.

    Returns (Uh, Vh, Wh, yu, dx, dz, solid) with solid[x, z, y] boolean."""
    yu = wall_refined_faces(ny)
    Uh, Vh, Wh, yu, dx, dz = projection_inputs(nx, ny, nz, seed=seed + 1, sigma=sigma, yu=yu)
    solid = solid_cells(rough_height_field(nx, nz, seed=seed), yu)
    for f in (Uh, Vh, Wh):
        f[1:-1, 1:-1, 1:-1][solid] = 0.0
    return Uh, Vh, Wh, yu, dx, dz, solid


def fill_halos(F: np.ndarray) -> np.ndarray:
    """Fill the halos of a halo'd [x+2, z+2, y+2] field in place: periodic images in x and z,
    and the wall ghost planes y = -1, ny as copies of y = 0, ny-1 (the P_per rule of
    mod_cfd_subroutines.f90:1087-1118).  Returns F."""
    F[0, :, :] = F[-2, :, :]
    F[-1, :, :] = F[1, :, :]
    F[:, 0, :] = F[:, -2, :]
    F[:, -1, :] = F[:, 1, :]
    F[:, :, 0] = F[:, :, 1]
    F[:, :, -1] = F[:, :, -2]
    return F


def vd_inputs(nx: int, ny: int, nz: int, seed: int = 4, beta: float = 2.0, rho_const=None):
    """Inputs of the variable-density projection: the channel predictor of projection_inputs,
    a density rho(y) = 1 - 0.6 (1 - (y-1)^2) (light core, dense walls) times 1 + N(0, 0.05),
    pressures P_now, P_old ~ N(0, 0.01) and div_now ~ N(0, 0.01), all halo'd with filled halos
    (draws from default_rng(seed + 1) after the predictor's default_rng(seed)).  With rho_const
    the density is that constant.

    Returns (Uh, Vh, Wh, rho, P_now, P_old, div_now, yu, dx, dz)."""
    Uh, Vh, Wh, yu, dx, dz = projection_inputs(nx, ny, nz, beta=beta, seed=seed)
    yp = (yu[:-1] + yu[1:]) / 2
    rng = np.random.default_rng(seed + 1)
    shape = (nx + 2, nz + 2, ny + 2)
    rho = np.zeros(shape, order="F")
    if rho_const is None:
        rho[1:-1, 1:-1, 1:-1] = (1.0 - 0.6 * (1.0 - (yp[None, None, :] - 1.0) ** 2)) * (
            1.0 + rng.normal(0.0, 0.05, size=(nx, nz, ny)))
    else:
        rho[1:-1, 1:-1, 1:-1] = rho_const
    P_now = np.zeros(shape, order="F")
    P_old = np.zeros(shape, order="F")
    div_now = np.zeros(shape, order="F")
    P_now[1:-1, 1:-1, 1:-1] = rng.normal(0.0, 0.01, size=(nx, nz, ny))
    P_old[1:-1, 1:-1, 1:-1] = rng.normal(0.0, 0.01, size=(nx, nz, ny))
    div_now[1:-1, 1:-1, 1:-1] = rng.normal(0.0, 0.01, size=(nx, nz, ny))
    for F in (rho, P_now, P_old, div_now):
        fill_halos(F)
    return Uh, Vh, Wh, rho, P_now, P_old, div_now, yu, dx, dz
