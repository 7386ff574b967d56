"""Seeded synthetic earth models, wavelets and acquisition geometry for the
TTI/VTI RTM workloads.

The reference ships no data: its simulator hard-codes a constant medium
(vp=1500 m/s, eps=delta=vs=theta=phi=0; simulator2/simulator2SetUp.h:45-55)
and an impulse at the centre.  These generators stand in for real models,
with the shapes, sizes and value ranges of the benchmark workloads:

* ``layered_vti``: flat layers at seeded random depths, vp ~ U[1500,4500],
  eps ~ U[0,0.3], delta ~ U[0, min(0.15, eps)], vs = 0, theta = phi = 0, rho = 1.
* ``smooth_tti``: Gaussian-correlated random fields (correlation length in
  metres) mapped to vp in [1500,5000], eps in [0,0.25], delta in [0,0.1]
  with delta <= eps, theta in [0,45] degrees, phi in [0,180] degrees.

Arrays are float32 with shape (nz, ny, nx) (x fastest in memory).
"""
from __future__ import annotations

import numpy as np


def layered_vti(nx, ny, nz, nlayers=6, seed=1234):
    rng = np.random.default_rng(seed)
    tops = np.sort(rng.choice(np.arange(1, nz), size=nlayers - 1, replace=False))
    bounds = np.concatenate([[0], tops, [nz]])
    vp1 = rng.uniform(1500.0, 4500.0, nlayers)
    eps1 = rng.uniform(0.0, 0.3, nlayers)
    delta1 = np.array([rng.uniform(0.0, min(0.15, e)) for e in eps1])
    vp = np.empty((nz, ny, nx), np.float32)
    eps = np.empty_like(vp)
    delta = np.empty_like(vp)
    for k in range(nlayers):
        sl = slice(bounds[k], bounds[k + 1])
        vp[sl] = vp1[k]
        eps[sl] = eps1[k]
        delta[sl] = delta1[k]
    zeros = np.zeros_like(vp)
    return dict(vp=vp, eps=eps, delta=delta, vs=zeros, theta=zeros.copy(), phi=zeros.copy(),
                rho=np.ones_like(vp))


def gaussian_field(shape, corr_cells, rng):
    """Unit-range smooth random field: white noise filtered by a Gaussian of
    the given correlation length (cells) in the Fourier domain, mapped to [0,1]."""
    noise = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) for n in shape]
    kz, ky, kx = np.meshgrid(*k, indexing="ij")
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2) * (corr_cells ** 2) / 4.0)
    f = np.real(np.fft.ifftn(np.fft.fftn(noise) * filt))
    f -= f.min()
    f /= max(f.max(), 1e-30)
    return f.astype(np.float32)


def smooth_tti(nx, ny, nz, dx=10.0, corr_m=300.0, seed=1234):
    rng = np.random.default_rng(seed)
    shape = (nz, ny, nx)
    c = corr_m / dx
    vp = 1500.0 + 3500.0 * gaussian_field(shape, c, rng)
    eps = 0.25 * gaussian_field(shape, c, rng)
    delta = np.minimum(0.1 * gaussian_field(shape, c, rng), eps)
    theta = np.deg2rad(45.0) * gaussian_field(shape, c, rng)
    phi = np.deg2rad(180.0) * gaussian_field(shape, c, rng)
    zeros = np.zeros(shape, np.float32)
    return dict(vp=vp.astype(np.float32), eps=eps.astype(np.float32), delta=delta.astype(np.float32),
                vs=zeros, theta=theta.astype(np.float32), phi=phi.astype(np.float32),
                rho=np.ones(shape, np.float32))


def add_velocity_blob(model, center, radius_cells, fraction=0.05):
    """Copy of ``model`` with vp raised by ``fraction`` inside a Gaussian blob."""
    m = {k: v.copy() for k, v in model.items()}
    nz, ny, nx = m["vp"].shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r2 = (x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2
    m["vp"] = (m["vp"] * (1.0 + fraction * np.exp(-r2 / (2.0 * radius_cells ** 2)))).astype(np.float32)
    return m


def cfl_dt(model, dx, cfl=0.4):
    """dt = cfl*dx / max(vp*sqrt(1+2*eps)) (the horizontal P speed)."""
    vmax = float(np.max(model["vp"] * np.sqrt(1.0 + 2.0 * model["eps"])))
    return float(cfl * dx / vmax)


def ricker(nt, dt, f0, t0=None):
    """Ricker wavelet of peak frequency f0, delayed by t0 (default 1.2/f0)."""
    t0 = 1.2 / f0 if t0 is None else t0
    t = np.arange(nt) * dt - t0
    a = (np.pi * f0 * t) ** 2
    return ((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)


def receiver_plane(nx, ny, iz):
    """Receivers on every (x, y) cell of plane iz: (nx*ny, 3) int32 of (ix, iy, iz)."""
    iy, ix = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    return np.stack([ix.ravel(), iy.ravel(), np.full(ix.size, iz)], axis=1).astype(np.int32)
