"""Shared helpers for the tests: seeded inputs in the reference layout and
comparison metrics."""
from __future__ import annotations

import os

import numpy as np

from oracle import DKEYS, Layout, RADIUS


def report_dir():
    """Directory for JSON reports of the GPU tests (TTI_REPORT_DIR), or None."""
    d = os.environ.get("TTI_REPORT_DIR")
    return d if d and os.path.isdir(d) else None


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)


def random_model(lay: Layout, rng, tti=True, halo_safe=True):
    """Random but physically plausible model volumes over the whole halo'd
    allocation (the reference kernels read model halos)."""
    sh = lay.shape
    vp = rng.uniform(1800.0, 3200.0, sh)
    eps = rng.uniform(0.0, 0.25, sh)
    delta = eps * rng.uniform(0.0, 0.6, sh)
    vs = rng.uniform(0.0, 400.0, sh)
    theta = rng.uniform(0.0, 0.8, sh) if tti else np.zeros(sh)
    phi = rng.uniform(0.0, 3.0, sh) if tti else np.zeros(sh)
    m1 = vp * vp * (1 + 2 * eps)
    m2 = np.sqrt((vp * vp - vs * vs) * (vp * vp * (1 + 2 * delta) - vs * vs))
    m = dict(m1=m1, m2=m2, m3=vp * vp, m4=vs * vs, rx=np.sin(theta) * np.cos(phi),
             ry=np.sin(theta) * np.sin(phi), rz=np.cos(theta),
             irho=1.0 / rng.uniform(1.0, 2.5, sh))
    return {k: np.ascontiguousarray(v, np.float32) for k, v in m.items()}


def random_field(lay: Layout, rng, scale=1.0, halo=True):
    a = (scale * rng.standard_normal(lay.shape)).astype(np.float32)
    if not halo:
        b = np.zeros_like(a)
        b[lay.interior] = a[lay.interior]
        a = b
    return a


def sponge_ab(n_alloc, rng, active=True):
    ab = np.ones((n_alloc, 2), np.float32)
    if active:
        ab[:, 0] = rng.uniform(0.9, 1.0, n_alloc)
        ab[:, 1] = rng.uniform(0.9, 1.0, n_alloc)
    return np.ascontiguousarray(ab.reshape(-1))


def sponge_profile(n: int, ldim: int, width: int, absorb_low: bool):
    """The simulator's sponge (A,B) pairs per global index (host logic mirror)."""
    ab = np.ones((ldim, 2), np.float32)
    for k in range(min(width, n)):
        g = np.float32(np.exp(-((0.3 * (width - k) / width) ** 2)))
        if absorb_low:
            ab[RADIUS + k] = g
        ab[RADIUS + n - 1 - k] = np.minimum(ab[RADIUS + n - 1 - k], g)
    return np.ascontiguousarray(ab.reshape(-1))


def sim_models(sim):
    names = ("irho", "model1", "model2", "model3", "model4", "rx", "ry", "rz")
    keys = ("irho", "m1", "m2", "m3", "m4", "rx", "ry", "rz")
    return {k: np.ascontiguousarray(sim.volume(n)) for k, n in zip(keys, names)}


def oracle_rtm(o, lay, m, ab, cfg, src, wavelet, rec, residual=None, adjoint=True):
    """Reference-order RTM with the oracle: forward with snapshots every
    xcorr_step steps, adjoint driven by residual traces, Vp image and density
    gradient at snapshot steps (simulator2SetUp.cu:517-782 with nsub = 1)."""
    from oracle import new_state

    dt = np.float32(cfg.dt)
    h = (cfg.dx, cfg.dy, cfg.dz)
    g = o.grid(lay, dt, h, free_surface=cfg.free_surface, sponge_active=cfg.sponge_width > 0)
    st = new_state(lay, o.dtype)
    nrec = len(rec)
    traces = np.zeros((cfg.nt, nrec), o.dtype)
    snaps = {}
    I = lay.interior
    for n in range(cfg.nt):
        row = np.zeros(nrec, o.dtype)
        o.fwd_step(g, st, m, ab, src, float(wavelet[n]), rec, row)
        traces[n] = row
        if adjoint and n % cfg.xcorr_step == 0:
            snaps[n] = [st[k][I].copy() for k in ("f3", "f4", "f1", "f2")]
    out = {"traces": traces, "f3": st["f3"].copy(), "f4": st["f4"].copy()}
    if not adjoint:
        return out
    res = traces if residual is None else residual.astype(o.dtype)
    adj = new_state(lay, o.dtype)
    n_in = lay.nx * lay.ny * lay.nz
    gvp = np.zeros(n_in, o.dtype)
    grho = np.zeros(n_in, o.dtype)
    for n in range(cfg.nt - 1, -1, -1):
        o.adj_step(g, adj, m, ab, rec, np.ascontiguousarray(res[n]))
        if n % cfg.xcorr_step == 0:
            s3, s4, s1, s2 = snaps[n]
            o.update_vp_gradient(lay, np.ascontiguousarray(s3.ravel()), np.ascontiguousarray(s4.ravel()),
                                 gvp, adj["f3"], adj["f4"])
            p, q = lay.zeros(o.dtype), lay.zeros(o.dtype)
            p[I] = s1
            q[I] = s2
            if cfg.free_surface:
                o.loop4(lay, p, q)
            d = {k: lay.zeros(o.dtype) for k in DKEYS}
            o.fwd_drv(lay, p, q, m["irho"], d, tuple(np.float32(1.0 / v) for v in h))
            if cfg.free_surface:
                o.loop4_derivatives(lay, d)
            o.rho_gradient(lay, grho, d, adj["f1"], adj["f2"], m, h, lay.nx, lay.ny)
    o.finalize_vp_gradient(lay, m["m3"], gvp, np.float32(cfg.dt * cfg.xcorr_step))
    out["grad_vp"] = gvp.reshape(lay.nz, lay.ny, lay.nx)
    out["grad_rho"] = grho.reshape(lay.nz, lay.ny, lay.nx)
    return out


def oracle_rtm_t1(o, lay, m, ab, cfg, src, wavelet, rec, residual=None):
    """RTM with the centred constant-density operator (scheme 1), composed
    from the oracle's type1 restatement in the simulator's step order:
    forward step: loop2, loop4, fwd_main_loop_2_1 (sponge form when the
    sponge is on), source, receivers; adjoint step: residual injection,
    adj_main_loop_2, loop2, loop4; Vp image (update_grad_loop) at snapshot
    steps, then the simulator's Vp finalisation."""
    dt = np.float32(cfg.dt)
    h = (cfg.dx, cfg.dy, cfg.dz)
    sponge = cfg.sponge_width > 0
    f1, f2, f3, f4 = (lay.zeros() for _ in range(4))
    nrec = len(rec)
    traces = np.zeros((cfg.nt, nrec), np.float32)
    snaps = {}
    I = lay.interior
    for n in range(cfg.nt):
        o.loop2(lay, f1, f2, f3, f4, ab[0], ab[1], ab[2], dt)
        if cfg.free_surface:
            o.loop4(lay, f1, f2)
        o.t1_fwd(lay, f3, f4, f1, f2, m, ab, dt, h, 1 if sponge else 0)
        if src >= 0:
            f3.flat[src] += np.float32(wavelet[n]) * dt
            f4.flat[src] += np.float32(wavelet[n]) * dt
        traces[n] = -(2 * f1.flat[rec] + f2.flat[rec]) / np.float32(3)
        if n % cfg.xcorr_step == 0:
            snaps[n] = (np.ascontiguousarray(f3[I].ravel()), np.ascontiguousarray(f4[I].ravel()))
    res = (traces if residual is None else residual).astype(np.float32)
    a1, a2, a3, a4 = (lay.zeros() for _ in range(4))
    gvp = np.zeros(lay.nx * lay.ny * lay.nz, np.float32)
    for n in range(cfg.nt - 1, -1, -1):
        a3.flat[rec] += np.float32(-2.0 / 3.0) * res[n]
        a4.flat[rec] += np.float32(-1.0 / 3.0) * res[n]
        o.t1_adj(lay, a3, a4, a1, a2, m, ab, dt, h, sponge)
        o.loop2(lay, a1, a2, a3, a4, ab[0], ab[1], ab[2], dt)
        if cfg.free_surface:
            o.loop4(lay, a1, a2)
        if n % cfg.xcorr_step == 0:
            o.t1_grad(lay, snaps[n][0], snaps[n][1], gvp, a3, a4)
    o.finalize_vp_gradient(lay, m["m3"], gvp, np.float32(cfg.dt * cfg.xcorr_step))
    return {"traces": traces, "f3": f3, "grad_vp": gvp.reshape(lay.nz, lay.ny, lay.nx)}
