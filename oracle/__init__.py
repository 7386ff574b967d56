"""CPU oracle for the TTI/VTI RTM hot path -- TEST INFRASTRUCTURE ONLY.

Python bindings (ctypes + numpy) over ``liboracle_tti.so``, the plain-C
restatement of the reference kernels in ``tti_oracle.c``.  Only the tests,
the smoke check and the CPU-baseline leg of ``bench.py`` may import this
package; the product library never does.

``Layout`` describes the reference volume layout (x fastest, radius-4 halo
on every axis, ``ldimx`` padded to 32 floats: infrastructure/axis.cpp:78-99,
utils/volume_index.h:20-23).  Volumes are numpy arrays of shape
``(ldimz, ldimy, ldimx)``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_tti.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref_tti.so")
RADIUS = 4


def pad32(n: int) -> int:
    return 32 * ((n - 1) // 32 + 1)


@dataclass(frozen=True)
class Layout:
    """Interior grid (nx, ny, nz) with the reference's halo/padding layout."""

    nx: int
    ny: int
    nz: int

    @property
    def ldimx(self) -> int:
        return pad32(self.nx + 2 * RADIUS)

    @property
    def ldimy(self) -> int:
        return self.ny + 2 * RADIUS

    @property
    def ldimz(self) -> int:
        return self.nz + 2 * RADIUS

    @property
    def shape(self):
        return (self.ldimz, self.ldimy, self.ldimx)

    @property
    def nvol(self) -> int:
        return self.ldimx * self.ldimy * self.ldimz

    @property
    def ranges(self):
        """(ixbeg, ixend, iybeg, iyend, izbeg, izend), inclusive, halo excluded."""
        r = RADIUS
        return (r, r + self.nx - 1, r, r + self.ny - 1, r, r + self.nz - 1)

    @property
    def interior(self):
        r = RADIUS
        return (slice(r, r + self.nz), slice(r, r + self.ny), slice(r, r + self.nx))

    def zeros(self, dtype=np.float32):
        return np.zeros(self.shape, dtype=dtype)

    def index(self, ix: int, iy: int, iz: int) -> int:
        """Flat index of an interior cell given 0-based interior coordinates."""
        r = RADIUS
        return ((iz + r) * self.ldimy + (iy + r)) * self.ldimx + (ix + r)


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


class OrcGrid(C.Structure):
    _fields_ = [
        ("ldimx", C.c_int), ("ldimy", C.c_int), ("ldimz", C.c_int),
        ("ixbeg", C.c_int), ("ixend", C.c_int), ("iybeg", C.c_int), ("iyend", C.c_int),
        ("izbeg", C.c_int), ("izend", C.c_int),
        ("free_surface", C.c_int), ("sponge_active", C.c_int),
        ("dt", C.c_float), ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
    ]


V, I, F, D, L = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_int64
_SIGS = {
    "orc_coefficients": [V, V, V],
    "orc_loop2": [V, V, V, V, I, I, I, I, I, I, I, I, V, V, V, F],
    "orc_loop4": [V, V, I, I, I],
    "orc_fwd_drv": [V] * 9 + [I] * 6 + [F] * 3 + [I, I],
    "orc_loop4_derivatives": [V] * 6 + [I, I, I],
    "orc_fwd_update": [V] * 18 + [I] * 8 + [F, D, D, D],
    "orc_adj_drv": [V] * 18 + [I] * 6 + [F] * 3 + [I, I] + [F] * 3,
    "orc_adj_update": [V] * 13 + [I] * 8 + [F, D, D, D, I],
    "orc_update_vp_gradient": [V] * 5 + [I] * 10,
    "orc_finalize_vp_gradient": [V, V] + [I] * 10 + [F],
    "orc_rho_gradient": [V] * 17 + [I] * 10 + [D, D, D],
    "orc_init_cijs": [V] * 13 + [L],
    "orc_pressure": [V, V, V, L],
    "orc_fwd_step": [C.POINTER(OrcGrid)] + [V] * 21 + [L, F, I, V, V],
    "orc_adj_step": [C.POINTER(OrcGrid)] + [V] * 23 + [I, V, V],
    "orc_t1_fwd": [V] * 14 + [I] * 10 + [F, D, D, D, I],
    "orc_t1_adj": [V] * 14 + [I] * 8 + [F, D, D, D, I],
    "orc_t1_grad": [V] * 5 + [I] * 10,
    "orc_num_threads": [],
}


class Oracle:
    """One precision of the C oracle: ``Oracle('f32')`` or ``Oracle('f64')``."""

    def __init__(self, precision: str = "f32"):
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle`")
        self.lib = C.CDLL(LIB_PATH)
        self.precision = precision
        self.dtype = np.float32 if precision == "f32" else np.float64
        self.fn = {}
        for name, sig in _SIGS.items():
            f = getattr(self.lib, f"{name}_{precision}")
            f.argtypes = sig
            f.restype = I if name == "orc_num_threads" else None
            self.fn[name] = f

    def _chk(self, *arrs):
        for a in arrs:
            if a is not None and a.dtype != self.dtype:
                raise TypeError(f"expected {self.dtype}, got {a.dtype}")

    @staticmethod
    def coefficients():
        c1 = np.zeros(5, np.float32)
        c2 = np.zeros(5, np.float32)
        cs = np.zeros(4, np.float32)
        lib = C.CDLL(LIB_PATH)
        f = lib.orc_coefficients_f32
        f.argtypes = [V, V, V]
        f(_p(c1), _p(c2), _p(cs))
        return c1, c2, cs

    def num_threads(self) -> int:
        return int(self.fn["orc_num_threads"]())

    # --- per-kernel restatements ------------------------------------------
    def loop2(self, lay: Layout, f1, f2, f3, f4, abx, aby, abz, dt):
        self._chk(f1, f2, f3, f4)
        self.fn["orc_loop2"](_p(f1), _p(f2), _p(f3), _p(f4), lay.ldimx, lay.ldimy, *lay.ranges,
                             _p(abx), _p(aby), _p(abz), dt)

    def loop4(self, lay: Layout, f1, f2):
        self._chk(f1, f2)
        self.fn["orc_loop4"](_p(f1), _p(f2), lay.ldimx, lay.ldimy, RADIUS)

    def fwd_drv(self, lay: Layout, f1, f2, irho, d, invd):
        """d: dict with keys d1x,d1y,d1z,d2x,d2y,d2z."""
        self._chk(f1, f2, irho, *d.values())
        self.fn["orc_fwd_drv"](_p(f1), _p(f2), _p(irho), _p(d["d1x"]), _p(d["d1y"]), _p(d["d1z"]),
                               _p(d["d2x"]), _p(d["d2y"]), _p(d["d2z"]), *lay.ranges, *invd,
                               lay.ldimx, lay.ldimy)

    def loop4_derivatives(self, lay: Layout, d):
        self.fn["orc_loop4_derivatives"](_p(d["d1x"]), _p(d["d1y"]), _p(d["d1z"]), _p(d["d2x"]),
                                         _p(d["d2y"]), _p(d["d2z"]), lay.ldimx, lay.ldimy, RADIUS)

    def fwd_update(self, lay: Layout, f3, f4, d, f1, f2, m, dt, h):
        """m: dict irho,m1,m2,m3,m4,rx,ry,rz; h = (dx, dy, dz)."""
        self._chk(f3, f4, f1, f2)
        self.fn["orc_fwd_update"](_p(f3), _p(f4), _p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]),
                                  _p(d["d2y"]), _p(d["d1z"]), _p(d["d2z"]), _p(f1), _p(f2),
                                  _p(m["irho"]), _p(m["m1"]), _p(m["m2"]), _p(m["m3"]), _p(m["m4"]),
                                  _p(m["rx"]), _p(m["ry"]), _p(m["rz"]), *lay.ranges, lay.ldimx,
                                  lay.ldimy, dt, *h)

    def adj_drv(self, lay: Layout, d, rhs3, rhs4, f1, f2, m, h):
        dx, dy, dz = h
        self._chk(rhs3, rhs4, f1, f2)
        self.fn["orc_adj_drv"](_p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]), _p(d["d2y"]), _p(d["d1z"]),
                               _p(d["d2z"]), _p(rhs3), _p(rhs4), _p(f1), _p(f2), _p(m["irho"]),
                               _p(m["m1"]), _p(m["m2"]), _p(m["m3"]), _p(m["m4"]), _p(m["rx"]),
                               _p(m["ry"]), _p(m["rz"]), *lay.ranges,
                               np.float32(1.0 / (4 * dx * dy)), np.float32(1.0 / (4 * dy * dz)),
                               np.float32(1.0 / (4 * dx * dz)), lay.ldimx, lay.ldimy,
                               np.float32(1.0 / dx), np.float32(1.0 / dy), np.float32(1.0 / dz))

    def adj_update(self, lay: Layout, f3, f4, d, rhs3, rhs4, abx, aby, abz, dt, h, sponge_active):
        self._chk(f3, f4, rhs3, rhs4)
        self.fn["orc_adj_update"](_p(f3), _p(f4), _p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]),
                                  _p(d["d2y"]), _p(d["d1z"]), _p(d["d2z"]), _p(rhs3), _p(rhs4),
                                  _p(abx), _p(aby), _p(abz), *lay.ranges, lay.ldimx, lay.ldimy, dt,
                                  *h, int(sponge_active))

    def update_vp_gradient(self, lay: Layout, snap3, snap4, grad, adj3, adj4):
        self.fn["orc_update_vp_gradient"](_p(snap3), _p(snap4), _p(grad), _p(adj3), _p(adj4),
                                          *lay.ranges, lay.nx, lay.ny, lay.ldimx, lay.ldimy)

    def finalize_vp_gradient(self, lay: Layout, model3, grad, dt_xcorr):
        self.fn["orc_finalize_vp_gradient"](_p(model3), _p(grad), *lay.ranges, lay.nx, lay.ny,
                                            lay.ldimx, lay.ldimy, dt_xcorr)

    def rho_gradient(self, lay: Layout, grad, fd, f1, f2, m, h, grad_ldimx=None, grad_ldimy=None):
        gx = lay.ldimx if grad_ldimx is None else grad_ldimx
        gy = lay.ldimy if grad_ldimy is None else grad_ldimy
        self.fn["orc_rho_gradient"](_p(grad), _p(fd["d1x"]), _p(fd["d2x"]), _p(fd["d1y"]),
                                    _p(fd["d2y"]), _p(fd["d1z"]), _p(fd["d2z"]), _p(f1), _p(f2),
                                    _p(m["irho"]), _p(m["m1"]), _p(m["m2"]), _p(m["m3"]),
                                    _p(m["m4"]), _p(m["rx"]), _p(m["ry"]), _p(m["rz"]), *lay.ranges,
                                    lay.ldimx, lay.ldimy, gx, gy, *h)

    # Type1 (constant density, centred): tests/test_type1*.py.
    def t1_fwd(self, lay: Layout, f3, f4, f1, f2, m, ab, dt, h, mode, out_ld=None):
        """mode 0: f3,f4 += dt*rhs; 1: sponge form; 2: rhs into halo-free f3,f4 (out_ld = (ldx, ldy))."""
        ox, oy = out_ld if out_ld else (lay.ldimx, lay.ldimy)
        self.fn["orc_t1_fwd"](_p(f3), _p(f4), _p(f1), _p(f2), _p(m["m1"]), _p(m["m2"]), _p(m["m3"]),
                              _p(m["m4"]), _p(m["rx"]), _p(m["ry"]), _p(m["rz"]), _p(ab[0]), _p(ab[1]),
                              _p(ab[2]), *lay.ranges, lay.ldimx, lay.ldimy, ox, oy, dt, *h, mode)

    def t1_adj(self, lay: Layout, f3, f4, f1, f2, m, ab, dt, h, sponge):
        self.fn["orc_t1_adj"](_p(f3), _p(f4), _p(f1), _p(f2), _p(m["m1"]), _p(m["m2"]), _p(m["m3"]),
                              _p(m["m4"]), _p(m["rx"]), _p(m["ry"]), _p(m["rz"]), _p(ab[0]), _p(ab[1]),
                              _p(ab[2]), *lay.ranges, lay.ldimx, lay.ldimy, dt, *h, int(sponge))

    def t1_grad(self, lay: Layout, snap_x, snap_z, grad, adj_x, adj_z):
        self.fn["orc_t1_grad"](_p(snap_x), _p(snap_z), _p(grad), _p(adj_x), _p(adj_z), *lay.ranges,
                               lay.nx, lay.ny, lay.ldimx, lay.ldimy)

    def init_cijs(self, vp, eps, delta, vs, theta, phi):
        n = vp.size
        out = [np.zeros(vp.shape, self.dtype) for _ in range(7)]
        args = [np.ascontiguousarray(a, np.float32) for a in (vp, eps, delta, vs, theta, phi)]
        self.fn["orc_init_cijs"](*[_p(a) for a in args], *[_p(o) for o in out], n)
        return out

    # --- step drivers ------------------------------------------------------
    def grid(self, lay: Layout, dt, h, free_surface=True, sponge_active=False) -> OrcGrid:
        return OrcGrid(lay.ldimx, lay.ldimy, lay.ldimz, *lay.ranges, int(free_surface),
                       int(sponge_active), dt, *h)

    def fwd_step(self, g: OrcGrid, st, m, ab, src_index=-1, src_amp=0.0, rec_index=None,
                 traces=None):
        d = st["d"]
        nrec = 0 if rec_index is None else len(rec_index)
        self.fn["orc_fwd_step"](C.byref(g), _p(st["f1"]), _p(st["f2"]), _p(st["f3"]), _p(st["f4"]),
                                _p(d["d1x"]), _p(d["d1y"]), _p(d["d1z"]), _p(d["d2x"]), _p(d["d2y"]),
                                _p(d["d2z"]), _p(m["irho"]), _p(m["m1"]), _p(m["m2"]), _p(m["m3"]),
                                _p(m["m4"]), _p(m["rx"]), _p(m["ry"]), _p(m["rz"]), _p(ab[0]),
                                _p(ab[1]), _p(ab[2]), int(src_index), float(src_amp), nrec,
                                _p(rec_index), _p(traces))

    def adj_step(self, g: OrcGrid, st, m, ab, rec_index=None, residual=None):
        d = st["d"]
        nrec = 0 if rec_index is None else len(rec_index)
        self.fn["orc_adj_step"](C.byref(g), _p(st["f1"]), _p(st["f2"]), _p(st["f3"]), _p(st["f4"]),
                                _p(d["d1x"]), _p(d["d1y"]), _p(d["d1z"]), _p(d["d2x"]), _p(d["d2y"]),
                                _p(d["d2z"]), _p(st["rhs3"]), _p(st["rhs4"]), _p(m["irho"]),
                                _p(m["m1"]), _p(m["m2"]), _p(m["m3"]), _p(m["m4"]), _p(m["rx"]),
                                _p(m["ry"]), _p(m["rz"]), _p(ab[0]), _p(ab[1]), _p(ab[2]), nrec,
                                _p(rec_index), _p(residual))


DKEYS = ("d1x", "d1y", "d1z", "d2x", "d2y", "d2z")
MKEYS = ("irho", "m1", "m2", "m3", "m4", "rx", "ry", "rz")


def extend_to_layout(lay: Layout, a) -> np.ndarray:
    """Interior array of shape (nz, ny, nx) spread over the halo'd layout by
    repeating the nearest interior cell on every axis (x padding included)."""
    a = np.asarray(a, np.float32).reshape(lay.nz, lay.ny, lay.nx)
    r = RADIUS
    return np.ascontiguousarray(np.pad(a, ((r, r), (r, r), (r, lay.ldimx - lay.nx - r)), mode="edge"))


def models_from_parameters(lay: Layout, vp, eps=None, delta=None, vs=None, theta=None, phi=None, rho=None,
                           dtype=np.float32) -> dict:
    """Model volumes (irho, m1..m4, rx, ry, rz) from interior parameter arrays
    of shape (nz, ny, nx), built on the host the way the simulator defines
    its model set-up: every parameter is extended into the halo'd layout by
    repeating the nearest interior cell, the reference's per-cell
    ``init_cijs`` (simulator2SetUp.cu:10-29) maps (vp, eps, delta, vs, theta,
    phi) to model1..model7, and the buoyancy is irho = 1/rho in FP32 (the
    reference never sets Model11, kernel_type2.cu:136-141).  Missing
    parameters default to 0 (rho to 1)."""
    shape = (lay.nz, lay.ny, lay.nx)
    par = [np.zeros(shape, np.float32) if a is None else a for a in (eps, delta, vs, theta, phi)]
    full = [extend_to_layout(lay, a) for a in (vp, *par)]
    m1, m2, m3, m4, rx, ry, rz = Oracle("f32").init_cijs(*full)
    rho = np.ones(shape, np.float32) if rho is None else np.asarray(rho, np.float32)
    irho = extend_to_layout(lay, np.float32(1.0) / rho)
    out = dict(irho=irho, m1=m1, m2=m2, m3=m3, m4=m4, rx=rx, ry=ry, rz=rz)
    return {k: np.ascontiguousarray(v, dtype) for k, v in out.items()}


def new_state(lay: Layout, dtype=np.float32):
    st = {k: lay.zeros(dtype) for k in ("f1", "f2", "f3", "f4", "rhs3", "rhs4")}
    st["d"] = {k: lay.zeros(dtype) for k in DKEYS}
    return st


def sponge_profile(n: int, ldim: int, width: int, absorb_low: bool):
    """The simulator's sponge (A,B) pairs per global index (host logic mirror)."""
    ab = np.ones((ldim, 2), np.float32)
    for k in range(min(width, n)):
        g = np.float32(np.exp(-((0.3 * (width - k) / width) ** 2)))
        if absorb_low:
            ab[RADIUS + k] = g
        ab[RADIUS + n - 1 - k] = np.minimum(ab[RADIUS + n - 1 - k], g)
    return np.ascontiguousarray(ab.reshape(-1))


def rtm_shot(o, lay, m, ab, cfg, src, wavelet, rec, residual=None, adjoint=True, observed=None):
    """Reference-order RTM with the oracle: forward with snapshots every
    xcorr_step steps, adjoint driven by residual traces, Vp image and density
    gradient at snapshot steps (simulator2SetUp.cu:517-782 with nsub = 1).
    With ``observed`` the residual is the oracle's own traces minus it (the
    simulator's adjoint_observed)."""
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
    if observed is not None:
        res = (traces - np.asarray(observed, o.dtype)).astype(o.dtype)
    else:
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


def rtm_shot_t1(o, lay, m, ab, cfg, src, wavelet, rec, residual=None):
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


# --- simulator3 (the elastic eTTI proxy) --------------------------------------
_E3_SIGS = {
    "orc_e3_vgplain": [V] * 10 + [I] * 5,
    "orc_e3_precompute": [V] * 3 + [I] * 8,
    "orc_e3_splain": [V] * 14 + [I] * 5,
    "orc_e3_vplain": [V] * 11 + [I] * 5,
    "orc_e3_mirror": [V, I, I, I, I],
    "orc_e3_update_gv": [V] * 5 + [I] * 7,
    "orc_e3_pressure": [V] * 7 + [L],
    "orc_e3_init_model": [V] * 3 + [I] * 4,
}


def _parr(vols):
    return (V * len(vols))(*[_p(v) for v in vols])


class ElasticOracle:
    """FP32 restatement of the simulator3 step kernels (``elastic_oracle.c``).

    Volumes are numpy arrays of ``Layout.shape``; ``M`` lists M1..M21 (or
    M1..M22), ``pre`` the twelve z-mixed volumes f10..f21."""

    def __init__(self):
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle`")
        self.lib = C.CDLL(LIB_PATH)
        self.fn = {}
        for name, sig in _E3_SIGS.items():
            f = getattr(self.lib, name)
            f.argtypes = sig
            f.restype = None
            self.fn[name] = f

    def vgplain(self, lay, f1, f2, f3, d, zprime):
        self.fn["orc_e3_vgplain"](_p(f1), _p(f2), _p(f3), *[_p(x) for x in d], _p(zprime), lay.nx, lay.ny, lay.nz,
                                  lay.ldimx, lay.ldimy)

    def precompute(self, lay, src, xz, yz, xs, ys, zs):
        self.fn["orc_e3_precompute"](_p(src), _p(xz), _p(yz), xs, ys, zs, lay.nx, lay.ny, lay.nz, lay.ldimx,
                                     lay.ldimy)

    def splain(self, lay, s, M, d, pre):
        """s = f4..f9, d = (d4..d9) as (f1_1, f1_2, f1_3, f2_2, f2_3, f3_3)."""
        m, p = _parr(M[:21]), _parr(pre)
        self.fn["orc_e3_splain"](*[_p(x) for x in s], C.addressof(m), *[_p(x) for x in d], C.addressof(p), lay.nx,
                                 lay.ny, lay.nz, lay.ldimx, lay.ldimy)

    def vplain(self, lay, v, s, M22, zprime):
        self.fn["orc_e3_vplain"](*[_p(x) for x in v], *[_p(x) for x in s], _p(M22), _p(zprime), lay.nx, lay.ny,
                                 lay.nz, lay.ldimx, lay.ldimy)

    def mirror(self, lay, fields, izbeg=RADIUS):
        f = _parr(fields)
        self.fn["orc_e3_mirror"](C.addressof(f), len(fields), lay.ldimx, lay.ldimy, izbeg)

    def update_gv(self, lay, g, s1, s3, a1, a3):
        self.fn["orc_e3_update_gv"](_p(g), _p(s1), _p(s3), _p(a1), _p(a3), lay.nx, lay.ny, lay.nz, lay.ldimx,
                                    lay.ldimy, lay.nx, lay.ny)

    def pressure(self, p, s):
        self.fn["orc_e3_pressure"](_p(p), *[_p(x) for x in s], p.size)

    def init_model(self, lay, M, d, zprime):
        m, dd = _parr(M), _parr(d)
        self.fn["orc_e3_init_model"](C.addressof(m), C.addressof(dd), _p(zprime), lay.nx, lay.ldimx, lay.ldimy,
                                     lay.ldimz)


def e3_execute(lay, niter, xcorr_step, press=500.0, adjoint=True, d123=(1.0, 1.0, 1.0)):
    """simulator3SetUp::execute (simulator3/simulator3SetUp.cu:2181-2657) on
    one subdomain, with the oracle: the stand-in model, the stress source at
    the grid centre, the forward steps (velocity update, free-surface
    mirrors, strains, stress update, pressure) with snapshots of the
    velocities every ``xcorr_step`` steps, then the adjoint steps in the
    reverse order with the velocity and density images.  Returns a dict of
    the final volumes and images."""
    e, o = ElasticOracle(), Oracle("f32")
    z = lay.zeros
    M = [z() for _ in range(22)]
    d = [z() for _ in range(6)]
    zprime = np.zeros(lay.ldimz, np.float32)
    e.init_model(lay, M, d, zprime)
    v = [z() for _ in range(3)]
    s = [z() for _ in range(6)]
    pre = [z() for _ in range(12)]
    p = z()
    c = tuple(n // 2 + RADIUS for n in (lay.nx, lay.ny, lay.nz))
    for k in range(6):  # init_src_kernel (:291-300)
        s[k][c[2], c[1], c[0]] = np.float32(press) * np.float32(k + 1)
    I = lay.interior
    snaps = {}
    nxt = 0
    for it in range(niter):
        e.vplain(lay, v, s, M[21], zprime)
        e.mirror(lay, s)
        e.mirror(lay, s)
        e.mirror(lay, v)
        e.mirror(lay, v)
        e.vgplain(lay, *v, d, zprime)
        e.splain(lay, s, M, d, pre)
        e.pressure(p, s)
        if adjoint and it == nxt:
            snaps[it] = (np.ascontiguousarray(v[0][I]), np.ascontiguousarray(v[2][I]))
            nxt += xcorr_step
    out = {"v": [x.copy() for x in v], "s": [x.copy() for x in s], "d": [x.copy() for x in d], "p": p.copy(),
           "pre": [x.copy() for x in pre]}
    if not adjoint:
        return out
    g1 = np.zeros((lay.nz, lay.ny, lay.nx), np.float32)
    g2 = np.zeros((lay.nz, lay.ny, lay.nx), np.float32)
    nxt -= xcorr_step
    for it in range(niter - 1, -1, -1):
        e.splain(lay, s, M, d, pre)
        e.vgplain(lay, *v, d, zprime)
        e.mirror(lay, s)
        e.mirror(lay, s)
        e.mirror(lay, v)
        e.mirror(lay, v)
        e.vplain(lay, v, s, M[21], zprime)
        if it == nxt:
            e.update_gv(lay, g1, snaps[it][0], snaps[it][1], v[0], v[2])
            # update_g_r_impl (:2091-2128): the TTI density gradient with
            # d4..d9, f4, f6, M18 (as 1/rho), M1..M4 and M5..M7 (as rx, ry, rz)
            o.rho_gradient(lay, g2, {"d1x": d[0], "d1y": d[1], "d1z": d[2], "d2x": d[3], "d2y": d[4], "d2z": d[5]},
                           s[0], s[2], {"irho": M[17], "m1": M[0], "m2": M[1], "m3": M[2], "m4": M[3], "rx": M[4],
                                        "ry": M[5], "rz": M[6]}, d123, lay.nx, lay.ny)
            nxt -= xcorr_step
    out.update({"v_adj": v, "s_adj": s, "g1": g1, "g2": g2})
    return out
