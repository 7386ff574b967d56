"""Shot server (include/tti_capi.h section 4): continuous batching of RTM
shots of different grid sizes on one B200.

The server itself is native (csrc/tti_serve.cu: a loader thread admitting
shots by HBM footprint and a scheduler thread that advances every resident
shot per batched, optionally graph-captured, launch).  This module is the
ctypes binding: requests hold their numpy arrays until the result is taken.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import OK, TTIError, lib

V, I, F, D, L64 = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_int64


class ServerConfig(C.Structure):
    _fields_ = [("max_active", I), ("hbm_budget", L64), ("round_ms", F), ("use_graphs", I),
                ("autotune", I), ("snap_precision", I), ("scheme", I)]


class ShotRequestC(C.Structure):
    _fields_ = [("nx", I), ("ny", I), ("nz", I), ("dx", D), ("dy", D), ("dz", D), ("dt", F),
                ("nt", I), ("xcorr_step", I), ("sponge_width", I), ("free_surface", I),
                ("vp", V), ("eps", V), ("delta", V), ("vs", V), ("theta", V), ("phi", V), ("rho", V),
                ("src_ix", I), ("src_iy", I), ("src_iz", I), ("wavelet", V), ("nrec", I),
                ("rec_ixyz", V), ("observed", V), ("image_vp", V), ("image_rho", V), ("traces", V)]


class ShotResultC(C.Structure):
    _fields_ = [("status", I), ("t_submit", D), ("t_admit", D), ("t_done", D), ("footprint", L64),
                ("checkpoint_every", I), ("units", L64), ("launches", L64)]


class ServerStatsC(C.Structure):
    _fields_ = [("rounds", L64), ("graph_updates", L64), ("graph_instantiations", L64),
                ("max_resident", I), ("busy_ms", D), ("gap_ms", D), ("build_ms", D), ("setup_ms", D),
                ("max_batched", I), ("setup_alloc_ms", D), ("setup_model_ms", D), ("setup_tune_ms", D)]


_declared = False


def _lib():
    global _declared
    l = lib()
    if not _declared:
        l.tti_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(V)]
        l.tti_server_submit.argtypes = [V, C.POINTER(ShotRequestC), C.POINTER(L64)]
        l.tti_server_wait.argtypes = [V, L64, D, C.POINTER(ShotResultC)]
        l.tti_server_stats_get.argtypes = [V, C.POINTER(ServerStatsC)]
        l.tti_server_now.argtypes = [V]
        l.tti_server_now.restype = D
        l.tti_server_destroy.argtypes = [V]
        l.tti_rtm_shot.argtypes = [C.POINTER(ShotRequestC), V]
        l.tti_rtm_shot.restype = I
        for n in ("tti_server_create", "tti_server_submit", "tti_server_wait", "tti_server_stats_get",
                  "tti_server_destroy"):
            getattr(l, n).restype = I
        _declared = True
    return l


PRECISIONS = {"fp32": 0, "fp16": 1, "bf16": 2}


def _f32(a, n):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
    if a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


@dataclass
class Shot:
    """One RTM shot: grid, model (interior arrays, x fastest), source,
    receivers and optional observed traces; outputs are filled in place."""

    nx: int
    ny: int
    nz: int
    dt: float
    nt: int
    vp: np.ndarray
    wavelet: np.ndarray
    source: tuple
    receivers: np.ndarray  # (nrec, 3) int: ix, iy, iz
    eps: Optional[np.ndarray] = None
    delta: Optional[np.ndarray] = None
    vs: Optional[np.ndarray] = None
    theta: Optional[np.ndarray] = None
    phi: Optional[np.ndarray] = None
    rho: Optional[np.ndarray] = None
    observed: Optional[np.ndarray] = None
    dx: float = 10.0
    dy: float = 10.0
    dz: float = 10.0
    xcorr_step: int = 4
    sponge_width: int = 0
    free_surface: bool = True
    want_traces: bool = True
    image_vp: np.ndarray = field(init=False)
    image_rho: np.ndarray = field(init=False)
    traces: Optional[np.ndarray] = field(init=False, default=None)

    def _c(self) -> ShotRequestC:
        n = self.nx * self.ny * self.nz
        keep = {}
        for k in ("vp", "eps", "delta", "vs", "theta", "phi", "rho"):
            keep[k] = _f32(getattr(self, k), n)
        keep["wavelet"] = _f32(np.asarray(self.wavelet)[: self.nt], self.nt)
        rec = np.ascontiguousarray(np.asarray(self.receivers, np.int32).reshape(-1, 3))
        keep["rec"] = rec
        nrec = rec.shape[0]
        keep["observed"] = _f32(self.observed, self.nt * nrec) if self.observed is not None else None
        self.image_vp = np.zeros((self.nz, self.ny, self.nx), np.float32)
        self.image_rho = np.zeros((self.nz, self.ny, self.nx), np.float32)
        self.traces = np.zeros((self.nt, nrec), np.float32) if (self.want_traces and nrec) else None
        self._keep = keep
        ptr = lambda a: a.ctypes.data if a is not None else None  # noqa: E731
        return ShotRequestC(self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, self.dt, self.nt,
                            self.xcorr_step, self.sponge_width, int(self.free_surface),
                            ptr(keep["vp"]), ptr(keep["eps"]), ptr(keep["delta"]), ptr(keep["vs"]),
                            ptr(keep["theta"]), ptr(keep["phi"]), ptr(keep["rho"]),
                            int(self.source[0]), int(self.source[1]), int(self.source[2]),
                            ptr(keep["wavelet"]), nrec, ptr(rec), ptr(keep["observed"]),
                            ptr(self.image_vp), ptr(self.image_rho), ptr(self.traces))


@dataclass
class Result:
    status: int
    t_submit: float
    t_admit: float
    t_done: float
    footprint: int
    checkpoint_every: int
    units: int
    launches: int

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


def rtm_shot(shot: Shot, opts=None) -> Shot:
    """One whole shot, synchronously (tti_rtm_shot): fills ``shot.image_vp``,
    ``shot.image_rho`` and ``shot.traces``.  ``opts`` is a
    ``miniappsforhpe_b200.Config`` whose fused, snap_precision,
    checkpoint_every, use_graphs, scheme and wave_precision fields are used
    (None: defaults)."""
    req = shot._c()
    cfg = opts.c_struct() if opts is not None else None
    rc = _lib().tti_rtm_shot(C.byref(req), C.byref(cfg) if cfg is not None else None)
    if rc != OK:
        raise TTIError(rc, "tti_rtm_shot")
    return shot


class Server:
    """Native shot server; ``submit`` returns a ticket, ``wait`` the result.

    ``max_active`` bounds the resident shots: two measured best on a mixed
    stream of 96^3 .. 320x320x200 shots, since one such shot nearly fills a
    B200 and each further resident shot adds the mapping of its stores."""

    def __init__(self, max_active: int = 2, hbm_budget: int = 0, round_ms: float = 50.0,
                 use_graphs: bool = True, autotune: bool = True, snap_precision: str = "fp16", scheme: int = 0):
        cfg = ServerConfig(max_active, hbm_budget, round_ms, int(use_graphs), int(autotune),
                           PRECISIONS[snap_precision], int(scheme))
        self._h = V()
        rc = _lib().tti_server_create(C.byref(cfg), C.byref(self._h))
        if rc != OK:
            raise TTIError(rc, "tti_server_create")
        self._shots = {}

    def now(self) -> float:
        return _lib().tti_server_now(self._h)

    def submit(self, shot: Shot) -> int:
        req = shot._c()
        t = L64()
        rc = _lib().tti_server_submit(self._h, C.byref(req), C.byref(t))
        if rc != OK:
            raise TTIError(rc, "tti_server_submit")
        self._shots[t.value] = shot
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0) -> Result:
        r = ShotResultC()
        rc = _lib().tti_server_wait(self._h, ticket, timeout, C.byref(r))
        if rc != OK:
            raise TTIError(rc, "tti_server_wait")
        self._shots.pop(ticket, None)
        return Result(r.status, r.t_submit, r.t_admit, r.t_done, r.footprint, r.checkpoint_every, r.units,
                      r.launches)

    def stats(self) -> dict:
        s = ServerStatsC()
        rc = _lib().tti_server_stats_get(self._h, C.byref(s))
        if rc != OK:
            raise TTIError(rc, "tti_server_stats_get")
        return {"rounds": s.rounds, "graph_updates": s.graph_updates,
                "graph_instantiations": s.graph_instantiations, "max_resident": s.max_resident,
                "busy_ms": s.busy_ms, "gap_ms": s.gap_ms, "build_ms": s.build_ms, "setup_ms": s.setup_ms,
                "max_batched": s.max_batched, "setup_alloc_ms": s.setup_alloc_ms,
                "setup_model_ms": s.setup_model_ms, "setup_tune_ms": s.setup_tune_ms}

    def close(self):
        if self._h:
            _lib().tti_server_destroy(self._h)
            self._h = V()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
