"""The reference's own kernels (built from its sources for sm_100a) against
this library's fused step kernels on the same B200, at 256^3.

One RTM time step of the reference = forward step (loop2, loop4, fwd_drv,
loop4_derivatives, fwd_main_loop_2), adjoint step (adj_drv,
loop4_derivatives, adj_main_loop_3, loop2, loop4) and a quarter of an
imaging step (update_Vp_gradient, fwd_drv on the snapshot, derivative
mirror, density gradient), simulator2SetUp.cu:517-814, kernel time only (the
reference's snapshot copies to host memory are not counted).  The fused path
is timed on the simulator's stream over a short shot.  The per-step times go
to reference_speed.json in the report directory (TTI_REPORT_DIR) when one
is set."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import miniappsforhpe_b200 as P
from oracle import DKEYS, REF_LIB_PATH, Layout
from tests.helpers import report_dir

N = 256
DX = 10.0
DT = 5e-4


def _ref_lib():
    lib = C.CDLL(REF_LIB_PATH)
    for name in ("ref_fwd_drv", "ref_fwd_update", "ref_adj_drv", "ref_adj_update", "ref_rho_gradient",
                 "ref_loop4_derivatives", "ref_update_vp_gradient", "ref_loop2", "ref_loop4", "ref_sync"):
        getattr(lib, name).restype = C.c_int
    return lib


def _p(t):
    return C.c_void_p(t.data_ptr())


def reference_step_ms(torch, reps=4):
    lib = _ref_lib()
    lay = Layout(N, N, N)
    r = lay.ranges
    dev = torch.device("cuda")
    vol = lambda v=0.0: torch.full(lay.shape, v, dtype=torch.float32, device=dev)  # noqa: E731
    g = torch.Generator(device=dev).manual_seed(3)
    f = {k: torch.randn(lay.shape, device=dev, generator=g) * 1e-3 for k in ("f1", "f2", "f3", "f4")}
    m = {"irho": vol(1.0), "m1": vol(9e6), "m2": vol(8e6), "m3": vol(7e6), "m4": vol(1e6),
         "rx": vol(0.3), "ry": vol(0.2), "rz": vol(0.93)}
    d = {k: vol() for k in DKEYS}
    r3, r4 = vol(), vol()
    ab = [torch.ones(2 * n, device=dev) for n in (lay.ldimx, lay.ldimy, lay.ldimz)]
    snap3 = torch.randn(N * N * N, device=dev, generator=g)
    snap4 = torch.randn(N * N * N, device=dev, generator=g)
    gvp = torch.zeros(N * N * N, device=dev)
    grho = torch.zeros(N * N * N, device=dev)
    fs = C.c_float

    def ok(rc):
        assert rc == 0

    def fwd():
        ok(lib.ref_loop2(_p(f["f1"]), _p(f["f2"]), _p(f["f3"]), _p(f["f4"]), lay.ldimx, lay.ldimy, *r,
                         _p(ab[0]), _p(ab[1]), _p(ab[2]), fs(DT)))
        ok(lib.ref_loop4(_p(f["f1"]), _p(f["f2"]), lay.ldimx, lay.ldimy, 4))
        ok(lib.ref_fwd_drv(_p(f["f1"]), _p(f["f2"]), _p(m["irho"]), *[_p(d[k]) for k in DKEYS], *r,
                           fs(1 / DX), fs(1 / DX), fs(1 / DX), lay.ldimx, lay.ldimy))
        ok(lib.ref_loop4_derivatives(*[_p(d[k]) for k in DKEYS], lay.ldimx, lay.ldimy, 4))
        ok(lib.ref_fwd_update(_p(f["f3"]), _p(f["f4"]), _p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]), _p(d["d2y"]),
                              _p(d["d1z"]), _p(d["d2z"]), _p(f["f1"]), _p(f["f2"]), *[_p(m[k]) for k in
                              ("irho", "m1", "m2", "m3", "m4", "rx", "ry", "rz")], *r, lay.ldimx, lay.ldimy,
                              fs(DT), C.c_double(DX), C.c_double(DX), C.c_double(DX)))

    def adj():
        ok(lib.ref_adj_drv(_p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]), _p(d["d2y"]), _p(d["d1z"]), _p(d["d2z"]),
                           _p(r3), _p(r4), _p(f["f1"]), _p(f["f2"]), *[_p(m[k]) for k in
                           ("irho", "m1", "m2", "m3", "m4", "rx", "ry", "rz")], *r, C.c_double(DX),
                           C.c_double(DX), C.c_double(DX), lay.ldimx, lay.ldimy, fs(DT)))
        ok(lib.ref_loop4_derivatives(*[_p(d[k]) for k in DKEYS], lay.ldimx, lay.ldimy, 4))
        ok(lib.ref_adj_update(_p(f["f3"]), _p(f["f4"]), _p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]), _p(d["d2y"]),
                              _p(d["d1z"]), _p(d["d2z"]), _p(r3), _p(r4), _p(ab[0]), _p(ab[1]), _p(ab[2]), *r,
                              lay.ldimx, lay.ldimy, fs(DT), C.c_double(DX), C.c_double(DX), C.c_double(DX), 0))
        ok(lib.ref_loop2(_p(f["f1"]), _p(f["f2"]), _p(f["f3"]), _p(f["f4"]), lay.ldimx, lay.ldimy, *r,
                         _p(ab[0]), _p(ab[1]), _p(ab[2]), fs(DT)))
        ok(lib.ref_loop4(_p(f["f1"]), _p(f["f2"]), lay.ldimx, lay.ldimy, 4))

    def img():
        ok(lib.ref_update_vp_gradient(_p(snap3), _p(snap4), _p(gvp), _p(f["f3"]), _p(f["f4"]), *r, N, N,
                                      lay.ldimx, lay.ldimy))
        ok(lib.ref_fwd_drv(_p(f["f1"]), _p(f["f2"]), _p(m["irho"]), *[_p(d[k]) for k in DKEYS], *r,
                           fs(1 / DX), fs(1 / DX), fs(1 / DX), lay.ldimx, lay.ldimy))
        ok(lib.ref_loop4_derivatives(*[_p(d[k]) for k in DKEYS], lay.ldimx, lay.ldimy, 4))
        ok(lib.ref_rho_gradient(_p(grho), _p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]), _p(d["d2y"]), _p(d["d1z"]),
                                _p(d["d2z"]), _p(f["f1"]), _p(f["f2"]), *[_p(m[k]) for k in
                                ("irho", "m1", "m2", "m3", "m4", "rx", "ry", "rz")], *r, lay.ldimx, lay.ldimy,
                                N, N, C.c_double(DX), C.c_double(DX), C.c_double(DX), 0))

    out = {}
    for name, fn in (("forward", fwd), ("adjoint", adj), ("imaging", img)):
        fn()  # warm-up (first-call attribute set-up)
        ok(lib.ref_sync())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()  # the reference launches on the legacy default stream
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    return out


def reference_type1_step_ms(torch, reps=4):
    """The reference's type1 launchers (kernels/kernel_type1_gpu_*.cu) in the
    simulator's step order: forward = loop2, loop4, fwd_main_loop_2_1 (sponge
    form); adjoint = adj_main_loop_2 (sponge form), loop2, loop4; imaging =
    update_grad_loop."""
    lib = _ref_lib()
    for name in ("ref_t1_fwd", "ref_t1_adj", "ref_t1_grad"):
        getattr(lib, name).restype = C.c_int
    lay = Layout(N, N, N)
    r = lay.ranges
    dev = torch.device("cuda")
    vol = lambda v=0.0: torch.full(lay.shape, v, dtype=torch.float32, device=dev)  # noqa: E731
    g = torch.Generator(device=dev).manual_seed(4)
    f = {k: torch.randn(lay.shape, device=dev, generator=g) * 1e-3 for k in ("f1", "f2", "f3", "f4")}
    m = [vol(v) for v in (9e6, 8e6, 7e6, 1e6, 0.3, 0.2, 0.93)]
    ab = [torch.ones(2 * n, device=dev) for n in (lay.ldimx, lay.ldimy, lay.ldimz)]
    snap3 = torch.randn(N * N * N, device=dev, generator=g)
    snap4 = torch.randn(N * N * N, device=dev, generator=g)
    gvp = torch.zeros(N * N * N, device=dev)
    fs, fd = C.c_float, C.c_double

    def ok(rc):
        assert rc == 0

    def loops():
        ok(lib.ref_loop2(_p(f["f1"]), _p(f["f2"]), _p(f["f3"]), _p(f["f4"]), lay.ldimx, lay.ldimy, *r,
                         _p(ab[0]), _p(ab[1]), _p(ab[2]), fs(DT)))
        ok(lib.ref_loop4(_p(f["f1"]), _p(f["f2"]), lay.ldimx, lay.ldimy, 4))

    def fwd():
        loops()
        ok(lib.ref_t1_fwd(_p(f["f3"]), _p(f["f4"]), _p(f["f1"]), _p(f["f2"]), *[_p(v) for v in m],
                          _p(ab[0]), _p(ab[1]), _p(ab[2]), *r, lay.ldimx, lay.ldimy, lay.ldimz, lay.ldimx,
                          lay.ldimy, lay.ldimz, fs(DT), fd(DX), fd(DX), fd(DX), 0, 1))

    def adj():
        ok(lib.ref_t1_adj(_p(f["f3"]), _p(f["f4"]), _p(f["f1"]), _p(f["f2"]), *[_p(v) for v in m],
                          _p(ab[0]), _p(ab[1]), _p(ab[2]), *r, lay.ldimx, lay.ldimy, lay.ldimz, fs(DT), fd(DX),
                          fd(DX), fd(DX), 1))
        loops()

    def img():
        ok(lib.ref_t1_grad(_p(snap3), _p(snap4), _p(gvp), _p(f["f3"]), _p(f["f4"]), *r, N, N, lay.ldimx,
                           lay.ldimy))

    out = {}
    for name, fn in (("forward", fwd), ("adjoint", adj), ("imaging", img)):
        fn()
        ok(lib.ref_sync())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    return out


def fused_step_ms(torch, nt=32, scheme=0):
    from miniappsforhpe_b200 import earth_models as EM

    model = EM.smooth_tti(N, N, N, dx=DX, corr_m=300.0, seed=5)
    dt = EM.cfl_dt(model, DX)
    cfg = P.Config(nx=N, ny=N, nz=N, dt=dt, nt=nt, xcorr_step=4, sponge_width=24, scheme=scheme)
    with P.Simulator(cfg) as sim:
        sim.set_model(**model)
        sim.set_source(N // 2, N // 2, 5, EM.ricker(nt, dt, 12.0))
        sim.set_receivers(EM.receiver_plane(N, N, 3))
        tr = sim.forward()
        sim.adjoint(tr)
        sim.set_profiling(True)
        tr = sim.forward()
        sim.adjoint(tr)
        t = sim.kernel_times()
    return {k: v[0] / max(v[1], 1) for k, v in t.items()}


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_LIB_PATH), reason="reference kernels not built")
def test_fused_step_is_faster_than_the_reference_kernels():
    import torch

    ref = reference_step_ms(torch)
    ours = fused_step_ms(torch)
    ref_step = ref["forward"] + ref["adjoint"] + ref["imaging"] / 4
    our_step = ours["forward"] + ours["adjoint"] + ours["imaging"] / 4
    rep = {"grid": [N, N, N], "reference_kernels_ms": ref, "fused_ms": ours,
           "reference_ms_per_rtm_step": ref_step, "fused_ms_per_rtm_step": our_step,
           "speedup": ref_step / our_step,
           "reference_gpts_per_s": N ** 3 / ref_step / 1e6, "fused_gpts_per_s": N ** 3 / our_step / 1e6}
    print(json.dumps(rep))
    if report_dir():
        with open(os.path.join(report_dir(), "reference_speed.json"), "w") as fh:
            json.dump(rep, fh, indent=1)
    assert our_step < ref_step


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_LIB_PATH), reason="reference kernels not built")
def test_fused_type1_step_is_faster_than_the_reference_type1_kernels():
    import torch

    ref = reference_type1_step_ms(torch)
    ours = fused_step_ms(torch, scheme=1)
    ref_step = ref["forward"] + ref["adjoint"] + ref["imaging"] / 4
    our_step = ours["forward"] + ours["adjoint"] + ours["imaging"] / 4
    rep = {"grid": [N, N, N], "operator": "centred constant-density (type1)", "reference_kernels_ms": ref,
           "fused_ms": ours, "reference_ms_per_rtm_step": ref_step, "fused_ms_per_rtm_step": our_step,
           "speedup": ref_step / our_step,
           "reference_gpts_per_s": N ** 3 / ref_step / 1e6, "fused_gpts_per_s": N ** 3 / our_step / 1e6}
    print(json.dumps(rep))
    if report_dir():
        with open(os.path.join(report_dir(), "reference_speed_type1.json"), "w") as fh:
            json.dump(rep, fh, indent=1)
    assert our_step < ref_step
