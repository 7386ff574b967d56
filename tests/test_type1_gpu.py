"""Type1 launchers on the GPU against the oracle and against the reference's
own type1 kernels (kernels/kernel_type1_gpu_{fwd,adj,grad}.cu, built from
the reference sources by oracle/Makefile), on the same seeded inputs:
forward in its three modes (accumulate, sponge, calc_snap), adjoint with and
without sponge, imaging.  Tolerance: relative L2 2e-6 (FP32 rounding of a
differently associated sum)."""
import ctypes as C
import os

import numpy as np
import pytest

import miniappsforhpe_b200 as P
from oracle import REF_LIB_PATH, Layout, Oracle
from tests.helpers import random_field, random_model, rel_l2, sponge_ab

H = (10.0, 12.5, 8.0)
DT = 1e-3
TOL = 2e-6
MKEYS = ("m1", "m2", "m3", "m4", "rx", "ry", "rz")


def inputs(nx=44, ny=37, nz=29, seed=7):
    lay = Layout(nx, ny, nz)
    rng = np.random.default_rng(seed)
    m = random_model(lay, rng, tti=True)
    ab = [sponge_ab(n, rng) for n in (lay.ldimx, lay.ldimy, lay.ldimz)]
    f = [random_field(lay, rng) for _ in range(4)]
    return lay, m, ab, f


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_product(lay, m, ab, f, what, mode=0, sponge=False):
    import torch

    t = {k: dev(v) for k, v in m.items()}
    a = [dev(x) for x in ab]
    f1, f2 = dev(f[0]), dev(f[1])
    r = lay.ranges
    if what == "fwd":
        if mode == 2:
            o3 = torch.zeros((lay.nz, lay.ny, lay.nx), device="cuda")
            o4 = torch.zeros_like(o3)
            ld = (lay.nx, lay.ny, lay.nz)
        else:
            o3, o4 = dev(f[2]), dev(f[3])
            ld = (lay.ldimx, lay.ldimy, lay.ldimz)
        P.launch_type1_fwd(o3, o4, f1, f2, *[t[k] for k in MKEYS], *a, *r, lay.ldimx, lay.ldimy, lay.ldimz, *ld,
                           DT, *H, calc_snap=(mode == 2), use_sponge=(mode == 1))
    else:
        o3, o4 = dev(f[2]), dev(f[3])
        P.launch_type1_adj(o3, o4, f1, f2, *[t[k] for k in MKEYS], *a, *r, lay.ldimx, lay.ldimy, lay.ldimz, DT,
                           *H, use_sponge=sponge)
    torch.cuda.synchronize()
    return o3.cpu().numpy(), o4.cpu().numpy()


def run_oracle(lay, m, ab, f, what, mode=0, sponge=False):
    o = Oracle("f32")
    if what == "fwd":
        if mode == 2:
            o3 = np.zeros((lay.nz, lay.ny, lay.nx), np.float32)
            o4 = np.zeros_like(o3)
            o.t1_fwd(lay, o3, o4, f[0], f[1], m, ab, np.float32(DT), H, 2, (lay.nx, lay.ny))
        else:
            o3, o4 = f[2].copy(), f[3].copy()
            o.t1_fwd(lay, o3, o4, f[0], f[1], m, ab, np.float32(DT), H, mode)
    else:
        o3, o4 = f[2].copy(), f[3].copy()
        o.t1_adj(lay, o3, o4, f[0], f[1], m, ab, np.float32(DT), H, sponge)
    return o3, o4


def run_reference(lay, m, ab, f, what, mode=0, sponge=False):
    import torch

    lib = C.CDLL(REF_LIB_PATH)
    for n in ("ref_t1_fwd", "ref_t1_adj"):
        getattr(lib, n).restype = C.c_int
    t = {k: dev(v) for k, v in m.items()}
    a = [dev(x) for x in ab]
    f1, f2 = dev(f[0]), dev(f[1])
    p = lambda x: C.c_void_p(x.data_ptr())  # noqa: E731
    r = lay.ranges
    if what == "fwd":
        if mode == 2:
            o3 = torch.zeros((lay.nz, lay.ny, lay.nx), device="cuda")
            o4 = torch.zeros_like(o3)
            ld = (lay.nx, lay.ny, lay.nz)
        else:
            o3, o4 = dev(f[2]), dev(f[3])
            ld = (lay.ldimx, lay.ldimy, lay.ldimz)
        rc = lib.ref_t1_fwd(p(o3), p(o4), p(f1), p(f2), *[p(t[k]) for k in MKEYS], *[p(x) for x in a], *r,
                            lay.ldimx, lay.ldimy, lay.ldimz, *ld, C.c_float(DT), *[C.c_double(h) for h in H],
                            int(mode == 2), int(mode == 1))
    else:
        o3, o4 = dev(f[2]), dev(f[3])
        rc = lib.ref_t1_adj(p(o3), p(o4), p(f1), p(f2), *[p(t[k]) for k in MKEYS], *[p(x) for x in a], *r,
                            lay.ldimx, lay.ldimy, lay.ldimz, C.c_float(DT), *[C.c_double(h) for h in H],
                            int(sponge))
    assert rc == 0
    torch.cuda.synchronize()
    return o3.cpu().numpy(), o4.cpu().numpy()


CASES = [("fwd", 0, False), ("fwd", 1, False), ("fwd", 2, False), ("adj", 0, False), ("adj", 0, True)]
IDS = ["fwd-accumulate", "fwd-sponge", "fwd-calc_snap", "adj", "adj-sponge"]


def _delta(got, base, what, mode):
    # compare the increments (outputs minus the inputs they update), which is
    # what the operator contributes
    if what == "fwd" and mode == 2:
        return got
    return [g - b for g, b in zip(got, base)]


@pytest.mark.gpu
@pytest.mark.parametrize("what,mode,sponge", CASES, ids=IDS)
def test_type1_product_matches_oracle(what, mode, sponge):
    lay, m, ab, f = inputs()
    got = run_product(lay, m, ab, f, what, mode, sponge)
    want = run_oracle(lay, m, ab, f, what, mode, sponge)
    for g, w in zip(_delta(got, f[2:], what, mode), _delta(want, f[2:], what, mode)):
        assert np.abs(w).max() > 0
        assert rel_l2(g, w) < TOL


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_LIB_PATH), reason="reference kernels not built")
@pytest.mark.parametrize("what,mode,sponge", CASES, ids=IDS)
def test_type1_product_matches_reference_kernels(what, mode, sponge):
    lay, m, ab, f = inputs(seed=11)
    got = run_product(lay, m, ab, f, what, mode, sponge)
    want = run_reference(lay, m, ab, f, what, mode, sponge)
    for g, w in zip(_delta(got, f[2:], what, mode), _delta(want, f[2:], what, mode)):
        assert np.abs(w).max() > 0
        assert rel_l2(g, w) < TOL


@pytest.mark.gpu
def test_type1_imaging_matches_oracle():
    import torch

    lay, m, ab, f = inputs(seed=13)
    rng = np.random.default_rng(13)
    n = lay.nx * lay.ny * lay.nz
    sx, sz, g0 = (rng.standard_normal(n).astype(np.float32) for _ in range(3))
    want = g0.copy()
    Oracle("f32").t1_grad(lay, sx, sz, want, f[0], f[1])
    g = dev(g0)
    P.launch_type1_update_grad(dev(sx), dev(sz), g, dev(f[0]), dev(f[1]), *lay.ranges, lay.nx, lay.ny, lay.ldimx,
                               lay.ldimy)
    torch.cuda.synchronize()
    assert rel_l2(g.cpu().numpy(), want) < 1e-6
