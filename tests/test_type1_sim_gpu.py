"""Simulator runs with the centred constant-density operator (scheme 1).

* The type1 kernel sequence (fused=False: loop2, loop4 and the type1
  forward launcher; the type1 adjoint launcher, loop2, loop4; the type1 Vp
  image) against the oracle's type1 restatement composed in the same order:
  traces and Vp image within 1e-5 relative L2.
* The fused type1 step kernels against that sequence, TTI and VTI, with and
  without the free surface, on a grid with partial tiles.
* FP16 snapshots and checkpointed recomputation on the fused type1 path.
* Adjoint consistency of the fused type1 pair (dot-product test).
"""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from oracle import Layout, Oracle
from tests.helpers import oracle_models, oracle_rtm_t1, rel_l2, sponge_profile


def make_sim(nx, ny, nz, tti, fused, fs=True, sponge=6, nt=40, xcorr=4, seed=7, **kw):
    if tti:
        model = EM.smooth_tti(nx, ny, nz, dx=10.0, corr_m=60.0, seed=seed)
    else:
        model = EM.layered_vti(nx, ny, nz, nlayers=4, seed=seed)
    dt = EM.cfl_dt(model, 10.0, cfl=0.4)
    cfg = P.Config(nx=nx, ny=ny, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt=dt, nt=nt, xcorr_step=xcorr,
                   sponge_width=sponge, free_surface=fs, fused=fused, scheme=1, **kw)
    sim = P.Simulator(cfg)
    sim.set_model(**model)  # density is unused by the constant-density operator
    w = EM.ricker(nt, dt, 25.0) * 1e3
    src = (nx // 2, ny // 2, 5)
    sim.set_source(*src, w)
    rec = EM.receiver_plane(nx, ny, 3)
    sim.set_receivers(rec)
    return sim, cfg, w, src, rec, model


def rtm(sim, residual=None):
    tr = sim.forward()
    sim.adjoint(tr if residual is None else residual)
    gvp, grho = sim.image()
    return tr, gvp, grho


@pytest.mark.gpu
@pytest.mark.parametrize("tti", [False, True], ids=["vti", "tti"])
def test_type1_sequence_matches_oracle(tti):
    nx, ny, nz = 36, 30, 28
    sim, cfg, w, src, rec, model = make_sim(nx, ny, nz, tti, fused=False, nt=32)
    tr = sim.forward()
    rng = np.random.default_rng(4)
    res = (tr * rng.uniform(0.5, 1.5, tr.shape)).astype(np.float32)
    sim.adjoint(res)
    gvp, grho = sim.image()
    lay = Layout(nx, ny, nz)
    m = oracle_models(lay, model)
    ab = (sponge_profile(nx, lay.ldimx, cfg.sponge_width, True),
          sponge_profile(ny, lay.ldimy, cfg.sponge_width, True),
          sponge_profile(nz, lay.ldimz, cfg.sponge_width, not cfg.free_surface))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm_t1(Oracle("f32"), lay, m, ab, cfg, lay.index(*src), w, rec_idx, residual=res)
    assert np.abs(want["traces"]).max() > 0 and np.abs(want["grad_vp"]).max() > 0
    assert rel_l2(tr, want["traces"]) < 1e-5
    assert rel_l2(gvp, want["grad_vp"]) < 1e-5
    assert not np.any(grho)  # the constant-density operator has no density image


@pytest.mark.gpu
@pytest.mark.parametrize("tti", [False, True], ids=["vti", "tti"])
@pytest.mark.parametrize("fs", [True, False], ids=["fs", "nofs"])
def test_type1_fused_matches_sequence(tti, fs):
    # partial CTA tiles in x and y, several z chunks; the forward kernel
    # computes x-neighbouring pairs: 70 puts the source on the second point
    # of a pair, 69 leaves the last pair of each row half outside
    nx = 70 if fs else 69
    out = {}
    for fused in (False, True):
        sim, *_ = make_sim(nx, 45, 90, tti, fused=fused, fs=fs, nt=36)
        tr = sim.forward()
        f3 = sim.volume("field3")
        sim.adjoint(tr)
        gvp, _ = sim.image()
        out[fused] = (tr, f3, gvp)
        sim.close()
    for a, b in zip(out[True], out[False]):
        assert np.all(np.isfinite(a)) and np.abs(b).max() > 0
        assert rel_l2(a, b) < 1e-5


@pytest.mark.gpu
def test_type1_fp16_snapshots_and_checkpoints():
    runs = {}
    for name, kw in (("f32", {}), ("f16", {"snap_precision": "fp16"}),
                     ("ckpt", {"snap_precision": "fp16", "checkpoint_every": 8})):
        sim, *_ = make_sim(64, 40, 48, True, fused=True, nt=40, **kw)
        runs[name] = rtm(sim)
        sim.close()
    # FP16 snapshots perturb only the image; traces are bit-identical
    assert np.array_equal(runs["f16"][0], runs["f32"][0])
    assert rel_l2(runs["f16"][1], runs["f32"][1]) < 2e-3
    # checkpointed recomputation reproduces the stored-snapshot run exactly
    for a, b in zip(runs["ckpt"], runs["f16"]):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("tti", [False, True], ids=["vti", "tti"])
def test_type1_dot_product(tti):
    """<F s, r> = <s, F^T r> for the receiver map of the fused type1 forward
    and adjoint (no free surface, no sponge)."""
    nt = 60
    sim, cfg, w, src, rec, _ = make_sim(48, 40, 44, tti, fused=True, fs=False, sponge=0, nt=nt)
    rng = np.random.default_rng(10)
    s = rng.standard_normal(nt).astype(np.float32)
    sim.set_source(*src, s)
    d = sim.forward().astype(np.float64)
    r = rng.standard_normal(d.shape).astype(np.float32)
    sim.adjoint(r)
    g = sim.source_gradient().astype(np.float64)
    lhs = float(np.sum(d * r.astype(np.float64)))
    rhs = float(np.sum(s.astype(np.float64) * g))
    assert abs(lhs - rhs) <= 1e-4 * max(abs(lhs), abs(rhs))
