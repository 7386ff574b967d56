"""Simulator-level parity on the GPU.

* The reference kernel sequence (fused=False) against the oracle's
  reference-order RTM: forward traces, Vp image and density gradient.
* The fused step kernels against the reference kernel sequence, TTI and VTI,
  with and without the free surface and the sponge.
* Adjoint consistency of the fused forward/adjoint pair: a dot-product test
  through the public API with FP64 reductions.
"""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from oracle import Layout, Oracle
from tests.helpers import oracle_models, oracle_rtm, rel_l2, sponge_profile


def make_sim(nx, ny, nz, tti, fused, fs=True, sponge=6, nt=48, xcorr=4, seed=5):
    if tti:
        model = EM.smooth_tti(nx, ny, nz, dx=10.0, corr_m=60.0, seed=seed)
    else:
        model = EM.layered_vti(nx, ny, nz, nlayers=4, seed=seed)
    dt = EM.cfl_dt(model, 10.0, cfl=0.4)
    cfg = P.Config(nx=nx, ny=ny, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt=dt, nt=nt, xcorr_step=xcorr,
                   sponge_width=sponge, free_surface=fs, fused=fused)
    sim = P.Simulator(cfg)
    sim.set_model(**model)
    w = EM.ricker(nt, dt, 25.0) * 1e3
    src = (nx // 2, ny // 2, 5)
    sim.set_source(*src, w)
    rec = EM.receiver_plane(nx, ny, 3)
    sim.set_receivers(rec)
    return sim, cfg, model, w, src, rec


@pytest.mark.gpu
@pytest.mark.parametrize("tti", [False, True], ids=["vti", "tti"])
def test_reference_sequence_matches_oracle(tti):
    nx, ny, nz = 36, 30, 28
    sim, cfg, model, w, src, rec = make_sim(nx, ny, nz, tti, fused=False)
    traces = sim.forward()
    rng = np.random.default_rng(2)
    res = (traces * rng.uniform(0.5, 1.5, traces.shape)).astype(np.float32)
    sim.adjoint(res)
    gvp, grho = sim.image()
    lay = Layout(nx, ny, nz)
    m = oracle_models(lay, model)
    ab = (sponge_profile(nx, lay.ldimx, cfg.sponge_width, True),
          sponge_profile(ny, lay.ldimy, cfg.sponge_width, True),
          sponge_profile(nz, lay.ldimz, cfg.sponge_width, not cfg.free_surface))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm(Oracle("f32"), lay, m, ab, cfg, lay.index(*src), w, rec_idx, residual=res)
    assert rel_l2(traces, want["traces"]) < 1e-5
    assert rel_l2(gvp, want["grad_vp"]) < 1e-5
    assert rel_l2(grho, want["grad_rho"]) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("tti", [False, True], ids=["vti", "tti"])
@pytest.mark.parametrize("fs", [True, False], ids=["fs", "nofs"])
def test_fused_matches_reference_sequence(tti, fs):
    # 70 x 45 x 90: partial CTA tiles in x and y, several z chunks
    out = {}
    for fused in (False, True):
        sim, cfg, *_ = make_sim(70, 45, 90, tti, fused=fused, fs=fs, nt=40)
        tr = sim.forward()
        f3 = sim.volume("field3")
        sim.adjoint(tr)
        gvp, grho = sim.image()
        out[fused] = (tr, f3, gvp, grho)
        sim.close()
    for a, b in zip(out[True], out[False]):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, b) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("tti", [False, True], ids=["vti", "tti"])
def test_dot_product_fused(tti):
    """<F s, r> = <s, F^T r> for the receiver map F of the fused forward and
    the fused adjoint, no free surface, no sponge (the cases where the
    reference's adjoint sequence is the exact transpose of its forward)."""
    nx, ny, nz, nt = 48, 40, 44, 60
    sim, cfg, model, w, src, rec = make_sim(nx, ny, nz, tti, fused=True, fs=False, sponge=0, nt=nt)
    rng = np.random.default_rng(9)
    s = rng.standard_normal(nt).astype(np.float32)
    sim.set_source(*src, s)
    d = sim.forward().astype(np.float64)
    r = rng.standard_normal(d.shape).astype(np.float32)
    sim.adjoint(r)
    g = sim.source_gradient().astype(np.float64)
    lhs = float(np.sum(d * r.astype(np.float64)))
    rhs = float(np.sum(s.astype(np.float64) * g))
    assert abs(lhs - rhs) <= 1e-4 * max(abs(lhs), abs(rhs))


@pytest.mark.gpu
def test_launch_counts_and_snapshot_capacity():
    sim, cfg, *_ = make_sim(40, 36, 30, True, fused=True, nt=20)
    sim.forward()
    # one fused step per time step (receivers on one plane are sampled inside
    # it), plus the step-0 p update
    assert sim.launch_count() == cfg.nt + 2
    with pytest.raises(P.TTIError) as e:
        P.Simulator(P.Config(nx=40, ny=36, nz=30, nt=20)).adjoint(np.zeros((20, 0), np.float32))
    assert e.value.status == P.ESTATE


def receiver_geometry(kind, nx, ny, nz):
    if kind == "two_planes":  # folded into the step kernels (two plane tables)
        return np.concatenate([EM.receiver_plane(nx, ny, 3), EM.receiver_plane(nx, ny, nz - 6)[::7]])
    # a vertical well through every plane: more planes than the step kernels
    # take, sampled and injected by separate kernels
    return np.array([[nx // 3, ny // 2, iz] for iz in range(nz)], np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["two_planes", "well"])
def test_receiver_geometries_fused_against_reference_sequence(kind):
    nx, ny, nz, nt = 44, 38, 40, 32
    out = {}
    for fused in (False, True):
        sim, cfg, model, w, src, _ = make_sim(nx, ny, nz, True, fused=fused, nt=nt)
        sim.set_receivers(receiver_geometry(kind, nx, ny, nz))
        tr = sim.forward()
        launches = sim.launch_count()
        sim.adjoint(tr)
        gvp, grho = sim.image()
        out[fused] = (tr, gvp, grho, sim.source_gradient())
        sim.close()
        if fused:  # separate receiver kernels only for the well
            assert launches == (2 * nt + 2 if kind == "well" else nt + 2)
    for a, b in zip(out[True], out[False]):
        assert np.all(np.isfinite(a)) and np.abs(b).max() > 0
        assert rel_l2(a, b) < 1e-5
