"""Reduced-precision snapshot storage (FP16 / BF16 with per-field power-of-two
scaling; stencils and time update stay FP32) against the FP64 oracle.

The forward wavefield does not depend on the snapshot precision (the traces
are bit-identical); the image and the density gradient carry the snapshot
quantisation error, which is reported and bounded here."""
import json
import os

import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from oracle import Layout, Oracle
from tests.helpers import oracle_models, oracle_rtm, rel_l2, report_dir, sponge_profile



def run(prec, model, nx, ny, nz, nt, dt, w, src, rec):
    cfg = P.Config(nx=nx, ny=ny, nz=nz, dt=dt, nt=nt, xcorr_step=4, sponge_width=8, fused=True,
                   snap_precision=prec)
    with P.Simulator(cfg) as sim:
        sim.set_model(**model)
        sim.set_source(*src, w)
        sim.set_receivers(rec)
        tr = sim.forward()
        sim.adjoint(tr)
        gv, gr = sim.image()
    return cfg, tr, gv, gr


@pytest.mark.gpu
def test_reduced_precision_snapshots_against_fp64_oracle():
    nx, ny, nz, nt = 48, 40, 40, 80
    model = EM.smooth_tti(nx, ny, nz, dx=10.0, corr_m=80.0, seed=21)
    dt = EM.cfl_dt(model, 10.0)
    w = EM.ricker(nt, dt, 25.0) * 1e3
    src = (nx // 2, ny // 2, 5)
    rec = EM.receiver_plane(nx, ny, 3)
    res = {p: run(p, model, nx, ny, nz, nt, dt, w, src, rec) for p in ("fp32", "fp16", "bf16")}
    cfg = res["fp32"][0]
    lay = Layout(nx, ny, nz)
    m64 = oracle_models(lay, model, np.float64)
    ab = (sponge_profile(nx, lay.ldimx, 8, True), sponge_profile(ny, lay.ldimy, 8, True),
          sponge_profile(nz, lay.ldimz, 8, False))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm(Oracle("f64"), lay, m64, ab, cfg, lay.index(*src), w.astype(np.float64), rec_idx)
    report = {}
    for p, (_, tr, gv, gr) in res.items():
        report[p] = {"traces": rel_l2(tr, want["traces"]), "image_vp": rel_l2(gv, want["grad_vp"]),
                     "grad_rho": rel_l2(gr, want["grad_rho"])}
    print(json.dumps(report))
    if report_dir():
        with open(os.path.join(report_dir(), "precision_report.json"), "w") as f:
            json.dump(report, f, indent=1)
    np.testing.assert_array_equal(res["fp16"][1], res["fp32"][1])
    np.testing.assert_array_equal(res["bf16"][1], res["fp32"][1])
    assert report["fp32"]["traces"] < 1e-5
    assert report["fp32"]["image_vp"] < 1e-5 and report["fp32"]["grad_rho"] < 1e-5
    assert report["fp16"]["image_vp"] < 1e-3 and report["fp16"]["grad_rho"] < 1e-3
    assert report["bf16"]["image_vp"] < 2e-2 and report["bf16"]["grad_rho"] < 2e-2


def run_wave(prec, model, nx, ny, nz, nt, dt, w, src, rec, **kw):
    cfg = P.Config(nx=nx, ny=ny, nz=nz, dt=dt, nt=nt, xcorr_step=4, sponge_width=8, fused=True,
                   snap_precision=prec, wave_precision=prec, **kw)
    with P.Simulator(cfg) as sim:
        sim.set_model(**model)
        sim.set_source(*src, w)
        sim.set_receivers(rec)
        tr = sim.forward()
        sim.adjoint(tr)
        gv, gr = sim.image()
    return tr, gv, gr


@pytest.mark.gpu
def test_reduced_precision_wavefields_against_fp64_oracle():
    """p and q rounded to FP16 / BF16 (per-field power-of-two scale) at every
    step, snapshots in the same format, stencils and pdot/qdot in FP32: the
    error of traces, image and gradient against the FP64 oracle."""
    nx, ny, nz, nt = 48, 40, 40, 80
    model = EM.smooth_tti(nx, ny, nz, dx=10.0, corr_m=80.0, seed=21)
    dt = EM.cfl_dt(model, 10.0)
    w = EM.ricker(nt, dt, 25.0) * 1e3
    src = (nx // 2, ny // 2, 5)
    rec = EM.receiver_plane(nx, ny, 3)
    cfg = run("fp32", model, nx, ny, nz, nt, dt, w, src, rec)[0]
    lay = Layout(nx, ny, nz)
    m64 = oracle_models(lay, model, np.float64)
    ab = (sponge_profile(nx, lay.ldimx, 8, True), sponge_profile(ny, lay.ldimy, 8, True),
          sponge_profile(nz, lay.ldimz, 8, False))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm(Oracle("f64"), lay, m64, ab, cfg, lay.index(*src), w.astype(np.float64), rec_idx)
    report = {}
    for p in ("fp16", "bf16"):
        tr, gv, gr = run_wave(p, model, nx, ny, nz, nt, dt, w, src, rec)
        assert np.all(np.isfinite(tr)) and np.all(np.isfinite(gv))
        report[p] = {"traces": rel_l2(tr, want["traces"]), "image_vp": rel_l2(gv, want["grad_vp"]),
                     "grad_rho": rel_l2(gr, want["grad_rho"])}
    print(json.dumps(report))
    if report_dir():
        with open(os.path.join(report_dir(), "precision_report_wavefields.json"), "w") as f:
            json.dump(report, f, indent=1)
    for k in ("traces", "image_vp", "grad_rho"):  # measured: fp16 <= 2.2e-3, bf16 <= 8.8e-3
        assert report["fp16"][k] < 5e-3
        assert report["bf16"][k] < 3e-2


@pytest.mark.gpu
def test_reduced_precision_wavefields_recompute_exactly():
    """Checkpointed recomputation restores the per-field scales from the
    restored state, so the rounded forward field is recomputed bit for bit."""
    nx, ny, nz, nt = 40, 32, 32, 44
    model = EM.smooth_tti(nx, ny, nz, dx=10.0, corr_m=80.0, seed=22)
    dt = EM.cfl_dt(model, 10.0)
    w = EM.ricker(nt, dt, 25.0) * 1e3
    args = (model, nx, ny, nz, nt, dt, w, (nx // 2, ny // 2, 5), EM.receiver_plane(nx, ny, 3))
    plain = run_wave("fp16", *args)
    ck = run_wave("fp16", *args, checkpoint_every=8)
    for a, b in zip(ck, plain):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_config3_128_vti_500_steps_against_fp64_oracle():
    """The forward configuration (128^3 layered VTI, 20-cell sponge, 15 Hz
    Ricker at (64, 64, 5), 500 steps, receivers on plane z = 3) as a full RTM
    shot (imaging every 4 steps, the traces as residual) in plain FP32, with
    FP16 / BF16 snapshots, and with FP16 / BF16 wavefields and snapshots,
    against one FP64 oracle run of the same shot.  Every error is reported."""
    n, nt = 128, 500
    model = EM.layered_vti(n, n, n, nlayers=6, seed=1234)
    dt = EM.cfl_dt(model, 10.0, cfl=0.4)
    w = EM.ricker(nt, dt, 15.0)
    src = (64, 64, 5)
    rec = EM.receiver_plane(n, n, 3)

    def shot(snap, wave):
        cfg = P.Config(nx=n, ny=n, nz=n, dt=dt, nt=nt, xcorr_step=4, sponge_width=20, fused=True,
                       snap_precision=snap, wave_precision=wave)
        with P.Simulator(cfg) as sim:
            sim.set_model(**model)
            sim.set_source(*src, w)
            sim.set_receivers(rec)
            tr = sim.forward()
            sim.adjoint(tr)
            gv, gr = sim.image()
        return cfg, tr, gv, gr

    forms = {"fp32": ("fp32", "fp32"), "snap_fp16": ("fp16", "fp32"), "snap_bf16": ("bf16", "fp32"),
             "wave_fp16": ("fp16", "fp16"), "wave_bf16": ("bf16", "bf16")}
    res = {k: shot(*v) for k, v in forms.items()}
    cfg = res["fp32"][0]
    lay = Layout(n, n, n)
    ab = (sponge_profile(n, lay.ldimx, 20, True), sponge_profile(n, lay.ldimy, 20, True),
          sponge_profile(n, lay.ldimz, 20, False))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm(Oracle("f64"), lay, oracle_models(lay, model, np.float64), ab, cfg, lay.index(*src),
                      w.astype(np.float64), rec_idx)
    report = {"config": "128^3 layered VTI, 500 steps, imaging every 4, vs FP64 oracle"}
    for k, (_, tr, gv, gr) in res.items():
        assert np.all(np.isfinite(tr)) and np.all(np.isfinite(gv)) and np.all(np.isfinite(gr)), k
        report[k] = {"traces": rel_l2(tr, want["traces"]), "image_vp": rel_l2(gv, want["grad_vp"]),
                     "grad_rho": rel_l2(gr, want["grad_rho"])}
    print(json.dumps(report))
    if report_dir():
        with open(os.path.join(report_dir(), "precision_report_config3.json"), "w") as f:
            json.dump(report, f, indent=1)
    assert max(report["fp32"].values()) < 1e-5
    assert report["snap_fp16"]["image_vp"] < 1e-3 and report["snap_fp16"]["grad_rho"] < 1e-3
    for k in ("snap_bf16", "wave_fp16", "wave_bf16"):
        assert max(report[k].values()) < 5e-2, (k, report[k])
