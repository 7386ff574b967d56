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
from tests.helpers import oracle_rtm, rel_l2, sim_models, sponge_profile

OUT = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gpurun_out")


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
        m = sim_models(sim)
    return cfg, tr, gv, gr, m


@pytest.mark.gpu
def test_reduced_precision_snapshots_against_fp64_oracle():
    nx, ny, nz, nt = 48, 40, 40, 80
    model = EM.smooth_tti(nx, ny, nz, dx=10.0, corr_m=80.0, seed=21)
    dt = EM.cfl_dt(model, 10.0)
    w = EM.ricker(nt, dt, 25.0) * 1e3
    src = (nx // 2, ny // 2, 5)
    rec = EM.receiver_plane(nx, ny, 3)
    res = {p: run(p, model, nx, ny, nz, nt, dt, w, src, rec) for p in ("fp32", "fp16", "bf16")}
    cfg, _, _, _, m32 = res["fp32"]
    lay = Layout(nx, ny, nz)
    m64 = {k: v.astype(np.float64) for k, v in m32.items()}
    ab = (sponge_profile(nx, lay.ldimx, 8, True), sponge_profile(ny, lay.ldimy, 8, True),
          sponge_profile(nz, lay.ldimz, 8, False))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm(Oracle("f64"), lay, m64, ab, cfg, lay.index(*src), w.astype(np.float64), rec_idx)
    report = {}
    for p, (_, tr, gv, gr, _) in res.items():
        report[p] = {"traces": rel_l2(tr, want["traces"]), "image_vp": rel_l2(gv, want["grad_vp"]),
                     "grad_rho": rel_l2(gr, want["grad_rho"])}
    print(json.dumps(report))
    if os.path.isdir(OUT):
        with open(os.path.join(OUT, "precision_report.json"), "w") as f:
            json.dump(report, f, indent=1)
    np.testing.assert_array_equal(res["fp16"][1], res["fp32"][1])
    np.testing.assert_array_equal(res["bf16"][1], res["fp32"][1])
    assert report["fp32"]["traces"] < 1e-5
    assert report["fp32"]["image_vp"] < 1e-5 and report["fp32"]["grad_rho"] < 1e-5
    assert report["fp16"]["image_vp"] < 1e-3 and report["fp16"]["grad_rho"] < 1e-3
    assert report["bf16"]["image_vp"] < 2e-2 and report["bf16"]["grad_rho"] < 2e-2
