"""Image error of the large single-shot configuration's method against an
FP64 oracle, on a 4x downsampled copy of the shot.

The full shot (512x512x400, dx = 12.5 m, 3000 steps, 10 Hz Ricker, layered
model, FP16 snapshots with FP32 checkpoints every 200 steps) is far beyond
what an FP64 host run can do.  The downsampled shot keeps its physics in
scaled units: 128x128x100 cells of 50 m, the same CFL number (so dt x4),
750 steps (the same duration), a 2.5 Hz Ricker (the same points per
wavelength and periods per shot), checkpoints every 48 steps (the multiple
of the imaging period nearest to 200/4), imaging every 4 steps, FP16
snapshots.  Its traces, Vp image and density gradient are
compared with one FP64 oracle run of the same downsampled shot, next to the
plain FP32 form (FP32 snapshots, no checkpoints)."""
import json
import os

import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from oracle import Layout, Oracle
from tests.helpers import oracle_models, oracle_rtm, rel_l2, report_dir, sponge_profile


@pytest.mark.gpu
def test_config5_method_downsampled_against_fp64_oracle():
    f = 4
    nx, ny, nz, nt = 512 // f, 512 // f, 400 // f, 3000 // f
    dx, f0, width = 12.5 * f, 10.0 / f, 24
    model = EM.layered_vti(nx, ny, nz, nlayers=6, seed=1234)
    dt = EM.cfl_dt(model, dx, cfl=0.4)
    w = EM.ricker(nt, dt, f0)
    src = (nx // 2, ny // 2, 5)
    rec = EM.receiver_plane(nx, ny, 3)

    def shot(snap, ckpt):
        cfg = P.Config(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dx, dt=dt, nt=nt, xcorr_step=4,
                       sponge_width=width, fused=True, snap_precision=snap, checkpoint_every=ckpt)
        with P.Simulator(cfg) as sim:
            sim.set_model(**model)
            sim.set_source(*src, w)
            sim.set_receivers(rec)
            tr = sim.forward()
            sim.adjoint(tr)
            gv, gr = sim.image()
        return cfg, tr, gv, gr

    res = {"c5_method_fp16_ckpt48": shot("fp16", 48), "plain_fp32": shot("fp32", 0)}
    cfg = res["plain_fp32"][0]
    lay = Layout(nx, ny, nz)
    ab = (sponge_profile(nx, lay.ldimx, width, True), sponge_profile(ny, lay.ldimy, width, True),
          sponge_profile(nz, lay.ldimz, width, False))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm(Oracle("f64"), lay, oracle_models(lay, model, np.float64), ab, cfg, lay.index(*src),
                      w.astype(np.float64), rec_idx)
    report = {"config": f"{nx}x{ny}x{nz}, dx {dx} m, {nt} steps, {f0} Hz (4x downsampled), vs FP64 oracle"}
    for k, (_, tr, gv, gr) in res.items():
        assert np.all(np.isfinite(gv)) and np.abs(gv).max() > 0, k
        report[k] = {"traces": rel_l2(tr, want["traces"]), "image_vp": rel_l2(gv, want["grad_vp"]),
                     "grad_rho": rel_l2(gr, want["grad_rho"])}
    print(json.dumps(report))
    if report_dir():
        with open(os.path.join(report_dir(), "precision_report_config5.json"), "w") as fh:
            json.dump(report, fh, indent=1)
    assert max(report["plain_fp32"].values()) < 1e-5
    c5 = report["c5_method_fp16_ckpt48"]
    assert c5["traces"] < 1e-5  # the forward field does not depend on the snapshot store
    assert c5["image_vp"] < 1e-3 and c5["grad_rho"] < 1e-3
