"""The full-RTM configuration at its full size, over a step subset: TTI,
256^3, dx = 10 m, 24-cell sponge, free surface, smooth Gaussian-random model
(300 m correlation, vp 1500-5000 m/s, eps 0-0.25, delta 0-0.1, theta 0-45
deg, phi 0-180 deg), 12 Hz Ricker at the centre of plane z = 5, receivers on
every cell of plane z = 3, observed traces from the same model plus a 5 % vp
blob, imaging every 4 steps.  The shot is cut to its first 200 time steps
(200 forward steps with 50 snapshots, 200 adjoint steps with 50 imaging
steps), so that the FP32 oracle finishes in a few minutes on the host.  In
200 steps the wave travels about 40 cells, so the blob sits under the
source (depth 10, radius 8 cells) where the observed traces differ from the
synthetic ones by more than rounding: a blob out of reach would leave a
residual of rounding noise, which no two FP32 implementations share.

The fused sm_100a path (autotuned work split) against the oracle's
reference-order RTM built from the same host parameters: traces, Vp image
and density gradient within 1e-5 relative L2."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from oracle import Layout, Oracle
from tests.helpers import oracle_models, oracle_rtm, rel_l2, sponge_profile


@pytest.mark.gpu
def test_config2_256_rtm_subset_matches_oracle():
    n, nt, xcorr, width = 256, 200, 4, 24
    model = EM.smooth_tti(n, n, n, dx=10.0, corr_m=300.0, seed=1234)
    true = EM.add_velocity_blob(model, (n // 2, n // 2, 10), radius_cells=8, fraction=0.05)
    dt = EM.cfl_dt(true, 10.0, cfl=0.4)
    w = EM.ricker(nt, dt, 12.0)
    src = (n // 2, n // 2, 5)
    rec = EM.receiver_plane(n, n, 3)
    cfg = P.Config(nx=n, ny=n, nz=n, dt=dt, nt=nt, xcorr_step=xcorr, sponge_width=width, free_surface=True,
                   fused=True)
    with P.Simulator(cfg) as sim:
        sim.set_source(*src, w)
        sim.set_receivers(rec)
        sim.set_model(**true)
        observed = sim.forward()
        sim.set_model(**model)
        sim.autotune(reps=1)
        traces = sim.forward()
        sim.adjoint_observed(observed)
        gvp, grho = sim.image()
    lay = Layout(n, n, n)
    ab = (sponge_profile(n, lay.ldimx, width, True), sponge_profile(n, lay.ldimy, width, True),
          sponge_profile(n, lay.ldimz, width, False))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm(Oracle("f32"), lay, oracle_models(lay, model), ab, cfg, lay.index(*src), w, rec_idx,
                      observed=observed)
    assert rel_l2(traces, observed) > 1e-2  # the residual is signal, not rounding
    for got, ref in ((traces, want["traces"]), (gvp, want["grad_vp"]), (grho, want["grad_rho"])):
        assert np.all(np.isfinite(got)) and np.abs(ref).max() > 0
    e = {"traces": rel_l2(traces, want["traces"]), "grad_vp": rel_l2(gvp, want["grad_vp"]),
         "grad_rho": rel_l2(grho, want["grad_rho"])}
    print(e)
    assert max(e.values()) < 1e-5, e
