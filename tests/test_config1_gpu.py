"""The reference's forward configuration at full size: VTI forward only,
128^3, dx = 10 m, 20-cell sponge, six seeded flat layers (vp 1500-4500 m/s,
eps 0-0.3, delta 0-0.15, delta <= eps), 15 Hz Ricker at (64, 64, 5), dt from
CFL 0.4, 500 steps, receivers on every cell of plane z = 3; pressure traces
of the fused sm_100a path against the oracle run of the same shot."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from oracle import Layout, Oracle
from tests.helpers import oracle_models, oracle_rtm, rel_l2, sponge_profile


@pytest.mark.gpu
def test_config1_vti_forward_traces_match_oracle():
    n, nt = 128, 500
    model = EM.layered_vti(n, n, n, nlayers=6, seed=1234)
    dt = EM.cfl_dt(model, 10.0, cfl=0.4)
    w = EM.ricker(nt, dt, 15.0)
    src = (64, 64, 5)
    rec = EM.receiver_plane(n, n, 3)
    cfg = P.Config(nx=n, ny=n, nz=n, dt=dt, nt=nt, sponge_width=20, fused=True, save_snapshots=False)
    with P.Simulator(cfg) as sim:
        sim.set_model(**model)
        sim.set_source(*src, w)
        sim.set_receivers(rec)
        tr = sim.forward()
    lay = Layout(n, n, n)
    m = oracle_models(lay, model)
    ab = (sponge_profile(n, lay.ldimx, 20, True), sponge_profile(n, lay.ldimy, 20, True),
          sponge_profile(n, lay.ldimz, 20, False))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    want = oracle_rtm(Oracle("f32"), lay, m, ab, cfg, lay.index(*src), w, rec_idx, adjoint=False)
    assert np.all(np.isfinite(tr))
    assert np.abs(tr).max() > 0
    assert rel_l2(tr, want["traces"]) < 1e-5
