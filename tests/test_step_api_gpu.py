"""Step-level calls (tti_sim_forward_begin / _step, tti_sim_adjoint_begin /
_step, tti_sim_image_step, tti_sim_adjoint_finish) and the run-level call
(tti_rtm_shot).  They launch the same kernels in the same order as the loop
calls (tti_sim_forward, tti_sim_adjoint), so results are bit-identical; calls
out of order are refused before anything is launched."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from miniappsforhpe_b200 import serve as S

NX, NY, NZ, NT = 40, 36, 30, 24


def setup(fused=True, scheme=0, **kw):
    model = EM.smooth_tti(NX, NY, NZ, dx=10.0, corr_m=60.0, seed=21)
    dt = EM.cfl_dt(model, 10.0)
    cfg = P.Config(nx=NX, ny=NY, nz=NZ, dt=dt, nt=NT, sponge_width=5, fused=fused, scheme=scheme, **kw)
    sim = P.Simulator(cfg)
    sim.set_model(**model)
    w = EM.ricker(NT, dt, 25.0) * 1e3
    sim.set_source(NX // 2, NY // 2, 5, w)
    rec = EM.receiver_plane(NX, NY, 3)
    sim.set_receivers(rec)
    return sim, cfg, model, w, rec


@pytest.mark.gpu
@pytest.mark.parametrize("fused,scheme", [(True, 0), (False, 0), (True, 1)], ids=["fused", "kernels", "type1"])
def test_step_calls_match_loop_calls(fused, scheme):
    sim, cfg, *_ = setup(fused, scheme)
    tr = sim.forward()
    res = (tr * 0.7).astype(np.float32)
    sim.adjoint(res)
    want = sim.image()

    sim.forward_begin()
    for n in range(cfg.nt):
        sim.forward_step(n)
    tr2 = sim.traces()
    sim.adjoint_begin(res)
    for n in range(cfg.nt - 1, -1, -1):
        sim.adjoint_step(n)
        if n % cfg.xcorr_step == 0:
            sim.image_step(n)
    sim.adjoint_finish()
    got = sim.image()
    np.testing.assert_array_equal(tr2, tr)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
    sim.close()


@pytest.mark.gpu
def test_step_calls_out_of_order_are_refused():
    sim, cfg, *_ = setup()
    with pytest.raises(P.TTIError) as e:
        sim.forward_step(0)  # no forward_begin
    assert e.value.status == P.ESTATE
    sim.forward_begin()
    with pytest.raises(P.TTIError) as e:
        sim.forward_step(1)
    assert e.value.status == P.ESTATE
    with pytest.raises(P.TTIError) as e:
        sim.adjoint_begin()  # forward not finished
    assert e.value.status == P.ESTATE
    for n in range(cfg.nt):
        sim.forward_step(n)
    sim.adjoint_begin()
    sim.adjoint_step(cfg.nt - 1)
    with pytest.raises(P.TTIError) as e:
        sim.image_step(cfg.nt - 1)  # not a snapshot step (nt - 1 = 23)
    assert e.value.status == P.EINVAL
    with pytest.raises(P.TTIError) as e:
        sim.adjoint_finish()  # steps left
    assert e.value.status == P.ESTATE
    sim.close()
    ck, *_ = setup(snap_precision="fp16", checkpoint_every=8)
    with pytest.raises(P.TTIError) as e:
        ck.forward_begin()
    assert e.value.status == P.EINVAL
    ck.close()


@pytest.mark.gpu
@pytest.mark.parametrize("observed", [True, False], ids=["observed", "self"])
def test_run_level_shot_matches_simulator(observed):
    sim, cfg, model, w, rec = setup()
    tr = sim.forward()
    obs = (tr * 0.5).astype(np.float32) if observed else None
    if observed:
        sim.adjoint_observed(obs)
    else:
        sim.adjoint(tr)
    want_vp, want_rho = sim.image()
    sim.close()
    shot = S.Shot(nx=NX, ny=NY, nz=NZ, dt=cfg.dt, nt=NT, vp=model["vp"], wavelet=w, source=(NX // 2, NY // 2, 5),
                  receivers=rec, eps=model.get("eps"), delta=model.get("delta"), vs=model.get("vs"),
                  theta=model.get("theta"), phi=model.get("phi"), rho=model.get("rho"), observed=obs,
                  xcorr_step=cfg.xcorr_step, sponge_width=cfg.sponge_width)
    S.rtm_shot(shot, P.Config(nx=NX, ny=NY, nz=NZ))
    np.testing.assert_array_equal(shot.traces, tr)
    np.testing.assert_array_equal(shot.image_vp, want_vp)
    np.testing.assert_array_equal(shot.image_rho, want_rho)
