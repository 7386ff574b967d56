"""Shot server: continuous batching of shots of different grid sizes.

Each shot's traces, Vp image and density gradient from the server (shots
resident together, advanced in batched rounds, graph-captured or not, with
autotuned z-chunks, admitted under an HBM budget that forces checkpointing)
are compared with the same shot run alone through the simulator API
(forward, adjoint_observed, image) at relative L2 <= 1e-6; the kernels and
their order per shot are the same, and no z-chunk choice changes an
accumulation order."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from miniappsforhpe_b200.serve import Server, Shot
from tests.helpers import rel_l2

SHOTS = [  # nx, ny, nz, nt, seed: enough steps that each shot outlasts the set-up of the next
    (48, 40, 40, 320, 1),
    (64, 48, 40, 400, 2),
    (40, 40, 48, 260, 3),
    (56, 40, 32, 360, 4),
]


def make_shot(nx, ny, nz, nt, seed):
    m = EM.smooth_tti(nx, ny, nz, dx=10.0, corr_m=60.0, seed=seed)
    dt = EM.cfl_dt(m, 10.0)
    w = EM.ricker(nt, dt, 25.0) * 1e3
    rec = EM.receiver_plane(nx, ny, 3)
    rng = np.random.default_rng(seed)
    obs = rng.standard_normal((nt, rec.shape[0])).astype(np.float32) * 1e-3
    return dict(nx=nx, ny=ny, nz=nz, dt=dt, nt=nt, vp=m["vp"], eps=m["eps"], delta=m["delta"],
                theta=m["theta"], phi=m["phi"], wavelet=w, source=(nx // 2 + seed, ny // 2, 4 + seed),
                receivers=rec, observed=obs, sponge_width=6)


def alone(s, prec, scheme=0):
    cfg = P.Config(nx=s["nx"], ny=s["ny"], nz=s["nz"], dt=s["dt"], nt=s["nt"], xcorr_step=4,
                   sponge_width=s["sponge_width"], fused=True, snap_precision=prec, scheme=scheme)
    with P.Simulator(cfg) as sim:
        sim.set_model(vp=s["vp"], eps=s["eps"], delta=s["delta"], theta=s["theta"], phi=s["phi"])
        sim.set_source(*s["source"], s["wavelet"])
        sim.set_receivers(s["receivers"])
        tr = sim.forward()
        sim.adjoint_observed(s["observed"])
        gv, gr = sim.image()
    return tr, gv, gr


@pytest.fixture(scope="module")
def shots():
    return [make_shot(*a) for a in SHOTS]


@pytest.fixture(scope="module")
def reference(shots):
    return [alone(s, "fp16") for s in shots]


@pytest.fixture(scope="module")
def reference_type1(shots):
    return [alone(s, "fp16", scheme=1) for s in shots]


def check(res, shots, reference):
    for sh, r, (tr, gv, gr) in zip(shots, res, reference):
        assert r.status == P.OK
        assert rel_l2(sh.traces, tr) <= 1e-6
        assert rel_l2(sh.image_vp, gv) <= 1e-6
        assert rel_l2(sh.image_rho, gr) <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False], ids=["graphs", "streams"])
def test_results_are_the_same_alone_and_in_the_mix(shots, reference, graphs):
    with Server(max_active=4, round_ms=0.3, use_graphs=graphs, autotune=True, snap_precision="fp16") as srv:
        objs = [Shot(**s) for s in shots]
        tickets = [srv.submit(o) for o in objs]
        res = [srv.wait(t, 300.0) for t in tickets]
        st = srv.stats()
    check(res, objs, reference)
    assert st["max_resident"] >= 2  # shots were resident together
    assert st["max_batched"] >= 2   # and advanced in the same rounds
    assert st["rounds"] > 4         # and advanced over several batched rounds
    assert all(r.units == 2 * s["nt"] for r, s in zip(res, shots))


@pytest.mark.gpu
def test_budget_forces_checkpointing_and_serial_admission(shots, reference):
    def server_footprint(s, K=0):  # simulator + receiver buffers + model-upload temporaries
        cfg = P.Config(nx=s["nx"], ny=s["ny"], nz=s["nz"], nt=s["nt"], snap_precision="fp16",
                       checkpoint_every=K)
        lx, ly, lz = 32 * ((s["nx"] + 7) // 32 + 1), s["ny"] + 8, s["nz"] + 8
        nrec = len(s["receivers"])
        return cfg.footprint_bytes() + nrec * (8 + 8 * s["nt"]) + 8 * lx * ly * lz * 4

    # a budget the largest shot fits only with checkpoints
    big = max(shots, key=server_footprint)
    full = server_footprint(big)
    least = min(server_footprint(big, K) for K in range(4, big["nt"], 4))
    assert least < full
    budget = (full + least) // 2
    with Server(max_active=4, hbm_budget=budget, round_ms=0.5, use_graphs=True, autotune=False,
                snap_precision="fp16") as srv:
        objs = [Shot(**s) for s in shots]
        tickets = [srv.submit(o) for o in objs]
        res = [srv.wait(t, 300.0) for t in tickets]
    check(res, objs, reference)
    assert any(r.checkpoint_every > 0 for r in res)
    for r, s in zip(res, shots):
        K = r.checkpoint_every
        if K:  # forward + adjoint + recomputation of every segment but the last
            assert r.units == 2 * s["nt"] + ((s["nt"] - 1) // K) * K


@pytest.mark.gpu
def test_centred_operator_served_in_the_mix(shots, reference_type1):
    """The same mix with the centred constant-density operator: every result
    equals the shot run alone (its density image stays zero)."""
    with Server(max_active=4, round_ms=0.3, use_graphs=True, autotune=False, snap_precision="fp16",
                scheme=1) as srv:
        objs = [Shot(**s) for s in shots]
        tickets = [srv.submit(o) for o in objs]
        res = [srv.wait(t, 300.0) for t in tickets]
        st = srv.stats()
    check(res, objs, reference_type1)
    assert st["max_batched"] >= 2
    assert all(not np.any(o.image_rho) for o in objs)
