"""Shot-parallel host logic on CPU ranks (gloo, world size 2): shot
assignment covers every shot once, and the stacked image equals the sum of
the per-shot images computed by the oracle on a tiny grid."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from miniappsforhpe_b200.shot_parallel import run_shot_stream, shots_for_rank


def test_assignment_covers_every_shot_once():
    for ws in (1, 2, 3, 8):
        got = sorted(s for r in range(ws) for s in shots_for_rank(11, ws, r))
        assert got == list(range(11))
    with pytest.raises(ValueError):
        shots_for_rank(4, 2, 2)


def _shot_image(shot):
    """A tiny oracle forward run per shot: the final pdot volume is the 'image'."""
    from oracle import Layout, Oracle, new_state
    from tests.helpers import random_model

    o = Oracle("f32")
    lay = Layout(12, 10, 10)
    m = random_model(lay, np.random.default_rng(100), tti=True)
    ab = [np.ones(2 * k, np.float32) for k in (lay.ldimx, lay.ldimy, lay.ldimz)]
    g = o.grid(lay, np.float32(1e-3), (10.0, 10.0, 10.0), free_surface=True)
    st = new_state(lay)
    src = lay.index(3 + shot, 5, 4)
    for n in range(6):
        o.fwd_step(g, st, m, ab, src, float(np.sin(n + shot)))
    return torch.from_numpy(st["f3"][lay.interior].copy())


def _worker(rank, ws, port, nshots, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        img = run_shot_stream(nshots, _shot_image, lambda: torch.zeros((10, 10, 12)), dist=dist)
        q.put((rank, img.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_gloo_two_ranks_stack_matches_serial_sum():
    ws, nshots = 2, 5
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, nshots, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = sum(_shot_image(s).numpy() for s in range(nshots))
    for r in range(ws):
        np.testing.assert_allclose(res[r], want, rtol=1e-5, atol=1e-6 * np.abs(want).max())


# --- serving across ranks: one server per rank, stacks per survey ---------

from miniappsforhpe_b200.shot_parallel import assign_by_cost, serve_stream  # noqa: E402


def test_cost_assignment_balances_and_covers_every_shot_once():
    costs = [5.0, 1.0, 4.0, 3.0, 3.0, 2.0, 8.0]
    parts = assign_by_cost(costs, 3)
    assert sorted(s for p in parts for s in p) == list(range(len(costs)))
    loads = sorted(sum(costs[s] for s in p) for p in parts)
    assert loads == [8.0, 9.0, 9.0]
    assert assign_by_cost(costs, 3) == parts  # deterministic
    assert assign_by_cost([1.0, 1.0], 4)[3] == []


class HostShot:
    """The fields serve_stream reads from a shot, plus its images."""

    def __init__(self, i, nx, ny, nz, nt, survey):
        self.i, self.nx, self.ny, self.nz, self.nt, self.survey = i, nx, ny, nz, nt, survey


class HostServer:
    """Host-side stand-in for one GPU's shot server: submit runs the shot as
    an RTM of the oracle on its tiny grid (the device step), wait returns."""

    def __init__(self):
        self.done = {}

    def submit(self, shot):
        from types import SimpleNamespace

        from oracle import Layout, Oracle, models_from_parameters, rtm_shot

        lay = Layout(shot.nx, shot.ny, shot.nz)
        rng = np.random.default_rng(7 + 13 * shot.survey)  # one model per survey
        vp = rng.uniform(1800.0, 2600.0, (shot.nz, shot.ny, shot.nx)).astype(np.float32)
        m = models_from_parameters(lay, vp)
        ab = [np.ones(2 * k, np.float32) for k in (lay.ldimx, lay.ldimy, lay.ldimz)]
        cfg = SimpleNamespace(nt=shot.nt, xcorr_step=2, dt=1e-3, dx=10.0, dy=10.0, dz=10.0, free_surface=True,
                              sponge_width=0)
        w = np.sin(np.arange(shot.nt) * (0.7 + 0.1 * shot.i)).astype(np.float32)
        rec = np.array([lay.index(ix, 1, 2) for ix in range(shot.nx)], np.int64)
        out = rtm_shot(Oracle("f32"), lay, m, ab, cfg, lay.index(1 + shot.i % (shot.nx - 2), 2, 3), w, rec)
        shot.image_vp, shot.image_rho = out["grad_vp"], out["grad_rho"]
        t = len(self.done)
        self.done[t] = shot.i
        return t

    def wait(self, ticket, timeout=-1.0):
        return self.done[ticket]


def host_stream():
    # two surveys on different grids, shots of different lengths
    spec = [(10, 8, 8, 6, 0), (12, 9, 8, 8, 1), (10, 8, 8, 10, 0), (12, 9, 8, 4, 1), (10, 8, 8, 8, 0)]
    return [HostShot(i, *s) for i, s in enumerate(spec)]


def _serve_worker(rank, ws, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        shots = host_stream()
        stacks, results = serve_stream(shots, HostServer(), lambda i: shots[i].survey, dist=dist)
        q.put((rank, {k: (v.numpy(), r.numpy()) for k, (v, r) in stacks.items()}, sorted(results)))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_serve_stream_stacks_each_survey():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(ws):
        rank, stacks, served = q.get(timeout=240)
        got[rank] = (stacks, served)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shots = host_stream()
    parts = assign_by_cost([s.nx * s.ny * s.nz * s.nt for s in shots], ws)
    assert [got[r][1] for r in range(ws)] == parts  # each rank served its share
    server = HostServer()
    want = {}
    for s in shots:
        server.submit(s)
        vp, rho = want.get(s.survey, (0.0, 0.0))
        want[s.survey] = (vp + s.image_vp, rho + s.image_rho)
    for r in range(ws):
        stacks = got[r][0]
        assert sorted(stacks) == [0, 1]
        for k, (vp, rho) in want.items():
            assert np.abs(vp).max() > 0
            np.testing.assert_allclose(stacks[k][0], vp, rtol=1e-5, atol=1e-6 * np.abs(vp).max())
            np.testing.assert_allclose(stacks[k][1], rho, rtol=1e-5, atol=1e-6 * np.abs(rho).max())
