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
