"""Checkpointed recomputation and captured CUDA graphs.

With ``checkpoint_every = K`` the forward pass keeps FP32 checkpoints of the
state every K steps and one K-step segment of snapshots; the adjoint pass
recomputes each earlier segment from its checkpoint.  The recomputed steps run
the same kernels on the same state, so traces, image and density gradient are
bit-identical to the run that keeps every snapshot (FP32 and FP16 stores).
Graph capture replays the same launches, so it is bit-identical too."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM

NX, NY, NZ, NT = 48, 40, 40, 80


def shot(**over):
    model = EM.smooth_tti(NX, NY, NZ, dx=10.0, corr_m=80.0, seed=31)
    dt = EM.cfl_dt(model, 10.0)
    w = EM.ricker(NT, dt, 25.0) * 1e3
    kw = dict(nx=NX, ny=NY, nz=NZ, dt=dt, nt=NT, xcorr_step=4, sponge_width=6, fused=True)
    kw.update(over)
    cfg = P.Config(**kw)
    with P.Simulator(cfg) as sim:
        sim.set_model(**model)
        sim.set_source(NX // 2, NY // 2, 5, w)
        sim.set_receivers(EM.receiver_plane(NX, NY, 3))
        out = []
        for _ in range(2):  # a second shot on the same simulator (graph reuse)
            tr = sim.forward()
            sim.adjoint(tr * 0.5)
            gv, gr = sim.image()
            out.append((tr, gv, gr))
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)
    return out[0]


@pytest.fixture(scope="module")
def plain():
    return {p: shot(snap_precision=p) for p in ("fp32", "fp16")}


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp16"])
@pytest.mark.parametrize("ckpt", [16, 24], ids=["even", "ragged"])
def test_checkpointed_recomputation_is_bit_identical(plain, prec, ckpt):
    got = shot(snap_precision=prec, checkpoint_every=ckpt)
    for a, b in zip(got, plain[prec]):
        np.testing.assert_array_equal(a, b)
    assert np.abs(got[1]).max() > 0 and np.abs(got[2]).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("ckpt", [0, 16])
def test_graph_capture_is_bit_identical(plain, ckpt):
    got = shot(snap_precision="fp16", checkpoint_every=ckpt, use_graphs=True)
    for a, b in zip(got, plain["fp16"]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_footprint_matches_device_allocation():
    import torch
    cfg = P.Config(nx=96, ny=96, nz=96, nt=200, snap_precision="fp16", checkpoint_every=40)
    want = cfg.footprint_bytes()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    sim = P.Simulator(cfg)
    free1, _ = torch.cuda.mem_get_info()
    sim.close()
    used = free0 - free1
    assert want <= used <= want + 64 * 2**20
