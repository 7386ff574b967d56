"""Edge shapes for the fused kernels: grids smaller than one tile in every
direction, fewer z planes than the z pipelines' lag, a single interior
plane in z, odd sizes; the fused path must match the reference kernel
sequence there too (both operators), and a shot with nt not a multiple of
the imaging cadence or of the checkpoint segment must give the same image
with and without checkpoints."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from tests.helpers import rel_l2


def run(nx, ny, nz, fused, scheme=0, nt=18, fs=True, **kw):
    model = EM.smooth_tti(nx, ny, nz, dx=10.0, corr_m=40.0, seed=nx * 7 + ny * 3 + nz)
    dt = EM.cfl_dt(model, 10.0, cfl=0.4)
    cfg = P.Config(nx=nx, ny=ny, nz=nz, dt=dt, nt=nt, xcorr_step=4, sponge_width=2, fused=fused,
                   scheme=scheme, free_surface=fs, **kw)
    with P.Simulator(cfg) as sim:
        sim.set_model(**model)
        sim.set_source(nx // 2, ny // 2, min(2, nz - 1), EM.ricker(nt, dt, 40.0) * 1e3)
        sim.set_receivers(EM.receiver_plane(nx, ny, 0))
        tr = sim.forward()
        sim.adjoint(tr)
        gv, gr = sim.image()
    return tr, gv, gr


@pytest.mark.gpu
@pytest.mark.parametrize("shape,fs", [((9, 5, 6), True), ((33, 17, 3), False), ((31, 15, 1), False),
                                      ((5, 40, 20), True)],
                         ids=["tiny", "one-past-tile", "one-plane", "narrow"])
@pytest.mark.parametrize("scheme", [0, 1], ids=["staggered", "centred"])
def test_fused_matches_sequence_on_edge_shapes(shape, fs, scheme):
    # a free surface needs more than four interior planes
    ref = run(*shape, fused=False, scheme=scheme, fs=fs)
    got = run(*shape, fused=True, scheme=scheme, fs=fs)
    for a, b in zip(got, ref):
        assert np.all(np.isfinite(a))
        if np.abs(b).max() == 0:
            assert np.abs(a).max() == 0
        else:
            assert rel_l2(a, b) < 1e-5


@pytest.mark.gpu
def test_checkpoints_with_ragged_segments():
    # nt = 22: the last imaging period and the last checkpoint segment are partial
    plain = run(40, 32, 24, True, nt=22, snap_precision="fp16")
    ck = run(40, 32, 24, True, nt=22, snap_precision="fp16", checkpoint_every=8)
    for a, b in zip(ck, plain):
        np.testing.assert_array_equal(a, b)
