"""Work split of the fused kernels and its autotuner.  Each CTA takes bz
consecutive planes of the grid's tile-major (tile, z) planes, in one or more
column segments; bz changes the launch shape, not the arithmetic, so every
choice gives bit-identical results.  The tuner records the fastest choice
for the grid."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM

NX, NY, NZ, NT = 64, 48, 40, 48


def run_shot():
    model = EM.smooth_tti(NX, NY, NZ, dx=10.0, corr_m=60.0, seed=9)
    dt = EM.cfl_dt(model, 10.0)
    cfg = P.Config(nx=NX, ny=NY, nz=NZ, dt=dt, nt=NT, sponge_width=6, snap_precision="fp16")
    with P.Simulator(cfg) as sim:
        sim.set_model(**model)
        sim.set_source(NX // 2, NY // 2, 5, EM.ricker(NT, dt, 25.0) * 1e3)
        sim.set_receivers(EM.receiver_plane(NX, NY, 3))
        tr = sim.forward()
        sim.adjoint(tr)
        gv, gr = sim.image()
    return tr, gv, gr


@pytest.mark.gpu
def test_chunk_length_does_not_change_results_and_tuner_records_a_choice():
    kinds = ("forward", "adjoint", "imaging")
    try:
        outs = []
        for bz in (8, 14, NZ, 100):  # 14 and 100: CTAs whose planes span two or more columns
            for k in kinds:
                P.tune_set(NX, NY, NZ, k, bz)
                assert P.tune_get(NX, NY, NZ, k) == bz
            outs.append(run_shot())
        for o in outs[1:]:
            for a, b in zip(o, outs[0]):
                np.testing.assert_array_equal(a, b)
        for k in kinds:
            P.tune_set(NX, NY, NZ, k, 0)
        model = EM.smooth_tti(NX, NY, NZ, dx=10.0, corr_m=60.0, seed=9)
        cfg = P.Config(nx=NX, ny=NY, nz=NZ, dt=EM.cfl_dt(model, 10.0), nt=NT, snap_precision="fp16")
        with P.Simulator(cfg) as sim:
            sim.set_model(**model)
            rep = sim.autotune(reps=2)
        assert rep["candidates"] >= 3
        for k in kinds:
            assert rep[k]["ms"] > 0 and rep[k]["ms"] <= rep[k]["model_ms"] * 1.0001
            assert P.tune_get(NX, NY, NZ, k) == rep[k]["bz"]
    finally:
        for k in kinds:
            P.tune_set(NX, NY, NZ, k, 0)
