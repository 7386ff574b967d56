"""Work split of the fused kernels and its autotuner.  Each CTA takes bz
consecutive planes of the grid's tile-major (tile, z) planes, in one or more
column segments, or (ztop > 0) the top ztop planes of one column or bz
planes of the columns' bottoms; the split changes the launch shape, not the
arithmetic, so every choice gives bit-identical results, for both operators.
The tuner records the fastest choice for the grid."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM

NX, NY, NZ, NT = 64, 48, 40, 48


# (bz, ztop): 14 and 100 span two or more columns; ztop > 0 are top/bottom
# splits of the 6 tile columns (bottom CTAs of one plane, of several
# bottoms, and tops of a single plane)
SPLITS = ((8, 0), (14, 0), (NZ, 0), (100, 0), (3, 17), (50, 30), (7, 1))


def run_shot(scheme=0):
    model = EM.smooth_tti(NX, NY, NZ, dx=10.0, corr_m=60.0, seed=9)
    dt = EM.cfl_dt(model, 10.0)
    cfg = P.Config(nx=NX, ny=NY, nz=NZ, dt=dt, nt=NT, sponge_width=6, snap_precision="fp16", scheme=scheme)
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
        for scheme, ks in ((0, kinds), (1, ("type1_forward", "type1_adjoint"))):
            outs = []
            for bz, zt in SPLITS:
                for k in ks:
                    P.tune_set(NX, NY, NZ, k, bz, zt)
                    assert P.tune_get_split(NX, NY, NZ, k) == (bz, zt)
                outs.append(run_shot(scheme))
            for o in outs[1:]:
                for a, b in zip(o, outs[0]):
                    np.testing.assert_array_equal(a, b)
            for k in ks:
                P.tune_set(NX, NY, NZ, k, 0)
        with pytest.raises(P.TTIError):  # the tops must leave bottoms
            P.tune_set(NX, NY, NZ, "forward", 4, NZ)
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
            assert P.tune_get_split(NX, NY, NZ, k) == (rep[k]["bz"], rep[k]["ztop"])
    finally:
        for k in P.TUNE_KINDS:
            P.tune_set(NX, NY, NZ, k, 0)
