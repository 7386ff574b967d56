"""Failure detection without a GPU fault: the bounded waits of the fused
kernels, run on a barrier that nothing completes, give up after their clock
limit and report TTI_ETIMEOUT; the context stays usable (a shot runs right
after and matches a shot run before)."""
import time

import numpy as np
import pytest

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM


def small_shot():
    nx = ny = nz = 32
    m = EM.layered_vti(nx, ny, nz, 3, seed=2)
    dt = EM.cfl_dt(m, 10.0)
    with P.Simulator(P.Config(nx=nx, ny=ny, nz=nz, dt=dt, nt=24, sponge_width=4)) as sim:
        sim.set_model(**m)
        sim.set_source(16, 16, 4, EM.ricker(24, dt, 25.0) * 1e3)
        sim.set_receivers(EM.receiver_plane(nx, ny, 3))
        tr = sim.forward()
        sim.adjoint(tr)
        return tr, sim.image()[0]


@pytest.mark.gpu
def test_bounded_wait_times_out_and_the_context_survives():
    before = small_shot()
    t0 = time.perf_counter()
    rc = P.lib().tti_selfcheck_bounded_wait(0.2, None)
    took = time.perf_counter() - t0
    assert rc == P.ETIMEOUT
    assert took < 5.0
    after = small_shot()
    for a, b in zip(before, after):
        np.testing.assert_array_equal(a, b)
    assert P.lib().tti_selfcheck_bounded_wait(0.0, None) == P.EINVAL
