"""Model set-up on the GPU against the oracle built from the same host
parameters.

* ``tti_launch_init_cijs`` (the reference's init_cijs, simulator2SetUp.cu:
  10-29) against the oracle's per-cell restatement on random parameters.
* ``tti_sim_set_model``: every model volume the step kernels read (irho,
  model1..model4, rx, ry, rz), halos and x padding included, against
  ``oracle.models_from_parameters`` (edge extension, init_cijs, irho = 1/rho)
  on a TTI model with variable vs and density and on a layered VTI model.

Tolerances: m3 = vp^2, m4 = vs^2 and irho = 1/rho are single IEEE operations
and must agree bit for bit; m1, m2 and the direction cosines go through
sqrtf/sinf/cosf and products the device compiler may contract into FMAs, so
they may differ by a few units in the last place (4 ulp of the volume's
largest magnitude).
"""
import numpy as np
import pytest
import torch

import miniappsforhpe_b200 as P
from miniappsforhpe_b200 import earth_models as EM
from oracle import Layout, Oracle, models_from_parameters

EXACT = ("irho", "m3", "m4")
NAMES = {"irho": "irho", "m1": "model1", "m2": "model2", "m3": "model3", "m4": "model4", "rx": "rx",
         "ry": "ry", "rz": "rz"}


def random_parameters(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    sh = (nz, ny, nx)
    eps = rng.uniform(0.0, 0.25, sh)
    return dict(vp=rng.uniform(1500.0, 5000.0, sh), eps=eps, delta=eps * rng.uniform(0.0, 0.6, sh),
                vs=rng.uniform(0.0, 600.0, sh), theta=rng.uniform(0.0, np.pi / 4, sh),
                phi=rng.uniform(0.0, np.pi, sh), rho=rng.uniform(1.0, 2.7, sh))


def check_close(name, got, want):
    assert got.shape == want.shape, name
    assert np.all(np.isfinite(got)), name
    if name in EXACT:
        np.testing.assert_array_equal(got, want, err_msg=name)
    else:
        scale = float(np.abs(want).max())
        np.testing.assert_allclose(got, want, rtol=0, atol=4 * np.spacing(np.float32(scale)), err_msg=name)


@pytest.mark.gpu
def test_init_cijs_launcher_matches_oracle():
    n = 100_003  # not a multiple of the block size
    p = {k: np.ascontiguousarray(v.ravel(), np.float32) for k, v in random_parameters(n, 1, 1, 3).items()}
    dev = {k: torch.from_numpy(p[k]).cuda() for k in ("vp", "eps", "delta", "vs", "theta", "phi")}
    out = [torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(7)]
    P.launch_init_cijs(dev["vp"], dev["eps"], dev["delta"], dev["vs"], dev["theta"], dev["phi"], *out, n)
    torch.cuda.synchronize()
    want = Oracle("f32").init_cijs(p["vp"], p["eps"], p["delta"], p["vs"], p["theta"], p["phi"])
    for name, g, w in zip(("m1", "m2", "m3", "m4", "rx", "ry", "rz"), out, want):
        check_close(name, g.cpu().numpy(), w)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["tti_random", "vti_layered"])
def test_set_model_volumes_match_host_build(kind):
    nx, ny, nz = 37, 29, 23  # ldimx = 64: 19 columns of x padding beyond the halo
    if kind == "tti_random":
        model = random_parameters(nx, ny, nz, 11)
    else:
        model = EM.layered_vti(nx, ny, nz, nlayers=4, seed=5)
    model = {k: np.ascontiguousarray(v, np.float32) for k, v in model.items()}
    lay = Layout(nx, ny, nz)
    want = models_from_parameters(lay, **model)
    cfg = P.Config(nx=nx, ny=ny, nz=nz, dt=1e-4, nt=4, save_snapshots=False)
    with P.Simulator(cfg) as sim:
        sim.set_model(**model)
        got = {k: sim.volume(n) for k, n in NAMES.items()}
    for k in NAMES:
        check_close(k, got[k], want[k])
    # the halo is the nearest interior cell: corners and the x padding
    assert got["m3"][0, 0, 0] == model["vp"][0, 0, 0] ** 2
    assert got["m3"][-1, -1, -1] == model["vp"][-1, -1, -1] ** 2
