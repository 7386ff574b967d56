"""Shared helpers for the tests: seeded inputs in the reference layout and
comparison metrics."""
from __future__ import annotations

import os

import numpy as np

from oracle import Layout, sponge_profile  # noqa: F401  (re-exported for the tests)
from oracle import rtm_shot as oracle_rtm  # noqa: F401
from oracle import rtm_shot_t1 as oracle_rtm_t1  # noqa: F401


def report_dir():
    """Directory for JSON reports of the GPU tests (TTI_REPORT_DIR), or None."""
    d = os.environ.get("TTI_REPORT_DIR")
    return d if d and os.path.isdir(d) else None


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)


def random_model(lay: Layout, rng, tti=True, halo_safe=True):
    """Random but physically plausible model volumes over the whole halo'd
    allocation (the reference kernels read model halos)."""
    sh = lay.shape
    vp = rng.uniform(1800.0, 3200.0, sh)
    eps = rng.uniform(0.0, 0.25, sh)
    delta = eps * rng.uniform(0.0, 0.6, sh)
    vs = rng.uniform(0.0, 400.0, sh)
    theta = rng.uniform(0.0, 0.8, sh) if tti else np.zeros(sh)
    phi = rng.uniform(0.0, 3.0, sh) if tti else np.zeros(sh)
    m1 = vp * vp * (1 + 2 * eps)
    m2 = np.sqrt((vp * vp - vs * vs) * (vp * vp * (1 + 2 * delta) - vs * vs))
    m = dict(m1=m1, m2=m2, m3=vp * vp, m4=vs * vs, rx=np.sin(theta) * np.cos(phi),
             ry=np.sin(theta) * np.sin(phi), rz=np.cos(theta),
             irho=1.0 / rng.uniform(1.0, 2.5, sh))
    return {k: np.ascontiguousarray(v, np.float32) for k, v in m.items()}


def random_field(lay: Layout, rng, scale=1.0, halo=True):
    a = (scale * rng.standard_normal(lay.shape)).astype(np.float32)
    if not halo:
        b = np.zeros_like(a)
        b[lay.interior] = a[lay.interior]
        a = b
    return a


def sponge_ab(n_alloc, rng, active=True):
    ab = np.ones((n_alloc, 2), np.float32)
    if active:
        ab[:, 0] = rng.uniform(0.9, 1.0, n_alloc)
        ab[:, 1] = rng.uniform(0.9, 1.0, n_alloc)
    return np.ascontiguousarray(ab.reshape(-1))


def sim_models(sim):
    """The simulator's model volumes read back from the device (for checking
    the model set-up itself; parity runs build theirs on the host)."""
    names = ("irho", "model1", "model2", "model3", "model4", "rx", "ry", "rz")
    keys = ("irho", "m1", "m2", "m3", "m4", "rx", "ry", "rz")
    return {k: np.ascontiguousarray(sim.volume(n)) for k, n in zip(keys, names)}


def oracle_models(lay, model, dtype=np.float32):
    """Model volumes the oracle runs on, built on the host from the same
    parameter arrays the simulator was given (init_cijs per cell after
    edge extension, irho = 1/rho)."""
    from oracle import models_from_parameters

    return models_from_parameters(lay, **model, dtype=dtype)
