"""The simulator3 (elastic eTTI proxy) oracle on the CPU.

The closed-form precompute of the oracle is checked bit for bit against a
numpy walk of the reference's register-queue loop (priming, then the
steady state, then the rotation: simulator3/simulator3SetUp.cu:47-187), on
a z extent that crosses one of its 64-plane blocks; the mirrors, the
pressure and the stand-in model against their formulas (:229-300,
:1387-1492); and the composed schedule (:2181-2657) for finite images.
"""
import os

import numpy as np
import pytest

from oracle import ElasticOracle, Layout, e3_execute

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INT = np.array([1.01, 2.01, 3.01, 4.01], np.float32)


def queue_walk_precompute(inp, XS, YS, ZS, lay):
    """The reference kernel's loop structure, per 64-plane block, in numpy."""
    nx, ny, nz = lay.nx, lay.ny, lay.nz
    X1, X2, Y1, Y2 = -3 - XS, 4 - XS, -3 - YS, 4 - YS
    xz, yz = lay.zeros(), lay.zeros()

    def sh(pl, dy, dx):
        return inp[pl, 4 + dy:4 + dy + ny, 4 + dx:4 + dx + nx]

    for b in range((nz - 1) // 64 + 1):
        iz = 64 * b
        p0 = iz + 1 - ZS
        qxz = [np.zeros((ny, nx), np.float32) for _ in range(8)]
        qyz = [np.zeros((ny, nx), np.float32) for _ in range(8)]
        for i in range(7):  # priming: the plane p0 + i arrives
            c = INT[max(3 - i, i - 4)]
            for j in range(i + 1):
                qxz[j] = qxz[j] + c * (sh(p0 + i, 0, X1 + i - j) + sh(p0 + i, 0, X2 - i + j))
                qyz[j] = qyz[j] + c * (sh(p0 + i, Y1 + i - j, 0) + sh(p0 + i, Y2 - i + j, 0))
        for zl in range(min(64, nz - iz)):
            pl = p0 + 7 + zl
            for i in range(8):
                c = INT[max(3 - i, i - 4)]
                qxz[i] = qxz[i] + c * (sh(pl, 0, X1 + i) + sh(pl, 0, X2 - i))
                qyz[i] = qyz[i] + c * (sh(pl, Y1 + i, 0) + sh(pl, Y2 - i, 0))
            xz[iz + 4 + zl, 4:4 + ny, 4:4 + nx] = np.float32(0.5) * qxz[0]
            yz[iz + 4 + zl, 4:4 + ny, 4:4 + nx] = np.float32(0.5) * qyz[0]
            qxz = qxz[1:] + [np.zeros((ny, nx), np.float32)]
            qyz = qyz[1:] + [np.zeros((ny, nx), np.float32)]
    return xz, yz


@pytest.mark.parametrize("shifts", [(1, 1, 1), (0, 0, 1), (0, 1, 0), (1, 0, 0)])
def test_precompute_closed_form_equals_the_queue_walk(shifts):
    lay = Layout(8, 5, 70)  # 70 planes: two 64-plane blocks, the second ragged
    inp = np.random.default_rng(3).standard_normal(lay.shape).astype(np.float32)
    xz, yz = lay.zeros(), lay.zeros()
    ElasticOracle().precompute(lay, inp, xz, yz, *shifts)
    wxz, wyz = queue_walk_precompute(inp, *shifts, lay)
    np.testing.assert_array_equal(xz, wxz)
    np.testing.assert_array_equal(yz, wyz)


def test_precompute_priming_weights_show_in_the_block_starts():
    """Planes m = 1..6 of each block weigh the early planes by the arriving
    plane's index: a constant input gives a different sum there than in the
    steady state."""
    lay = Layout(4, 4, 70)
    inp = np.ones(lay.shape, np.float32)
    xz, yz = lay.zeros(), lay.zeros()
    ElasticOracle().precompute(lay, inp, xz, yz, 1, 1, 1)
    col = xz[4:4 + lay.nz, 6, 6]
    steady = np.float32(0.5) * 2 * 2 * INT.sum()  # each weight twice, pairs of ones
    assert np.isclose(col[0], steady) and np.isclose(col[7], steady) and np.isclose(col[64], steady)
    assert not np.isclose(col[1], steady) and not np.isclose(col[65], steady)


def test_mirror_pressure_and_update_gv_formulas():
    e, lay = ElasticOracle(), Layout(6, 5, 12)
    rng = np.random.default_rng(4)
    f = [rng.standard_normal(lay.shape).astype(np.float32) for _ in range(6)]
    want = [x.copy() for x in f]
    for w in want:
        w[4] = 0.0
        for iz in range(4):
            w[iz] = -w[8 - iz]
    e.mirror(lay, f)
    for a, b in zip(f, want):
        np.testing.assert_array_equal(a, b)
    p = lay.zeros()
    e.pressure(p, f)
    w = -(2 * f[0] + 3 * f[1] + 4 * f[2] + 5 * f[3] + 6 * f[4] + 7 * f[5]) / np.float32(27)
    np.testing.assert_allclose(p, w, rtol=1e-6, atol=1e-6)
    g = rng.standard_normal((lay.nz, lay.ny, lay.nx)).astype(np.float32)
    s1, s3 = (rng.standard_normal(g.shape).astype(np.float32) for _ in range(2))
    g0 = g.copy()
    e.update_gv(lay, g, s1, s3, f[0], f[2])
    I = lay.interior
    np.testing.assert_allclose(g, g0 + f[0][I] * s1 + f[2][I] * s3, rtol=1e-6, atol=1e-6)


def test_stand_in_model_formulas():
    e, lay = ElasticOracle(), Layout(5, 4, 6)
    M = [lay.zeros() for _ in range(22)]
    d = [lay.zeros() for _ in range(6)]
    zp = np.zeros(lay.ldimz, np.float32)
    e.init_model(lay, M, d, zp)
    iz, iy, ix = np.meshgrid(np.arange(lay.ldimz), np.arange(lay.ldimy), np.arange(4, 4 + lay.nx), indexing="ij")
    iz, iy, ix = (a.astype(np.float32) for a in (iz, iy, ix))
    args = [2 * iz + iy + ix, iz + 2 * iy + ix, iz + iy + 2 * ix, 3 * iz + iy + ix, iz + 3 * iy + ix,
            iz + iy + 3 * ix, 4 * iz + iy + ix, iz + 4 * iy + ix, iz + iy + 4 * ix, 5 * iz + iy + ix,
            iz + 5 * iy + ix]
    for k, a in enumerate(args):
        np.testing.assert_allclose(M[2 * k][:, :, 4:4 + lay.nx], np.cos(a), atol=2e-6)
        np.testing.assert_allclose(M[2 * k + 1][:, :, 4:4 + lay.nx], np.sin(a), atol=2e-6)
    np.testing.assert_allclose(d[2][:, :, 4:4 + lay.nx], np.cos(6 * iz + iy + ix), atol=2e-6)
    np.testing.assert_allclose(zp, np.cos(6 * np.arange(lay.ldimz, dtype=np.float32)), atol=2e-6)
    assert not M[0][:, :, :4].any() and not M[0][:, :, 4 + lay.nx:].any()  # x halo left unset


def test_composed_schedule_images():
    """Three forward and three adjoint steps: the velocity image is finite
    everywhere; the density image is finite away from the x edges (the
    stand-in model leaves the x halo at zero, so 1/M18 there is infinite)."""
    lay = Layout(32, 16, 70)
    out = e3_execute(lay, 3, 1, press=1.0)
    assert np.isfinite(out["g1"]).all() and np.abs(out["g1"]).max() > 0
    inner = out["g2"][:, :, 4:lay.nx - 4]
    assert np.isfinite(inner).all() and np.abs(inner).max() > 0


def test_bench_cpu_sample_of_the_elastic_steps():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    d = bench.elastic_cpu_sample(n=24, steps=1)
    assert d["value"] > 0 and d["kind"] == "port" and d["cores"] >= 1
