"""Type1 (constant density, centred second derivatives) oracle on the CPU.

Pins of the restatement of kernels/kernel_type1_gpu_{fwd,adj,grad}.cu:
* FP64: the adjoint launcher is the exact transpose of the forward launcher
  (both without sponge): <dt*M D x, y> = <x, dt*D M^T y> for inputs
  supported on the interior, to 1e-12; a wrong tap, sign, weight or
  coefficient breaks it;
* FP32 agrees with FP64 to rounding;
* the imaging kernel is the plain product-sum it restates."""
import numpy as np

from oracle import Layout, Oracle
from tests.helpers import random_field, random_model, rel_l2, sponge_ab

H = (10.0, 12.5, 8.0)
DT = np.float32(1e-3)


def _setup(o, nx=20, ny=17, nz=15, seed=3):
    lay = Layout(nx, ny, nz)
    rng = np.random.default_rng(seed)
    m = {k: v.astype(o.dtype) for k, v in random_model(lay, rng, tti=True).items()}
    ab = [sponge_ab(n, rng) for n in (lay.ldimx, lay.ldimy, lay.ldimz)]
    return lay, rng, m, ab


def _interior(lay, a):
    b = np.zeros_like(a)
    b[lay.interior] = a[lay.interior]
    return b


def test_type1_adjoint_is_the_transpose_of_the_forward_fp64():
    o = Oracle("f64")
    lay, rng, m, ab = _setup(o)
    x1 = _interior(lay, random_field(lay, rng).astype(np.float64))
    x2 = _interior(lay, random_field(lay, rng).astype(np.float64))
    y1 = _interior(lay, random_field(lay, rng).astype(np.float64))
    y2 = _interior(lay, random_field(lay, rng).astype(np.float64))
    a3, a4 = lay.zeros(np.float64), lay.zeros(np.float64)
    o.t1_fwd(lay, a3, a4, x1, x2, m, ab, DT, H, 0)
    b3, b4 = lay.zeros(np.float64), lay.zeros(np.float64)
    o.t1_adj(lay, b3, b4, y1, y2, m, ab, DT, H, False)
    lhs = float(np.sum(a3 * y1) + np.sum(a4 * y2))
    rhs = float(np.sum(x1 * b3) + np.sum(x2 * b4))
    assert abs(lhs) > 0
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_type1_fp32_matches_fp64():
    o32, o64 = Oracle("f32"), Oracle("f64")
    lay, rng, m, ab = _setup(o32, seed=5)
    f1, f2, f3, f4 = (random_field(lay, rng) for _ in range(4))
    m64 = {k: v.astype(np.float64) for k, v in m.items()}
    for mode in (0, 1, 2):
        ld = (lay.nx, lay.ny) if mode == 2 else None
        shape = (lay.nz, lay.ny, lay.nx) if mode == 2 else lay.shape
        r32 = [np.zeros(shape, np.float32) if mode == 2 else f.copy() for f in (f3, f4)]
        r64 = [np.zeros(shape, np.float64) if mode == 2 else f.astype(np.float64) for f in (f3, f4)]
        o32.t1_fwd(lay, *r32, f1, f2, m, ab, DT, H, mode, ld)
        o64.t1_fwd(lay, *r64, f1.astype(np.float64), f2.astype(np.float64), m64, ab, DT, H, mode, ld)
        for a, b in zip(r32, r64):
            assert rel_l2(a, b) < 1e-5
    for sponge in (False, True):
        r32 = [f3.copy(), f4.copy()]
        r64 = [f3.astype(np.float64), f4.astype(np.float64)]
        o32.t1_adj(lay, *r32, f1, f2, m, ab, DT, H, sponge)
        o64.t1_adj(lay, *r64, f1.astype(np.float64), f2.astype(np.float64), m64, ab, DT, H, sponge)
        for a, b in zip(r32, r64):
            assert rel_l2(a, b) < 1e-5


def test_type1_imaging_is_the_product_sum():
    o = Oracle("f32")
    lay, rng, _, _ = _setup(o, seed=9)
    n = lay.nx * lay.ny * lay.nz
    sx, sz, g = (rng.standard_normal(n).astype(np.float32) for _ in range(3))
    ax, az = random_field(lay, rng), random_field(lay, rng)
    want = g + ax[lay.interior].ravel() * sx + az[lay.interior].ravel() * sz
    o.t1_grad(lay, sx, sz, g, ax, az)
    np.testing.assert_allclose(g, want, rtol=1e-6, atol=1e-6)
