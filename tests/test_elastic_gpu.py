"""The simulator3 (elastic eTTI proxy) step kernels on the GPU against the
oracle: each launcher on seeded inputs over a z extent that crosses the
reference's 64-plane blocks (nx 64, ny 32, nz 80), and the composed
forward/adjoint schedule with its two images.

FP32 throughout; the kernels and the oracle sum in the same order but the
GPU contracts multiply-adds, so volumes agree to a max-normalised error of
1e-5 per launch and 1e-4 after the composed schedule (its values grow by
about 1e4 per step: the reference's stand-in coefficients are not a stable
scheme)."""
import numpy as np
import pytest
import torch

from oracle import ElasticOracle, Layout, e3_execute

pytestmark = pytest.mark.gpu

LAY = Layout(64, 32, 80)


def maxerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def vols(n, rng, lay=LAY):
    return [rng.standard_normal(lay.shape).astype(np.float32) for _ in range(n)]


def dev(a):
    return [torch.from_numpy(x).cuda() for x in a]


def host(a):
    return [x.cpu().numpy() for x in a]


def zprime_of(lay):
    return np.cos(6 * np.arange(lay.ldimz, dtype=np.float32)).astype(np.float32)


def test_vgplain():
    from miniappsforhpe_b200 import elastic as E

    rng = np.random.default_rng(10)
    v, zp = vols(3, rng), zprime_of(LAY)
    d = [LAY.zeros() for _ in range(6)]
    ElasticOracle().vgplain(LAY, *v, d, zp)
    gv, gd = dev(v), dev([LAY.zeros() for _ in range(6)])
    E.launch_vgplain(*gv, *gd, torch.from_numpy(zp).cuda(), LAY.nx, LAY.ny, LAY.nz, LAY.ldimx, LAY.ldimy)
    torch.cuda.synchronize()
    for a, b in zip(host(gd), d):
        assert maxerr(a, b) < 1e-5


def test_splain_with_the_blocked_precomputes():
    from miniappsforhpe_b200 import elastic as E

    rng = np.random.default_rng(11)
    s, M, d = vols(6, rng), vols(21, rng), vols(6, rng)
    pre = [LAY.zeros() for _ in range(12)]
    gs, gM, gd, gpre = dev(s), dev(M), dev(d), dev(pre)
    s_o = [x.copy() for x in s]
    ElasticOracle().splain(LAY, s_o, M, d, pre)
    E.launch_splain(*gs, gM, *gd, gpre, LAY.nx, LAY.ny, LAY.nz, LAY.ldimx, LAY.ldimy)
    torch.cuda.synchronize()
    I = LAY.interior
    for a, b in zip(host(gpre), pre):
        assert maxerr(a[I], b[I]) < 1e-5
    for a, b in zip(host(gs), s_o):
        assert maxerr(a, b) < 1e-5


def test_vplain_and_mirrors():
    from miniappsforhpe_b200 import elastic as E

    rng = np.random.default_rng(12)
    v, s, (M22,), zp = vols(3, rng), vols(6, rng), vols(1, rng), zprime_of(LAY)
    gv, gs = dev(v), dev(s)
    v_o = [x.copy() for x in v]
    e = ElasticOracle()
    e.vplain(LAY, v_o, s, M22, zp)
    E.launch_vplain(*gv, *gs, torch.from_numpy(M22).cuda(), torch.from_numpy(zp).cuda(), LAY.nx, LAY.ny, LAY.nz,
                    LAY.ldimx, LAY.ldimy)
    torch.cuda.synchronize()
    for a, b in zip(host(gv), v_o):
        assert maxerr(a, b) < 1e-5
    s_o = [x.copy() for x in s]
    e.mirror(LAY, s_o)
    E.launch_mirror(gs, LAY.ldimx, LAY.ldimy, 4, LAY.ldimz)
    torch.cuda.synchronize()
    for a, b in zip(host(gs), s_o):
        np.testing.assert_array_equal(a, b)


def test_mirror_rejects_a_surface_without_room_for_its_image():
    from miniappsforhpe_b200 import TTIError
    from miniappsforhpe_b200 import elastic as E

    lay = Layout(8, 8, 1)  # ldimz 9: the mirror of plane 0 about 4 is plane 8, about 5 it would be 10
    f = dev([lay.zeros()])
    E.launch_mirror(f, lay.ldimx, lay.ldimy, 4, lay.ldimz)
    with pytest.raises(TTIError):
        E.launch_mirror(f, lay.ldimx, lay.ldimy, 5, lay.ldimz)


def test_pressure_update_gv_and_model():
    from miniappsforhpe_b200 import elastic as E

    rng = np.random.default_rng(13)
    s = vols(6, rng)
    e = ElasticOracle()
    p = LAY.zeros()
    e.pressure(p, s)
    gp = torch.zeros(LAY.shape, device="cuda")
    E.launch_compute_p(gp, *dev(s), gp.numel())
    g = rng.standard_normal((LAY.nz, LAY.ny, LAY.nx)).astype(np.float32)
    s1, s3 = (rng.standard_normal(g.shape).astype(np.float32) for _ in range(2))
    gg = torch.from_numpy(g).cuda()
    e.update_gv(LAY, g, s1, s3, s[0], s[2])
    ds = dev(s)
    E.launch_update_gv(gg, *dev([s1, s3]), ds[0], ds[2], LAY.nx, LAY.ny, LAY.nz, LAY.ldimx, LAY.ldimy)
    M = [LAY.zeros() for _ in range(22)]
    d = [LAY.zeros() for _ in range(6)]
    zp = np.zeros(LAY.ldimz, np.float32)
    e.init_model(LAY, M, d, zp)
    gM, gd = dev([LAY.zeros() for _ in range(22)]), dev([LAY.zeros() for _ in range(6)])
    gz = torch.zeros(LAY.ldimz, device="cuda")
    E.launch_init_model(gM, gd, gz, LAY.nx, LAY.ldimx, LAY.ldimy, LAY.ldimz)
    torch.cuda.synchronize()
    assert maxerr(gp.cpu().numpy(), p) < 1e-6
    assert maxerr(gg.cpu().numpy(), g) < 1e-6
    for a, b in zip(host(gM) + host(gd) + [gz.cpu().numpy()], M + d + [zp]):
        np.testing.assert_allclose(a, b, atol=4e-6)


def test_composed_schedule_against_the_oracle():
    from miniappsforhpe_b200.elastic import ElasticProxy

    lay = Layout(32, 16, 70)
    want = e3_execute(lay, 3, 1, press=1.0)
    sim = ElasticProxy(lay.nx, lay.ny, lay.nz)
    assert sim.ldimx == lay.ldimx
    sim.execute(3, 1, press=1.0)
    torch.cuda.synchronize()
    for a, b in zip(host(sim.v), want["v_adj"]):
        assert maxerr(a, b) < 1e-4
    for a, b in zip(host(sim.s), want["s_adj"]):
        assert maxerr(a, b) < 1e-4
    assert maxerr(sim.g1.cpu().numpy(), want["g1"]) < 1e-4
    inner = (slice(None), slice(None), slice(4, lay.nx - 4))  # 1/M18 is infinite at the zeroed x halo
    g2 = sim.g2.cpu().numpy()[inner]
    assert np.isfinite(g2).all()
    assert maxerr(g2, want["g2"][inner]) < 1e-4
    assert sim.launches == 3 * 8 + 3 * 7 + 3 * 2


class OddLayout:
    """A halo'd layout whose rows are not a multiple of four floats (the
    launchers then stage their tiles with 4-byte copies)."""

    def __init__(self, nx, ny, nz):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.ldimx, self.ldimy, self.ldimz = nx + 9, ny + 8, nz + 8
        self.shape = (self.ldimz, self.ldimy, self.ldimx)

    def zeros(self):
        return np.zeros(self.shape, np.float32)


def test_velocity_kernels_on_rows_of_odd_length():
    from miniappsforhpe_b200 import elastic as E

    lay = OddLayout(40, 20, 70)
    rng = np.random.default_rng(14)
    v, s, (M22,) = vols(3, rng, lay), vols(6, rng, lay), vols(1, rng, lay)
    zp = np.cos(6 * np.arange(lay.ldimz, dtype=np.float32)).astype(np.float32)
    e = ElasticOracle()
    d = [lay.zeros() for _ in range(6)]
    e.vgplain(lay, *v, d, zp)
    v_o = [x.copy() for x in v]
    e.vplain(lay, v_o, s, M22, zp)
    gv, gd, gz = dev(v), dev([lay.zeros() for _ in range(6)]), torch.from_numpy(zp).cuda()
    E.launch_vgplain(*gv, *gd, gz, lay.nx, lay.ny, lay.nz, lay.ldimx, lay.ldimy)
    E.launch_vplain(*gv, *dev(s), torch.from_numpy(M22).cuda(), gz, lay.nx, lay.ny, lay.nz, lay.ldimx, lay.ldimy)
    torch.cuda.synchronize()
    for a, b in zip(host(gd), d):
        assert maxerr(a, b) < 1e-5
    for a, b in zip(host(gv), v_o):
        assert maxerr(a, b) < 1e-5


def test_stress_update_on_rows_of_odd_length():
    from miniappsforhpe_b200 import elastic as E

    lay = OddLayout(40, 20, 70)
    rng = np.random.default_rng(15)
    s, M, d = vols(6, rng, lay), vols(21, rng, lay), vols(6, rng, lay)
    pre = [lay.zeros() for _ in range(12)]
    gs, gpre = dev(s), dev(pre)
    s_o = [x.copy() for x in s]
    ElasticOracle().splain(lay, s_o, M, d, pre)
    E.launch_splain(*gs, dev(M), *dev(d), gpre, lay.nx, lay.ny, lay.nz, lay.ldimx, lay.ldimy)
    torch.cuda.synchronize()
    I = (slice(4, 4 + lay.nz), slice(4, 4 + lay.ny), slice(4, 4 + lay.nx))
    for a, b in zip(host(gpre), pre):
        assert maxerr(a[I], b[I]) < 1e-5
    for a, b in zip(host(gs), s_o):
        assert maxerr(a, b) < 1e-5
