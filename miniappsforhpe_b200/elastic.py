"""Elastic step kernels of the reference's simulator3 (its eTTI proxy):
ctypes bindings of include/tti_capi.h section 5.

Arguments are CUDA tensors (or raw device pointers) in the halo'd layout of
the simulator (FP32, x fastest, radius-4 halo, interior [4, 4+n-1] per
axis).  The constants are the reference's stand-ins; see the header.
"""
from __future__ import annotations

import ctypes as C

from . import _ptr, _call

V = C.c_void_p


def _arr(vols):
    ptrs = (V * len(vols))(*[_ptr(v) for v in vols])
    return ptrs


def launch_vgplain(f1, f2, f3, d4, d5, d6, d7, d8, d9, zprime, nx, ny, nz, ldimx, ldimy, stream=None):
    """vgPlainLoop (simulator3/simulator3SetUp.cu:1364-1386)."""
    _call("tti_e3_launch_vgplain", f1, f2, f3, d4, d5, d6, d7, d8, d9, zprime, nx, ny, nz, ldimx, ldimy, stream)


def launch_splain(f4, f5, f6, f7, f8, f9, M, f1_1, f1_2, f1_3, f2_2, f2_3, f3_3, f10_21, nx, ny, nz, ldimx, ldimy,
                  stream=None):
    """sPlainLoop (simulator3/simulator3SetUp.cu:1127-1216); M = [M1..M21],
    f10_21 = the 12 precompute outputs f10 .. f21."""
    if len(M) != 21 or len(f10_21) != 12:
        raise ValueError("expected 21 model volumes and 12 precompute volumes")
    m, p = _arr(M), _arr(f10_21)
    _call("tti_e3_launch_splain", f4, f5, f6, f7, f8, f9, C.addressof(m), f1_1, f1_2, f1_3, f2_2, f2_3, f3_3,
          C.addressof(p), nx, ny, nz, ldimx, ldimy, stream)


def launch_vplain(f1, f2, f3, f4, f5, f6, f7, f8, f9, M22, zprime, nx, ny, nz, ldimx, ldimy, stream=None):
    """vPlainLoop (simulator3/simulator3SetUp.cu:1105-1125)."""
    _call("tti_e3_launch_vplain", f1, f2, f3, f4, f5, f6, f7, f8, f9, M22, zprime, nx, ny, nz, ldimx, ldimy, stream)


def launch_mirror(fields, ldimx, ldimy, izbeg, ldimz, stream=None):
    """mirror_s / mirror_v (simulator3/simulator3SetUp.cu:1425-1492)."""
    f = _arr(fields)
    _call("tti_e3_launch_mirror", C.addressof(f), len(fields), ldimx, ldimy, ldimz, izbeg, stream)


def launch_compute_p(p, f4, f5, f6, f7, f8, f9, n, stream=None):
    """compute_p_kernel (simulator3/simulator3SetUp.cu:275-289)."""
    _call("tti_e3_launch_compute_p", p, f4, f5, f6, f7, f8, f9, n, stream)


def launch_init_model(M22, d4_9, zprime, nx, ldimx, ldimy, ldimz, stream=None):
    """init_cijs_kernel (simulator3/simulator3SetUp.cu:229-273); M22 = [M1..M22], d4_9 = [d4..d9]."""
    m, d = _arr(M22), _arr(d4_9)
    _call("tti_e3_launch_init_model", C.addressof(m), C.addressof(d), zprime, nx, ldimx, ldimy, ldimz, stream)


def launch_update_gv(g1, snap_v1, snap_v3, a_v1, a_v3, nx, ny, nz, ldimx, ldimy, g_ldimx=None, g_ldimy=None,
                     stream=None):
    """update_gv / update_g_v (simulator3/simulator3SetUp.cu:1494-1538)."""
    _call("tti_e3_launch_update_gv", g1, snap_v1, snap_v3, a_v1, a_v3, nx, ny, nz, ldimx, ldimy,
          nx if g_ldimx is None else g_ldimx, ny if g_ldimy is None else g_ldimy, stream)


class ElasticProxy:
    """One subdomain of the reference's simulator3 on one device: the
    velocities f1..f3, stresses f4..f9, strains d4..d9, z-mixed volumes
    f10..f21, the stand-in model M1..M22 and zprime, the pressure, and the
    velocity (g1) and density (g2) images, with the step schedule of
    simulator3SetUp::execute (simulator3/simulator3SetUp.cu:2181-2657).

    Volumes are CUDA tensors of shape (nz+8, ny+8, ldimx) with ldimx = nx+8
    padded to 32 floats (x fastest, radius-4 halo); the images are halo-free
    (nz, ny, nx)."""

    RADIUS = 4

    def __init__(self, nx, ny, nz, device="cuda", d123=(1.0, 1.0, 1.0)):
        import torch

        self.nx, self.ny, self.nz = nx, ny, nz
        self.ldimx = 32 * ((nx + 8 - 1) // 32 + 1)
        self.ldimy, self.ldimz = ny + 8, nz + 8
        self.d123 = d123
        shape = (self.ldimz, self.ldimy, self.ldimx)

        def z():
            return torch.zeros(shape, dtype=torch.float32, device=device)

        self.v = [z() for _ in range(3)]
        self.s = [z() for _ in range(6)]
        self.d = [z() for _ in range(6)]
        self.pre = [z() for _ in range(12)]
        self.M = [z() for _ in range(22)]
        self.p = z()
        self.zprime = torch.zeros(self.ldimz, dtype=torch.float32, device=device)
        self.g1 = torch.zeros((nz, ny, nx), dtype=torch.float32, device=device)
        self.g2 = torch.zeros((nz, ny, nx), dtype=torch.float32, device=device)
        self.snaps = {}
        self.launches = 0  # calls of the C-ABI step launchers
        self._stream = torch.cuda.current_stream(device).cuda_stream
        launch_init_model(self.M, self.d, self.zprime, nx, self.ldimx, self.ldimy, self.ldimz, self._stream)

    @property
    def _g(self):
        return (self.nx, self.ny, self.nz, self.ldimx, self.ldimy)

    def init_source(self, press=500.0):
        """init_src_kernel (:291-300): stress k at the grid centre = press * k."""
        c = tuple(n // 2 + self.RADIUS for n in (self.nx, self.ny, self.nz))
        for k in range(6):
            self.s[k][c[2], c[1], c[0]] = float(press) * (k + 1)

    def _mirrors(self):
        st = self._stream
        for fields in (self.s, self.s, self.v, self.v):
            launch_mirror(fields, self.ldimx, self.ldimy, self.RADIUS, self.ldimz, st)
        self.launches += 4

    def _vplain(self):
        launch_vplain(*self.v, *self.s, self.M[21], self.zprime, *self._g, stream=self._stream)

    def _vgplain(self):
        launch_vgplain(*self.v, *self.d, self.zprime, *self._g, stream=self._stream)

    def _splain(self):
        launch_splain(*self.s, self.M[:21], *self.d, self.pre, *self._g, stream=self._stream)

    def forward_step(self):
        """One forward step (:2196-2411): velocity update, free-surface
        mirrors, strains, stress update, pressure."""
        self._vplain()
        self._mirrors()
        self._vgplain()
        self._splain()
        launch_compute_p(self.p, *self.s, self.p.numel(), self._stream)
        self.launches += 4

    def adjoint_step(self):
        """One adjoint step (:2424-2585): stress update, strains, mirrors, velocity update."""
        self._splain()
        self._vgplain()
        self._mirrors()
        self._vplain()
        self.launches += 3

    def image(self, it):
        """The images at snapshot step it (:2586-2611): g1 from the
        velocities, g2 the density gradient with the elastic volumes."""
        from . import launch_update_rho_gradient_rho

        s1, s3 = self.snaps[it]
        launch_update_gv(self.g1, s1, s3, self.v[0], self.v[2], *self._g, stream=self._stream)
        r = self.RADIUS
        d, M = self.d, self.M
        launch_update_rho_gradient_rho(self.g2, d[0], d[3], d[1], d[4], d[2], d[5], self.s[0], self.s[2], M[17],
                                       M[0], M[1], M[2], M[3], M[4], M[5], M[6], r, r + self.nx - 1, r,
                                       r + self.ny - 1, r, r + self.nz - 1, self.ldimx, self.ldimy, self.nx, self.ny,
                                       *self.d123, stream=self._stream)
        self.launches += 2

    def execute(self, niter, xcorr_step, press=500.0, adjoint=True):
        """simulator3SetUp::execute on this subdomain: the forward steps with
        velocity snapshots every xcorr_step steps, then (adjoint=True) the
        adjoint steps in reverse with the images at the snapshot steps."""
        r = self.RADIUS
        sl = (slice(r, r + self.nz), slice(r, r + self.ny), slice(r, r + self.nx))
        self.init_source(press)
        nxt = 0
        for it in range(niter):
            self.forward_step()
            if adjoint and it == nxt:
                self.snaps[it] = (self.v[0][sl].contiguous(), self.v[2][sl].contiguous())
                nxt += xcorr_step
        if not adjoint:
            return
        nxt -= xcorr_step
        for it in range(niter - 1, -1, -1):
            self.adjoint_step()
            if it == nxt:
                self.image(it)
                nxt -= xcorr_step
