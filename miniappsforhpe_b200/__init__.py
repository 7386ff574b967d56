"""B200-native TTI/VTI pseudo-acoustic RTM (the simulator2 / kernels path of
MiniAppsForHPE) -- Python bindings over the C ABI of ``libtti_b200.so``.

The compute path is the in-tree CUDA library built for sm_100a
(``python -m miniappsforhpe_b200.build``).  Importing this package never
falls back to anything else: if the library is missing, ``lib()`` raises.

Two levels, matching ``include/tti_capi.h``:

* per-kernel launchers with the reference launchers' argument lists
  (``launch_fwd_kernel2_drv`` ... ``launch_kernel_loop4``), taking device
  pointers (ints) or CUDA tensors;
* ``Simulator``, the ``simulator2SetUp`` call surface: model, source,
  receivers, forward and adjoint time loops, image readback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtti_b200.so")
RADIUS = 4

OK, EINVAL, ENOMEM, ELAUNCH, ETIMEOUT, ESTATE, ERANGE, ETOOBIG = range(8)


class TTIError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


_lib = None


def lib() -> C.CDLL:
    """The loaded ``libtti_b200.so``; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m miniappsforhpe_b200.build`")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


V, I, F, D, L64 = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_int64


class SimConfig(C.Structure):
    _fields_ = [
        ("nx", I), ("ny", I), ("nz", I),
        ("dx", D), ("dy", D), ("dz", D),
        ("dt", F), ("nt", I), ("xcorr_step", I), ("sponge_width", I),
        ("free_surface", I), ("fused", I), ("save_snapshots", I), ("snap_precision", I),
        ("checkpoint_every", I), ("use_graphs", I), ("scheme", I), ("wave_precision", I),
    ]


class TuneReport(C.Structure):
    _fields_ = [("bz", I * 3), ("ztop", I * 3), ("ms", F * 3), ("model_ms", F * 3), ("ncand", I)]


_SIGS = {
    "tti_launch_fwd_kernel2_drv": [V] * 9 + [I] * 6 + [F] * 3 + [I, I, I, V],
    "tti_launch_update_rho_fwd_main_loop_2_1": [V] * 30 + [I] * 8 + [F, D, D, D, I, I, I, I, I, V],
    "tti_launch_adj_kernel2_drv": [V] * 18 + [I] * 6 + [F] * 6 + [I, I, I, F, F, F, F, V],
    "tti_launch_update_adj_kernel_main_3": [V] * 13 + [I] * 8 + [F, D, D, D, I, I, I, I, I, V],
    "tti_launch_update_rho_gradient_rho": [V] * 17 + [I] * 10 + [D, D, D, I, I, V],
    "tti_launch_kernel_loop4_derivatives": [V] * 6 + [I, I, I, V],
    "tti_launch_update_Vp_gradient": [V] * 5 + [I] * 10 + [V],
    "tti_launch_finalize_Vp_gradient": [V, V] + [I] * 10 + [F, V],
    "tti_launch_kernel_loop2": [V] * 4 + [I] * 8 + [V] * 3 + [F, V],
    "tti_launch_kernel_loop4": [V, V, I, I, I, V],
    "tti_launch_init_cijs": [V] * 13 + [L64, V],
    "tti_launch_compute_pressure": [V, V, V, L64, V],
    "tti_launch_type1_fwd": [V] * 14 + [I] * 12 + [F, D, D, D, I, V, I, I, I],
    "tti_launch_type1_adj": [V] * 14 + [I] * 9 + [F, D, D, D, I, V, I, I],
    "tti_launch_type1_update_grad": [V] * 5 + [I] * 10 + [V],
    "tti_sim_create": [C.POINTER(SimConfig), C.POINTER(V)],
    "tti_sim_footprint_bytes": [C.POINTER(SimConfig), C.POINTER(L64)],
    "tti_sim_destroy": [V],
    "tti_sim_set_model": [V] * 8,
    "tti_sim_set_source": [V, I, I, I, V, I],
    "tti_sim_set_receivers": [V, I, V],
    "tti_sim_forward": [V, V, I],
    "tti_sim_adjoint": [V, V, I],
    "tti_sim_get_image": [V, V, V, I],
    "tti_sim_source_gradient": [V, V],
    "tti_sim_adjoint_observed": [V, V, I],
    "tti_sim_forward_begin": [V],
    "tti_sim_forward_step": [V, I],
    "tti_sim_get_traces": [V, V, I],
    "tti_sim_adjoint_begin": [V, V, I],
    "tti_sim_adjoint_step": [V, I],
    "tti_sim_image_step": [V, I],
    "tti_sim_adjoint_finish": [V],
    "tti_sim_sync": [V],
    "tti_sim_set_profiling": [V, I],
    "tti_sim_kernel_times": [V, V, V],
    "tti_sim_autotune": [V, I, C.POINTER(TuneReport)],
    "tti_tune_set": [I, I, I, I, I],
    "tti_tune_set_split": [I, I, I, I, I, I],
    "tti_tune_get_split": [I, I, I, I, V, V],
    "tti_selfcheck_bounded_wait": [D, V],
    "tti_tune_get": [I, I, I, I],
    "tti_sim_volume": [V, I, C.POINTER(V)],
    "tti_sim_read_volume": [V, I, V],
    "tti_sim_layout": [V, C.POINTER(I), C.POINTER(I), C.POINTER(I)],
    "tti_snap_create": [I, V, I, C.POINTER(V)],
    "tti_snap_create_tiered": [I, V, I, I, C.POINTER(V)],
    "tti_snap_destroy": [V],
    "tti_snap_lock_for_write": [V],
    "tti_snap_start_write": [V, V, V],
    "tti_snap_start_read": [V, V, V],
    "tti_snap_finish_read": [V, V],
    "tti_snap_count": [V],
    "tti_e3_launch_vgplain": [V] * 10 + [I] * 5 + [V],
    "tti_e3_launch_splain": [V] * 14 + [I] * 5 + [V],
    "tti_e3_launch_vplain": [V] * 11 + [I] * 5 + [V],
    "tti_e3_launch_mirror": [V, I, I, I, I, I, V],
    "tti_e3_launch_update_gv": [V] * 5 + [I] * 7 + [V],
    "tti_e3_launch_compute_p": [V] * 7 + [L64, V],
    "tti_e3_launch_init_model": [V] * 3 + [I] * 4 + [V],
}


def _declare(l: C.CDLL) -> None:
    for name, sig in _SIGS.items():
        f = getattr(l, name)
        f.argtypes = sig
        f.restype = I
    l.tti_status_string.argtypes = [I]
    l.tti_status_string.restype = C.c_char_p
    l.tti_version.argtypes = []
    l.tti_version.restype = C.c_char_p
    l.tti_sim_launch_count.argtypes = [V]
    l.tti_sim_launch_count.restype = L64
    l.tti_sim_stream.argtypes = [V]
    l.tti_sim_stream.restype = V


def status_string(status: int) -> str:
    return lib().tti_status_string(status).decode()


def version() -> str:
    return lib().tti_version().decode()


def _ptr(x):
    """Device pointer of a CUDA tensor, or an int pointer, or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("expected a CUDA tensor")
        if not x.is_contiguous():
            raise ValueError("expected a contiguous tensor")
        return x.data_ptr()
    raise TypeError(f"cannot take a device pointer of {type(x)}")


def _call(name: str, *args):
    f = getattr(lib(), name)
    conv = []
    for a, t in zip(args, f.argtypes):
        conv.append(_ptr(a) if t is V else a)
    rc = f(*conv)
    if rc != OK:
        raise TTIError(rc, name)
    return rc


# ---------------------------------------------------------------------------
# Per-kernel launchers (reference names, reference argument order).
def launch_fwd_kernel2_drv(field1, field2, Model11, dfield1dx, dfield1dy, dfield1dz, dfield2dx,
                           dfield2dy, dfield2dz, ixbeg, ixend, iybeg, iyend, izbeg, izend, invdx,
                           invdy, invdz, ldimx, ldimy, order=8, stream=None):
    """kernels/kernel_type2_fwd_drv.h:7-11."""
    _call("tti_launch_fwd_kernel2_drv", field1, field2, Model11, dfield1dx, dfield1dy, dfield1dz,
          dfield2dx, dfield2dy, dfield2dz, ixbeg, ixend, iybeg, iyend, izbeg, izend, invdx, invdy,
          invdz, ldimx, ldimy, order, stream)


def launch_update_rho_fwd_main_loop_2_1(field3, field4, field1_dx, field2_dx, field1_dy, field2_dy,
                                        field1_dz, field2_dz, field1, field2, irho, model1, model2,
                                        model3, model4, rx, ry, rz, ixbeg, ixend, iybeg, iyend,
                                        izbeg, izend, ldimx, ldimy, dt, dx, dy, dz, order=8,
                                        stream=None):
    """kernels/kernel_type2_fwd.h:6-14 (PML and sponge arguments fixed to off)."""
    _call("tti_launch_update_rho_fwd_main_loop_2_1", field3, field4, field1_dx, field2_dx, field1_dy,
          field2_dy, field1_dz, field2_dz, field1, field2, irho, model1, model2, model3, model4, rx,
          ry, rz, None, None, None, None, None, None, None, None, None, None, None, None, ixbeg,
          ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy, dt, dx, dy, dz, 0, order, 0, 0, 0, stream)


def launch_adj_kernel2_drv(dfield1dx, dfield2dx, dfield1dy, dfield2dy, dfield1dz, dfield2dz,
                           field3_rhs, field4_rhs, field1, field2, Model11, model1, model2, model3,
                           model4, model5, model6, model7, ixbeg, ixend, iybeg, iyend, izbeg, izend,
                           invdxx, invdyy, invdzz, invdxy, invdyz, invdzx, ldimx, ldimy, order, dt,
                           invdx, invdy, invdz, stream=None):
    """kernels/kernel_type2_grad_snap.h:7-12."""
    _call("tti_launch_adj_kernel2_drv", dfield1dx, dfield2dx, dfield1dy, dfield2dy, dfield1dz,
          dfield2dz, field3_rhs, field4_rhs, field1, field2, Model11, model1, model2, model3, model4,
          model5, model6, model7, ixbeg, ixend, iybeg, iyend, izbeg, izend, invdxx, invdyy, invdzz,
          invdxy, invdyz, invdzx, ldimx, ldimy, order, dt, invdx, invdy, invdz, stream)


def launch_type1_fwd(field3, field4, field1, field2, model1, model2, model3, model4, model5, model6,
                     model7, ABx, ABy, ABz, ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx_in, ldimy_in,
                     ldimz_in, ldimx_out, ldimy_out, ldimz_out, dt, dx, dy, dz, order=8, stream=None,
                     calc_snap=False, use_sponge=False, simple=False):
    """kernels/kernel_type1_gpu_fwd.h:6-9 (fwd_main_loop_2_1_inner_gpu::launch)."""
    _call("tti_launch_type1_fwd", field3, field4, field1, field2, model1, model2, model3, model4, model5,
          model6, model7, ABx, ABy, ABz, ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx_in, ldimy_in,
          ldimz_in, ldimx_out, ldimy_out, ldimz_out, dt, dx, dy, dz, order, stream, int(calc_snap),
          int(use_sponge), int(simple))


def launch_type1_adj(field3, field4, field1, field2, model1, model2, model3, model4, model5, model6,
                     model7, ABx, ABy, ABz, ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy, ldimz, dt,
                     dx, dy, dz, order=8, stream=None, use_sponge=False, simple=False):
    """kernels/kernel_type1_gpu_adj.h:6-9 (adj_main_loop_2_inner_gpu::launch)."""
    _call("tti_launch_type1_adj", field3, field4, field1, field2, model1, model2, model3, model4, model5,
          model6, model7, ABx, ABy, ABz, ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy, ldimz, dt, dx,
          dy, dz, order, stream, int(use_sponge), int(simple))


def launch_type1_update_grad(snap_x, snap_z, grad_Vp, adj_x, adj_z, ixbeg, ixend, iybeg, iyend, izbeg, izend,
                             snap_ldimx, snap_ldimy, ldimx, ldimy, stream=None):
    """kernels/kernel_type1_gpu_grad.h:4-7 (launch_update_grad_loop_kernel)."""
    _call("tti_launch_type1_update_grad", snap_x, snap_z, grad_Vp, adj_x, adj_z, ixbeg, ixend, iybeg, iyend,
          izbeg, izend, snap_ldimx, snap_ldimy, ldimx, ldimy, stream)


def launch_update_adj_kernel_main_3(field3, field4, field1_dx, field2_dx, field1_dy, field2_dy,
                                    field1_dz, field2_dz, field3_rhs, field4_rhs, ab_xx, ab_yy,
                                    ab_zz, ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy,
                                    dt, dx, dy, dz, order=8, sponge_active=False, stream=None):
    """kernels/kernel_type2_adj.h:8-14 (no PML)."""
    _call("tti_launch_update_adj_kernel_main_3", field3, field4, field1_dx, field2_dx, field1_dy,
          field2_dy, field1_dz, field2_dz, field3_rhs, field4_rhs, ab_xx, ab_yy, ab_zz, ixbeg, ixend,
          iybeg, iyend, izbeg, izend, ldimx, ldimy, dt, dx, dy, dz, 0, 0, 0, order,
          int(sponge_active), stream)


def launch_update_rho_gradient_rho(grad, fwd_field1_dx, fwd_field2_dx, fwd_field1_dy, fwd_field2_dy,
                                   fwd_field1_dz, fwd_field2_dz, field1, field2, irho, model1,
                                   model2, model3, model4, rx, ry, rz, ixbeg, ixend, iybeg, iyend,
                                   izbeg, izend, ldimx, ldimy, grad_ldimx, grad_ldimy, dx, dy, dz,
                                   order=8, simple_gradient=False, stream=None):
    """kernels/kernel_type2_grad.h:22-32."""
    _call("tti_launch_update_rho_gradient_rho", grad, fwd_field1_dx, fwd_field2_dx, fwd_field1_dy,
          fwd_field2_dy, fwd_field1_dz, fwd_field2_dz, field1, field2, irho, model1, model2, model3,
          model4, rx, ry, rz, ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy, grad_ldimx,
          grad_ldimy, dx, dy, dz, order, int(simple_gradient), stream)


def launch_kernel_loop4_derivatives(dfield1dx, dfield1dy, dfield1dz, dfield2dx, dfield2dy, dfield2dz,
                                    xtot, ytot, izbeg, stream=None):
    """kernels/kernel_type2_small.h:8-9 with the launch of kernel_type2.cu:278-293."""
    _call("tti_launch_kernel_loop4_derivatives", dfield1dx, dfield1dy, dfield1dz, dfield2dx,
          dfield2dy, dfield2dz, xtot, ytot, izbeg, stream)


def launch_update_Vp_gradient(snap_field3, snap_field4, grad_Vp, adj_field3, adj_field4, ixbeg,
                              ixend, iybeg, iyend, izbeg, izend, snx, sny, ldimx, ldimy, stream=None):
    """kernels/kernel_type2_small.h:11-14 with the launch of kernel_type2.cu:305-330."""
    _call("tti_launch_update_Vp_gradient", snap_field3, snap_field4, grad_Vp, adj_field3,
          adj_field4, ixbeg, ixend, iybeg, iyend, izbeg, izend, snx, sny, ldimx, ldimy, stream)


def launch_finalize_Vp_gradient(model3, grad_Vp, ixbeg, ixend, iybeg, iyend, izbeg, izend, snx, sny,
                                ldimx, ldimy, dt_xcorr, stream=None):
    """kernels/kernel_type2_small.h:16-18."""
    _call("tti_launch_finalize_Vp_gradient", model3, grad_Vp, ixbeg, ixend, iybeg, iyend, izbeg,
          izend, snx, sny, ldimx, ldimy, dt_xcorr, stream)


def launch_kernel_loop2(field1, field2, field3, field4, ldimx, ldimy, ixbeg, ixend, iybeg, iyend,
                        izbeg, izend, ab_x, ab_y, ab_z, dt, stream=None):
    """kernel_base::kernel_loop2_inner (kernels/kernel_base.cu:82-140)."""
    _call("tti_launch_kernel_loop2", field1, field2, field3, field4, ldimx, ldimy, ixbeg, ixend,
          iybeg, iyend, izbeg, izend, ab_x, ab_y, ab_z, dt, stream)


def launch_kernel_loop4(field1, field2, ldimx, ldimy, izbeg, stream=None):
    """kernel_base::kernel_loop4_inner (kernels/kernel_base.cu:142-187)."""
    _call("tti_launch_kernel_loop4", field1, field2, ldimx, ldimy, izbeg, stream)


def launch_init_cijs(vp, eps, delta, vs, theta, phi, model1, model2, model3, model4, model5, model6,
                     model7, n, stream=None):
    """simulator2SetUp.cu:10-29, per cell."""
    _call("tti_launch_init_cijs", vp, eps, delta, vs, theta, phi, model1, model2, model3, model4,
          model5, model6, model7, n, stream)


def launch_compute_pressure(pressure, field1, field2, n, stream=None):
    """simulator2SetUp.cu:31-42."""
    _call("tti_launch_compute_pressure", pressure, field1, field2, n, stream)


# ---------------------------------------------------------------------------
@dataclass
class Config:
    """Simulator configuration (tti_sim_config)."""

    nx: int
    ny: int
    nz: int
    dx: float = 10.0
    dy: float = 10.0
    dz: float = 10.0
    dt: float = 1e-3
    nt: int = 100
    xcorr_step: int = 4
    sponge_width: int = 0
    free_surface: bool = True
    fused: bool = True
    save_snapshots: bool = True
    snap_precision: str = "fp32"  # "fp32" | "fp16" | "bf16"
    checkpoint_every: int = 0  # >0: FP32 checkpoints every K steps, snapshots recomputed per segment
    use_graphs: bool = False  # capture each time loop into a CUDA graph
    scheme: int = 0  # 0: staggered variable-density operator; 1: centred constant-density (type1)
    wave_precision: str = "fp32"  # p/q rounded each step to "fp16" | "bf16" (per-field scale)

    def c_struct(self) -> SimConfig:
        prec = {"fp32": 0, "fp16": 1, "bf16": 2}[self.snap_precision]
        return SimConfig(self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, self.dt, self.nt,
                         self.xcorr_step, self.sponge_width, int(self.free_surface), int(self.fused),
                         int(self.save_snapshots), prec, int(self.checkpoint_every), int(self.use_graphs),
                         int(self.scheme), {"fp32": 0, "fp16": 1, "bf16": 2}[self.wave_precision])

    def footprint_bytes(self) -> int:
        """Device bytes ``tti_sim_create`` allocates for this configuration."""
        c = self.c_struct()
        out = L64()
        rc = lib().tti_sim_footprint_bytes(C.byref(c), C.byref(out))
        if rc != OK:
            raise TTIError(rc, "tti_sim_footprint_bytes")
        return out.value


VOLUMES = ("field1", "field2", "field3", "field4", "irho", "model1", "model2", "model3", "model4",
           "rx", "ry", "rz")


def _host_f32(a, n):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
    if a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def _host_out(a, n):
    """A caller's host output array: float32, C-contiguous, n values."""
    if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"] or a.size != n:
        raise ValueError(f"host output must be a C-contiguous float32 numpy array of {n} values")
    return a


class Simulator:
    """The ``simulator2SetUp`` call surface on one B200 (include/tti_capi.h section 2)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self._h = V()
        c = cfg.c_struct()
        rc = lib().tti_sim_create(C.byref(c), C.byref(self._h))
        if rc != OK:
            raise TTIError(rc, "tti_sim_create")
        self.n = cfg.nx * cfg.ny * cfg.nz
        lx, ly, lz = I(), I(), I()
        lib().tti_sim_layout(self._h, C.byref(lx), C.byref(ly), C.byref(lz))
        self.layout = (lx.value, ly.value, lz.value)
        self.nrec = 0

    def close(self):
        if self._h:
            lib().tti_sim_destroy(self._h)
            self._h = V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chk(self, rc, what):
        if rc != OK:
            raise TTIError(rc, what)

    def set_model(self, vp, eps=None, delta=None, vs=None, theta=None, phi=None, rho=None):
        arrs = [_host_f32(a, self.n) for a in (vp, eps, delta, vs, theta, phi, rho)]
        self._keep = arrs
        ptrs = [None if a is None else a.ctypes.data_as(V) for a in arrs]
        self._chk(lib().tti_sim_set_model(self._h, *ptrs), "tti_sim_set_model")

    def set_source(self, ix, iy, iz, wavelet):
        w = _host_f32(wavelet, self.cfg.nt)
        self._chk(lib().tti_sim_set_source(self._h, ix, iy, iz, w.ctypes.data_as(V), self.cfg.nt),
                  "tti_sim_set_source")

    def set_receivers(self, ixyz):
        r = np.ascontiguousarray(ixyz, dtype=np.int32).reshape(-1, 3)
        self._chk(lib().tti_sim_set_receivers(self._h, len(r), r.ctypes.data_as(V)),
                  "tti_sim_set_receivers")
        self.nrec = len(r)

    def forward(self, traces_out=None):
        """Forward loop; returns the (nt, nrec) pressure traces as numpy, or
        writes them into ``traces_out``: a CUDA tensor, or a C-contiguous
        float32 numpy array of nt*nrec values (host memory, pinned or not)."""
        if traces_out is not None and hasattr(traces_out, "data_ptr"):
            self._chk(lib().tti_sim_forward(self._h, _ptr(traces_out), 1), "tti_sim_forward")
            return traces_out
        out = np.zeros((self.cfg.nt, self.nrec), np.float32) if traces_out is None else _host_out(
            traces_out, self.cfg.nt * self.nrec)
        p = out.ctypes.data_as(V) if self.nrec else None
        self._chk(lib().tti_sim_forward(self._h, p, 0), "tti_sim_forward")
        return out

    def adjoint(self, residual):
        """Adjoint loop driven by (nt, nrec) residual traces (numpy or CUDA tensor)."""
        if hasattr(residual, "data_ptr"):
            self._chk(lib().tti_sim_adjoint(self._h, _ptr(residual), 1), "tti_sim_adjoint")
            return
        r = np.ascontiguousarray(residual, np.float32).reshape(self.cfg.nt, self.nrec)
        self._chk(lib().tti_sim_adjoint(self._h, r.ctypes.data_as(V), 0), "tti_sim_adjoint")

    def adjoint_observed(self, observed):
        """Adjoint loop with residual = last synthetic traces - observed (numpy or CUDA tensor)."""
        if hasattr(observed, "data_ptr"):
            self._chk(lib().tti_sim_adjoint_observed(self._h, _ptr(observed), 1), "tti_sim_adjoint_observed")
            return
        o = np.ascontiguousarray(observed, np.float32).reshape(self.cfg.nt, self.nrec)
        self._chk(lib().tti_sim_adjoint_observed(self._h, o.ctypes.data_as(V), 0), "tti_sim_adjoint_observed")

    # Step-level calls (tti_sim_forward_begin ... tti_sim_adjoint_finish): the
    # same kernels as forward()/adjoint(), one time step per call.
    def forward_begin(self):
        self._chk(lib().tti_sim_forward_begin(self._h), "tti_sim_forward_begin")

    def forward_step(self, n: int):
        self._chk(lib().tti_sim_forward_step(self._h, int(n)), "tti_sim_forward_step")

    def traces(self) -> np.ndarray:
        out = np.zeros((self.cfg.nt, self.nrec), np.float32)
        if self.nrec:
            self._chk(lib().tti_sim_get_traces(self._h, out.ctypes.data_as(V), 0), "tti_sim_get_traces")
        return out

    def adjoint_begin(self, residual=None):
        if residual is None:
            self._chk(lib().tti_sim_adjoint_begin(self._h, None, 0), "tti_sim_adjoint_begin")
            return
        self._resid = np.ascontiguousarray(residual, np.float32).reshape(self.cfg.nt, self.nrec)
        self._chk(lib().tti_sim_adjoint_begin(self._h, self._resid.ctypes.data_as(V), 0), "tti_sim_adjoint_begin")

    def adjoint_step(self, n: int):
        self._chk(lib().tti_sim_adjoint_step(self._h, int(n)), "tti_sim_adjoint_step")

    def image_step(self, n: int):
        self._chk(lib().tti_sim_image_step(self._h, int(n)), "tti_sim_image_step")

    def adjoint_finish(self):
        self._chk(lib().tti_sim_adjoint_finish(self._h), "tti_sim_adjoint_finish")

    def set_profiling(self, enable: bool):
        self._chk(lib().tti_sim_set_profiling(self._h, int(enable)), "tti_sim_set_profiling")

    def kernel_times(self):
        """{'forward'|'adjoint'|'imaging': (total_ms, launches)} since profiling was enabled."""
        ms = (C.c_double * 3)()
        n = (C.c_int64 * 3)()
        self._chk(lib().tti_sim_kernel_times(self._h, C.cast(ms, V), C.cast(n, V)), "tti_sim_kernel_times")
        return {k: (ms[i], n[i]) for i, k in enumerate(("forward", "adjoint", "imaging"))}

    def autotune(self, reps: int = 3) -> dict:
        """Time every z-chunk candidate of the fused kernels on this grid and
        record the fastest (include/tti_capi.h, tti_sim_autotune).  With the
        centred scheme the 'forward' and 'adjoint' entries are its type1
        kernels."""
        r = TuneReport()
        self._chk(lib().tti_sim_autotune(self._h, int(reps), C.byref(r)), "tti_sim_autotune")
        kinds = ("forward", "adjoint", "imaging")
        return {k: {"bz": r.bz[i], "ztop": r.ztop[i], "ms": r.ms[i], "model_ms": r.model_ms[i]}
                for i, k in enumerate(kinds) if r.bz[i] > 0} | {"candidates": r.ncand}

    def image(self, out_vp=None, out_rho=None):
        """(grad_vp, grad_rho), each (nz, ny, nx): new numpy arrays, or the
        given outputs (CUDA tensors, or C-contiguous float32 numpy arrays)."""
        if out_vp is not None and hasattr(out_vp, "data_ptr"):
            self._chk(lib().tti_sim_get_image(self._h, _ptr(out_vp), _ptr(out_rho), 1),
                      "tti_sim_get_image")
            return out_vp, out_rho
        c = self.cfg
        n = c.nx * c.ny * c.nz
        gv = np.zeros((c.nz, c.ny, c.nx), np.float32) if out_vp is None else _host_out(out_vp, n)
        gr = np.zeros((c.nz, c.ny, c.nx), np.float32) if out_rho is None else _host_out(out_rho, n)
        self._chk(lib().tti_sim_get_image(self._h, gv.ctypes.data_as(V), gr.ctypes.data_as(V), 0),
                  "tti_sim_get_image")
        return gv, gr

    def source_gradient(self) -> np.ndarray:
        """dt*(adjoint p+q) at the source cell per step of the last adjoint run."""
        out = np.zeros(self.cfg.nt, np.float32)
        self._chk(lib().tti_sim_source_gradient(self._h, out.ctypes.data_as(V)), "tti_sim_source_gradient")
        return out

    def volume(self, name: str) -> np.ndarray:
        """Host copy of an internal halo'd volume, shape (ldimz, ldimy, ldimx)."""
        lx, ly, lz = self.layout
        out = np.zeros((lz, ly, lx), np.float32)
        self._chk(lib().tti_sim_read_volume(self._h, VOLUMES.index(name), out.ctypes.data_as(V)),
                  "tti_sim_read_volume")
        return out

    def launch_count(self) -> int:
        return int(lib().tti_sim_launch_count(self._h))

    def stream_handle(self) -> int:
        return int(lib().tti_sim_stream(self._h) or 0)


TUNE_KINDS = ("forward", "adjoint", "imaging", "type1_forward", "type1_adjoint")


def tune_set(nx: int, ny: int, nz: int, kind: str, bz: int, ztop: int = 0) -> None:
    """Record (bz > 0) or clear (bz = 0) the work split of a fused kernel
    kind (TUNE_KINDS) on an nx*ny*nz grid (current device); ztop > 0 is a
    top/bottom split (tti_tune_set_split)."""
    k = TUNE_KINDS.index(kind)
    rc = lib().tti_tune_set_split(nx, ny, nz, k, bz, ztop)
    if rc != OK:
        raise TTIError(rc, "tti_tune_set_split")


def tune_get(nx: int, ny: int, nz: int, kind: str) -> int:
    k = TUNE_KINDS.index(kind)
    v = lib().tti_tune_get(nx, ny, nz, k)
    if v < 0:
        raise TTIError(-v, "tti_tune_get")
    return v


def tune_get_split(nx: int, ny: int, nz: int, kind: str) -> tuple:
    """(bz, ztop) of the split in effect for a kernel kind on this grid."""
    bz, zt = I(), I()
    rc = lib().tti_tune_get_split(nx, ny, nz, TUNE_KINDS.index(kind), C.byref(bz), C.byref(zt))
    if rc != OK:
        raise TTIError(rc, "tti_tune_get_split")
    return bz.value, zt.value


class SnapshotStore:
    """LIFO snapshot store with the rtm_snap call sequence: ``capacity``
    slots in HBM, then ``host_capacity`` slots in pinned host memory."""

    def __init__(self, nelems, capacity, host_capacity=0):
        arr = (C.c_int64 * len(nelems))(*nelems)
        self.nvol = len(nelems)
        self._h = V()
        rc = lib().tti_snap_create_tiered(len(nelems), C.cast(arr, V), capacity, host_capacity,
                                          C.byref(self._h))
        if rc != OK:
            raise TTIError(rc, "tti_snap_create")

    def _vols(self, vols):
        a = (C.c_void_p * self.nvol)(*[_ptr(v) for v in vols])
        return C.cast(a, V)

    def lock_for_write(self):
        _chk(lib().tti_snap_lock_for_write(self._h), "lock_for_write")

    def start_write(self, vols, stream=None):
        _chk(lib().tti_snap_start_write(self._h, self._vols(vols), stream), "start_write")

    def start_read(self, vols, stream=None):
        _chk(lib().tti_snap_start_read(self._h, self._vols(vols), stream), "start_read")

    def finish_read(self, stream=None):
        _chk(lib().tti_snap_finish_read(self._h, stream), "finish_read")

    def count(self) -> int:
        return int(lib().tti_snap_count(self._h))

    def close(self):
        if self._h:
            lib().tti_snap_destroy(self._h)
            self._h = V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _chk(rc, what):
    if rc != OK:
        raise TTIError(rc, what)
