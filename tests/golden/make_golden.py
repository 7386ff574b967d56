"""Golden vectors of the reference's own TTI kernels, and the same cases run
through the oracle and through the product.

The reference has no tests and ships no fixtures for this path, so the
golden vectors are produced here: each case builds seeded inputs in the
reference layout and runs the reference kernels (compiled unmodified from
the reference sources for sm_100a into oracle/_ref/libref_tti.so, see
oracle/Makefile) on a B200.  ``python tests/golden/make_golden.py OUT_DIR``
writes ``reference_kernels.npz``; the committed copy lives next to this file.

``oracle_outputs(case)`` (CPU) and ``product_outputs(case)`` (GPU) run the
same cases through the C oracle and through libtti_b200.so.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import DKEYS, Layout, Oracle, REF_LIB_PATH  # noqa: E402

DX, DY, DZ = 10.0, 12.5, 8.0
DT = 1.0e-3


def _lay():
    return Layout(20, 16, 12)


CASES = [
    dict(name="fwd_drv", seed=101),
    dict(name="fwd_update_tti", seed=102, tti=True),
    dict(name="fwd_update_vti", seed=103, tti=False),
    dict(name="adj_drv_tti", seed=104, tti=True),
    dict(name="adj_update", seed=105, sponge=False),
    dict(name="adj_update_sponge", seed=106, sponge=True),
    dict(name="rho_grad", seed=107),
    dict(name="loop2", seed=108),
    dict(name="loop4", seed=109),
    dict(name="loop4_drv", seed=110),
    dict(name="vp_grad", seed=111),
    dict(name="steps", seed=112, nsteps=24),
]


def make_inputs(case):
    """Seeded inputs; every array is float32 and C-contiguous."""
    lay = _lay()
    rng = np.random.default_rng(case["seed"])
    sh = lay.shape
    tti = case.get("tti", True)
    vp = rng.uniform(1800.0, 3200.0, sh)
    eps = rng.uniform(0.0, 0.25, sh)
    delta = eps * rng.uniform(0.0, 0.6, sh)
    vs = rng.uniform(0.0, 400.0, sh)
    theta = rng.uniform(0.0, 0.8, sh) if tti else np.zeros(sh)
    phi = rng.uniform(0.0, 3.0, sh) if tti else np.zeros(sh)
    m = dict(m1=vp * vp * (1 + 2 * eps),
             m2=np.sqrt((vp * vp - vs * vs) * (vp * vp * (1 + 2 * delta) - vs * vs)),
             m3=vp * vp, m4=vs * vs, rx=np.sin(theta) * np.cos(phi), ry=np.sin(theta) * np.sin(phi),
             rz=np.cos(theta), irho=1.0 / rng.uniform(1.0, 2.5, sh))
    f = lambda s=1.0: (s * rng.standard_normal(sh)).astype(np.float32)  # noqa: E731
    inp = {k: np.ascontiguousarray(v, np.float32) for k, v in m.items()}
    inp.update(f1=f(), f2=f(), f3=f(), f4=f(), rhs3=f(1e6), rhs4=f(1e6))
    inp.update({k: f(0.1) for k in DKEYS})
    inp.update({"fd" + k[1:]: f(0.1) for k in DKEYS})
    n = lay.nx * lay.ny * lay.nz
    inp.update(snap3=(rng.standard_normal(n)).astype(np.float32),
               snap4=(rng.standard_normal(n)).astype(np.float32),
               grad=(rng.standard_normal(n)).astype(np.float32))
    act = case.get("sponge", True)
    for ax, nn in (("abx", lay.ldimx), ("aby", lay.ldimy), ("abz", lay.ldimz)):
        ab = np.ones((nn, 2), np.float32)
        if act:
            ab[:] = rng.uniform(0.9, 1.0, (nn, 2))
        inp[ax] = np.ascontiguousarray(ab.reshape(-1))
    if case["name"] == "steps":
        for k in ("f1", "f2", "f3", "f4"):
            inp[k] = np.zeros(sh, np.float32)
        inp["wavelet"] = np.sin(np.arange(case["nsteps"]) * 0.4).astype(np.float32) * 1e3
        inp["src"] = np.int64(lay.index(9, 8, 5))
        inp["rec"] = np.array([lay.index(ix, iy, 2) for iy in range(lay.ny) for ix in range(lay.nx)],
                              np.int64)
    return lay, inp


def _d(inp, prefix="d"):
    return {k: inp[prefix + k[1:]].copy() for k in DKEYS}


def oracle_outputs(case):
    o = Oracle("f32")
    lay, inp = make_inputs(case)
    h = (DX, DY, DZ)
    invd = (np.float32(1 / DX), np.float32(1 / DY), np.float32(1 / DZ))
    name = case["name"]
    m = {k: inp[k] for k in ("irho", "m1", "m2", "m3", "m4", "rx", "ry", "rz")}
    out = {}
    if name == "fwd_drv":
        d = {k: lay.zeros() for k in DKEYS}
        o.fwd_drv(lay, inp["f1"], inp["f2"], inp["irho"], d, invd)
        out.update(d)
    elif name.startswith("fwd_update"):
        f3, f4 = inp["f3"].copy(), inp["f4"].copy()
        o.fwd_update(lay, f3, f4, _d(inp), inp["f1"], inp["f2"], m, DT, h)
        out.update(f3=f3, f4=f4)
    elif name.startswith("adj_drv"):
        d = {k: lay.zeros() for k in DKEYS}
        r3, r4 = lay.zeros(), lay.zeros()
        o.adj_drv(lay, d, r3, r4, inp["f1"], inp["f2"], m, h)
        out.update(d)
        out.update(rhs3=r3, rhs4=r4)
    elif name.startswith("adj_update"):
        f3, f4 = inp["f3"].copy(), inp["f4"].copy()
        o.adj_update(lay, f3, f4, _d(inp), inp["rhs3"], inp["rhs4"], inp["abx"], inp["aby"], inp["abz"],
                     DT, h, case.get("sponge", False))
        out.update(f3=f3, f4=f4)
    elif name == "rho_grad":
        g = inp["grad"].copy()
        o.rho_gradient(lay, g, _d(inp, "fd"), inp["f1"], inp["f2"], m, h, lay.nx, lay.ny)
        out.update(grad=g)
    elif name == "loop2":
        f1, f2 = inp["f1"].copy(), inp["f2"].copy()
        o.loop2(lay, f1, f2, inp["f3"], inp["f4"], inp["abx"], inp["aby"], inp["abz"], DT)
        out.update(f1=f1, f2=f2)
    elif name == "loop4":
        f1, f2 = inp["f1"].copy(), inp["f2"].copy()
        o.loop4(lay, f1, f2)
        out.update(f1=f1, f2=f2)
    elif name == "loop4_drv":
        d = _d(inp)
        o.loop4_derivatives(lay, d)
        out.update(d)
    elif name == "vp_grad":
        g = inp["grad"].copy()
        o.update_vp_gradient(lay, inp["snap3"], inp["snap4"], g, inp["f3"], inp["f4"])
        out.update(grad=g)
    elif name == "steps":
        out.update(_oracle_steps(o, lay, inp, m, case))
    return out


def _oracle_steps(o, lay, inp, m, case):
    from oracle import new_state

    st = new_state(lay)
    g = o.grid(lay, DT, (DX, DY, DZ), free_surface=True, sponge_active=True)
    ab = (inp["abx"], inp["aby"], inp["abz"])
    nrec = len(inp["rec"])
    tr = np.zeros((case["nsteps"], nrec), np.float32)
    for n in range(case["nsteps"]):
        row = np.zeros(nrec, np.float32)
        o.fwd_step(g, st, m, ab, int(inp["src"]), float(inp["wavelet"][n]), inp["rec"], row)
        tr[n] = row
    out = {"traces": tr}
    out.update({k: st[k].copy() for k in ("f1", "f2", "f3", "f4")})
    for n in range(case["nsteps"] - 1, -1, -1):
        o.adj_step(g, st, m, ab, inp["rec"], tr[n].copy())
    out.update({"adj_" + k: st[k].copy() for k in ("f1", "f2", "f3", "f4")})
    return out


# ---------------------------------------------------------------------------
# GPU runners (reference kernels / product), via torch device memory.
def _dev(inp):
    import torch

    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in inp.items()
            if isinstance(v, np.ndarray) and v.dtype == np.float32}


def _ref_lib():
    if not os.path.exists(REF_LIB_PATH):
        raise FileNotFoundError(REF_LIB_PATH)
    lib = C.CDLL(REF_LIB_PATH)
    for name in ("ref_fwd_drv", "ref_fwd_update", "ref_adj_drv", "ref_adj_update", "ref_rho_gradient",
                 "ref_loop4_derivatives", "ref_update_vp_gradient", "ref_loop2", "ref_loop4", "ref_sync"):
        getattr(lib, name).restype = C.c_int
    return lib


def _p(t):
    return C.c_void_p(t.data_ptr())


def reference_outputs(case):
    """Run one case through the reference's own kernels (GPU)."""
    lib = _ref_lib()
    return _gpu_run(case, _RefKernels(lib))


def product_outputs(case):
    """Run one case through libtti_b200.so's per-kernel launchers (GPU)."""
    return _gpu_run(case, _ProductKernels())


class _RefKernels:
    def __init__(self, lib):
        self.lib = lib

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} returned {rc}")

    def fwd_drv(self, lay, t, d):
        r = lay.ranges
        self._ok(self.lib.ref_fwd_drv(_p(t["f1"]), _p(t["f2"]), _p(t["irho"]), *[_p(d[k]) for k in DKEYS], *r,
                                      C.c_float(1 / DX), C.c_float(1 / DY), C.c_float(1 / DZ), lay.ldimx,
                                      lay.ldimy), "ref_fwd_drv")

    def fwd_update(self, lay, t, d, f3, f4):
        self._ok(self.lib.ref_fwd_update(
            _p(f3), _p(f4), _p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]), _p(d["d2y"]), _p(d["d1z"]),
            _p(d["d2z"]), _p(t["f1"]), _p(t["f2"]), _p(t["irho"]), _p(t["m1"]), _p(t["m2"]), _p(t["m3"]),
            _p(t["m4"]), _p(t["rx"]), _p(t["ry"]), _p(t["rz"]), *lay.ranges, lay.ldimx, lay.ldimy,
            C.c_float(DT), C.c_double(DX), C.c_double(DY), C.c_double(DZ)), "ref_fwd_update")

    def adj_drv(self, lay, t, d, r3, r4):
        self._ok(self.lib.ref_adj_drv(
            _p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]), _p(d["d2y"]), _p(d["d1z"]), _p(d["d2z"]), _p(r3),
            _p(r4), _p(t["f1"]), _p(t["f2"]), _p(t["irho"]), _p(t["m1"]), _p(t["m2"]), _p(t["m3"]),
            _p(t["m4"]), _p(t["rx"]), _p(t["ry"]), _p(t["rz"]), *lay.ranges, C.c_double(DX),
            C.c_double(DY), C.c_double(DZ), lay.ldimx, lay.ldimy, C.c_float(DT)), "ref_adj_drv")

    def adj_update(self, lay, t, d, r3, r4, f3, f4, sponge):
        self._ok(self.lib.ref_adj_update(
            _p(f3), _p(f4), _p(d["d1x"]), _p(d["d2x"]), _p(d["d1y"]), _p(d["d2y"]), _p(d["d1z"]),
            _p(d["d2z"]), _p(r3), _p(r4), _p(t["abx"]), _p(t["aby"]), _p(t["abz"]), *lay.ranges, lay.ldimx,
            lay.ldimy, C.c_float(DT), C.c_double(DX), C.c_double(DY), C.c_double(DZ), int(sponge)),
            "ref_adj_update")

    def rho_grad(self, lay, t, fd, g):
        self._ok(self.lib.ref_rho_gradient(
            _p(g), _p(fd["d1x"]), _p(fd["d2x"]), _p(fd["d1y"]), _p(fd["d2y"]), _p(fd["d1z"]), _p(fd["d2z"]),
            _p(t["f1"]), _p(t["f2"]), _p(t["irho"]), _p(t["m1"]), _p(t["m2"]), _p(t["m3"]), _p(t["m4"]),
            _p(t["rx"]), _p(t["ry"]), _p(t["rz"]), *lay.ranges, lay.ldimx, lay.ldimy, lay.nx, lay.ny,
            C.c_double(DX), C.c_double(DY), C.c_double(DZ), 0), "ref_rho_gradient")

    def loop2(self, lay, t, f1, f2, f3, f4):
        self._ok(self.lib.ref_loop2(_p(f1), _p(f2), _p(f3), _p(f4), lay.ldimx, lay.ldimy, *lay.ranges,
                                    _p(t["abx"]), _p(t["aby"]), _p(t["abz"]), C.c_float(DT)), "ref_loop2")

    def loop4(self, lay, f1, f2):
        self._ok(self.lib.ref_loop4(_p(f1), _p(f2), lay.ldimx, lay.ldimy, 4), "ref_loop4")

    def loop4_drv(self, lay, d):
        self._ok(self.lib.ref_loop4_derivatives(*[_p(d[k]) for k in DKEYS], lay.ldimx, lay.ldimy, 4),
                 "ref_loop4_derivatives")

    def vp_grad(self, lay, t, g):
        self._ok(self.lib.ref_update_vp_gradient(_p(t["snap3"]), _p(t["snap4"]), _p(g), _p(t["f3"]),
                                                 _p(t["f4"]), *lay.ranges, lay.nx, lay.ny, lay.ldimx,
                                                 lay.ldimy), "ref_update_vp_gradient")

    def sync(self):
        self._ok(self.lib.ref_sync(), "ref_sync")


class _ProductKernels:
    def __init__(self):
        import miniappsforhpe_b200 as P

        self.P = P

    def fwd_drv(self, lay, t, d):
        self.P.launch_fwd_kernel2_drv(t["f1"], t["f2"], t["irho"], *[d[k] for k in DKEYS], *lay.ranges,
                                      1 / DX, 1 / DY, 1 / DZ, lay.ldimx, lay.ldimy)

    def fwd_update(self, lay, t, d, f3, f4):
        self.P.launch_update_rho_fwd_main_loop_2_1(
            f3, f4, d["d1x"], d["d2x"], d["d1y"], d["d2y"], d["d1z"], d["d2z"], t["f1"], t["f2"], t["irho"],
            t["m1"], t["m2"], t["m3"], t["m4"], t["rx"], t["ry"], t["rz"], *lay.ranges, lay.ldimx, lay.ldimy,
            DT, DX, DY, DZ)

    def adj_drv(self, lay, t, d, r3, r4):
        self.P.launch_adj_kernel2_drv(
            d["d1x"], d["d2x"], d["d1y"], d["d2y"], d["d1z"], d["d2z"], r3, r4, t["f1"], t["f2"], t["irho"],
            t["m1"], t["m2"], t["m3"], t["m4"], t["rx"], t["ry"], t["rz"], *lay.ranges, 1 / DX ** 2,
            1 / DY ** 2, 1 / DZ ** 2, 1 / (4 * DX * DY), 1 / (4 * DY * DZ), 1 / (4 * DX * DZ), lay.ldimx,
            lay.ldimy, 8, DT, 1 / DX, 1 / DY, 1 / DZ)

    def adj_update(self, lay, t, d, r3, r4, f3, f4, sponge):
        self.P.launch_update_adj_kernel_main_3(
            f3, f4, d["d1x"], d["d2x"], d["d1y"], d["d2y"], d["d1z"], d["d2z"], r3, r4, t["abx"], t["aby"],
            t["abz"], *lay.ranges, lay.ldimx, lay.ldimy, DT, DX, DY, DZ, sponge_active=sponge)

    def rho_grad(self, lay, t, fd, g):
        self.P.launch_update_rho_gradient_rho(
            g, fd["d1x"], fd["d2x"], fd["d1y"], fd["d2y"], fd["d1z"], fd["d2z"], t["f1"], t["f2"], t["irho"],
            t["m1"], t["m2"], t["m3"], t["m4"], t["rx"], t["ry"], t["rz"], *lay.ranges, lay.ldimx, lay.ldimy,
            lay.nx, lay.ny, DX, DY, DZ)

    def loop2(self, lay, t, f1, f2, f3, f4):
        self.P.launch_kernel_loop2(f1, f2, f3, f4, lay.ldimx, lay.ldimy, *lay.ranges, t["abx"], t["aby"],
                                   t["abz"], DT)

    def loop4(self, lay, f1, f2):
        self.P.launch_kernel_loop4(f1, f2, lay.ldimx, lay.ldimy, 4)

    def loop4_drv(self, lay, d):
        self.P.launch_kernel_loop4_derivatives(*[d[k] for k in DKEYS], lay.ldimx, lay.ldimy, 4)

    def vp_grad(self, lay, t, g):
        self.P.launch_update_Vp_gradient(t["snap3"], t["snap4"], g, t["f3"], t["f4"], *lay.ranges, lay.nx,
                                         lay.ny, lay.ldimx, lay.ldimy)

    def sync(self):
        import torch

        torch.cuda.synchronize()


def _gpu_run(case, K):
    import torch

    lay, inp = make_inputs(case)
    t = _dev(inp)
    name = case["name"]
    d = {k: t[k].clone() for k in DKEYS}
    fd = {k: t["fd" + k[1:]].clone() for k in DKEYS}
    zeros = lambda: torch.zeros(lay.shape, dtype=torch.float32, device="cuda")  # noqa: E731
    out = {}
    if name == "fwd_drv":
        dz = {k: zeros() for k in DKEYS}
        K.fwd_drv(lay, t, dz)
        out.update(dz)
    elif name.startswith("fwd_update"):
        f3, f4 = t["f3"].clone(), t["f4"].clone()
        K.fwd_update(lay, t, d, f3, f4)
        out.update(f3=f3, f4=f4)
    elif name.startswith("adj_drv"):
        dz = {k: zeros() for k in DKEYS}
        r3, r4 = zeros(), zeros()
        K.adj_drv(lay, t, dz, r3, r4)
        out.update(dz)
        out.update(rhs3=r3, rhs4=r4)
    elif name.startswith("adj_update"):
        f3, f4 = t["f3"].clone(), t["f4"].clone()
        K.adj_update(lay, t, d, t["rhs3"], t["rhs4"], f3, f4, case.get("sponge", False))
        out.update(f3=f3, f4=f4)
    elif name == "rho_grad":
        g = t["grad"].clone()
        K.rho_grad(lay, t, fd, g)
        out.update(grad=g)
    elif name == "loop2":
        f1, f2 = t["f1"].clone(), t["f2"].clone()
        K.loop2(lay, t, f1, f2, t["f3"], t["f4"])
        out.update(f1=f1, f2=f2)
    elif name == "loop4":
        f1, f2 = t["f1"].clone(), t["f2"].clone()
        K.loop4(lay, f1, f2)
        out.update(f1=f1, f2=f2)
    elif name == "loop4_drv":
        K.loop4_drv(lay, d)
        out.update(d)
    elif name == "vp_grad":
        g = t["grad"].clone()
        K.vp_grad(lay, t, g)
        out.update(grad=g)
    elif name == "steps":
        out.update(_gpu_steps(K, lay, t, inp, case))
    K.sync()
    return {k: v.cpu().numpy() if hasattr(v, "cpu") else v for k, v in out.items()}


def _gpu_steps(K, lay, t, inp, case):
    """The reference step order (simulator2SetUp.cu:530-651 forward,
    :654-720 adjoint) with the point source and pressure receivers of this
    build applied between kernels, exactly as in the oracle's step drivers."""
    import torch

    f1, f2, f3, f4 = (torch.zeros(lay.shape, dtype=torch.float32, device="cuda") for _ in range(4))
    d = {k: torch.zeros(lay.shape, dtype=torch.float32, device="cuda") for k in DKEYS}
    r3 = torch.zeros_like(f1)
    r4 = torch.zeros_like(f1)
    src = int(inp["src"])
    rec = torch.from_numpy(inp["rec"]).cuda()
    nt = case["nsteps"]
    traces = torch.zeros((nt, len(inp["rec"])), dtype=torch.float32, device="cuda")
    dtf = np.float32(DT)
    flat = lambda v: v.view(-1)  # noqa: E731
    for n in range(nt):
        K.loop2(lay, t, f1, f2, f3, f4)
        K.loop4(lay, f1, f2)
        K.fwd_drv(lay, {**t, "f1": f1, "f2": f2}, d)
        K.loop4_drv(lay, d)
        K.fwd_update(lay, {**t, "f1": f1, "f2": f2}, d, f3, f4)
        amp = np.float32(inp["wavelet"][n]) * dtf
        flat(f3)[src] += float(amp)
        flat(f4)[src] += float(amp)
        traces[n] = -(2 * flat(f1)[rec] + flat(f2)[rec]) / 3
    out = {"traces": traces.clone(), "f1": f1.clone(), "f2": f2.clone(), "f3": f3.clone(), "f4": f4.clone()}
    for n in range(nt - 1, -1, -1):
        res = traces[n]
        flat(f3)[rec] += np.float32(-2.0 / 3.0) * res
        flat(f4)[rec] += np.float32(-1.0 / 3.0) * res
        K.adj_drv(lay, {**t, "f1": f1, "f2": f2}, d, r3, r4)
        K.loop4_drv(lay, d)
        K.adj_update(lay, t, d, r3, r4, f3, f4, True)
        K.loop2(lay, t, f1, f2, f3, f4)
        K.loop4(lay, f1, f2)
    out.update(adj_f1=f1, adj_f2=f2, adj_f3=f3, adj_f4=f4)
    return out


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    res = {}
    for case in CASES:
        for k, v in reference_outputs(case).items():
            res[f"{case['name']}/{k}"] = v.astype(np.float32)
    path = os.path.join(out_dir, "reference_kernels.npz")
    np.savez_compressed(path, **res)
    print(path, len(res), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
