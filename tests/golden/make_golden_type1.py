"""Golden vectors of the reference's own type1 kernels
(kernels/kernel_type1_gpu_{fwd,adj,grad}.cu, compiled unmodified from the
reference sources into oracle/_ref/libref_tti.so).

``python tests/golden/make_golden_type1.py OUT_DIR`` runs the seeded cases
of ``CASES`` on a B200 and writes ``reference_type1.npz`` (per case the
interior of the two output volumes, and the Vp image of the imaging case;
the kernels write nothing outside the interior); the committed copy
lives next to this file.  ``case_inputs`` rebuilds the same inputs on the
CPU, so the oracle can be checked against the file without a GPU."""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import Layout  # noqa: E402
from tests.helpers import random_field, random_model, sponge_ab  # noqa: E402

H = (10.0, 12.5, 8.0)
DT = 1e-3
MKEYS = ("m1", "m2", "m3", "m4", "rx", "ry", "rz")
# (name, operator, forward mode: 0 accumulate / 1 sponge / 2 calc_snap, adjoint sponge, seed)
CASES = [("fwd_accumulate", "fwd", 0, False, 31), ("fwd_sponge", "fwd", 1, False, 32),
         ("fwd_calc_snap", "fwd", 2, False, 33), ("adj", "adj", 0, False, 34), ("adj_sponge", "adj", 0, True, 35),
         ("grad", "grad", 0, False, 36)]


def case_inputs(seed, nx=24, ny=20, nz=16):
    lay = Layout(nx, ny, nz)
    rng = np.random.default_rng(seed)
    m = random_model(lay, rng, tti=True)
    ab = [sponge_ab(n, rng) for n in (lay.ldimx, lay.ldimy, lay.ldimz)]
    f = [random_field(lay, rng) for _ in range(4)]
    n = lay.nx * lay.ny * lay.nz
    g = [rng.standard_normal(n).astype(np.float32) for _ in range(3)]  # snap_x, snap_z, image
    return lay, m, ab, f, g


def reference_case(name, what, mode, sponge, seed):
    import torch

    from oracle import REF_LIB_PATH

    lib = C.CDLL(REF_LIB_PATH)
    for fn in ("ref_t1_fwd", "ref_t1_adj", "ref_t1_grad"):
        getattr(lib, fn).restype = C.c_int
    lay, m, ab, f, g = case_inputs(seed)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    p = lambda x: C.c_void_p(x.data_ptr())  # noqa: E731
    t = {k: dev(v) for k, v in m.items()}
    a = [dev(x) for x in ab]
    f1, f2 = dev(f[0]), dev(f[1])
    r = lay.ranges
    hs = [C.c_double(h) for h in H]
    if what == "grad":
        sx, sz, img = dev(g[0]), dev(g[1]), dev(g[2])
        rc = lib.ref_t1_grad(p(sx), p(sz), p(img), p(f1), p(f2), *r, lay.nx, lay.ny, lay.ldimx, lay.ldimy)
        assert rc == 0
        torch.cuda.synchronize()
        return {"image": img.cpu().numpy()}
    if what == "fwd":
        if mode == 2:
            o3 = torch.zeros((lay.nz, lay.ny, lay.nx), device="cuda")
            o4 = torch.zeros_like(o3)
            ld = (lay.nx, lay.ny, lay.nz)
        else:
            o3, o4 = dev(f[2]), dev(f[3])
            ld = (lay.ldimx, lay.ldimy, lay.ldimz)
        rc = lib.ref_t1_fwd(p(o3), p(o4), p(f1), p(f2), *[p(t[k]) for k in MKEYS], *[p(x) for x in a], *r,
                            lay.ldimx, lay.ldimy, lay.ldimz, *ld, C.c_float(DT), *hs, int(mode == 2),
                            int(mode == 1))
    else:
        o3, o4 = dev(f[2]), dev(f[3])
        rc = lib.ref_t1_adj(p(o3), p(o4), p(f1), p(f2), *[p(t[k]) for k in MKEYS], *[p(x) for x in a], *r,
                            lay.ldimx, lay.ldimy, lay.ldimz, C.c_float(DT), *hs, int(sponge))
    assert rc == 0
    torch.cuda.synchronize()
    return {"f3": o3.cpu().numpy(), "f4": o4.cpu().numpy()}


def oracle_case(name, what, mode, sponge, seed):
    from oracle import Oracle

    o = Oracle("f32")
    lay, m, ab, f, g = case_inputs(seed)
    if what == "grad":
        img = g[2].copy()
        o.t1_grad(lay, g[0], g[1], img, f[0], f[1])
        return {"image": img}
    if what == "fwd":
        if mode == 2:
            o3 = np.zeros((lay.nz, lay.ny, lay.nx), np.float32)
            o4 = np.zeros_like(o3)
            o.t1_fwd(lay, o3, o4, f[0], f[1], m, ab, np.float32(DT), H, 2, (lay.nx, lay.ny))
        else:
            o3, o4 = f[2].copy(), f[3].copy()
            o.t1_fwd(lay, o3, o4, f[0], f[1], m, ab, np.float32(DT), H, mode)
    else:
        o3, o4 = f[2].copy(), f[3].copy()
        o.t1_adj(lay, o3, o4, f[0], f[1], m, ab, np.float32(DT), H, sponge)
    return {"f3": o3, "f4": o4}


def interior(case, arrays):
    """Interior of halo'd outputs (calc_snap outputs and the image are already dense)."""
    lay = case_inputs(case[4])[0]
    if case[1] == "grad" or (case[1] == "fwd" and case[2] == 2):
        return arrays
    return {k: np.ascontiguousarray(v[lay.interior]) for k, v in arrays.items()}


def main(out_dir):
    gold = {}
    for case in CASES:
        for k, v in interior(case, reference_case(*case)).items():
            gold[f"{case[0]}/{k}"] = v
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "reference_type1.npz"), **gold)
    print(f"wrote {len(gold)} arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
