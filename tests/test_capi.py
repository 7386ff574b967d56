"""The C ABI: the library loads, exports every entry point include/tti_capi.h
declares, and rejects bad arguments with status codes (no GPU needed: the
argument checks run before any CUDA call)."""
import ctypes as C
import os
import re

import pytest

import miniappsforhpe_b200 as P

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "tti_capi.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tti_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("tti_launch_fwd_kernel2_drv", "tti_launch_update_rho_fwd_main_loop_2_1",
                 "tti_launch_adj_kernel2_drv", "tti_launch_update_adj_kernel_main_3",
                 "tti_launch_update_rho_gradient_rho", "tti_sim_create", "tti_sim_forward",
                 "tti_sim_adjoint", "tti_snap_start_write", "tti_snap_start_read"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(P.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version():
    assert P.status_string(P.OK) == "ok"
    assert P.status_string(P.ETIMEOUT) == "timed out"
    assert re.match(r"\d+\.\d+\.\d+", P.version())


def test_unsupported_order_is_rejected():
    with pytest.raises(P.TTIError) as e:
        P.launch_fwd_kernel2_drv(1, 1, 1, 1, 1, 1, 1, 1, 1, 4, 35, 4, 35, 4, 35, 0.1, 0.1, 0.1, 64, 40,
                                 order=16)
    assert e.value.status == P.EINVAL


def test_bad_ranges_are_rejected():
    with pytest.raises(P.TTIError) as e:  # ldimx leaves no radius-4 halo after ixend
        P.launch_fwd_kernel2_drv(1, 1, 1, 1, 1, 1, 1, 1, 1, 4, 30, 4, 35, 4, 35, 0.1, 0.1, 0.1, 32, 40)
    assert e.value.status == P.EINVAL
    with pytest.raises(P.TTIError) as e:  # null volume
        P.launch_fwd_kernel2_drv(None, 1, 1, 1, 1, 1, 1, 1, 1, 4, 20, 4, 20, 4, 20, 0.1, 0.1, 0.1, 32, 29)
    assert e.value.status == P.EINVAL


def test_pml_is_rejected():
    lib = P.lib()
    args = [C.c_void_p(1)] * 18 + [C.c_void_p(1)] + [None] * 11 + [4, 20, 4, 20, 4, 20, 32, 29,
                                                                    C.c_float(1e-3), 10.0, 10.0, 10.0,
                                                                    0, 8, 0, 0, 0, None]
    assert lib.tti_launch_update_rho_fwd_main_loop_2_1(*args) == P.EINVAL


def test_sim_config_is_validated():
    with pytest.raises(P.TTIError) as e:
        P.Simulator(P.Config(nx=0, ny=8, nz=8))
    assert e.value.status == P.EINVAL
    with pytest.raises(P.TTIError):
        P.Simulator(P.Config(nx=8, ny=8, nz=8, dt=-1.0))


def test_reduced_precision_snapshots_need_the_fused_path():
    with pytest.raises(P.TTIError) as e:
        P.Simulator(P.Config(nx=48, ny=40, nz=40, nt=8, fused=False, snap_precision="fp16"))
    assert e.value.status == P.EINVAL
    with pytest.raises(P.TTIError) as e:  # nx not a multiple of 8
        P.Simulator(P.Config(nx=44, ny=40, nz=40, nt=8, snap_precision="bf16"))
    assert e.value.status == P.EINVAL


def test_checkpoint_config_is_validated():
    base = dict(nx=32, ny=24, nz=24, nt=40, xcorr_step=4)
    for bad in (dict(checkpoint_every=6), dict(checkpoint_every=8, fused=False),
                dict(checkpoint_every=8, save_snapshots=False), dict(checkpoint_every=-4)):
        with pytest.raises(P.TTIError) as e:
            P.Config(**base, **bad).footprint_bytes()
        assert e.value.status == P.EINVAL


def test_footprint_accounts_for_snapshots_and_checkpoints():
    """The footprint query needs no device: it is the creation plan's sum."""
    n = 64 * 64 * 64
    lay = (96, 72, 72)
    vol = lay[0] * lay[1] * lay[2] * 4
    cfg = dict(nx=64, ny=64, nz=64, nt=400, xcorr_step=4)
    full = P.Config(**cfg).footprint_bytes()
    nsnap = 100
    assert full >= 14 * vol + nsnap * 4 * n * 4
    half = P.Config(**cfg, snap_precision="fp16").footprint_bytes()
    assert full - half == nsnap * 4 * n * 2 + 0  # same plan but 2-byte slots
    ck = P.Config(**cfg, snap_precision="fp16", checkpoint_every=40).footprint_bytes()
    # 10 FP32 checkpoints + one 10-slot segment + the recompute state
    assert ck < half
    assert ck - (half - nsnap * 4 * n * 2) == pytest.approx(
        10 * 4 * n * 4 + 10 * 4 + 10 * 4 * n * 2 + 6 * vol, abs=4096)
    no_snap = P.Config(**cfg, save_snapshots=False).footprint_bytes()
    assert no_snap < ck
    # the reference kernel sequence needs its derivative volumes and scratch
    # (14 volumes); the fused path keeps the model a second time, interleaved
    # in float4 cells (8 volumes)
    assert P.Config(**cfg, save_snapshots=False, fused=False).footprint_bytes() - no_snap == 14 * vol - 8 * vol


def test_scheme_is_validated_and_type1_needs_no_derivative_volumes():
    base = dict(nx=64, ny=64, nz=64, nt=40, xcorr_step=4, save_snapshots=False)
    for bad in (-1, 2):
        with pytest.raises(P.TTIError) as e:
            P.Config(**base, scheme=bad).footprint_bytes()
        assert e.value.status == P.EINVAL
    vol = 96 * 72 * 72 * 4
    fused = P.Config(**base).footprint_bytes()
    # the centred operator's kernel sequence works on p, q, pdot, qdot alone,
    # and neither of its paths keeps the staggered adjoint's interleaved model
    assert P.Config(**base, scheme=1, fused=False).footprint_bytes() == fused - 8 * vol
    assert P.Config(**base, scheme=1).footprint_bytes() == fused - 8 * vol


def test_type1_snapshot_slots_hold_two_fields():
    n = 64 * 64 * 64
    cfg = dict(nx=64, ny=64, nz=64, nt=400, xcorr_step=4, scheme=1)
    none = P.Config(**cfg, save_snapshots=False).footprint_bytes()
    for prec, elt in (("fp32", 4), ("fp16", 2)):
        full = P.Config(**cfg, snap_precision=prec).footprint_bytes()
        # 100 slots of pdot and qdot, their scales, the running maxima
        assert full - none == 100 * (2 * n * elt + 16) + 16


def test_work_split_table_round_trip():
    """The split table is host state: it records (bz, ztop) per grid and
    kernel kind and rejects a top that leaves no bottoms."""
    try:
        P.tune_set(64, 48, 40, "adjoint", 3, 17)
        assert P.tune_get_split(64, 48, 40, "adjoint") == (3, 17)
        assert P.tune_get(64, 48, 40, "adjoint") == 3
        P.tune_set(64, 48, 40, "type1_forward", 12)
        assert P.tune_get_split(64, 48, 40, "type1_forward") == (12, 0)
        for bad in ((4, 40), (4, -1)):
            with pytest.raises(P.TTIError) as e:
                P.tune_set(64, 48, 40, "forward", *bad)
            assert e.value.status == P.EINVAL
    finally:
        for k in P.TUNE_KINDS:
            P.tune_set(64, 48, 40, k, 0)


def test_wave_precision_is_validated_and_costs_only_its_scales():
    base = dict(nx=64, ny=64, nz=64, nt=40, xcorr_step=4, save_snapshots=False)
    with pytest.raises(P.TTIError) as e:
        P.Config(**base, fused=False, wave_precision="fp16").footprint_bytes()
    assert e.value.status == P.EINVAL
    plain = P.Config(**base).footprint_bytes()
    assert P.Config(**base, wave_precision="bf16").footprint_bytes() == plain + 16


def _vp(n):
    return [C.c_void_p(1)] * n  # never dereferenced: the checks come first


def test_type1_launchers_reject_bad_arguments():
    """Order, ranges, missing volumes and the sponge/calc_snap combination are
    refused before anything reaches the device (the reference aborts)."""
    lib = P.lib()
    fwd, adj = lib.tti_launch_type1_fwd, lib.tti_launch_type1_adj
    fwd.restype = adj.restype = C.c_int
    dims = [4, 27, 4, 23, 4, 19, 32, 28, 24]  # ranges, ldimx/y/z
    tail = [C.c_float(1e-3), C.c_double(10.0), C.c_double(10.0), C.c_double(10.0)]
    ok_fwd = _vp(14) + dims + [32, 28, 24] + tail
    assert fwd(*ok_fwd, 16, None, 0, 0, 0) == P.EINVAL                       # order
    assert fwd(*ok_fwd, 8, None, 1, 1, 0) == P.EINVAL                        # calc_snap with the sponge
    assert fwd(*(_vp(14) + [4, 27, 4, 23, 4, 19, 28, 28, 24] + [32, 28, 24] + tail), 8, None, 0, 0, 0) == P.EINVAL
    assert fwd(*([None] + _vp(13) + dims + [32, 28, 24] + tail), 8, None, 0, 0, 0) == P.EINVAL
    assert fwd(*(_vp(11) + [None] * 3 + dims + [32, 28, 24] + tail), 8, None, 0, 1, 0) == P.EINVAL
    ok_adj = _vp(14) + dims + tail
    assert adj(*ok_adj, 12, None, 0, 0) == P.EINVAL
    assert adj(*(_vp(4) + [None] + _vp(9) + dims + tail), 8, None, 0, 0) == P.EINVAL


def test_noalloc_launcher_rejects_a_range_beyond_its_array():
    lib = P.lib()
    f = lib.tti_launch_adj_kernel2_drv_noalloc
    f.restype = C.c_int
    one = C.c_float(1.0)
    # 120 x 120 x 80 interior: 160 * 128 * 88 cells > 2^20
    args = _vp(18) + [4, 123, 4, 123, 4, 83] + [one] * 6 + [160, 128, 8] + [one] * 4 + [None]
    assert f(*args) == P.ETOOBIG
    args = _vp(18) + [4, 123, 4, 123, 4, 83] + [one] * 6 + [160, 128, 6] + [one] * 4 + [None]
    assert f(*args) == P.EINVAL  # order checked first


def test_step_and_run_level_calls_reject_missing_objects():
    lib = P.lib()
    for name, extra in (("tti_sim_forward_begin", []), ("tti_sim_forward_step", [0]),
                        ("tti_sim_adjoint_step", [0]), ("tti_sim_image_step", [0]),
                        ("tti_sim_adjoint_finish", []), ("tti_sim_sync", [])):
        assert getattr(lib, name)(None, *extra) == P.EINVAL, name
    lib.tti_rtm_shot.restype = C.c_int
    assert lib.tti_rtm_shot(None, None) == P.EINVAL


def test_server_config_is_validated():
    from miniappsforhpe_b200 import serve as S

    for kw in (dict(max_active=0), dict(round_ms=0.0), dict(scheme=2)):
        with pytest.raises(P.TTIError) as e:
            S.Server(**kw)
        assert e.value.status == P.EINVAL


def test_header_is_plain_c(tmp_path):
    """include/tti_capi.h compiles as C99 on its own (the drop-in boundary is
    a C header, not a C++ one)."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    src = tmp_path / "use.c"
    src.write_text('#include "tti_capi.h"\nint main(void) { tti_sim_config c = {0}; (void)c; return 0; }\n')
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-pedantic", "-fsyntax-only",
                        "-I" + os.path.dirname(HEADER), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
