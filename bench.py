"""Benchmark: TTI RTM shot throughput on B200 (Gpts/s of forward+adjoint+imaging).

Workload (the reference's full-RTM configuration): TTI pseudo-acoustic RTM,
256^3 grid, dx = 10 m, 24-cell absorbing sponge, smooth Gaussian-random TTI
model (300 m correlation; vp 1500-5000 m/s, eps 0-0.25, delta 0-0.1,
theta 0-45 deg, phi 0-180 deg), 12 Hz Ricker source, 2000 steps, snapshot and
imaging every 4 steps, receivers on every cell of plane z = 3; observed data
from the same model plus a 5 % vp blob.  One bench "step" is one full shot:
forward with snapshots, adjoint driven by the residual, Vp image and density
gradient.  value = interior points x time steps / shot time (device time,
CUDA events on the simulator's stream, max over ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one shot stream per GPU (independent shots, images stacked with
one NCCL all-reduce per shot); launch it under torch.distributed.run.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TTI fwd+adj+grad Gpts/s & HBM % of peak; shots/hr, p50/p99 at fixed image error"
# Algorithmic bytes per interior point per time step (FP32, each array once):
# forward TTI 64, adjoint TTI 64, imaging 16 per imaging step, snapshot 8 per
# snapshot step; the fused kernels' per-launch figure is 64 B/pt.
B_FWD, B_ADJ, B_IMG, B_SNAP = 64, 64, 16, 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256, help="grid points per axis")
    ap.add_argument("--nt", type=int, default=2000)
    ap.add_argument("--xcorr", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--per-kernel", action="store_true", help="reference kernel sequence instead of fused")
    ap.add_argument("--snap-precision", choices=["fp32", "fp16", "bf16"], default="fp32",
                    help="snapshot storage (the stencils and time update stay FP32)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload(args, rank):
    from miniappsforhpe_b200 import earth_models as EM

    n = args.n
    model = EM.smooth_tti(n, n, n, dx=10.0, corr_m=300.0, seed=1234 + rank)
    true = EM.add_velocity_blob(model, (n // 2, n // 2, n // 2), radius_cells=max(2, n // 12), fraction=0.05)
    dt = EM.cfl_dt(true, 10.0, cfl=0.4)
    w = EM.ricker(args.nt, dt, 12.0)
    src = (n // 2 + (rank * 17) % max(1, n // 4), n // 2, 5)
    rec = EM.receiver_plane(n, n, 3)
    desc = {
        "workload": f"TTI RTM shot {n}^3, dx=10m, sponge 24, {args.nt} steps, imaging every {args.xcorr}",
        "grid": [n, n, n], "nt": args.nt, "xcorr_step": args.xcorr, "sponge_width": 24,
        "model": "smooth Gaussian-random TTI (300 m), observed = model + 5% vp blob",
        "source": "12 Hz Ricker", "receivers": f"{n * n} (plane z=3)",
        "l2": "inputs larger than L2 (every step streams >1 GB through HBM)",
    }
    return model, true, dt, w, src, rec, desc


def sample_clocks(path):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        f = open(path, "w")
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms",
                                 "200"], stdout=f, stderr=subprocess.DEVNULL), f
    except Exception:
        return None, None


def summarize_clocks(path, gpu_index):
    try:
        rows = [r.split(",") for r in open(path).read().strip().splitlines()]
    except Exception:
        return None
    rows = [[c.strip() for c in r] for r in rows if len(r) >= 9 and r[0].strip() == str(gpu_index)]
    if not rows:
        return None
    sm = [float(r[1]) for r in rows]
    mx = float(rows[0][2])
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the fused kernels from the committed ncu summary, if any."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "fused_kernels_traffic.json")))
    except Exception:
        return {}


# ---------------------------------------------------------------------------
def cpu_sample(args, model_np, dt, nsteps=2):
    """The oracle (C restatement of the reference kernels, OpenMP on all host
    cores) on the same grid: nsteps forward steps, nsteps adjoint steps and one
    imaging step, extrapolated to a full shot."""
    from miniappsforhpe_b200 import earth_models as EM  # noqa: F401
    from oracle import DKEYS, Layout, Oracle, new_state

    o = Oracle("f32")
    n = args.n
    lay = Layout(n, n, n)
    m = {}
    ext = lambda a: np.pad(a, 4, mode="edge")  # noqa: E731
    vp, eps, delta = model_np["vp"], model_np["eps"], model_np["delta"]
    vs, th, ph = model_np["vs"], model_np["theta"], model_np["phi"]
    pars = [np.ascontiguousarray(ext(a)) for a in (vp, eps, delta, vs, th, ph)]
    full = []
    for a in pars:
        b = np.zeros(lay.shape, np.float32)
        b[:, :, : a.shape[2]] = a
        full.append(b)
    m1, m2, m3, m4, m5, m6, m7 = o.init_cijs(*full)
    m = dict(m1=m1, m2=m2, m3=m3, m4=m4, rx=m5, ry=m6, rz=m7, irho=np.ones(lay.shape, np.float32))
    ab = [np.ones(2 * k, np.float32) for k in (lay.ldimx, lay.ldimy, lay.ldimz)]
    g = o.grid(lay, np.float32(dt), (10.0, 10.0, 10.0), free_surface=True, sponge_active=True)
    st = new_state(lay)
    st["f1"][lay.interior] = np.random.default_rng(0).standard_normal((n, n, n)).astype(np.float32)
    t0 = time.perf_counter()
    for _ in range(nsteps):
        o.fwd_step(g, st, m, ab)
    t_fwd = (time.perf_counter() - t0) / nsteps
    t0 = time.perf_counter()
    for _ in range(nsteps):
        o.adj_step(g, st, m, ab)
    t_adj = (time.perf_counter() - t0) / nsteps
    t0 = time.perf_counter()
    d = {k: lay.zeros() for k in DKEYS}
    o.fwd_drv(lay, st["f1"], st["f2"], m["irho"], d, (np.float32(0.1),) * 3)
    o.loop4_derivatives(lay, d)
    grho = np.zeros(n * n * n, np.float32)
    o.rho_gradient(lay, grho, d, st["f1"], st["f2"], m, (10.0, 10.0, 10.0), n, n)
    gvp = np.zeros(n * n * n, np.float32)
    s3 = np.ascontiguousarray(st["f3"][lay.interior].ravel())
    o.update_vp_gradient(lay, s3, s3, gvp, st["f3"], st["f4"])
    t_img = time.perf_counter() - t0
    t_shot = args.nt * (t_fwd + t_adj) + (args.nt // args.xcorr) * t_img
    pts = float(n) ** 3 * args.nt
    return {
        "value": pts / t_shot / 1e9, "unit": "Gpts/s", "cores": o.num_threads(), "kind": "port",
        "sample": (f"oracle FP32 on {n}^3: {nsteps} forward + {nsteps} adjoint steps + 1 imaging step, "
                   f"extrapolated to {args.nt} steps ({t_fwd:.2f}s/fwd, {t_adj:.2f}s/adj, {t_img:.2f}s/img)"),
        "shot_s": t_shot,
    }


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from miniappsforhpe_b200 import earth_models as EM  # noqa: F401

    model, true, dt, w, src, rec, desc = workload(args, 0)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_sample(args, model, dt, nsteps=1)
        if i >= args.warmup:
            vals.append(r["value"])
    v = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gpts/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(r["shot_s"] * 1e3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": desc,
        "cpu_baseline": {"value": v, "unit": "Gpts/s", "cores": r["cores"], "kind": "port",
                         "sample": r["sample"] + "; per step: one such sample"},
        "e2e": {"value": v, "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    import miniappsforhpe_b200 as P

    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    model, true, dt, w, src, rec, desc = workload(args, rank)
    n = args.n
    cfg = P.Config(nx=n, ny=n, nz=n, dx=10.0, dy=10.0, dz=10.0, dt=dt, nt=args.nt, xcorr_step=args.xcorr,
                   sponge_width=24, free_surface=True, fused=not args.per_kernel, save_snapshots=True,
                   snap_precision=args.snap_precision)
    sim = P.Simulator(cfg)
    sim.set_source(*src, w)
    sim.set_receivers(rec)
    nrec = len(rec)
    # observed data: forward on the true model (outside the timed region)
    sim.set_model(**true)
    observed = torch.empty((args.nt, nrec), dtype=torch.float32, device=dev)
    sim.forward(observed)
    sim.set_model(**model)
    gvp = torch.empty((n, n, n), dtype=torch.float32, device=dev)
    grho = torch.empty_like(gvp)
    synth = torch.empty_like(observed)
    stack = torch.zeros_like(gvp)
    stream = torch.cuda.ExternalStream(sim.stream_handle(), device=dev)

    def shot():
        sim.forward(synth)
        l1 = sim.launch_count()
        sim.adjoint_observed(observed)
        l2 = sim.launch_count()
        sim.image(gvp, grho)
        if dist is not None:
            dist.all_reduce(gvp)
        stack.add_(gvp)
        return l1 + l2

    for _ in range(args.warmup):
        shot()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clk_proc, clk_file = sample_clocks(os.path.join(ROOT, "gpurun_out", f"clocks_rank{rank}.csv")) \
        if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else sample_clocks(f"/tmp/clocks_rank{rank}.csv")
    sim.set_profiling(True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    launches = 0
    for _ in range(args.steps):
        launches += shot()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    times = sim.kernel_times()
    sim.set_profiling(False)
    if clk_proc is not None:
        clk_proc.terminate()
        clk_proc.wait()
        clk_file.close()
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    pts = float(n) ** 3 * args.nt
    value = pts * args.steps * ws / (ms / 1e3) / 1e9
    ms_per_step = ms / args.steps

    # roofline of the dominant step kernel
    peak, peak_kind = peaks()
    kind = max(("forward", "adjoint"), key=lambda k: times[k][0])
    kms, kn = times[kind]
    per_launch_s = (kms / max(kn, 1)) / 1e3
    alg_bytes = (B_FWD if kind == "forward" else B_ADJ) * float(n) ** 3
    achieved = alg_bytes / per_launch_s / 1e9 if kn else None
    traffic = ncu_traffic().get(f"{kind}_dram_bytes_per_launch_{n}")
    roofline = {"kernel": f"fused {kind} step", "bound": "hbm", "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                "avg_launch_ms": per_launch_s * 1e3, "launches": kn}
    passes = {k: {"total_ms": v[0] / args.steps, "launches_per_shot": v[1] / args.steps}
              for k, v in times.items()}
    step_bytes = (B_FWD + B_ADJ + B_IMG / args.xcorr + B_SNAP / args.xcorr) * float(n) ** 3
    hbm_frac = step_bytes * args.nt / (ms_per_step / 1e3) / 1e9 / peak

    # end to end through the host-buffer API
    e2e = None
    if not args.no_e2e:
        host_model = {k: np.ascontiguousarray(v) for k, v in model.items()}
        obs_host = observed.cpu().numpy()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sim.set_model(**host_model)
            tr = sim.forward()
            sim.adjoint_observed(obs_host)
            gv, gr = sim.image()
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([el], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        h2d = 7 * n ** 3 * 4 + args.nt * nrec * 4
        d2h = args.nt * nrec * 4 + 2 * n ** 3 * 4
        e2e = {"value": pts * args.steps * ws / el / 1e9, "unit": "Gpts/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "timer": "wall clock, synchronized on both sides"}
        del tr, gv, gr

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        r = cpu_sample(args, model, dt)
        cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")}

    clocks = summarize_clocks(clk_file.name if clk_file else "", local)
    line = {
        "metric": METRIC, "value": value, "unit": "Gpts/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, see config)",
        "config": {**desc, "parallelism": f"shot-parallel x{ws}" if ws > 1 else "single GPU",
                   "path": "reference kernel sequence" if args.per_kernel else "fused step kernels",
                   "snapshots": args.snap_precision},
        "roofline": roofline, "hbm_frac_alg_134B": hbm_frac,
        "shots_per_hour": 3600.0 * 1e3 / ms_per_step * ws,
        "passes_ms_per_shot": passes, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
