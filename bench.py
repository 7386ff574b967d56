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

N > 1 runs one shot stream per GPU (independent shots; the image stack is
summed over the GPUs with one NCCL all-reduce at the end of the stream);
launch it under torch.distributed.run.
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
B_VTI = 52  # forward or adjoint step on a VTI model: rx, ry, rz are not read
# Centred constant-density operator (--scheme 1), per interior point: a
# forward or adjoint step reads p, q, m1..m4, rx, ry, rz and pdot, qdot and
# writes pdot, qdot and the next p, q: 60 B (48 on a VTI model); the Vp image
# reads two snapshot fields and the adjoint pdot, qdot and updates the image:
# 2*elt + 16 B per imaging step; the snapshot writes 2*elt B.
B_T1, B_T1_VTI = 60, 48


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
    ap.add_argument("--scheme", type=int, choices=[0, 1], default=0,
                    help="0: staggered variable-density operator; 1: centred constant-density (type1)")
    ap.add_argument("--snap-precision", choices=["fp32", "fp16", "bf16"], default="fp32",
                    help="snapshot storage (the stencils and time update stay FP32)")
    ap.add_argument("--checkpoint", type=int, default=0,
                    help="checkpointed recomputation: FP32 checkpoints every K steps")
    ap.add_argument("--grid", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                    help="non-cubic grid (overrides --n)")
    ap.add_argument("--f0", type=float, default=12.0, help="Ricker peak frequency (Hz)")
    ap.add_argument("--dx", type=float, default=10.0)
    ap.add_argument("--model", choices=["smooth", "layered"], default="smooth",
                    help="smooth Gaussian-random TTI (full RTM workload) or layered VTI")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the modelled work split instead of timing the candidates first")
    ap.add_argument("--bz", type=int, nargs=3, default=None, metavar=("FWD", "ADJ", "IMG"),
                    help="fixed planes per CTA of the forward, adjoint and imaging kernels (implies --no-autotune)")
    ap.add_argument("--ztop", type=int, nargs=3, default=[0, 0, 0], metavar=("FWD", "ADJ", "IMG"),
                    help="with --bz: top/bottom split depth per kernel (0: plain tile-major split)")
    ap.add_argument("--serve", action="store_true",
                    help="served batch: Poisson stream of RTM shots through the shot server, "
                         "against the same stream run one shot at a time in plain FP32")
    ap.add_argument("--shots", type=int, default=64)
    ap.add_argument("--rate", type=float, default=2.0, help="mean arrivals per second")
    ap.add_argument("--nt-range", type=int, nargs=2, default=[1000, 3000])
    ap.add_argument("--max-active", type=int, default=2,
                    help="resident shots in the served mode (2 measured best on the C4 stream: 8, 4, 2 gave 2691, 2995, 3230 shots/hour)")
    ap.add_argument("--round-ms", type=float, default=50.0)
    ap.add_argument("--serve-modes", default="served,plain",
                    help="served: the shot server; plain: the run-level call shot by shot in FP32; "
                         "sequential: the server with one resident shot, FP32")
    ap.add_argument("--elastic", action="store_true",
                    help="the elastic simulator3 proxy: forward + adjoint steps of its step kernels")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def grid_of(args):
    return tuple(args.grid) if args.grid else (args.n, args.n, args.n)


def workload(args, rank):
    from miniappsforhpe_b200 import earth_models as EM

    nx, ny, nz = grid_of(args)
    if args.model == "layered":
        model = EM.layered_vti(nx, ny, nz, nlayers=6, seed=1234 + rank)
        mdesc = "layered VTI (6 flat layers), observed = model + 5% vp blob"
    else:
        model = EM.smooth_tti(nx, ny, nz, dx=args.dx, corr_m=300.0, seed=1234 + rank)
        mdesc = "smooth Gaussian-random TTI (300 m), observed = model + 5% vp blob"
    true = EM.add_velocity_blob(model, (nx // 2, ny // 2, nz // 2), radius_cells=max(2, min(nx, ny, nz) // 12),
                                fraction=0.05)
    dt = EM.cfl_dt(true, args.dx, cfl=0.4)
    w = EM.ricker(args.nt, dt, args.f0)
    src = (nx // 2 + (rank * 17) % max(1, nx // 4), ny // 2, 5)
    rec = EM.receiver_plane(nx, ny, 3)
    gname = f"{nx}^3" if nx == ny == nz else f"{nx}x{ny}x{nz}"
    op = ", centred constant-density operator" if args.scheme == 1 else ""
    desc = {
        "workload": (f"TTI RTM shot {gname}{op}, dx={args.dx:g}m, sponge 24, {args.nt} steps, imaging every "
                     f"{args.xcorr}"),
        "grid": [nx, ny, nz], "nt": args.nt, "xcorr_step": args.xcorr, "sponge_width": 24, "dx": args.dx,
        "model": mdesc, "source": f"{args.f0:g} Hz Ricker", "receivers": f"{nx * ny} (plane z=3)",
        "l2": "inputs larger than L2 (every step streams >1 GB through HBM)",
    }
    if args.checkpoint:
        desc["checkpoint_every"] = args.checkpoint
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
CPU_SAMPLE_STEPS = 20  # the shot's first 20 time steps: 20 forward, 20 adjoint, 5 imaging steps


def cpu_sample(args, model_np, dt, w, src, rec, nsteps=CPU_SAMPLE_STEPS):
    """The oracle (C restatement of the reference kernels, FP32, OpenMP on all
    host cores) running the first nsteps time steps of the same shot in the
    reference order: forward from rest with the source, the receivers and a
    snapshot every xcorr steps, adjoint from rest driven by its own traces,
    imaging at the snapshot steps (one per xcorr steps, the shot's share), on
    the shot's own model (host-built like the simulator's), sponge and free
    surface.  Gpts/s = interior points x nsteps / wall time of that run."""
    from types import SimpleNamespace

    from oracle import Layout, Oracle, models_from_parameters, rtm_shot, rtm_shot_t1, sponge_profile

    o = Oracle("f32")
    nsteps = min(nsteps, args.nt)
    nx, ny, nz = grid_of(args)
    lay = Layout(nx, ny, nz)
    m = models_from_parameters(lay, **model_np)
    cfg = SimpleNamespace(nt=nsteps, xcorr_step=args.xcorr, dt=dt, dx=args.dx, dy=args.dx, dz=args.dx,
                          free_surface=True, sponge_width=24)
    ab = (sponge_profile(nx, lay.ldimx, 24, True), sponge_profile(ny, lay.ldimy, 24, True),
          sponge_profile(nz, lay.ldimz, 24, False))
    rec_idx = np.array([lay.index(*r) for r in rec], np.int64)
    run = rtm_shot_t1 if getattr(args, "scheme", 0) == 1 else rtm_shot
    t0 = time.perf_counter()
    run(o, lay, m, ab, cfg, lay.index(*src), w[:nsteps], rec_idx)
    el = time.perf_counter() - t0
    op = "type1 " if getattr(args, "scheme", 0) == 1 else ""
    return {
        "value": float(nx) * ny * nz * nsteps / el / 1e9, "unit": "Gpts/s", "cores": o.num_threads(),
        "kind": "port",
        "sample": (f"oracle {op}FP32 on {nx}x{ny}x{nz}: the shot's first {nsteps} time steps ({nsteps} forward, "
                   f"{nsteps} adjoint, {(nsteps + args.xcorr - 1) // args.xcorr} imaging steps) on its own model, "
                   f"sponge and source, {el:.2f} s"),
        "sample_s": el,
    }


def run_reference(args):
    """The reference arm: the reference has no CPU implementation of this path
    (its only CPU code is the elastic proxy), so the oracle port of its
    kernels stands in, on all host cores.  One step = one bounded sample (the
    shot's first 20 time steps); ms_per_step is that sample's wall time."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    model, true, dt, w, src, rec, desc = workload(args, 0)
    vals, secs = [], []
    for i in range(args.warmup + args.steps):
        r = cpu_sample(args, model, dt, w, src, rec)
        if i >= args.warmup:
            vals.append(r["value"])
            secs.append(r["sample_s"])
    v = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gpts/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(secs) * 1e3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": desc,
        "cpu_baseline": {"value": v, "unit": "Gpts/s", "cores": r["cores"], "kind": "port",
                         "sample": r["sample"] + "; one bench step = one such sample"},
        "e2e": {"value": v, "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Elastic proxy (simulator3): algorithmic bytes per interior point of each
# launcher call (FP32, each array once): velocity gradients R f1..f3, W d4..d9;
# velocity update R f4..f9, M22, RW f1..f3; stress update (six z-mixed
# precomputes R 1 W 2 each, then R M1..M21, d4..d9, f10..f21, RW f4..f9);
# pressure R f4..f9 W p over the whole allocation.
E3_BYTES = {"vgplain": 36, "vplain": 52, "splain": 276, "compute_p": 28}


def run_elastic(args):
    """One bench step = one forward and one adjoint step of simulator3's
    schedule (simulator3/simulator3SetUp.cu:2196-2585) on an n^3 subdomain:
    velocity update, free-surface mirrors, strains, stress update with the
    z-mixed precomputes, pressure; then stress update, strains, mirrors,
    velocity update.  value = interior points x 2 passes / step time."""
    import torch

    from miniappsforhpe_b200.elastic import ElasticProxy, launch_compute_p

    torch.cuda.set_device(0)
    n = args.n
    sim = ElasticProxy(n, n, n)
    sim.init_source(1e-30)  # the stand-in scheme grows ~1e4 per step; start small
    st = torch.cuda.current_stream()
    calls = {
        "vplain": sim._vplain, "mirrors": sim._mirrors, "vgplain": sim._vgplain, "splain": sim._splain,
        "compute_p": lambda: launch_compute_p(sim.p, *sim.s, sim.p.numel(), sim._stream),
    }
    order = ["vplain", "mirrors", "vgplain", "splain", "compute_p", "splain", "vgplain", "mirrors", "vplain"]
    for _ in range(args.warmup):
        for k in order:
            calls[k]()
    torch.cuda.synchronize()
    ev = {k: [] for k in calls}
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(st)
    for _ in range(args.steps):
        for k in order:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            calls[k]()
            b.record(st)
            ev[k].append((a, b))
    t1.record(st)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / args.steps
    pts = n ** 3
    hbm, kind = peaks()
    kern = {}
    for k, lst in ev.items():
        per = sum(a.elapsed_time(b) for a, b in lst) / len(lst)
        row = {"avg_call_ms": per, "calls_per_step": len(lst) // args.steps}
        if k in E3_BYTES:
            cells = sim.p.numel() if k == "compute_p" else pts
            gbs = E3_BYTES[k] * cells / (per * 1e-3) / 1e9
            row.update({"alg_bytes_per_pt": E3_BYTES[k], "achieved_gbs": gbs, "frac": gbs / hbm})
        kern[k] = row
    top = max((k for k in kern if k in E3_BYTES), key=lambda k: kern[k]["avg_call_ms"] * kern[k]["calls_per_step"])
    line = {
        "metric": "elastic proxy (simulator3) forward+adjoint step Gpts/s", "value": 2 * pts / (ms * 1e-3) / 1e9,
        "unit": "Gpts/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (the reference's own cos/sin stand-in model)",
        "config": {"workload": f"simulator3 elastic proxy {n}^3, one forward + one adjoint step",
                   "grid": [n, n, n], "l2": "inputs larger than L2 (~50 volumes of the grid)"},
        "roofline": {"kernel": top, "bound": "hbm", "achieved": kern[top]["achieved_gbs"], "peak": hbm,
                     "peak_kind": kind, "unit": "GB/s", "frac": kern[top]["frac"], "traffic": None},
        "kernels": kern,
        # kernels per step: velocity updates 2, mirrors 8, strains 2, stress updates 2 x 7, pressure 1
        "gpu_launches": 27 * args.steps,
        "cpu_baseline": None if args.no_cpu_baseline else elastic_cpu_sample(),
    }
    print(json.dumps(line), flush=True)


def elastic_cpu_sample(n=96, steps=8):
    """The oracle's restatement of the same steps on the host (all cores), on
    a 96^3 subdomain: Gpts/s of forward + adjoint step pairs."""
    from oracle import ElasticOracle, Layout

    e, lay = ElasticOracle(), Layout(n, n, n)
    z = lay.zeros
    M, d, v, s, pre, p = [z() for _ in range(22)], [z() for _ in range(6)], [z() for _ in range(3)], \
        [z() for _ in range(6)], [z() for _ in range(12)], z()
    zp = np.zeros(lay.ldimz, np.float32)
    e.init_model(lay, M, d, zp)
    s[0][lay.ldimz // 2, lay.ldimy // 2, lay.ldimx // 2] = 1e-30
    t = time.perf_counter()
    for _ in range(steps):
        e.vplain(lay, v, s, M[21], zp)
        for f in (s, s, v, v):
            e.mirror(lay, f)
        e.vgplain(lay, *v, d, zp)
        e.splain(lay, s, M, d, pre)
        e.pressure(p, s)
        e.splain(lay, s, M, d, pre)
        e.vgplain(lay, *v, d, zp)
        for f in (s, s, v, v):
            e.mirror(lay, f)
        e.vplain(lay, v, s, M[21], zp)
    dt = time.perf_counter() - t
    return {"value": 2 * n ** 3 * steps / dt / 1e9, "unit": "Gpts/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{steps} forward + adjoint step pairs on a {n}^3 subdomain (the oracle, OpenMP)"}


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
    nx, ny, nz = grid_of(args)
    npts = float(nx) * ny * nz
    cfg = P.Config(nx=nx, ny=ny, nz=nz, dx=args.dx, dy=args.dx, dz=args.dx, dt=dt, nt=args.nt,
                   xcorr_step=args.xcorr, sponge_width=24, free_surface=True, fused=not args.per_kernel,
                   save_snapshots=True, snap_precision=args.snap_precision, checkpoint_every=args.checkpoint,
                   scheme=args.scheme)
    sim = P.Simulator(cfg)
    sim.set_source(*src, w)
    sim.set_receivers(rec)
    nrec = len(rec)
    # observed data: forward on the true model (outside the timed region)
    sim.set_model(**true)
    observed = torch.empty((args.nt, nrec), dtype=torch.float32, device=dev)
    sim.forward(observed)
    sim.set_model(**model)
    tuned = None
    if args.bz:
        kinds = ("type1_forward", "type1_adjoint") if args.scheme == 1 else ("forward", "adjoint", "imaging")
        for kind, b, zt in zip(kinds, args.bz, args.ztop):
            P.tune_set(nx, ny, nz, kind, b, zt)
        tuned = {k: {"bz": b, "ztop": zt} for k, b, zt in zip(kinds[:2] + ("imaging",), args.bz, args.ztop)}
    elif not args.per_kernel and not args.no_autotune:
        tuned = sim.autotune(reps=2)  # outside the timed region; picks the work split per kernel
    gvp = torch.empty((nz, ny, nx), dtype=torch.float32, device=dev)
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
        stack.add_(gvp)
        return l1 + l2

    def reduce_stack():
        # the stream's one collective: the image stack summed over the ranks
        if dist is not None:
            dist.all_reduce(stack)

    for _ in range(args.warmup):
        shot()
    reduce_stack()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    rdir = os.environ.get("TTI_REPORT_DIR")  # where the clock samples are kept, if set
    clk_proc, clk_file = sample_clocks(os.path.join(rdir if rdir and os.path.isdir(rdir) else "/tmp",
                                                    f"clocks_rank{rank}.csv"))
    sim.set_profiling(True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    launches = 0
    for _ in range(args.steps):
        launches += shot()
    reduce_stack()
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
    pts = npts * args.nt
    value = pts * args.steps * ws / (ms / 1e3) / 1e9
    ms_per_step = ms / args.steps

    # roofline of the dominant step kernel
    peak, peak_kind = peaks()
    kind = max(("forward", "adjoint"), key=lambda k: times[k][0])
    kms, kn = times[kind]
    per_launch_s = (kms / max(kn, 1)) / 1e3
    vti = args.model == "layered"
    t1 = args.scheme == 1
    if t1:
        b_step = B_T1_VTI if vti else B_T1
    else:
        b_step = B_VTI if vti else (B_FWD if kind == "forward" else B_ADJ)
    alg_bytes = b_step * npts
    achieved = alg_bytes / per_launch_s / 1e9 if kn else None
    # DRAM bytes per launch from the committed ncu capture at this run's work
    # split (the traffic depends on it: L2 keeps the halos neighbouring
    # columns share only when their CTAs run side by side)
    tkey = f"{'type1_' if t1 else ''}{kind}"
    sp = (tuned or {}).get(tkey)
    split = [sp["bz"], sp.get("ztop", 0)] if isinstance(sp, dict) else None
    traffic = (ncu_traffic().get(f"{tkey}_dram_bytes_per_launch_{nx}x{ny}x{nz}_{split[0]}x{split[1]}")
               if split else None)
    roofline = {"kernel": f"fused {'type1 ' if t1 else ''}{kind} step", "bound": "hbm", "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                "traffic": traffic, "traffic_split": split,
                "alg_bytes_per_launch": alg_bytes,
                "avg_launch_ms": per_launch_s * 1e3, "launches": kn}
    passes = {k: {"total_ms": v[0] / args.steps, "launches_per_shot": v[1] / args.steps}
              for k, v in times.items()}
    if t1:
        elt = {"fp32": 4, "fp16": 2, "bf16": 2}[args.snap_precision]
        step_bytes = (2 * b_step + (2 * elt + 16) / args.xcorr + 2 * elt / args.xcorr) * npts
    else:
        step_bytes = ((2 * B_VTI if vti else B_FWD + B_ADJ) + B_IMG / args.xcorr + B_SNAP / args.xcorr) * npts
    hbm_frac = step_bytes * args.nt / (ms_per_step / 1e3) / 1e9 / peak

    # end to end through the host-buffer API
    e2e = None
    if not args.no_e2e:
        # the caller's host buffers, pinned: model parameters and observed
        # traces in, traces and images out
        def pinned(a=None, shape=None):
            h = torch.empty(a.shape if a is not None else shape, dtype=torch.float32, pin_memory=True).numpy()
            if a is not None:
                h[...] = a
            return h

        host_model = {k: pinned(v) for k, v in model.items()}
        obs_host = pinned(observed.cpu().numpy())
        tr, gv, gr = pinned(shape=(args.nt, nrec)), pinned(shape=(nz, ny, nx)), pinned(shape=(nz, ny, nx))
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sim.set_model(**host_model)
            sim.forward(tr)
            sim.adjoint_observed(obs_host)
            sim.image(gv, gr)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([el], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        h2d = int(len(host_model) * npts * 4 + args.nt * nrec * 4)
        d2h = int(args.nt * nrec * 4 + 2 * npts * 4)
        e2e = {"value": pts * args.steps * ws / el / 1e9, "unit": "Gpts/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "timer": "wall clock, synchronized on both sides",
               "host_buffers": "pinned"}
        del tr, gv, gr

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        r = cpu_sample(args, model, dt, w, src, rec)
        cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")}

    clocks = summarize_clocks(clk_file.name if clk_file else "", local)
    line = {
        "metric": METRIC, "value": value, "unit": "Gpts/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, see config)",
        "config": {**desc, "parallelism": f"shot-parallel x{ws}" if ws > 1 else "single GPU",
                   "path": "reference kernel sequence" if args.per_kernel else "fused step kernels",
                   "operator": ("centred constant-density (type1 kernels)" if args.scheme == 1
                                else "staggered variable-density (type2 kernels)"),
                   "snapshots": args.snap_precision,
                   "work_split": ({k.replace("type1_", ""): [v["bz"], v.get("ztop", 0)]
                                   for k, v in tuned.items() if isinstance(v, dict)}
                                  if tuned else "modelled")},
        "roofline": roofline, "hbm_frac_alg_per_step": hbm_frac,
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


# ---------------------------------------------------------------------------
SERVE_SIZES = [(96, 96, 96), (160, 160, 160), (224, 224, 160), (320, 320, 200)]


def serve_stream(args):
    """The served batch: arrival time, grid, steps, source and model seed per shot."""
    rng = np.random.default_rng(2024)
    t = np.cumsum(rng.exponential(1.0 / args.rate, args.shots))
    t -= t[0]
    out = []
    for i in range(args.shots):
        nx, ny, nz = SERVE_SIZES[rng.integers(len(SERVE_SIZES))]
        nt = int(rng.integers(args.nt_range[0], args.nt_range[1] + 1))
        src = (int(rng.integers(0, nx)), int(rng.integers(0, ny)), 2)
        out.append(dict(i=i, arrival=float(t[i]), nx=nx, ny=ny, nz=nz, nt=nt, src=src, seed=1000 + i))
    return out


def serve_shot(spec, keep_traces=False):
    """Shot object for one stream entry: layered VTI model of the seed (6 flat
    layers, vp 1500-4500, eps U[0,0.3], delta U[0,min(0.15,eps)]), 20-cell
    sponge, 15 Hz Ricker, dt from CFL 0.4, receivers every 4th cell of z=3."""
    from miniappsforhpe_b200 import earth_models as EM
    from miniappsforhpe_b200.serve import Shot

    nx, ny, nz, nt = spec["nx"], spec["ny"], spec["nz"], spec["nt"]
    m = EM.layered_vti(nx, ny, nz, nlayers=6, seed=spec["seed"])
    dt = EM.cfl_dt(m, 10.0, cfl=0.4)
    w = EM.ricker(nt, dt, 15.0) * 1e3
    rec = EM.receiver_plane(nx, ny, 3)
    rec = rec[(rec[:, 0] % 4 == 0) & (rec[:, 1] % 4 == 0)]
    return Shot(nx=nx, ny=ny, nz=nz, dt=dt, nt=nt, vp=m["vp"], eps=m["eps"], delta=m["delta"], wavelet=w,
                source=spec["src"], receivers=rec, sponge_width=20, want_traces=keep_traces)


def serve_run(args, stream, mode, keep):
    """Play the stream against a server; returns per-shot records."""
    import threading

    from miniappsforhpe_b200.serve import Server

    if mode == "served":
        srv = Server(max_active=args.max_active, round_ms=args.round_ms, use_graphs=True, autotune=True,
                     snap_precision="fp16")
    else:
        srv = Server(max_active=1, round_ms=200.0, use_graphs=False, autotune=False, snap_precision="fp32")
    # warm-up: one short shot per grid size (first-sight tuning and cost model)
    warm = []
    for k, (nx, ny, nz) in enumerate(SERVE_SIZES):
        spec = dict(i=-1, arrival=0.0, nx=nx, ny=ny, nz=nz, nt=16, src=(nx // 2, ny // 2, 2), seed=77 + k)
        sh = serve_shot(spec)
        warm.append((srv.submit(sh), sh))
    for t, _ in warm:
        srv.wait(t)
    tickets = {}
    errors = []

    def client():
        t0 = time.perf_counter()
        for spec in stream:
            sh = serve_shot(spec)
            dly = spec["arrival"] - (time.perf_counter() - t0)
            if dly > 0:
                time.sleep(dly)
            try:
                tickets[spec["i"]] = (srv.submit(sh), sh)
            except Exception as e:  # noqa: BLE001
                errors.append(repr(e))
                return

    th = threading.Thread(target=client)
    th.start()
    recs = []
    for spec in stream:
        while spec["i"] not in tickets:
            if errors:
                raise RuntimeError(errors[0])
            time.sleep(0.002)
        t, sh = tickets[spec["i"]]
        r = srv.wait(t)
        if r.status != 0:
            raise RuntimeError(f"shot {spec['i']} failed with status {r.status}")
        rec = dict(i=spec["i"], t_submit=r.t_submit, t_admit=r.t_admit, t_done=r.t_done, latency=r.latency,
                   ckpt=r.checkpoint_every, units=r.units, footprint=r.footprint)
        if spec["i"] in keep:
            rec["image"] = (sh.image_vp.copy(), sh.image_rho.copy())
        recs.append(rec)
        tickets[spec["i"]] = None
    th.join()
    stats = srv.stats()
    srv.close()
    return recs, stats


def plain_run(args, stream, keep):
    """The same stream one shot at a time in plain FP32 through the run-level
    call (tti_rtm_shot: a simulator created for the shot, fused FP32 kernels,
    FP32 snapshots, no graphs, no autotuning; checkpoints only for a shot
    whose snapshots would not fit the free HBM), in arrival order."""
    import torch

    import miniappsforhpe_b200 as P
    from miniappsforhpe_b200.serve import rtm_shot

    def options(spec):
        base = dict(nx=spec["nx"], ny=spec["ny"], nz=spec["nz"], nt=spec["nt"], xcorr_step=4, sponge_width=20)
        free = torch.cuda.mem_get_info()[0] - (2 << 30)
        full = P.Config(**base).footprint_bytes()
        if full <= free:
            return P.Config(**base), 0
        best = min(range(4, spec["nt"], 4), key=lambda k: P.Config(**base, checkpoint_every=k).footprint_bytes())
        return P.Config(**base, checkpoint_every=best), best

    for k, (nx, ny, nz) in enumerate(SERVE_SIZES):  # warm-up, as for the server
        spec = dict(i=-1, arrival=0.0, nx=nx, ny=ny, nz=nz, nt=16, src=(nx // 2, ny // 2, 2), seed=77 + k)
        rtm_shot(serve_shot(spec), options(spec)[0])
    shots = {spec["i"]: serve_shot(spec) for spec in stream}  # built ahead, as the client thread would
    recs = []
    busy = 0.0
    t0 = time.perf_counter()
    for spec in stream:
        now = time.perf_counter() - t0
        if now < spec["arrival"]:
            time.sleep(spec["arrival"] - now)
        sh = shots.pop(spec["i"])
        opts, ck = options(spec)
        ts = time.perf_counter()
        rtm_shot(sh, opts)
        te = time.perf_counter()
        busy += te - ts
        rec = dict(i=spec["i"], t_submit=spec["arrival"], t_admit=ts - t0, t_done=te - t0,
                   latency=te - t0 - spec["arrival"], ckpt=ck, units=0, footprint=opts.footprint_bytes())
        if spec["i"] in keep:
            rec["image"] = (sh.image_vp.copy(), sh.image_rho.copy())
        recs.append(rec)
    return recs, {"busy_ms": None, "wall_in_calls_s": busy}


def serve_summary(recs, stats, stream):
    if stats.get("busy_ms") is None:  # the plain loop: no server
        lat = np.array([r["latency"] for r in recs])
        span = max(r["t_done"] for r in recs) - min(r["t_submit"] for r in recs)
        pts = sum(s["nx"] * s["ny"] * s["nz"] * s["nt"] for s in stream)
        return {"shots": len(recs), "shots_per_hour": len(recs) / span * 3600.0, "makespan_s": span,
                "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                "mean_latency_s": float(lat.mean()), "gpts_per_s": pts / span / 1e9,
                "checkpointed_shots": int(sum(1 for r in recs if r["ckpt"])),
                "time_in_shot_calls_s": stats["wall_in_calls_s"]}
    lat = np.array([r["latency"] for r in recs])
    span = max(r["t_done"] for r in recs) - min(r["t_submit"] for r in recs)
    pts = sum(s["nx"] * s["ny"] * s["nz"] * s["nt"] for s in stream)
    return {"shots": len(recs), "shots_per_hour": len(recs) / span * 3600.0, "makespan_s": span,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()), "gpts_per_s": pts / span / 1e9,
            "checkpointed_shots": int(sum(1 for r in recs if r["ckpt"])),
            "device_busy_frac": stats["busy_ms"] / 1e3 / span, "rounds": stats["rounds"],
            "graph_updates": stats["graph_updates"], "graph_instantiations": stats["graph_instantiations"],
            "max_resident": stats["max_resident"], "device_gap_s": stats.get("gap_ms", 0.0) / 1e3,
            "host_round_build_s": stats.get("build_ms", 0.0) / 1e3, "host_setup_s": stats.get("setup_ms", 0.0) / 1e3,
            "host_setup_split_s": {k: stats.get(f"setup_{k}_ms", 0.0) / 1e3 for k in ("alloc", "model", "tune")}}


def run_serve(args):
    stream = serve_stream(args)
    keep = {s["i"] for s in stream if s["i"] % 4 == 0}
    modes = [m for m in args.serve_modes.split(",") if m]
    out, images = {}, {}
    for mode in modes:
        recs, stats = plain_run(args, stream, keep) if mode == "plain" else serve_run(args, stream, mode, keep)
        out[mode] = serve_summary(recs, stats, stream)
        images[mode] = {r["i"]: r["image"] for r in recs if "image" in r}
    line = {"metric": METRIC, "mode": "serve", "unit": "shots/hour",
            "value": out.get("served", out.get(modes[0]))["shots_per_hour"], "higher_is_better": True,
            "n_gpus": 1, "dtype": "f32 stencils, fp16 snapshots (served) / fp32 (plain, sequential)",
            "data": "synthetic (seeded)",
            "config": {"workload": f"served batch: {args.shots} TTI RTM shots, Poisson arrivals {args.rate}/s",
                       "sizes": SERVE_SIZES, "nt_range": args.nt_range, "max_active": args.max_active,
                       "round_ms": args.round_ms, "model": "layered VTI per shot seed (6 layers), 15 Hz Ricker",
                       "receivers": "every 4th cell of plane z=3", "sponge_width": 20,
                       "observed": "zero (residual = synthetic traces; work does not depend on the values)"},
            **out}
    base = "plain" if "plain" in out else "sequential"
    if "served" in out and "sequential" in out:
        line["served_vs_server_one_at_a_time"] = out["served"]["shots_per_hour"] / out["sequential"]["shots_per_hour"]
    if "served" in out and base in out:
        line["speedup_shots_per_hour"] = out["served"]["shots_per_hour"] / out[base]["shots_per_hour"]
        e = []
        for i, (gv, gr) in images["served"].items():
            rv, rr = images[base][i]
            e.append((float(np.linalg.norm((gv - rv).astype(np.float64)) / max(np.linalg.norm(rv), 1e-30)),
                      float(np.linalg.norm((gr - rr).astype(np.float64)) / max(np.linalg.norm(rr), 1e-30))))
        line["image_rel_l2_served_vs_fp32"] = {"shots_compared": len(e), "max_vp": max(x[0] for x in e),
                                               "max_rho": max(x[1] for x in e)}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.serve:
        run_serve(args)
        return
    if args.elastic:
        run_elastic(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
