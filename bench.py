#!/usr/bin/env python
"""Benchmark of x3div's Euler-timestep hot path on B200.

Workload (one "step"): the plain derivative sweep of a 512^3 periodic box --
u, v, w = Taylor-Green field + seeded Gaussian noise (amplitude 1e-3), and
for each field and each direction the six compact operator families (first
derivative, second derivative, staggered derivative v->p and p->v,
interpolation v->p and p->v), each an explicit stencil + cyclic Thomas solve
over all 512^2 lines of the direction: 54 operator applications per step.

  value    : derivative Gpts/s of the FP32-mixed path (FP32 fields and
             sweeps; operator coefficients computed in FP64), inputs
             resident in HBM, CUDA events on the launching stream, max over
             ranks.  The plain FP64 path's figure is under "fp64", and the
             full Euler step (transeq + int_time + divergence + FP64 Poisson
             + gradp + cor_vel) in ms under "euler_step_ms".
  e2e      : the same sweep through x3d_apply_batch with pinned HOST buffers:
             each field uploaded once, all 18 of its outputs downloaded.
  roofline : the dominant line-solve kernel, algorithmic bytes (one read +
             one write of the field per application) / its average launch
             time, against the measured HBM copy bandwidth.

--impl reference times the reference's algorithm on the host cores: the
reference (Fortran + MPI + 2decomp&FFT) cannot be built in this image, so
this is the FP64 C restatement in oracle/ (OpenMP, all host threads) on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "derivative Gpts/s and Euler-step ms at 512^3: FP32-mixed vs FP64, 1 B200"
KINDS = [("der", ("derx", "dery", "derz")), ("der2", ("derxx", "deryy", "derzz")),
         ("dervp", ("derxvp", "deryvp", "derzvp")), ("derpv", ("derxpv", "derypv", "derzpv")),
         ("intvp", ("intxvp", "intyvp", "intzvp")), ("intpv", ("intxpv", "intypv", "intzpv"))]
FAMILY = {0: "ls_stage_x", 1: "ls_stage_yz(y)", 2: "ls_stage_yz(z)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--no-euler", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--profile-timed", nargs="?", const="sweep", default=None,
                    choices=["sweep", "euler", "euler64", "b48", "poisson"],
                    help="bracket the timed FP32 sweep (or the FP32-mixed Euler steps, the FP64 ones, the "
                         "batch replays, or the --poisson-times solves through the own x transforms) with "
                         "cudaProfilerStart/Stop, for ncu --profile-from-start off")
    ap.add_argument("--poisson-times", action="store_true",
                    help="only time the FP64 Poisson solve on an n^3 box, through the library's own x "
                         "transforms and through cuFFT's 2-D (x, y) transforms, and print one JSON line")
    ap.add_argument("--kernel-config", type=int, default=None,
                    help="force one kernel configuration (x3d_ctx_set_kernel) instead of autotuning")
    ap.add_argument("--no-b48", action="store_true")
    ap.add_argument("--b48-count", type=int, default=48,
                    help="boxes in the batching workload (the first of the same seeded draw; 48 by default)")
    ap.add_argument("--no-c5", action="store_true",
                    help="skip the 768^3 long run (20 Euler steps, FP32-mixed and FP64, reported under c5)")
    return ap.parse_args()


def tg_noise(n, seed, amp=1e-3):
    """Taylor-Green velocity + N(0, amp^2) noise on an n^3 box of side 2 pi,
    returned as a C-contiguous (z, y, x) float64 array (= Fortran (x, y, z))."""
    rng = np.random.default_rng(seed)
    x = np.arange(n) * (2 * np.pi / n)
    s, c = np.sin(x), np.cos(x)
    comp = seed % 3
    if comp == 0:      # u = sin x cos y cos z
        f = c[:, None, None] * c[None, :, None] * s[None, None, :]
    elif comp == 1:    # v = -cos x sin y cos z
        f = -c[:, None, None] * s[None, :, None] * c[None, None, :]
    else:              # w = 0
        f = np.zeros((n, n, n))
    f = f + amp * rng.standard_normal((n, n, n))
    return np.ascontiguousarray(f)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = [r.split(",") for r in out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # each reason column reads "Active" or "Not Active"
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        load = [v for v in sm if mx and v > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of each line-solve kernel from the committed ncu
    summary (profiles/linesolve_traffic.json), scaled to this size."""
    p = os.path.join(ROOT, "profiles", "linesolve_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    elif args.impl == "b200":
        torch.cuda.set_device(local)
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------
def sample_ops(s):
    """(oracle kind, direction) of the three applications of CPU sample step s."""
    return [(KINDS[(s + 2 * d) % 6][0], d) for d in range(3)]


def cpu_sample(n, reps=1, start=0):
    """The oracle on a bounded sample of the sweep: per step three of the 54
    applications, one per direction, on one n^3 FP64 field with all host
    threads.  Step s applies family (s + 2 d) mod 6 along direction d, so six
    consecutive steps visit all 18 family x direction pairs once (the
    sweep's operator mix); start is the first step's index."""
    from oracle import oracle as O
    O.lib()
    f = np.asfortranarray(tg_noise(n, 0).transpose(2, 1, 0))
    d = 2 * np.pi / n
    times = []
    for s in range(start, start + reps):
        t0 = time.perf_counter()
        for kind, di in sample_ops(s):
            O.apply(kind, di, f, d)
        times.append(time.perf_counter() - t0)
    pts = 3.0 * n ** 3
    return pts, times


ROTATION = ("step s applies operator family (s + 2 d) mod 6 of (der, der2, dervp, derpv, intvp, intpv) "
            "along direction d, so every 6 steps visit all 18 family x direction pairs of the sweep once")


def cpu_threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def run_reference(args, world, rank):
    if rank != 0:
        return
    n = args.n
    sample = (f"oracle/ (FP64 C restatement, OpenMP) applying 3 of the 54 applications of a sweep step "
              f"to one {n}^3 field per step, one per direction, rotating: {ROTATION}")
    pts, _ = cpu_sample(n, reps=max(1, args.warmup), start=0)
    pts, times = cpu_sample(n, reps=args.steps, start=0)
    t = sum(times)
    val = pts * args.steps / t / 1e9
    cores = cpu_threads()
    line = {
        "metric": METRIC, "value": round(val, 4), "unit": "Gpts/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t / args.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"periodic compact derivative sweep, {n}^3, TG + 1e-3 noise",
                   "sample": sample, "parallelism": f"{cores} host threads"},
        "cpu_baseline": {"value": round(val, 4), "unit": "Gpts/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(val, 4), "unit": "Gpts/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "reference Fortran/MPI build unavailable (no gfortran, MPI or 2decomp&FFT); "
                "timed the oracle restatement of its algorithm",
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
def sweep_groups(ctx, fields, outs, fused):
    """The 54 applications of one step, as (direction, [(op, in, out), ...])
    groups: with fused=True the six operator families of one field and one
    direction form one group (one multi-output launch), else one group per
    application."""
    groups = []
    k = 0
    for f in fields:
        for d in range(3):
            g = []
            for kind, names in KINDS:
                g.append((ctx.op(names[d]), f, outs[k % len(outs)]))
                k += 1
            if fused:
                groups.append((d, g))
            else:
                groups.extend((d, [it]) for it in g)
    return groups


# Lines per tile (W) of each chunked configuration (x3d_ctx_set_kernel 0..15
# and 17..20; 16 is one thread per line).
CONFIG_W = [16, 32, 16, 8, 32, 8, 16, 32, 16, 8, 32, 8, 32, 16, 32, 32, 1, 16, 8, 8, 16]


def config_pattern(cfg, d):
    """The roofline probe pattern with the access order of configuration cfg
    along y (d = 1) or z (d = 2): whole-line tiles of W columns taken in
    order -- claimed from a counter by the persistent configurations, and
    dispatched in block order by the hardware for the one-CTA-per-tile ones,
    which keeps the tiles in flight a window of consecutive tiles as well."""
    w = CONFIG_W[cfg] if 0 <= cfg < len(CONFIG_W) and cfg != 16 else 16
    return f"claim_w{w}" if d == 1 else f"claimz_w{w}"


def pattern_ceilings(ctx, torch, src, outs):
    """Bandwidth of one read and six writes with no arithmetic
    (x3d_roofline_probe), flat, in the y stage kernels' tile order for
    W = 8 .. 128 columns over whole lines, over blocks of 128 rows, and with
    the tiles claimed in order from a counter as the persistent stage kernels
    take them, along y lines (claim_w) and along z lines (claimz_w): what the
    sweep launches' traffic mix and access order can reach on this GPU
    (best over 1, 2, 4 and 8 CTAs per SM of 5 timed launches after 3 warm-up
    ones)."""
    nz, ny, nx = src.shape
    bytes_moved = 7 * src.numel() * src.element_size()
    res = {}
    cases = [("flat", 0, 0)] + [(f"tile_w{w}", 1, w) for w in (8, 16, 32, 64, 128)] + \
            [(f"block128_w{w}", 2, w) for w in (32, 64, 128)] + [(f"claim_w{w}", 5, w) for w in (8, 16, 32)] + \
            [(f"claimz_w{w}", 6, w) for w in (8, 16, 32)]
    for key, pattern, w in cases:
        rt = 16 if w == 128 else 32
        rows = 128 if pattern == 2 else ny
        if pattern and (nx % w or ny % rows or rows % rt or (w // max(1, w // 32)) * (rows // rt) > 512):
            continue
        best = None
        for per_sm in (1, 2, 4, 8):
            run = lambda: ctx.roofline_probe(pattern, w, src, outs, per_sm)  # noqa: E731
            for _ in range(3):
                run()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            for _ in range(5):
                a.record()
                run()
                b.record()
                b.synchronize()
                ms = a.elapsed_time(b)
                best = ms if best is None else min(best, ms)
        res[key] = round(bytes_moved / (best * 1e-3) / 1e9, 1)
    return res


def timed_sweep(ctx, torch, fields, outs, steps, warmup, world, fused=True, per_launch=True, profile=False):
    from x3div_b200._capi import Work
    groups = sweep_groups(ctx, fields, outs, fused)
    stream = torch.cuda.current_stream()
    L = ctx.L
    h = ctx.handle
    arrs = []
    for d, g in groups:
        arr = (Work * len(g))()
        for k, (op, src, dst) in enumerate(g):
            arr[k].op, arr[k].in_, arr[k].out = op.handle, src.data_ptr(), dst.data_ptr()
        arrs.append((d, arr, len(g)))

    def run(arr, n):
        rc = L.x3d_apply_batch(h, arr, n)
        if rc:
            ctx._check(rc)

    for _ in range(warmup):
        for d, arr, n in arrs:
            run(arr, n)
    ctx.sync()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps * len(arrs))] if per_launch else []
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0 = ctx.launch_count()
    if profile:
        torch.cuda.profiler.start()
    t0.record(stream)
    k = 0
    for _ in range(steps):
        for d, arr, n in arrs:
            if per_launch:
                ev[k][0].record(stream)
            run(arr, n)
            if per_launch:
                ev[k][1].record(stream)
            k += 1
    t1.record(stream)
    torch.cuda.synchronize()
    ctx.sync()
    if profile:
        torch.cuda.profiler.stop()
    launches = ctx.launch_count() - c0
    ms = t0.elapsed_time(t1)
    fam = {}
    if per_launch:
        for k, (d, arr, n) in enumerate(arrs * steps):
            fam.setdefault(d, []).append(ev[k][0].elapsed_time(ev[k][1]))
    barrier(world)
    group = len(groups[0][1])
    return ms, fam, sum(len(g) for _, g in groups), launches, group


def poisson_times(torch, n, steps, warmup, profile=False, seed=7):
    """One FP64 x3d_poisson solve on an n^3 periodic box of side 2 pi (a
    seeded N(0, 1) right-hand side, solved in place), timed with CUDA events
    over `steps` solves after `warmup`: through the library's own x
    transforms (the default) and through cuFFT's 2-D (x, y) transforms
    around the same fused z kernel (stage choice poisson_x = 0)."""
    from x3div_b200 import Context
    gen = torch.Generator(device="cuda").manual_seed(seed)
    base = torch.randn(n, n, n, dtype=torch.float64, device="cuda", generator=gen)
    out = {}
    for name, choice in (("own_x_transforms", -1), ("cufft_2d_xy", 0)):
        ctx = Context(n, n, n, lengths=(2 * np.pi,) * 3, precision="f64", stream=torch.cuda.current_stream())
        ctx.set_stage_choice("poisson_x", choice)
        rhs = base.clone()
        for _ in range(warmup):
            ctx.poisson(rhs)
        torch.cuda.synchronize()
        prof = profile and choice == -1
        if prof:
            torch.cuda.profiler.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            ctx.poisson(rhs)
        e1.record()
        torch.cuda.synchronize()
        if prof:
            torch.cuda.profiler.stop()
        out[name] = round(e0.elapsed_time(e1) / steps, 4)
        ctx.close()
        del rhs
    return {"poisson_ms": out, "grid": [n, n, n], "steps": steps, "warmup": warmup, "dtype": "f64"}


def run_c5(torch, n=768, steps=20, dt=5e-4, seed=5):
    """Long-run check at 768^3: 20 Euler steps (dt = 5e-4) from the same
    Taylor-Green + N(0, (1e-3)^2) field with FP32 derivatives (FP64 Poisson)
    and with the FP64 path, after the autotuner and the Poisson solve's
    one-time setup.  Reports ms per step, the divergence left after
    the last step (max |div u|) and the kinetic-energy drift of each, and the
    FP32-mixed / FP64 divergence ratio (the bar is <= 10)."""
    from x3div_b200 import Context
    out = {"grid": [n, n, n], "steps": steps, "dt": dt}
    x = torch.arange(n, device="cuda", dtype=torch.float64) * (2 * np.pi / n)
    g = torch.Generator(device="cuda")
    res = {}
    for prec, dtype in (("f32_mixed", torch.float32), ("f64", torch.float64)):
        c = Context(n, n, n, lengths=(2 * np.pi,) * 3, precision="f32" if dtype == torch.float32 else "f64",
                    stream=torch.cuda.current_stream())
        c.autotune(1)
        tg = [torch.cos(x)[:, None, None] * torch.cos(x)[None, :, None] * torch.sin(x)[None, None, :],
              -torch.cos(x)[:, None, None] * torch.sin(x)[None, :, None] * torch.cos(x)[None, None, :],
              torch.zeros(n, n, n, device="cuda", dtype=torch.float64)]
        U = []
        for f in range(3):
            g.manual_seed(seed * 10 + f)
            U.append((tg[f] + 1e-3 * torch.randn(n, n, n, device="cuda", dtype=torch.float64,
                                                  generator=g)).to(dtype).contiguous())
        del tg
        du = [torch.empty_like(U[0]) for _ in range(3)]
        pg = [torch.empty_like(U[0]) for _ in range(3)]
        pp3 = torch.zeros((n, n, n), dtype=torch.float64, device="cuda")
        # the solve's one-time setup (spectrum, cuFFT plan, tables) before the
        # timed steps: a solve on the scratch pressure, which every step
        # overwrites with the divergence
        c.poisson(pp3)
        ke = lambda: 0.5 * sum(float((u.double() ** 2).mean()) for u in U)
        ke0 = ke()
        c.sync()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            c.euler_step(*U, *du, pp3, *pg, dt)
        b.record()
        torch.cuda.synchronize()
        c.sync()
        c.divergence(pp3, *U)
        mx, _ = c.div_stats(pp3)
        res[prec] = {"ms_per_step": round(a.elapsed_time(b) / steps, 2), "div_max_after": mx,
                     "ke_drift": (ke() - ke0) / ke0}
        c.close()
        del U, du, pg, pp3
        torch.cuda.empty_cache()
    out.update(res)
    out["div_ratio_f32_over_f64"] = res["f32_mixed"]["div_max_after"] / max(res["f64"]["div_max_after"], 1e-300)
    return out


def run_b48(args, world, rank, local, torch):
    """The batching workload: 48 seeded uneven periodic boxes (this rank's LPT
    share), 3 FP32 fields each (Taylor-Green + N(0, (1e-2)^2)), all 54 operator
    applications per box in one persistent launch, its chunk length and tile
    width tuned per box shape and direction (x3d_batch_autotune), replayed
    from a CUDA graph."""
    from x3div_b200 import Batch, b48_boxes, box_points, shard_boxes
    boxes = b48_boxes(count=args.b48_count)
    mine = shard_boxes(boxes, world)[rank]
    my = [boxes[i] for i in mine]
    g = torch.Generator(device="cuda")
    fields, outs = [], []
    for i, b in zip(mine, my):
        nx, ny, nz = b
        x = torch.arange(nx, device="cuda", dtype=torch.float64) * (2 * np.pi / nx)
        y = torch.arange(ny, device="cuda", dtype=torch.float64) * (2 * np.pi / ny)
        z = torch.arange(nz, device="cuda", dtype=torch.float64) * (2 * np.pi / nz)
        tg = [torch.cos(z)[:, None, None] * torch.cos(y)[None, :, None] * torch.sin(x)[None, None, :],
              -torch.cos(z)[:, None, None] * torch.sin(y)[None, :, None] * torch.cos(x)[None, None, :],
              torch.zeros(nz, ny, nx, device="cuda", dtype=torch.float64)]
        fs = []
        for f in range(3):
            g.manual_seed(1000 * i + f)
            fs.append((tg[f] + 1e-2 * torch.randn(nz, ny, nx, device="cuda", dtype=torch.float64,
                                                   generator=g)).to(torch.float32).contiguous())
        fields.append(fs)
        outs.append([[[torch.empty_like(fs[0]) for _ in range(6)] for _ in range(3)] for _ in range(3)])
    batch = Batch(my, precision="f32", device=local, stream=torch.cuda.current_stream())
    batch.bind_sweep(fields, outs)
    batch.autotune()
    info = batch.info()
    # per box shape: (chunk length, lines per tile) along x, y, z
    choices = {}
    for k, b in enumerate(my):
        key = "x".join(str(v) for v in b[:3])
        if key not in choices:
            choices[key] = [list(batch.choice(k, d)) for d in range(3)]
    batch.capture()
    for _ in range(args.warmup):
        batch.replay()
    batch.sync()
    torch.cuda.synchronize()
    barrier(world)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.profile_timed == "b48":
        torch.cuda.profiler.start()
    a.record()
    for _ in range(args.steps):
        batch.replay()
    b.record()
    torch.cuda.synchronize()
    if args.profile_timed == "b48":
        torch.cuda.profiler.stop()
    batch.sync()
    ms = max_over_ranks(a.elapsed_time(b), world)
    pts = torch.tensor([float(info["points"])], dtype=torch.float64, device="cuda")
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(pts, op=dist.ReduceOp.SUM)
    tot_points = float(pts.item())
    res = {"value": round(tot_points * args.steps / (ms * 1e-3) / 1e9, 2), "unit": "Gpts/s",
           "ms_per_step": round(ms / args.steps, 3), "boxes": len(boxes), "boxes_this_rank": len(my),
           "points_per_step": int(tot_points), "tiles_per_launch": info["tiles"],
           "jobs_in_persistent_launch": info["jobs"], "fallback_jobs": info["fallback_jobs"],
           "launches_per_step": (1 if info["jobs"] else 0) + info["fallback_jobs"],
           "cuda_graph": True,
           "tuned_per_shape_chunk_and_lines_xyz": choices,
           "bytes_per_step": int(tot_points / 6 * 4 * (1 + 6))}
    batch.close()
    del fields, outs
    torch.cuda.empty_cache()
    return res


def run_b200(args, world, rank, local):
    import torch

    from x3div_b200 import Context
    n = args.n
    npts = n ** 3
    peak, peak_kind = measured_peak()
    clocks = Clocks(local)
    out = {}

    # ---- FP32-mixed sweep (headline) ---------------------------------------
    ctx = Context(n, n, n, lengths=(2 * np.pi,) * 3, precision="f32", device=local,
                  stream=torch.cuda.current_stream())
    if args.kernel_config is not None:
        ctx.set_kernel(args.kernel_config)
    elif not args.no_autotune:
        ctx.autotune(6)
    host = [tg_noise(n, s + 3 * rank) for s in range(3)]
    fields = [torch.from_numpy(h).to(device="cuda", dtype=torch.float32) for h in host]
    outs = [torch.empty_like(fields[0]) for _ in range(18)]
    clocks.start()
    ms, fam, nitems, launches, group = timed_sweep(ctx, torch, fields, outs, args.steps,
                                                   args.warmup, world, fused=True,
                                                   profile=args.profile_timed == "sweep")
    ms = max_over_ranks(ms, world)
    pts_step = nitems * npts
    value = world * pts_step * args.steps / (ms * 1e-3) / 1e9
    es = 4
    per_launch_bytes = (1 + group) * npts * es  # one read, one write per operator
    fam_stats = {}
    for d, ts in fam.items():
        avg = sum(ts) / len(ts)
        fam_stats[FAMILY[d]] = {"launches": len(ts), "avg_ms": round(avg, 4),
                                "gbs": round(per_launch_bytes / (avg * 1e-3) / 1e9, 1),
                                "share": round(sum(ts) / sum(sum(v) for v in fam.values()), 3),
                                "config": ctx.autotune_choice(d, group)}
    dom_d = max(fam, key=lambda d: sum(fam[d]))
    dom = fam_stats[FAMILY[dom_d]]
    traffic = profiled_traffic().get(f"{FAMILY[dom_d]}:f32:group{group}")
    traffic_bytes = traffic["bytes_per_point"] * npts if traffic else None
    roofline = {"bound": "hbm", "achieved": dom["gbs"], "peak": peak, "unit": "GB/s",
                "frac": round(dom["gbs"] / peak, 3), "traffic": traffic_bytes,
                "kernel": FAMILY[dom_d] + f" ({group} operators per launch)",
                "algorithmic_bytes_per_launch": per_launch_bytes, "peak_source": peak_kind}
    # the same traffic with no arithmetic, in the dominant launch's order
    ceil = pattern_ceilings(ctx, torch, fields[0], outs[:6])
    if ceil:
        cfg = dom["config"]
        key = "flat" if FAMILY[dom_d] == "ls_stage_x" else config_pattern(cfg, dom_d)
        if key in ceil:
            roofline["pattern_ceiling_gbs"] = ceil[key]
            roofline["pattern"] = key
            roofline["frac_of_pattern"] = round(dom["gbs"] / ceil[key], 3)
    out["ceilings"] = ceil
    out.update(value=value, ms=ms, fam=fam_stats, roofline=roofline, launches=launches)
    # the same 54 applications one operator per launch
    ms1, fam1, _, launches1, _ = timed_sweep(ctx, torch, fields, outs, args.steps, args.warmup,
                                             world, fused=False)
    ms1 = max_over_ranks(ms1, world)
    out["unfused"] = {"value": round(world * pts_step * args.steps / (ms1 * 1e-3) / 1e9, 2),
                      "ms_per_step": round(ms1 / args.steps, 3), "launches": launches1,
                      "kernels": {FAMILY[d]: {"avg_ms": round(sum(ts) / len(ts), 4),
                                              "gbs": round(2 * npts * es / (sum(ts) / len(ts) * 1e-3) / 1e9, 1),
                                              "config": ctx.autotune_choice(d, 1)}
                                  for d, ts in fam1.items()}}

    # ---- e2e: host buffers through x3d_apply_batch ---------------------------
    if not args.no_e2e:
        pin_in = [torch.from_numpy(h.astype(np.float32)).pin_memory() for h in host]
        pin_out = [torch.empty((n, n, n), dtype=torch.float32).pin_memory() for _ in range(18)]
        e2e_steps = max(1, min(args.steps, 2))

        def e2e_step():
            for f in pin_in:
                items = []
                k = 0
                for kind, names in KINDS:
                    for name in names:
                        items.append((ctx.op(name), f.numpy(), pin_out[k].numpy()))
                        k += 1
                ctx.apply_batch(items)

        e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        t = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        el = max_over_ranks(time.perf_counter() - t, world)
        out["e2e"] = {"value": round(world * pts_step * e2e_steps / el / 1e9, 3), "unit": "Gpts/s",
                      "h2d_bytes_per_step": 3 * npts * 4, "d2h_bytes_per_step": nitems * npts * 4,
                      "api": "x3d_apply_batch with pinned host buffers"}
        del pin_in, pin_out
    del fields, outs

    # ---- Euler step, FP32-mixed ---------------------------------------------
    def euler_ms(c, dt_torch, profile=False):
        U = [torch.from_numpy(h).to(device="cuda", dtype=dt_torch) for h in host]
        du = [torch.empty_like(U[0]) for _ in range(3)]
        pg = [torch.empty_like(U[0]) for _ in range(3)]
        pp3 = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
        for _ in range(2):
            c.euler_step(*U, *du, pp3, *pg, 5e-4)
        c.sync()
        barrier(world)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        if profile:
            torch.cuda.profiler.start()
        a.record()
        for _ in range(reps):
            c.euler_step(*U, *du, pp3, *pg, 5e-4)
        b.record()
        torch.cuda.synchronize()
        if profile:
            torch.cuda.profiler.stop()
        c.sync()
        c.divergence(pp3, *U)
        mx, mean = c.div_stats(pp3)
        stages = c.stage_choices()
        return max_over_ranks(a.elapsed_time(b) / reps, world), mx, stages

    if not args.no_euler:
        out["euler_f32"] = euler_ms(ctx, torch.float32, profile=args.profile_timed == "euler")
    ctx.close()
    torch.cuda.empty_cache()

    # ---- plain FP64 path -------------------------------------------------------
    if not args.no_fp64:
        ctx64 = Context(n, n, n, lengths=(2 * np.pi,) * 3, precision="f64", device=local,
                        stream=torch.cuda.current_stream())
        if args.kernel_config is not None:
            ctx64.set_kernel(args.kernel_config)
        elif not args.no_autotune:
            ctx64.autotune(6)
        fields = [torch.from_numpy(h).to(device="cuda") for h in host]
        outs = [torch.empty_like(fields[0]) for _ in range(18)]
        ms64, fam64, _, l64, g64 = timed_sweep(ctx64, torch, fields, outs, args.steps, args.warmup,
                                               world, fused=True)
        ms64 = max_over_ranks(ms64, world)
        f64 = {"value": round(world * pts_step * args.steps / (ms64 * 1e-3) / 1e9, 2),
               "ms_per_step": round(ms64 / args.steps, 3), "launches": l64}
        f64["kernels"] = {FAMILY[d]: {"avg_ms": round(sum(ts) / len(ts), 4),
                                      "gbs": round((1 + g64) * npts * 8 / (sum(ts) / len(ts) * 1e-3) / 1e9, 1),
                                      "config": ctx64.autotune_choice(d, g64)}
                          for d, ts in fam64.items()}
        ms64u, _, _, l64u, _ = timed_sweep(ctx64, torch, fields, outs, args.steps, args.warmup,
                                           world, fused=False, per_launch=False)
        ms64u = max_over_ranks(ms64u, world)
        f64["unfused"] = {"value": round(world * pts_step * args.steps / (ms64u * 1e-3) / 1e9, 2),
                          "ms_per_step": round(ms64u / args.steps, 3), "launches": l64u}
        out["fp64"] = f64
        del fields, outs
        if not args.no_euler:
            out["euler_f64"] = euler_ms(ctx64, torch.float64, profile=args.profile_timed == "euler64")
        ctx64.close()
    if not args.no_b48:
        out["b48"] = run_b48(args, world, rank, local, torch)
    out["clocks"] = clocks.stop()
    if not args.no_c5 and rank == 0:
        out["c5"] = run_c5(torch)
    return out, pts_step


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.poisson_times:
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps(poisson_times(torch, args.n, args.steps, args.warmup,
                                           profile=args.profile_timed == "poisson")), flush=True)
        return
    res, pts_step = run_b200(args, world, rank, local)
    if rank == 0:
        n = args.n
        sample_n = min(n, 512)
        pts, times = cpu_sample(sample_n, reps=6)
        cpu_val = pts * len(times) / sum(times) / 1e9
        line = {
            "metric": METRIC,
            "value": round(res["value"], 2),
            "unit": "Gpts/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(res["ms"] / args.steps, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (operator coefficients computed in f64)",
            "data": "synthetic",
            "config": {"workload": f"periodic compact derivative sweep, {n}^3 per GPU, 3 fields x "
                                   "6 operator families x 3 directions = 54 line-solve applications "
                                   "per step, the 6 families of one field and direction fused into "
                                   "one launch", "grid": [n, n, n], "fields": "Taylor-Green + seeded N(0, (1e-3)^2) noise",
                       "l2": "inputs (0.5 GB per field) larger than L2; no flush",
                       "parallelism": f"{world} independent box(es), one per GPU"},
            "gpu_launches": res["launches"],
            "roofline": res["roofline"],
            "pattern_ceilings_gbs": res.get("ceilings"),
            "kernels": res["fam"],
            "unfused": res["unfused"],
            "cpu_baseline": {"value": round(cpu_val, 4), "unit": "Gpts/s", "cores": cpu_threads(),
                             "kind": "port",
                             "sample": f"oracle (FP64 C, OpenMP) on one {sample_n}^3 field, 6 steps of 3 "
                                       f"applications: {ROTATION}"},
        }
        if "e2e" in res:
            line["e2e"] = res["e2e"]
        if "fp64" in res:
            line["fp64"] = res["fp64"]
        em = {}
        if "euler_f32" in res:
            em["f32_mixed"] = round(res["euler_f32"][0], 2)
            em["f32_mixed_div_after_max"] = res["euler_f32"][1]
            em["f32_stage_configs"] = res["euler_f32"][2]
        if "euler_f64" in res:
            em["f64"] = round(res["euler_f64"][0], 2)
            em["f64_div_after_max"] = res["euler_f64"][1]
            em["f64_stage_configs"] = res["euler_f64"][2]
        if em:
            line["euler_step_ms"] = em
        if "b48" in res:
            line["b48"] = res["b48"]
        if "c5" in res:
            line["c5"] = res["c5"]
        if res.get("clocks"):
            line["clocks"] = res["clocks"]
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
