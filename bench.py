"""Benchmark of the SE3P k-space solve on B200 (one JSON line on stdout).

Workload (default, the configuration the headline metric is quoted on):
SE3P FORCE, N = 100,000 charges uniform in the unit box, charges uniform in
[-1, 1] shifted to zero sum, M = 128^3, P = 16, xi = 20, m = 0.94 sqrt(pi P);
FP32 spread/interpolation with compensated accumulation, FP64 FFT and
Green's-function scaling.  A step is one full solve (sort, spread + fold,
D2Z, scaling, Z2D, unfold + interpolation) of that system.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c1|c2|c3|c4|c5] [--no-extra]

Timing: W untimed steps, then K steps each timed with CUDA events on the
solve's stream; a 256 MiB buffer is written between steps so every step
starts with a cold L2 (the inputs, 3.2 MB, and grids, 50 MB, would fit in it).
The solves replay their CUDA graph (se_plan_set_graph, the repeated-solve
launch mode); `direct_launch_ms_per_step` times the same solves launched
one kernel at a time.
Under torchrun every rank solves its own replica (weak scaling); the time is
the max over ranks.  `e2e` repeats the measurement through se_solve_host with
pinned host buffers (H2D of x, q and D2H of the forces inside the timed
region).  `--impl reference` times SE_fast_gridding's own CPU spectral_ewald()
(built from its sources) on all host cores instead.

On one GPU the line also carries the other configurations of the metric as
sub-records, each with its own timing, accuracy and roofline: `c3` (256
batched POTENTIAL systems), `c4` (the serving loop under Poisson arrivals:
solves/s, p50/p99) and `c5` (16M clustered FORCE particles, M = 512).
`--workload cN` prints that configuration alone as its own line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(N=100_000, M=128, P=16, L=1.0, xi=20.0, mode="force", precision="fp32",
                charges="uniform", seed=1)
METRIC = "SE3P particles/s at rel-RMS<=1e-6 vs FP64 oracle; serve solves/s, p50/p99"
FALLBACK_HBM_GBS = 6650.0
STAGES = ("sort", "spread", "kspace", "interp")


def workload_name(w):
    return (f"SE3P {w['mode'].upper()} N={w['N']} M={w['M']}^3 P={w['P']} xi={w['xi']} "
            f"L={w['L']}, rel-RMS<=1e-6 vs the FP64 path")


def workload_config(w):
    """The configuration both arms report (what is solved, not how)."""
    return {"workload": workload_name(w), "N": w["N"], "M": w["M"], "P": w["P"],
            "xi": w["xi"], "L": w["L"], "mode": w["mode"],
            "l2": "GPU arm: flushed between steps (256 MiB write); CPU arm: not applicable"}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference(args, procs, threads, steps, warmup, w):
    cmd = [sys.executable, os.path.join(ROOT, "oracle", "ref_bench.py"),
           "--N", str(w["N"]), "--M", str(w["M"]), "--P", str(w["P"]), "--L", str(w["L"]),
           "--xi", str(w["xi"]), "--mode", w["mode"], "--charges", w["charges"],
           "--seed", str(w["seed"]), "--procs", str(procs), "--threads", str(threads),
           "--steps", str(steps), "--warmup", str(warmup)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    return json.loads(r.stdout.strip().splitlines()[-1])


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        for ln in self.lines:
            f = [s.strip() for s in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic():
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


_FMA_PEAK = None


def fma_peak():
    global _FMA_PEAK
    if _FMA_PEAK is None:
        from se_fast_gridding_b200 import solver
        _FMA_PEAK = solver.fma_peak_tflops()
    return _FMA_PEAK


def kernel_work(stage, systems, precision):
    """Algorithmic bytes and flops of one launch of the spread or the
    interpolation over `systems` ((N, M, P, mode) tuples):
      spread  bytes N (3 + 1) 8 (positions, charge) + M^3 8 (the FP64 grid,
              written once, fold fused); flops 2 P^3 N (one FMA per point);
      interp  bytes M^3 s (the grid, s = 4 on the FP32 path, which reads its
              FP32 copy) + N 32 + N 8 w (w = 1 POTENTIAL, 3 FORCE);
              flops 2 P^3 N POTENTIAL, 4 P^3 N FORCE (two FMAs per point:
              the value and the derivative-weighted sum along z)."""
    s_grid = 4 if precision.startswith("fp32") else 8
    b = f = 0.0
    for N, M, P, mode in systems:
        w = 3 if mode == "force" else 1
        if stage == "spread":
            b += N * 32 + M ** 3 * 8
            f += 2.0 * P ** 3 * N
        else:
            b += M ** 3 * s_grid + N * 32 + N * 8 * w
            f += (4.0 if mode == "force" else 2.0) * P ** 3 * N
    return b, f


def roofline_of(stage_ms, systems, precision, kname, traffic=None):
    """Rooflines of the dominant kernel (spread or interpolation, whichever
    took longer): HBM (algorithmic bytes / stage time) against the measured
    copy bandwidth, and FP32 FMA (algorithmic flops / stage time) against
    the measured FMA-chain peak."""
    hbm, kind = measured_peaks()
    dom = max(("spread", "interp"), key=lambda k: stage_ms[k])
    b, f = kernel_work(dom, systems, precision)
    t = stage_ms[dom] * 1e-3
    peak_f = fma_peak()
    return ({"kernel": kname(dom), "bound": "hbm", "achieved": b / t / 1e9, "peak": hbm,
             "unit": "GB/s", "frac": b / t / 1e9 / hbm,
             "traffic": None if traffic is None else traffic.get(dom),
             "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured"
             else "fallback 6650 GB/s", "algorithmic_bytes": b},
            {"kernel": kname(dom), "bound": "fp32_fma", "achieved": f / t / 1e12, "peak": peak_f,
             "unit": "TFLOP/s", "frac": f / t / 1e12 / peak_f, "algorithmic_flops": f,
             "peak_source": "measured FMA-chain kernel (se_probe_fma_tflops)"})


def tile_kernels(M, P):
    return M % 16 == 0 and M >= 32 and P <= 16


def avg_stages(stages):
    return {k: sum(d[k] for d in stages) / len(stages) for k in STAGES}


# ------------------------------------------------------------------- C3 --

def c3_record(args, dev, pg=None, rank=0, world=1):
    """256 systems per step, one sort / spread / interpolation launch and one
    batched cuFFT plan for all of them (FP32 gridding, FP64 k-space); the same
    systems as an FP64 batch and one by one on FP64 single-system plans."""
    import torch
    from se_fast_gridding_b200 import shard, solver
    from se_fast_gridding_b200 import workloads as W
    t_start = time.perf_counter()
    allsys = W.c3_systems()
    mine = shard.partition([solver.System(s["N"], s["M"], s["P"], s["L"], s["xi"]) for s in allsys],
                           world)[rank]
    systems = [solver.System(allsys[i]["N"], 64, allsys[i]["P"], allsys[i]["L"], allsys[i]["xi"])
               for i in mine]
    xs, qs = [], []
    for i in mine:
        s = allsys[i]
        x, q = W.synthetic_system(s["N"], s["L"], seed=s["seed"])
        xs.append(x)
        qs.append(q)
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed_batch(prec, steps, warmup):
        b = solver.BatchSolver(systems, precision=prec)
        x, q = b.pack(xs, qs, device=dev)
        out = torch.empty(int(b.out_off[-1]), dtype=torch.float64, device=dev)
        b.set_timing(True)
        for _ in range(warmup):
            b.solve(x, q, out)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        ms, st, launches = [], [], 0
        for k in range(steps):
            flush.fill_(float(k))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.solve(x, q, out)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            launches += b.launches
            st.append(b.stage_ms())
        outs = [o.cpu().numpy() for o in b.split(out)]
        b.close()
        t = sum(ms) / len(ms)
        if pg:
            t = shard.max_over_ranks(t)
        return t, avg_stages(st), launches, outs

    t32, st32, launches, o32 = timed_batch("fp32", args.steps, max(args.warmup, 3))
    t64b, st64b, _, o64 = timed_batch("fp64", 5, 3)
    # the plain FP64 single-system path: one plan per system, the systems
    # solved one after another (L2 flushed first)
    plans = [solver.SpectralEwald(s.M, s.P, s.L, s.xi, None, "potential", "fp64", s.N)
             for s in systems]
    xd = [torch.tensor(v, device=dev) for v in xs]
    qd = [torch.tensor(v, device=dev) for v in qs]
    od = [torch.empty(s.N, dtype=torch.float64, device=dev) for s in systems]
    for se, a, c, o in zip(plans, xd, qd, od):
        se.solve(a, c, o)
    t64 = []
    for k in range(3):
        flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for se, a, c, o in zip(plans, xd, qd, od):
            se.solve(a, c, o)
        e1.record(stream)
        e1.synchronize()
        t64.append(e0.elapsed_time(e1))
    fp64_ms = sum(t64) / len(t64)
    if pg:
        fp64_ms = shard.max_over_ranks(fp64_ms)
    errs = [W.rel_rms(a, b) for a, b in zip(o32, o64)]
    for se in plans:
        se.close()
    ntot_all = sum(s["N"] for s in allsys)
    info = [(s.N, s.M, s.P, "potential") for s in systems]
    roof, roof_fma = roofline_of(st32, info, "fp32", lambda d: f"k_{d}2")
    return {
        "workload": "256 batched SE3P POTENTIAL systems: N log-uniform [1e3, 6.4e4], L in [1,4], "
                    "M=64, P in {8,12,16}, xi=8/L, FP32 gridding, FP64 k-space, one launch set",
        "systems": 256, "particles": ntot_all, "ms_per_step": t32,
        "particles_per_s": ntot_all / (t32 * 1e-3), "solves_per_s": 256 / (t32 * 1e-3),
        "stage_ms": st32, "gpu_launches": launches, "steps": args.steps,
        "warmup": max(args.warmup, 3), "l2": "flushed between steps (256 MiB write)",
        "accuracy": {"rel_rms_fp32_vs_fp64_max_over_systems": max(errs)},
        "fp64_batch": {"ms_per_step": t64b, "stage_ms": st64b,
                       "fp32_speedup": t64b / t32},
        "fp64_plain": {"ms_per_step": fp64_ms, "fp32_batched_speedup": fp64_ms / t32,
                       "note": "the same systems solved one by one on FP64 single-system "
                               "plans (3 steps, L2 flushed)"},
        "roofline": roof, "roofline_fma": roof_fma,
        "wall_s": time.perf_counter() - t_start,
    }


# ------------------------------------------------------------------- C5 --

def c5_record(args, dev, rank=0):
    """One clustered FORCE system, N = 16M (64 Gaussian clusters of width
    0.02 L), M = 512^3, P = 12, xi = 60, FP32 gridding, FP64 k-space; its
    inputs (512 MB) exceed L2, so no flush is needed between steps."""
    import torch
    from se_fast_gridding_b200 import solver
    from se_fast_gridding_b200 import workloads as W
    t_start = time.perf_counter()
    c = W.C5
    N, M, P, xi = c["N"], c["M"], c["P"], c["xi"]
    x_np, q_np = W.synthetic_system(N, c["L"], seed=c["seed"] + rank, charges="pm1",
                                    clusters=c["clusters"], sigma=c["sigma"])
    x, q = torch.tensor(x_np, device=dev), torch.tensor(q_np, device=dev)
    del x_np, q_np
    stream = torch.cuda.current_stream(dev)

    def timed(prec, steps, warmup):
        se = solver.SpectralEwald(M, P, c["L"], xi, None, "force", prec, N)
        out = torch.empty(3 * N, dtype=torch.float64, device=dev)
        se.set_timing(True)
        for _ in range(warmup):
            se.solve(x, q, out)
        ms, st = [], []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            se.solve(x, q, out)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            st.append(se.stage_ms())
        launches = se.launches
        se.close()
        return sum(ms) / len(ms), avg_stages(st), out, launches

    steps = max(3, min(args.steps, 10))
    t32, st32, f32, launches = timed("fp32", steps, 3)
    t64, st64, f64, _ = timed("fp64", 3, 1)
    idx = torch.arange(0, N, N // 2000, device=dev)[:2000]
    sub32 = torch.cat([f32[idx + d * N] for d in range(3)]).cpu().numpy()
    sub64 = torch.cat([f64[idx + d * N] for d in range(3)]).cpu().numpy()
    err = W.rel_rms(sub32, sub64)
    del f32, f64, x, q
    torch.cuda.empty_cache()
    roof, roof_fma = roofline_of(st32, [(N, M, P, "force")], "fp32", lambda d: f"k_{d}2")
    return {
        "workload": "clustered SE3P FORCE N=16e6 (64 Gaussian clusters, sigma 0.02 L) M=512^3 "
                    "P=12 xi=60, FP32 gridding, FP64 k-space",
        "N": N, "M": M, "P": P, "ms_per_step": t32, "particles_per_s": N / (t32 * 1e-3),
        "stage_ms": st32, "gpu_launches": launches, "steps": steps, "warmup": 3,
        "l2": "inputs (512 MB) and grid (1 GB) exceed L2",
        "accuracy": {"rel_rms_fp32_vs_fp64_2000": err},
        "fp64": {"ms_per_step": t64, "stage_ms": st64, "fp32_speedup": t64 / t32},
        "roofline": roof, "roofline_fma": roof_fma,
        "wall_s": time.perf_counter() - t_start,
    }


# ------------------------------------------------------------------- C4 --

def c4_record(args, dev, rank=0):
    """Poisson arrivals of POTENTIAL/FORCE solves (50/50), N log-uniform in
    [500, 2e6], P in {8, 12, 16}, through the native request loop (8 slots,
    120 GB budget), host (pinned) inputs and outputs; the results go to one
    pinned buffer made before any replay.  Each trace is replayed once untimed
    (plan cache warm) and once timed; latency is submit to result-in-host-
    memory on the host clock.  `capacity` submits a whole trace at once (the
    throughput the loop sustains when requests never wait to arrive), and
    `fp64_plain` solves the trace's first requests one by one on FP64
    single-system plans (device buffers, device time) for comparison."""
    import torch
    from se_fast_gridding_b200 import serve, solver
    t_start = time.perf_counter()
    xs, qs = serve.particle_pool()
    rates = [2000.0] if args.serve_rates is None else [float(r) for r in args.serve_rates.split(",")]
    traces = [(literal, rate, serve.poisson_trace(rate, args.serve_seconds, seed=4 + rank,
                                                  literal_grid=literal))
              for literal in (False, True) for rate in rates]
    arena = serve.output_arena(max((t for _, _, t in traces),
                                   key=lambda tr: sum(r.system.out_width * r.system.N
                                                      for r in tr)))
    runs, capacity = [], []
    with serve.Server(slots=args.serve_slots, precision="fp32", hbm_budget=120 * 10 ** 9) as srv:
        for literal, rate, trace in traces:
            serve.replay(srv, trace, xs, qs, arena)                       # warm
            comps, _, wall, lag = serve.replay(srv, trace, xs, qs, arena)  # timed
            parts = sum(r.system.N for r in trace)
            lat = serve.latency_summary(comps)
            grid = "M=64 for all" if literal else "M=64*2^ceil(log2(N/16000)/3) <= 256"
            runs.append({"grid": grid, "offered_req_s": rate, "requests": len(trace),
                         "solves_per_s": len(comps) / wall, "particles_per_s": parts / wall,
                         "wall_s": wall, "max_submit_lag_ms": lag * 1e3, **lat})
            if rate == rates[0]:
                burst = [serve.TraceRequest(0.0, r.system, r.offset) for r in trace]
                comps, _, wall, _ = serve.replay(srv, burst, xs, qs, arena)
                capacity.append({"grid": grid, "requests": len(burst),
                                 "solves_per_s": len(comps) / wall,
                                 "particles_per_s": parts / wall, "wall_s": wall})
        st = srv.stats()
    # the plain FP64 single-system path on the first requests of the
    # M-from-N trace: device buffers, one plan per (M, P, mode), device time
    trace = traces[0][2][:128]
    stream = torch.cuda.current_stream(dev)
    plans = {}
    xd = xs.to(dev)
    qd = qs.to(dev)
    outs = {}
    for r in trace:
        s = r.system
        key = (s.M, s.P, s.mode)
        cap = max(rr.system.N for rr in trace if (rr.system.M, rr.system.P, rr.system.mode) == key)
        if key not in plans:
            plans[key] = solver.SpectralEwald(s.M, s.P, s.L, s.xi, None, s.mode, "fp64", cap)
        outs.setdefault(key, torch.empty(3 * cap, dtype=torch.float64, device=dev))

    def run_plain():
        for r in trace:
            s = r.system
            key = (s.M, s.P, s.mode)
            plans[key].solve_system(s, xd[r.offset:r.offset + 3 * s.N], qd[r.offset:r.offset + s.N],
                                    outs[key][:s.out_width * s.N])
    run_plain()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run_plain()
    e1.record(stream)
    e1.synchronize()
    t64 = e0.elapsed_time(e1) * 1e-3
    parts64 = sum(r.system.N for r in trace)
    for p in plans.values():
        p.close()
    del xd, qd, outs
    head = runs[0]
    cap0 = capacity[0]
    offered = cap0["particles_per_s"] * cap0["wall_s"] / args.serve_seconds
    limit = {
        "offered_particles_per_s": offered,
        "capacity_particles_per_s": cap0["particles_per_s"],
        "note": "the M-from-N trace offers this many particles/s of spread and interpolation "
                "(its requests with N > 128k on M=256 grids); the capacity, the whole trace "
                "submitted at once, is below it, so kernel throughput and not admission bounds "
                "the served rate" if offered > cap0["particles_per_s"] else
                "the capacity exceeds the offered particle rate",
    }
    return {
        "workload": f"serving: Poisson {head['offered_req_s']:.0f} req/s for {args.serve_seconds} s, "
                    "POTENTIAL/FORCE 50/50, N log-uniform [500, 2e6], P in {8,12,16}, L=1, "
                    f"xi=8M/64, FP32 gridding, {args.serve_slots} slots, 120 GB budget, "
                    "pinned host I/O",
        "latency_clock": "host steady clock, submit to result in host memory",
        "solves_per_s": head["solves_per_s"], "p50_ms": head["p50_ms"], "p99_ms": head["p99_ms"],
        "particles_per_s": head["particles_per_s"], "runs": runs, "capacity": capacity,
        "limit": limit,
        "fp64_plain": {"requests": len(trace), "particles_per_s": parts64 / t64,
                       "solves_per_s": len(trace) / t64,
                       "served_capacity_speedup": cap0["particles_per_s"] / (parts64 / t64),
                       "note": "the first 128 requests of the M-from-N trace solved one by one "
                               "on FP64 single-system plans, device buffers, device time"},
        "server": {k: st[k] for k in ("plans", "plans_created", "plans_evicted", "hbm_peak")},
        "wall_s": time.perf_counter() - t_start,
    }


# ------------------------------------------------------------------- C1 --

def c1_record(args, dev):
    """Plain SE3P POTENTIAL FP64, N=100 charges +-1 in the unit box, M=32,
    P=21, xi=8, m=0.94 sqrt(pi P) -- the reference's CPU-runnable case.  A
    solve this small is bound by launches: timed directly, replayed from a
    CUDA graph (se_plan_set_graph), through host buffers, and the reference's
    own spectral_ewald() on one core for the same system."""
    import torch
    from se_fast_gridding_b200 import solver
    from se_fast_gridding_b200 import workloads as W
    N, M, P, xi = 100, 32, 21, 8.0
    x_np, q_np = W.synthetic_system(N, 1.0, seed=0, charges="pm1")
    m = 0.94 * (3.14159265358979323846 * P) ** 0.5
    s = torch.cuda.Stream(dev)
    res = {}
    with torch.cuda.stream(s):
        x, q = torch.tensor(x_np, device=dev), torch.tensor(q_np, device=dev)
        out = torch.empty(N, dtype=torch.float64, device=dev)
        for name, graph in (("direct", False), ("graph", True)):
            se = solver.SpectralEwald(M, P, 1.0, xi, m, "potential", "fp64", N)
            se.set_graph(graph)
            for _ in range(max(args.warmup, 3)):
                se.solve(x, q, out, stream=s)
            s.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            for _ in range(args.steps):
                se.solve(x, q, out, stream=s)
            b.record(s)
            b.synchronize()
            res[name] = a.elapsed_time(b) / args.steps
            se.close()
        se = solver.SpectralEwald(M, P, 1.0, xi, m, "potential", "fp64", N)
        xh, qh = torch.tensor(x_np).pin_memory(), torch.tensor(q_np).pin_memory()
        oh = torch.empty(N, dtype=torch.float64).pin_memory()
        for _ in range(3):
            se.solve_host_ptr(N, xh.data_ptr(), qh.data_ptr(), oh.data_ptr(), stream=s)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            se.solve_host_ptr(N, xh.data_ptr(), qh.data_ptr(), oh.data_ptr(), stream=s)
        res["host_buffers"] = 1e3 * (time.perf_counter() - t0) / args.steps
        se.close()
    cpu = None
    if not args.no_cpu_baseline:
        w = dict(N=N, M=M, P=P, L=1.0, xi=xi, mode="potential", precision="fp64",
                 charges="pm1", seed=0)
        try:
            r = cpu_reference(args, 1, 1, 20, 2, w)
            cpu = {"ms_per_solve": 1e3 * sum(r["step_s"]) / len(r["step_s"]), "cores": 1,
                   "kind": r["kind"], "sample": r["sample"]}
        except Exception as e:   # reported, not required
            cpu = {"sample": f"failed: {e}"[:200]}
    return {"us_per_solve": {k: 1e3 * v for k, v in res.items()}, "cpu_reference": cpu,
            "ms_per_step": res["graph"], "steps": args.steps, "warmup": max(args.warmup, 3),
            "workload": "SE3P POTENTIAL FP64 N=100 M=32^3 P=21 xi=8 L=1",
            "particles_per_s": N / (res["graph"] * 1e-3)}


def sub_line(rec, value_key, unit, n_gpus, dtype):
    """A standalone JSON line for one configuration's record."""
    return {"metric": METRIC, "value": rec[value_key] * n_gpus, "unit": unit, "n_gpus": n_gpus,
            "steps": rec.get("steps", 1), "warmup": rec.get("warmup", 1),
            "ms_per_step": rec["ms_per_step"] if "ms_per_step" in rec else rec["wall_s"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic (seeded)", "config": {"workload": rec["workload"]},
            **{k: v for k, v in rec.items() if k != "workload"}}


# ------------------------------------------------------------ reference --

def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    w = WORKLOAD
    ncpu = os.cpu_count() or 1
    procs = max(1, min(ncpu, args.ref_procs or ncpu))
    res = cpu_reference(args, procs, 1, args.steps, args.warmup, w)
    value = res["value"]
    ms = 1e3 * sum(res["step_s"]) / len(res["step_s"])
    fft = res.get("fft")
    excl = None
    if fft:
        excl = {"value": procs * w["N"] / (fft["solve_s"] - fft["fft_s_per_solve"]),
                "unit": "particles/s", "fft_share": fft["share"],
                "fft_s_per_solve": fft["fft_s_per_solve"], "solve_s": fft["solve_s"],
                "note": "the same solves with the time inside fftw_execute (the project's own "
                        "mixed-radix CPU FFT standing in for the absent FFTW) taken out"}
    line = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded uniform charges and positions)",
        "config": workload_config(w),
        "impl": "reference",
        "arithmetic": "FP64 gridding and FFT (the reference's AVX path, -DFGG_SPLIT -DFORCE)",
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": res["cores"],
                         "kind": res["kind"], "sample": res["sample"]},
        "excluding_fft": excl,
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- C2 --

def timed_solves(se, x, q, out, stream, flush, steps):
    import torch
    ms, st = [], []
    for k in range(steps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        se.solve(x, q, out)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
        st.append(se.stage_ms())
    return sum(ms) / len(ms), avg_stages(st)


def timed_host(se, N, xh, qh, oh, stream, flush, steps, warmup):
    import torch
    for _ in range(max(warmup, 1)):
        se.solve_host_ptr(N, xh.data_ptr(), qh.data_ptr(), oh.data_ptr())
    ms = []
    for k in range(steps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        se.solve_host_ptr(N, xh.data_ptr(), qh.data_ptr(), oh.data_ptr())
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    return sum(ms) / len(ms)


def run_c2(args):
    import numpy as np
    import torch
    from se_fast_gridding_b200 import solver
    from se_fast_gridding_b200 import workloads as O

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist
    w = WORKLOAD
    N = w["N"]
    x_np, q_np = O.synthetic_system(N, w["L"], seed=w["seed"] + rank, charges=w["charges"])
    m = solver.default_m(w["P"])
    # every solve runs on a side stream and replays its CUDA graph (the
    # repeated-solve launch mode, se_plan_set_graph); the direct launches are
    # timed beside it
    torch.cuda.set_stream(torch.cuda.Stream(dev))
    stream = torch.cuda.current_stream(dev)
    se = solver.SpectralEwald(w["M"], w["P"], w["L"], w["xi"], m, w["mode"], w["precision"], N)
    se.set_graph(True)
    x = torch.tensor(x_np, device=dev)
    q = torch.tensor(q_np, device=dev)
    out = torch.empty(3 * N, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    xh = torch.tensor(x_np).pin_memory()
    qh = torch.tensor(q_np).pin_memory()
    oh = torch.empty(3 * N, dtype=torch.float64).pin_memory()

    # accuracy (rank 0, outside the timed region): FP32 vs the FP64 path and
    # vs the FP64 direct k-space sum on the 1,000-particle subset; the plain
    # FP64 path and the FP32-FFT mode timed the same way
    accuracy = fp64 = fft32 = None
    if rank == 0:
        se.solve(x, q, out)
        f32 = out.cpu().numpy()
        s64 = solver.SpectralEwald(w["M"], w["P"], w["L"], w["xi"], m, w["mode"], "fp64", N)
        s64.set_graph(True)
        s64.set_timing(True)
        f64 = s64.solve(x, q).cpu().numpy()
        o64 = torch.empty(3 * N, dtype=torch.float64, device=dev)
        for _ in range(3):
            s64.solve(x, q, o64)
        t64, st64 = timed_solves(s64, x, q, o64, stream, flush, 5)
        s64.set_timing(False)
        e2e64 = timed_host(s64, N, xh, qh, oh, stream, flush, 5, 3)
        fp64 = {"ms_per_step": t64, "stage_ms": st64,
                "e2e": {"value": N / (e2e64 * 1e-3), "unit": "particles/s", "ms_per_step": e2e64,
                        "h2d_bytes_per_step": 4 * N * 8, "d2h_bytes_per_step": 3 * N * 8},
                "note": "the FP64 path on the same inputs, same timing (5 steps, L2 flushed); "
                        "e2e through se_solve_host with pinned host buffers"}
        s3 = solver.SpectralEwald(w["M"], w["P"], w["L"], w["xi"], m, w["mode"], "fp32-fft32", N)
        s3.set_graph(True)
        o3 = torch.empty(3 * N, dtype=torch.float64, device=dev)
        s3.set_timing(True)
        for _ in range(3):
            s3.solve(x, q, o3)
        t3, st3 = timed_solves(s3, x, q, o3, stream, flush, 10)
        f3 = o3.cpu().numpy()
        fft32 = {"ms_per_step": t3, "value": N / (t3 * 1e-3), "stage_ms": st3,
                 "rel_rms_vs_fp64": O.rel_rms(f3, f64)}
        s3.close()
        del o64, o3
        s64.close()
        accuracy = {"rel_rms_fp32_vs_fp64": O.rel_rms(f32, f64)}
        gpath = os.path.join(ROOT, "tests", "golden", "c2.npz")
        if os.path.exists(gpath):
            g = np.load(gpath)
            t = g["targets"]
            sub = np.concatenate([f32[t + d * N] for d in range(3)])
            accuracy["rel_rms_vs_direct_1000"] = O.rel_rms(sub, g["force_direct"])
            sub64 = np.concatenate([f64[t + d * N] for d in range(3)])
            accuracy["rel_rms_fp64_vs_direct_1000"] = O.rel_rms(sub64, g["force_direct"])
            sub3 = np.concatenate([f3[t + d * N] for d in range(3)])
            fft32["rel_rms_vs_direct_1000"] = O.rel_rms(sub3, g["force_direct"])

    se.set_timing(True)
    for _ in range(max(args.warmup, 3)):
        flush.fill_(1.0)
        se.solve(x, q, out)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    stage = []
    launches = 0
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        se.solve(x, q, out)
        ev[k][1].record(stream)
        launches += se.launches
        stage.append(se.stage_ms())
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms = sum(step_ms) / len(step_ms)
    clk = clocks.stop()
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
        pg.barrier()
    value = world * N / (ms * 1e-3)
    stage_avg = avg_stages(stage)

    # the same solves launched directly (no graph), for comparison
    se.set_graph(False)
    se.set_timing(False)
    direct = []
    for k in range(max(args.warmup, 1) + args.steps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        se.solve(x, q, out)
        b.record(stream)
        b.synchronize()
        if k >= max(args.warmup, 1):
            direct.append(a.elapsed_time(b))
    direct_ms = sum(direct) / len(direct)

    # end to end through the host-buffer entry point, pinned buffers
    e2e = timed_host(se, N, xh, qh, oh, stream, flush, args.steps, args.warmup)
    if pg:
        t = torch.tensor([e2e], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e = float(t.item())
    se.close()

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return

    tr = ncu_traffic()
    traffic = tr if (tr and tr.get("workload") == workload_name(w)) else None
    P, M = w["P"], w["M"]
    tiles = tile_kernels(M, P)
    roofline, roofline_fma = roofline_of(stage_avg, [(N, M, P, w["mode"])], w["precision"],
                                         lambda d: f"k_{d}2" if tiles else f"k_{d}", traffic)
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            res = cpu_reference(args, 1, 1, 1, 0, w)
            cpu = {"value": res["value"], "unit": "particles/s", "cores": res["cores"],
                   "kind": res["kind"], "sample": res["sample"], "fft": res.get("fft")}
        except Exception as e:   # the baseline is reported, not required
            cpu = {"value": None, "unit": "particles/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {e}"[:200]}
    line = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform charges and positions, one replica per GPU)",
        "config": workload_config(w),
        "arithmetic": "FP32 spread/interpolation with compensated (FP64-folded) sums, FP64 FFT "
                      "and Green's-function scaling",
        "parallelism": f"replicas x{world}",
        "launch": "CUDA graph replay on a side stream (se_plan_set_graph); e2e: se_solve_host",
        "roofline": roofline, "roofline_fma": roofline_fma,
        "stage_ms": stage_avg, "direct_launch_ms_per_step": direct_ms, "cpu_baseline": cpu,
        "e2e": {"value": world * N / (e2e * 1e-3), "unit": "particles/s",
                "h2d_bytes_per_step": 4 * N * 8, "d2h_bytes_per_step": 3 * N * 8,
                "ms_per_step": e2e},
        "gpu_launches": launches,
        "clocks": clk, "accuracy": accuracy, "wall_s_timed": wall,
        "fp32_fft32": fft32,
        "fp64_plain": None if fp64 is None else dict(fp64, fp32_speedup=fp64["ms_per_step"] / ms),
    }
    if world == 1 and not args.no_extra:
        torch.cuda.empty_cache()
        line["c3"] = c3_record(args, dev)
        line["c4"] = c4_record(args, dev)
        line["c5"] = c5_record(args, dev)
    print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-procs", type=int, default=0,
                    help="CPU processes for --impl reference (default: all cores)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="C2 line only, without the c3 / c4 / c5 sub-records")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the headline single FORCE system (with c3/c4/c5 sub-records); "
                         "c3: 256 batched systems; c4: the serving loop under Poisson "
                         "arrivals; c5: 16M clustered particles; c1: the 100-particle FP64 case")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--serve-rates", default=None, help="comma-separated req/s (default 2000)")
    ap.add_argument("--serve-slots", type=int, default=8)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "c2":
        return run_c2(args)
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if args.workload == "c3" and world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    if args.workload == "c1":
        rec, key, unit, dtype = c1_record(args, dev), "particles_per_s", "particles/s", "f64"
    elif args.workload == "c3":
        rec, key, unit, dtype = c3_record(args, dev, pg, rank, world), "particles_per_s", \
            "particles/s", "f32"
    elif args.workload == "c4":
        rec, key, unit, dtype = c4_record(args, dev, rank), "solves_per_s", "solves/s", "f32"
    else:
        rec, key, unit, dtype = c5_record(args, dev, rank), "particles_per_s", "particles/s", "f32"
    if rank == 0:
        n = 1 if args.workload == "c3" else world   # c3: the systems are shared out
        print(json.dumps(sub_line(rec, key, unit, n, dtype)), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
