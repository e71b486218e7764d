"""Benchmark of the SE3P k-space solve on B200 (one JSON line on stdout).

Workload (default, the configuration the headline metric is quoted on):
SE3P FORCE, N = 100,000 charges uniform in the unit box, charges uniform in
[-1, 1] shifted to zero sum, M = 128^3, P = 16, xi = 20, m = 0.94 sqrt(pi P);
FP32 spread/interpolation with compensated accumulation, FP64 FFT and
Green's-function scaling.  A step is one full solve (sort, spread + fold,
D2Z, scaling, Z2D, unfold + interpolation) of that system.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

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


def workload_name(w):
    return (f"SE3P {w['mode'].upper()} N={w['N']} M={w['M']}^3 P={w['P']} xi={w['xi']} "
            f"L={w['L']}, {w['precision'].upper()} gridding (compensated), FP64 FFT+scaling")


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


def c3_systems(seed=3):
    """256 independent POTENTIAL systems: N log-uniform in [1e3, 6.4e4], L in
    [1, 4], M = 64 (h = L/64), P from {8, 12, 16}, xi = 8/L, charges +-1."""
    import numpy as np
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(256):
        N = int(round(np.exp(rng.uniform(np.log(1e3), np.log(6.4e4)))))
        L = float(rng.uniform(1.0, 4.0))
        P = int(rng.choice([8, 12, 16]))
        out.append(dict(N=N, M=64, P=P, L=L, xi=8.0 / L, seed=1000 + i))
    return out


def run_batched(args):
    """C3: 256 systems per step, one sort / spread / interpolation launch and
    one batched cuFFT plan for all of them (FP32 gridding, FP64 k-space)."""
    import numpy as np
    import torch
    from se_fast_gridding_b200 import shard, solver
    from se_fast_gridding_b200 import workloads as O
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    allsys = c3_systems()
    mine = shard.partition([solver.System(s["N"], s["M"], s["P"], s["L"], s["xi"]) for s in allsys],
                           world)[rank]
    systems = [solver.System(allsys[i]["N"], 64, allsys[i]["P"], allsys[i]["L"], allsys[i]["xi"])
               for i in mine]
    xs, qs = [], []
    for i in mine:
        s = allsys[i]
        x, q = O.synthetic_system(s["N"], s["L"], seed=s["seed"])
        xs.append(x)
        qs.append(q)
    b = solver.BatchSolver(systems, precision="fp32")
    x, q = b.pack(xs, qs, device=dev)
    out = torch.empty(int(b.out_off[-1]), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    b.set_timing(True)
    for _ in range(args.warmup):
        b.solve(x, q, out)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ms = []
    stage = {"sort": [], "spread": [], "kspace": [], "interp": []}
    launches = 0
    for k in range(args.steps):
        flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.solve(x, q, out)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        launches += b.launches
        for kk, v in b.stage_ms().items():
            stage[kk].append(v)
    t = sum(ms) / len(ms)
    if pg:
        t = shard.max_over_ranks(t)
    ntot_all = sum(s["N"] for s in allsys)
    # the plain FP64 single-system path on the same inputs: one plan per
    # system, the systems solved one after another (L2 flushed first); and the
    # accuracy of the FP32 batch against it
    errs = []
    outs = b.split(out)
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
    for j in range(len(systems)):
        errs.append(O.rel_rms(outs[j].cpu().numpy(), od[j].cpu().numpy()))
    for se in plans:
        se.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": ntot_all / (t * 1e-3), "unit": "particles/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": "C3 batched SE3P POTENTIAL: 256 systems, N log-uniform "
                                   "[1e3, 6.4e4], L in [1,4], M=64, P in {8,12,16}, xi=8/L, "
                                   "FP32 gridding, FP64 k-space, one launch set",
                       "systems": 256, "particles": ntot_all,
                       "l2": "flushed between steps (256 MiB write)"},
            "solves_per_s": 256 / (t * 1e-3), "stage_ms": {k: sum(v) / len(v) for k, v in stage.items()},
            "gpu_launches": launches,
            "accuracy": {"rel_rms_fp32_vs_fp64_max_over_systems": max(errs)},
            "fp64_plain": {"ms_per_step": fp64_ms, "fp32_batched_speedup": fp64_ms / t,
                           "note": "the same systems solved one by one on FP64 single-system "
                                   "plans (3 steps, L2 flushed)"},
        }
        print(json.dumps(line), flush=True)
    b.close()
    if pg:
        pg.destroy_process_group()


def run_large(args):
    """C5: one clustered FORCE system, N = 16M (64 Gaussian clusters of width
    0.02 L), M = 512^3, P = 12, xi = 60, FP32 gridding, FP64 k-space."""
    import numpy as np
    import torch
    from se_fast_gridding_b200 import solver
    from se_fast_gridding_b200 import workloads as O
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N, M, P, xi = 16_000_000, 512, 12, 60.0
    x_np, q_np = O.synthetic_system(N, 1.0, seed=5 + rank, charges="pm1", clusters=64, sigma=0.02)
    x, q = torch.tensor(x_np, device=dev), torch.tensor(q_np, device=dev)
    se = solver.SpectralEwald(M, P, 1.0, xi, None, "force", "fp32", N)
    out = torch.empty(3 * N, dtype=torch.float64, device=dev)
    se.set_timing(True)
    stream = torch.cuda.current_stream(dev)
    for _ in range(max(1, args.warmup)):
        se.solve(x, q, out)
    ms, stage = [], {"sort": [], "spread": [], "kspace": [], "interp": []}
    for k in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        se.solve(x, q, out)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        for kk, v in se.stage_ms().items():
            stage[kk].append(v)
    t = sum(ms) / len(ms)
    # accuracy on a 2,000-particle subset: FP32 vs the FP64 path
    s64 = solver.SpectralEwald(M, P, 1.0, xi, None, "force", "fp64", N)
    f64 = s64.solve(x, q)
    idx = torch.arange(0, N, N // 2000, device=dev)[:2000]
    sub32 = torch.cat([out[idx + d * N] for d in range(3)]).cpu().numpy()
    sub64 = torch.cat([f64[idx + d * N] for d in range(3)]).cpu().numpy()
    err = O.rel_rms(sub32, sub64)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": world * N / (t * 1e-3), "unit": "particles/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded clustered)",
            "config": {"workload": "C5 clustered SE3P FORCE N=16e6 (64 clusters, sigma 0.02 L) "
                                   "M=512^3 P=12 xi=60, FP32 gridding, FP64 k-space",
                       "N": N, "M": M, "P": P},
            "stage_ms": {k: sum(v) / len(v) for k, v in stage.items()},
            "accuracy": {"rel_rms_fp32_vs_fp64_2000": err},
        }), flush=True)


def run_serve(args):
    """C4: Poisson arrivals of POTENTIAL/FORCE solves (50/50), N log-uniform in
    [500, 2e6], P in {8, 12, 16}, through the native request loop (8 slots,
    120 GB budget), host (pinned) inputs and outputs; the results go to one
    pinned buffer made before any replay.  Each trace is replayed once untimed
    (plan cache warm) and once timed; latency is submit to result-in-host-
    memory on the host clock."""
    import torch
    from se_fast_gridding_b200 import serve
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    xs, qs = serve.particle_pool()
    rates = [2000.0] if args.serve_rates is None else [float(r) for r in args.serve_rates.split(",")]
    runs = []
    traces = [(literal, rate, serve.poisson_trace(rate, args.serve_seconds, seed=4 + rank,
                                                  literal_grid=literal))
              for literal in (False, True) for rate in rates]
    # pinned result buffers for the largest trace, made before any replay
    arena = serve.output_arena(max((t for _, _, t in traces),
                                   key=lambda tr: sum(r.system.out_width * r.system.N
                                                      for r in tr)))
    with serve.Server(slots=args.serve_slots, precision="fp32", hbm_budget=120 * 10 ** 9) as srv:
        for literal, rate, trace in traces:
            serve.replay(srv, trace, xs, qs, arena)                       # warm
            comps, _, wall, lag = serve.replay(srv, trace, xs, qs, arena)  # timed
            parts = sum(r.system.N for r in trace)
            lat = serve.latency_summary(comps)
            runs.append({"grid": "M=64 for all" if literal else "M=64*2^ceil(log2(N/16000)/3) <= 256",
                         "offered_req_s": rate, "requests": len(trace),
                         "solves_per_s": len(comps) / wall, "particles_per_s": parts / wall,
                         "wall_s": wall, "max_submit_lag_ms": lag * 1e3, **lat})
        st = srv.stats()
    head = runs[rates.index(2000.0) if 2000.0 in rates else 0]
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": head["solves_per_s"] * world, "unit": "solves/s",
            "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": head["wall_s"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Poisson trace; particles sliced from a uniform pool)",
            "config": {"workload": f"C4 serving: Poisson {head['offered_req_s']:.0f} req/s for "
                                   f"{args.serve_seconds} s, POTENTIAL/FORCE 50/50, N log-uniform "
                                   "[500, 2e6], P in {8,12,16}, L=1, xi=8M/64, FP32 gridding, "
                                   f"{args.serve_slots} slots, 120 GB budget, pinned host I/O",
                       "latency_clock": "host steady clock, submit to result in host memory"},
            "p50_ms": head["p50_ms"], "p99_ms": head["p99_ms"],
            "particles_per_s": head["particles_per_s"], "runs": runs,
            "server": {k: st[k] for k in ("plans", "plans_created", "plans_evicted", "hbm_peak")},
        }), flush=True)


def run_c1(args):
    """C1: plain SE3P POTENTIAL FP64, N=100 charges +-1 in the unit box, M=32,
    P=21, xi=8, m=0.94 sqrt(pi P) -- the reference's CPU-runnable case.  A
    solve this small is bound by launches: timed directly, replayed from a
    CUDA graph (se_plan_set_graph), through host buffers, and the reference's
    own spectral_ewald() on one core for the same system."""
    import torch
    from se_fast_gridding_b200 import solver
    from se_fast_gridding_b200 import workloads as W
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
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
    if rank == 0:
        best = res["graph"]
        print(json.dumps({
            "metric": METRIC, "value": N / (best * 1e-3), "unit": "particles/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": best,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded, charges +-1)",
            "config": {"workload": "C1 SE3P POTENTIAL FP64 N=100 M=32^3 P=21 xi=8 L=1",
                       "timing": "CUDA events over back-to-back solves on one stream"},
            "us_per_solve": {k: 1e3 * v for k, v in res.items()},
            "cpu_reference": cpu,
        }), flush=True)


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
    line = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded uniform charges and positions)",
        "config": {"workload": workload_name(dict(w, precision="fp64")) + " (CPU reference)",
                   "N": w["N"], "M": w["M"], "P": w["P"], "xi": w["xi"]},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": res["cores"],
                         "kind": res["kind"], "sample": res["sample"]},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-procs", type=int, default=0,
                    help="CPU processes for --impl reference (default: all cores)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the headline single FORCE system; c3: 256 batched systems; "
                         "c4: the serving loop under Poisson arrivals; c5: 16M clustered particles")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--serve-rates", default=None, help="comma-separated req/s (default 2000)")
    ap.add_argument("--serve-slots", type=int, default=8)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "c1":
        return run_c1(args)
    if args.workload == "c3":
        return run_batched(args)
    if args.workload == "c4":
        return run_serve(args)
    if args.workload == "c5":
        return run_large(args)

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

    # accuracy (rank 0, outside the timed region): FP32 vs the FP64 path and
    # vs the FP64 direct k-space sum on the 1,000-particle subset
    accuracy = None
    fp64_ms = None
    fft32 = None
    if rank == 0:
        se.solve(x, q, out)
        f32 = out.cpu().numpy()
        s64 = solver.SpectralEwald(w["M"], w["P"], w["L"], w["xi"], m, w["mode"], "fp64", N)
        s64.set_graph(True)
        f64 = s64.solve(x, q).cpu().numpy()
        # the plain FP64 path on the same inputs, timed the same way (the
        # FP32 path is measured against it)
        fl = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
        o64 = torch.empty(3 * N, dtype=torch.float64, device=dev)
        for _ in range(3):
            s64.solve(x, q, o64)
        t64 = []
        for k in range(5):
            fl.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s64.solve(x, q, o64)
            b.record(stream)
            b.synchronize()
            t64.append(a.elapsed_time(b))
        fp64_ms = sum(t64) / len(t64)
        # the FP32-FFT mode on the same inputs, timed the same way
        s3 = solver.SpectralEwald(w["M"], w["P"], w["L"], w["xi"], m, w["mode"], "fp32-fft32", N)
        s3.set_graph(True)
        o3 = torch.empty(3 * N, dtype=torch.float64, device=dev)
        s3.set_timing(True)
        for _ in range(3):
            s3.solve(x, q, o3)
        t3, st3 = [], []
        for k in range(10):
            fl.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s3.solve(x, q, o3)
            b.record(stream)
            b.synchronize()
            t3.append(a.elapsed_time(b))
            st3.append(s3.stage_ms())
        f3 = o3.cpu().numpy()
        fft32 = {"ms_per_step": sum(t3) / len(t3), "value": N / (sum(t3) / len(t3) * 1e-3),
                 "stage_ms": {k: sum(d[k] for d in st3) / len(st3) for k in st3[0]},
                 "rel_rms_vs_fp64": O.rel_rms(f3, f64)}
        s3.close()
        del fl, o64, o3
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

    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    se.set_timing(True)
    for _ in range(args.warmup):
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
    stage = {"sort": [], "spread": [], "kspace": [], "interp": []}
    launches = 0
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        se.solve(x, q, out)
        ev[k][1].record(stream)
        launches += se.launches
        for key, v in se.stage_ms().items():
            stage[key].append(v)
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
    stage_avg = {k: sum(v) / len(v) for k, v in stage.items()}

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
    xh = torch.tensor(x_np).pin_memory()
    qh = torch.tensor(q_np).pin_memory()
    oh = torch.empty(3 * N, dtype=torch.float64).pin_memory()
    se.set_timing(False)
    for _ in range(max(args.warmup, 1)):
        se.solve_host_ptr(N, xh.data_ptr(), qh.data_ptr(), oh.data_ptr())
    e2e_ms = []
    for k in range(args.steps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        se.solve_host_ptr(N, xh.data_ptr(), qh.data_ptr(), oh.data_ptr())
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e = sum(e2e_ms) / len(e2e_ms)
    if pg:
        t = torch.tensor([e2e], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e = float(t.item())

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return

    # roofline of the dominant kernel
    hbm, hbm_kind = measured_peaks()
    fma = solver.fma_peak_tflops()
    s = 4 if w["precision"] == "fp32" else 8
    P, M = w["P"], w["M"]
    dom = max(("spread", "interp"), key=lambda k: stage_avg[k])
    if dom == "spread":
        alg_bytes = N * 4 * 8 + M ** 3 * 8      # x, q in; M^3 FP64 grid out
        flops = 2.0 * P ** 3 * N
    else:
        alg_bytes = M ** 3 * 8 + N * 4 * 8 + 3 * N * 8
        flops = 8.0 * P ** 3 * N
    t_dom = stage_avg[dom] * 1e-3
    tr = ncu_traffic()
    traffic = None
    if tr and tr.get("workload") == workload_name(w):
        traffic = tr.get(dom)
    kname = f"k_{dom}2" if (M % 16 == 0 and M >= 32 and P <= 16) else f"k_{dom}"
    roofline = {"kernel": kname, "bound": "hbm", "achieved": alg_bytes / t_dom / 1e9,
                "peak": hbm, "unit": "GB/s", "frac": alg_bytes / t_dom / 1e9 / hbm,
                "traffic": traffic, "peak_source": f"{hbm_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if hbm_kind == "measured" else "fallback 6650 GB/s",
                "algorithmic_bytes": alg_bytes}
    roofline_fma = {"kernel": kname, "bound": "fp32_fma", "achieved": flops / t_dom / 1e12,
                    "peak": fma, "unit": "TFLOP/s", "frac": flops / t_dom / 1e12 / fma,
                    "peak_source": "measured FMA-chain kernel (se_probe_fma_tflops)"}
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            res = cpu_reference(args, 1, 1, 1, 0, w)
            cpu = {"value": res["value"], "unit": "particles/s", "cores": res["cores"],
                   "kind": res["kind"], "sample": res["sample"]}
        except Exception as e:   # the baseline is reported, not required
            cpu = {"value": None, "unit": "particles/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {e}"[:200]}
    line = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform charges and positions, one replica per GPU)",
        "config": {"workload": workload_name(w), "N": N, "M": M, "P": P, "xi": w["xi"],
                   "L": w["L"], "precision": w["precision"], "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (256 MiB write)",
                   "launch": "CUDA graph replay on a side stream (se_plan_set_graph); "
                             "e2e: se_solve_host"},
        "roofline": roofline, "roofline_fma": roofline_fma,
        "stage_ms": stage_avg, "direct_launch_ms_per_step": direct_ms, "cpu_baseline": cpu,
        "e2e": {"value": world * N / (e2e * 1e-3), "unit": "particles/s",
                "h2d_bytes_per_step": 4 * N * 8, "d2h_bytes_per_step": 3 * N * 8,
                "ms_per_step": e2e},
        "gpu_launches": launches,
        "clocks": clk, "accuracy": accuracy, "wall_s_timed": wall,
        "fp32_fft32": fft32,
        "fp64_plain": None if fp64_ms is None else {
            "ms_per_step": fp64_ms, "fp32_speedup": fp64_ms / ms,
            "note": "the FP64 path on the same inputs, same timing (5 steps, L2 flushed)"},
    }
    print(json.dumps(line), flush=True)
    se.close()
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
