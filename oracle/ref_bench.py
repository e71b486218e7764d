"""Time the reference's CPU implementation of the SE k-space solve.

TEST/BASELINE INFRASTRUCTURE ONLY (the CPU-baseline leg of bench.py).  Runs
SE_fast_gridding's own spectral_ewald() (spectral_ewald.c:20-182), built from
its sources into oracle/_ref/libse_ref_{pot,force}.so with FFTW replaced by
oracle/fftw_cpu.c, on seeded synthetic inputs.  When that build is absent it
times the oracle port instead and says so (kind "port").

    python oracle/ref_bench.py --N 100000 --M 128 --P 16 --xi 20 --mode force \
        --procs 1 --threads 1 --steps 2 --warmup 0

Each step, every one of --procs worker processes (each with --threads OpenMP
threads) solves the whole system once; the step time is the wall time from a
common start barrier to the last worker's finish.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def _worker(rank, args, barrier, q_out):
    try:
        _work(rank, args, barrier, q_out)
    except BaseException as e:   # the parent must not wait for a worker that died
        barrier.abort()
        q_out.put((rank, "error", repr(e)))


def _work(rank, args, barrier, q_out):
    os.environ["OMP_NUM_THREADS"] = str(args.threads)
    sys.path.insert(0, HERE)
    import numpy as np
    import oracle as O
    kind = "reference"
    lib = O.ref_lib("force" if args.mode == "force" else "pot")
    if lib is None:
        kind = "port"
    x, q = O.synthetic_system(args.N, args.L, seed=args.seed + rank, charges=args.charges)
    m = 0.94 * np.sqrt(O.PI * args.P)
    width = 3 if args.mode == "force" else 1
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    times = []
    if kind == "reference":
        import ctypes as C
        lib.fc_fft_seconds.restype = C.c_double
    for step in range(args.warmup + args.steps):
        barrier.wait()
        if kind == "reference":
            lib.fc_fft_reset()
        t0 = time.perf_counter()
        os.dup2(devnull, 1)          # the reference prints dispatcher lines
        try:
            if kind == "reference":
                O.ref_spectral_ewald(lib, x, q, args.M, args.P, m, args.L, args.xi, width * args.N)
            else:
                O.spectral_ewald(x, q, args.M, args.P, m, args.L, args.xi, args.mode)
        finally:
            os.dup2(saved, 1)
        t1 = time.perf_counter()
        fft = lib.fc_fft_seconds() if kind == "reference" else None
        barrier.wait()
        if step >= args.warmup:
            times.append((t0, t1, fft))
    q_out.put((rank, kind, times))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=100_000)
    ap.add_argument("--M", type=int, default=128)
    ap.add_argument("--P", type=int, default=16)
    ap.add_argument("--L", type=float, default=1.0)
    ap.add_argument("--xi", type=float, default=20.0)
    ap.add_argument("--mode", default="force")
    ap.add_argument("--charges", default="uniform")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--procs", type=int, default=1)
    ap.add_argument("--threads", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=0)
    args = ap.parse_args(argv)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(args.procs)
    q_out = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, args, barrier, q_out)) for r in range(args.procs)]
    for p in procs:
        p.start()
    results = [q_out.get() for _ in procs]
    for p in procs:
        p.join()
    errors = [r for r in results if r[1] == "error"]
    if errors:
        sys.exit(f"reference worker failed: {errors[0][2]}")
    kind = results[0][1]
    step_s = []
    for s in range(args.steps):
        starts = [r[2][s][0] for r in results]
        ends = [r[2][s][1] for r in results]
        step_s.append(max(ends) - min(starts))
    per_step = sum(step_s) / len(step_s)
    value = args.procs * args.N / per_step
    # the FFT's share of one solve (time inside fftw_execute, the project's
    # own CPU FFT standing in for FFTW), averaged over workers and steps
    solve_s = [t1 - t0 for r in results for (t0, t1, _) in r[2]]
    fft_s = [f for r in results for (_, _, f) in r[2] if f is not None]
    fft = None
    if fft_s:
        fft = {"fft_s_per_solve": sum(fft_s) / len(fft_s),
               "solve_s": sum(solve_s) / len(solve_s),
               "share": sum(fft_s) / sum(solve_s)}
    print(json.dumps({
        "value": value, "unit": "particles/s", "kind": kind,
        "cores": args.procs * args.threads, "procs": args.procs, "threads": args.threads,
        "step_s": step_s, "fft": fft,
        "sample": (f"{args.procs} x spectral_ewald() ({args.mode}, N={args.N}, M={args.M}, "
                   f"P={args.P}, xi={args.xi}) per step, {args.steps} steps"),
    }))


if __name__ == "__main__":
    main()
