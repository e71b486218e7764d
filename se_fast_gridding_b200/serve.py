"""Serving: a request loop of Spectral Ewald solves on one GPU (se_server_*).

The loop itself is native (csrc/se_serve.cu): requests are queued as they
arrive and admitted first come, first served whenever a solve slot (a CUDA
stream) is free and the plan they need fits the device-memory budget; plans
(grid, spectrum, particle buffers, cuFFT plans) are cached by (M, P, mode,
capacity class) and stay resident; admitted solves overlap on the device.
This module wraps it for numpy arrays and torch tensors, and generates the
Poisson request traces the benchmark replays.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import check, lib
from .solver import System, _prec


@dataclass
class Completion:
    ticket: int
    status: int
    queue_s: float
    latency_s: float

    @property
    def ok(self) -> bool:
        return self.status == _lib.SE_OK


def request_bytes(system: System, precision="fp32") -> int:
    """Device bytes the server charges for the plan a request needs."""
    s = system.c_struct()
    return int(lib().se_server_request_bytes(C.byref(s), _prec(precision)))


class Server:
    """se_server_create / submit / poll / drain / destroy for Python callers.

    Inputs and outputs are torch tensors (CUDA tensors make a device request,
    CPU tensors a host request; pin them for overlap) or numpy arrays (host).
    The server keeps each request's tensors referenced until it completes.
    """

    def __init__(self, slots: int = 8, precision="fp32", hbm_budget: int = 120 * 10 ** 9,
                 max_queue: int = 0):
        cfg = _lib.se_server_config(slots=slots, precision=_prec(precision),
                                    hbm_budget=int(hbm_budget), max_queue=max_queue)
        self.precision = precision
        self._s = C.c_void_p()
        check(lib().se_server_create(C.byref(self._s), C.byref(cfg)), "se_server_create")
        self._live: dict[int, tuple] = {}

    def reserve(self, systems) -> None:
        arr = (_lib.se_system * len(systems))(*[s.c_struct() for s in systems])
        check(lib().se_server_reserve(self._s, arr, len(systems)), "se_server_reserve")

    @staticmethod
    def _addr(a):
        if isinstance(a, torch.Tensor):
            if a.dtype != torch.float64 or not a.is_contiguous():
                raise ValueError("tensors must be contiguous float64")
            return a.data_ptr(), a.is_cuda
        if isinstance(a, np.ndarray):
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("arrays must be contiguous float64")
            return a.ctypes.data, False
        raise TypeError(type(a))

    def submit(self, system: System, x, q, out) -> int:
        """Queue one solve: x (3N SoA), q (N) in, out (N or 3N) written when it
        completes.  Returns the ticket."""
        (xp, xd), (qp, qd), (op, od) = self._addr(x), self._addr(q), self._addr(out)
        if not (xd == qd == od):
            raise ValueError("x, q and out must all be host or all be device memory")
        n = system.N
        if x.shape[0] != 3 * n or q.shape[0] != n or out.shape[0] != system.out_width * n:
            raise ValueError("x, q, out sizes do not match N")
        req = _lib.se_request(sys=system.c_struct(), x=xp, q=qp, out=op,
                              where=_lib.SE_WHERE_DEVICE if xd else _lib.SE_WHERE_HOST)
        t = C.c_longlong()
        check(lib().se_server_submit(self._s, C.byref(req), C.byref(t)), "se_server_submit")
        self._live[t.value] = (x, q, out)
        return t.value

    def poll(self, max_n: int = 4096) -> list[Completion]:
        buf = (_lib.se_completion * max_n)()
        n = C.c_int()
        check(lib().se_server_poll(self._s, buf, max_n, C.byref(n)), "se_server_poll")
        out = []
        for i in range(n.value):
            c = buf[i]
            self._live.pop(c.ticket, None)
            out.append(Completion(c.ticket, c.status, c.queue_s, c.latency_s))
        return out

    def drain(self, timeout: float | None = None) -> None:
        check(lib().se_server_drain(self._s, -1.0 if timeout is None else float(timeout)),
              "se_server_drain")

    def stats(self) -> dict:
        st = _lib.se_server_stats()
        check(lib().se_server_get_stats(self._s, C.byref(st)), "se_server_get_stats")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def close(self) -> None:
        if self._s:
            lib().se_server_destroy(self._s)
            self._s = C.c_void_p()
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------- traces ----

def grid_for(N: int, n0: int = 16000, m_min: int = 64, m_cap: int = 256) -> int:
    """Grid size of a served request: M = 64 * 2^ceil(log2(N / n0) / 3), at
    least 64 and at most 256, so the particles per grid cell stay within a
    factor of 8 as N grows."""
    if N <= n0:
        return m_min
    return min(m_cap, m_min * 2 ** math.ceil(math.log2(N / n0) / 3))


@dataclass
class TraceRequest:
    t: float           # arrival time, seconds from the start of the trace
    system: System
    offset: int        # where its positions start in the particle pool


def poisson_trace(rate: float, duration: float, seed: int = 4, n_min: int = 500,
                  n_max: int = 2_000_000, L: float = 1.0, literal_grid: bool = False,
                  pool: int = 6_000_000) -> list[TraceRequest]:
    """Arrivals of a Poisson process at `rate` per second over `duration`:
    POTENTIAL or FORCE with equal odds, N log-uniform in [n_min, n_max], P
    from {8, 12, 16}, M from grid_for(N) (M = 64 for every request with
    literal_grid), xi = 8 M / (64 L) so that xi h is that of M = 64, xi = 8/L."""
    rng = np.random.Generator(np.random.Philox(seed))
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        N = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        M = 64 if literal_grid else grid_for(N)
        P = int(rng.choice([8, 12, 16]))
        mode = "force" if rng.random() < 0.5 else "potential"
        xi = 8.0 * M / (64.0 * L)
        off = int(rng.integers(0, pool - 3 * N + 1))
        out.append(TraceRequest(t, System(N, M, P, L, xi, None, mode), off))
    return out


def particle_pool(size: int = 6_000_000, L: float = 1.0, seed: int = 7, pin: bool = True):
    """Uniform coordinates in [0, L) and charges +-1, as host tensors.  Any
    3N consecutive coordinates are the SoA positions of N uniform particles
    and any N consecutive charges their charges, so each request is a slice."""
    rng = np.random.Generator(np.random.Philox(seed))
    xs = torch.from_numpy(rng.random(size) * L)
    qs = torch.from_numpy(np.where(rng.random(size) < 0.5, -1.0, 1.0))
    if pin:
        xs, qs = xs.pin_memory(), qs.pin_memory()
    return xs, qs


def output_arena(trace: list[TraceRequest], pin: bool = True) -> torch.Tensor:
    """One host buffer holding every request's output of a trace back to back
    (pinned: allocating pinned memory while the GPU is busy can wait for it
    to go idle, so a server's result buffers are set up beforehand)."""
    n = sum(r.system.out_width * r.system.N for r in trace)
    return torch.empty(max(n, 1), dtype=torch.float64, pin_memory=pin)


def replay(server: Server, trace: list[TraceRequest], xs: torch.Tensor, qs: torch.Tensor,
           arena: torch.Tensor | None = None, keep_outputs: bool = False):
    """Submit each request at its arrival time (real time), collect the
    completions.  Outputs go to consecutive slices of `arena` (one is made when
    none is given; it must hold every output of the trace).  Returns
    (completions by ticket, outputs by ticket or None, wall seconds from the
    first arrival to the last completion, the largest lag of a submission
    behind its arrival)."""
    if arena is None:
        arena = output_arena(trace, pin=xs.is_pinned())
    tickets, outs, comps = {}, {}, {}
    off = 0
    start = time.perf_counter()
    lag = 0.0
    for k, r in enumerate(trace):
        while True:
            now = time.perf_counter() - start
            if now >= r.t:
                break
            for c in server.poll():
                comps[c.ticket] = c
            if r.t - now > 2e-4:
                time.sleep(min(r.t - now - 1e-4, 1e-3))
        lag = max(lag, time.perf_counter() - start - r.t)
        s = r.system
        x = xs[r.offset:r.offset + 3 * s.N]
        q = qs[r.offset:r.offset + s.N]
        w = s.out_width * s.N
        out = arena[off:off + w]
        off += w
        t = server.submit(s, x, q, out)
        tickets[t] = k
        if keep_outputs:
            outs[t] = out
    server.drain()
    end = time.perf_counter()
    for c in server.poll():
        comps[c.ticket] = c
    return comps, (outs if keep_outputs else None), end - start, lag


def latency_summary(comps) -> dict:
    lat = np.array([c.latency_s for c in comps.values()])
    qd = np.array([c.queue_s for c in comps.values()])
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "max_ms": float(lat.max() * 1e3),
            "queue_p50_ms": float(np.percentile(qd, 50) * 1e3),
            "queue_p99_ms": float(np.percentile(qd, 99) * 1e3),
            "failed": int(sum(1 for c in comps.values() if not c.ok))}
