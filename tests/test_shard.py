"""Host-side logic of the multi-GPU path, on CPU: assignment of independent
systems to ranks, admission by device-memory footprint, and the gather of
per-system results across a world-size-2 gloo group (the per-system compute
here is the CPU oracle; on GPUs it is a BatchSolver per rank)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from se_fast_gridding_b200 import shard


class Sys:
    def __init__(self, N, M, P):
        self.N, self.M, self.P = N, M, P


def test_partition_is_balanced_and_complete():
    rng = np.random.Generator(np.random.Philox(1))
    systems = [Sys(int(rng.integers(1000, 64000)), 64, int(rng.choice([8, 12, 16])))
               for _ in range(256)]
    for world in (1, 2, 4, 8):
        shards = shard.partition(systems, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(256))
        loads = [sum(shard.system_cost(systems[i]) for i in s) for s in shards]
        assert max(loads) <= 1.05 * (sum(loads) / world) + max(shard.system_cost(s) for s in systems)
        assert shards == shard.partition(systems, world)   # deterministic


def test_admit_by_footprint():
    items = [5, 3, 8, 1, 4]
    taken, rest = shard.admit(items, 10, footprint=lambda b: b)
    assert taken == [0, 1, 3] and rest == [2, 4]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, result_q):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle as O
    from se_fast_gridding_b200 import shard as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    systems = [Sys(40 + 10 * i, 8 + 2 * (i % 3), 4 + (i % 2)) for i in range(6)]
    mine = S.partition(systems, world)[rank]
    outs = []
    for i in mine:
        s = systems[i]
        x, q = O.synthetic_system(s.N, 1.0, seed=i)
        outs.append(O.spectral_ewald(x, q, s.M, s.P, 0.9 * np.sqrt(O.PI * s.P), 1.0, 4.0))
    allout = S.gather_outputs(mine, outs, len(systems))
    t = S.max_over_ranks(float(rank + 1))
    if rank == 0:
        result_q.put((allout, t))
    dist.destroy_process_group()


def test_sharded_results_equal_single_process(oracle_mod):
    O = oracle_mod
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    allout, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert tmax == 2.0
    for i in range(6):
        s = Sys(40 + 10 * i, 8 + 2 * (i % 3), 4 + (i % 2))
        x, qq = O.synthetic_system(s.N, 1.0, seed=i)
        ref = O.spectral_ewald(x, qq, s.M, s.P, 0.9 * np.sqrt(O.PI * s.P), 1.0, 4.0)
        np.testing.assert_array_equal(allout[i], ref)
