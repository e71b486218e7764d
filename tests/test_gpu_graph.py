"""Repeated solves replayed from a CUDA graph (se_plan_set_graph,
se_batch_set_graph, and the host-buffer entry point's own graph) give exactly
the direct solves' results: positions that change in place between steps, a
new particle count (a new capture), new box parameters between replays, and
batches."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from se_fast_gridding_b200 import solver, workloads
    return torch, solver, workloads


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("M,P", [(32, 8), (24, 6)])   # tile-aligned kernels and the others
def test_graph_replay_equals_direct(env, prec, M, P):
    torch, S, W = env
    s = torch.cuda.Stream()
    N = 3000
    g = S.SpectralEwald(M, P, 1.0, 8.0, None, "force", prec, N)
    d = S.SpectralEwald(M, P, 1.0, 8.0, None, "force", prec, N)
    g.set_graph(True)
    with torch.cuda.stream(s):
        x = torch.empty(3 * N, dtype=torch.float64, device="cuda")
        q = torch.empty(N, dtype=torch.float64, device="cuda")
        out = torch.empty(3 * N, dtype=torch.float64, device="cuda")
        launches = []
        for step in range(5):
            xs, qs = W.synthetic_system(N, 1.0, seed=100 + step, charges="uniform")
            x.copy_(torch.from_numpy(xs))
            q.copy_(torch.from_numpy(qs))
            g.solve(x, q, out, stream=s)
            ref = d.solve(x, q, stream=s)
            s.synchronize()
            np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())
            launches.append(g.launches)
        assert launches[2:] == [d.launches] * 3     # replays launch the same kernels
        # a smaller particle count on the same buffers: a new capture
        n2 = 1700
        g.solve(x[:3 * n2].contiguous(), q[:n2], out[:3 * n2], stream=s)
        for _ in range(2):
            x2, q2 = x[:3 * n2].contiguous(), q[:n2].contiguous()
            o2 = out[:3 * n2]
            g.solve(x2, q2, o2, stream=s)
            r2 = d.solve(x2, q2, stream=s)
            s.synchronize()
            np.testing.assert_array_equal(o2.cpu().numpy(), r2.cpu().numpy())
        # other box parameters between replays (read from the device table)
        xl = torch.empty_like(x)
        for L in (1.5, 2.0, 2.5, 3.0):   # direct, capture, replay, replay
            sysL = S.System(N=N, M=M, P=P, L=L, xi=8.0 / L, mode="force")
            xl.copy_(x * L)
            g.solve_system(sysL, xl, q, out, stream=s)
            ref = S.SpectralEwald(M, P, L, 8.0 / L, None, "force", prec, N).solve(xl, q,
                                                                                 stream=s)
            s.synchronize()
            np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())
    # stage timing inside replays
    g.set_timing(True)
    for _ in range(3):
        g.solve(x, q, out, stream=s)
    ms = g.stage_ms()
    assert all(v > 0 for v in ms.values()), ms
    g.close()
    d.close()


def test_batch_graph_equals_direct(env):
    torch, S, W = env
    s = torch.cuda.Stream()
    systems = [S.System(N=900 + 300 * i, M=(32, 24)[i % 2], P=(8, 12, 16)[i % 3],
                        L=1.0 + 0.5 * i, xi=8.0 / (1.0 + 0.5 * i),
                        mode=("potential", "force")[i % 2]) for i in range(5)]
    bg = S.BatchSolver(systems, "fp32")
    bd = S.BatchSolver(systems, "fp32")
    bg.set_graph(True)
    with torch.cuda.stream(s):
        xs, qs = zip(*[W.synthetic_system(t.N, t.L, seed=7 + i) for i, t in enumerate(systems)])
        x, q = bg.pack(xs, qs)
        out = torch.empty(int(bg.out_off[-1]), dtype=torch.float64, device="cuda")
        for step in range(4):
            x.mul_(0.999)                                  # every particle moves, in place
            bg.solve(x, q, out, stream=s)
            ref = bd.solve(x, q, stream=s)
            s.synchronize()
            np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())
    bg.close()
    bd.close()


@pytest.mark.parametrize("prec", ["fp32", "fp64", "fp32-fft32"])
def test_host_entry_replays_equal_device_solves(env, prec):
    """se_solve_host captures its solve on the second call with a given N and
    replays it after that: new host buffers and contents every call, pinned or
    pageable, a caller stream or the default one, N changing back and forth,
    and an input error reported from a replay."""
    torch, S, W = env
    from se_fast_gridding_b200 import _lib
    N = 2500
    se = S.SpectralEwald(32, 8, 1.0, 8.0, None, "force", prec, N)
    ref = S.SpectralEwald(32, 8, 1.0, 8.0, None, "force", prec, N)
    side = torch.cuda.Stream()
    for step, n in enumerate([N, N, N, 1200, 1200, N, 1200, 1200]):
        xs, qs = W.synthetic_system(n, 1.0, seed=300 + step, charges="uniform")
        if step % 2:
            xh, qh = torch.tensor(xs).pin_memory(), torch.tensor(qs).pin_memory()
            oh = torch.empty(3 * n, dtype=torch.float64).pin_memory()
            se.solve_host_ptr(n, xh.data_ptr(), qh.data_ptr(), oh.data_ptr(),
                              stream=side if step % 4 == 1 else None)
            got = oh.numpy()
        else:
            got = se.solve_host(xs, qs)
        want = ref.solve(torch.tensor(xs, device="cuda"), torch.tensor(qs, device="cuda"))
        np.testing.assert_array_equal(got, want.cpu().numpy())
    bad = W.synthetic_system(1200, 1.0, seed=9)[0]
    bad[5] = np.nan
    for _ in range(3):   # direct, captured and replayed with this N: reported every time
        with pytest.raises(_lib.SEError):
            se.solve_host(bad, np.ones(1200))
    xs, qs = W.synthetic_system(1200, 1.0, seed=10)
    np.testing.assert_array_equal(se.solve_host(xs, qs), ref.solve(
        torch.tensor(xs, device="cuda"), torch.tensor(qs, device="cuda")).cpu().numpy())
    se.close()
    ref.close()
