"""The serving loop (se_server_*) and plan re-pointing (se_solve_system).

Each served result must be bit-identical to the same system solved alone on
a plan made for it: alone or in a mix, on one slot or many, whether its plan
was cached, new or rebuilt after an eviction, with host or device buffers.
FP64 results are also within 1e-12 relative RMS of the CPU oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from se_fast_gridding_b200 import serve, solver
    return serve, solver


def mixed_requests(S, n, seed, n_max=20000, grids=(32, 64)):
    import oracle as O
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(n):
        N = int(np.exp(rng.uniform(np.log(200), np.log(n_max))))
        M = int(rng.choice(grids))
        P = int(rng.choice([8, 12, 16]))
        L = float(rng.uniform(1, 3))
        mode = "force" if rng.random() < 0.5 else "potential"
        s = S.System(N=N, M=M, P=P, L=L, xi=8.0 * M / (64 * L), mode=mode)
        x, q = O.synthetic_system(N, L, seed=seed * 1000 + i)
        out.append((s, x, q))
    return out


def solve_alone(S, s, x, q, prec):
    import torch
    se = S.SpectralEwald(s.M, s.P, s.L, s.xi, s.m, s.mode, prec, s.N)
    o = se.solve(torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda")).cpu().numpy()
    se.close()
    return o


def serve_all(serve, reqs, prec, slots, budget, device=False, one_at_a_time=False):
    import torch
    outs = []
    with serve.Server(slots=slots, precision=prec, hbm_budget=budget) as srv:
        tickets = []
        for s, x, q in reqs:
            if device:
                xt, qt = torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda")
                ot = torch.empty(s.out_width * s.N, dtype=torch.float64, device="cuda")
            else:
                xt = torch.tensor(x).pin_memory()
                qt = torch.tensor(q).pin_memory()
                ot = torch.empty(s.out_width * s.N, dtype=torch.float64).pin_memory()
            tickets.append(srv.submit(s, xt, qt, ot))
            outs.append(ot)
            if one_at_a_time:
                srv.drain()
        srv.drain()
        comps = {c.ticket: c for c in srv.poll()}
        stats = srv.stats()
    assert sorted(comps) == sorted(tickets)
    assert all(c.ok for c in comps.values()), [c.status for c in comps.values()]
    assert all(c.latency_s >= c.queue_s >= 0 for c in comps.values())
    return [o.cpu().numpy() for o in outs], stats


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_solve_system_repoints_plan(env, prec):
    """One plan per (M, P, mode) serves systems of other N, L and xi."""
    import torch
    serve, S = env
    reqs = mixed_requests(S, 12, seed=3, n_max=5000, grids=(32,))
    reqs = [r for r in reqs if r[0].P == 12 and r[0].mode == "force"] or reqs[:1]
    s0 = reqs[0][0]
    big = S.SpectralEwald(s0.M, s0.P, 1.0, 8.0, None, s0.mode, prec, 8192)
    for s, x, q in reqs + reqs[::-1]:
        if (s.M, s.P, s.mode) != (s0.M, s0.P, s0.mode):
            continue
        got = big.solve_system(s, torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda"))
        np.testing.assert_array_equal(got.cpu().numpy(), solve_alone(S, s, x, q, prec))
    big.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_served_results_equal_alone_and_in_mix(env, prec):
    import oracle as O
    serve, S = env
    reqs = mixed_requests(S, 24, seed=11)
    alone = [solve_alone(S, s, x, q, prec) for s, x, q in reqs]
    one, st1 = serve_all(serve, reqs, prec, slots=1, budget=40 << 30, one_at_a_time=True)
    mix, st8 = serve_all(serve, reqs, prec, slots=8, budget=40 << 30)
    for a, b, c in zip(alone, one, mix):
        np.testing.assert_array_equal(b, a)
        np.testing.assert_array_equal(c, a)
    assert st8["completed"] == len(reqs) and st8["failed"] == 0
    assert st8["plans_created"] <= st8["completed"]
    if prec == "fp64":
        for (s, x, q), a in list(zip(reqs, alone))[:4]:
            ref = O.spectral_ewald(x, q, s.M, s.P, S.default_m(s.P), s.L, s.xi, s.mode)
            assert O.rel_rms(a, ref) < FP64_TOL


def test_tight_budget_evicts_and_stays_exact(env):
    serve, S = env
    reqs = mixed_requests(S, 16, seed=12)
    need = max(serve.request_bytes(s, "fp32") for s, _, _ in reqs)
    budget = int(2.2 * need)
    alone = [solve_alone(S, s, x, q, "fp32") for s, x, q in reqs]
    got, st = serve_all(serve, reqs, "fp32", slots=4, budget=budget)
    for a, b in zip(alone, got):
        np.testing.assert_array_equal(b, a)
    assert st["plans_evicted"] > 0
    assert st["hbm_peak"] <= budget


def test_device_requests_equal_host_requests(env):
    serve, S = env
    reqs = mixed_requests(S, 10, seed=13)
    host_out, _ = serve_all(serve, reqs, "fp32", slots=4, budget=40 << 30)
    dev_out, _ = serve_all(serve, reqs, "fp32", slots=4, budget=40 << 30, device=True)
    for a, b in zip(host_out, dev_out):
        np.testing.assert_array_equal(a, b)


def test_server_errors(env):
    import torch
    from se_fast_gridding_b200 import _lib
    serve, S = env
    reqs = mixed_requests(S, 3, seed=14, n_max=2000)
    with serve.Server(slots=2, precision="fp32", hbm_budget=8 << 30) as srv:
        # a non-finite position fails that request only
        s, x, q = reqs[0]
        xb = x.copy()
        xb[5] = np.nan
        bad = srv.submit(s, torch.tensor(xb).pin_memory(), torch.tensor(q).pin_memory(),
                         torch.empty(s.out_width * s.N, dtype=torch.float64).pin_memory())
        good = []
        for s, x, q in reqs[1:]:
            good.append(srv.submit(s, torch.tensor(x).pin_memory(), torch.tensor(q).pin_memory(),
                                   torch.empty(s.out_width * s.N, dtype=torch.float64)
                                   .pin_memory()))
        srv.drain(timeout=60)
        comps = {c.ticket: c for c in srv.poll()}
        assert comps[bad].status == _lib.SE_ERR_INPUT
        assert all(comps[t].ok for t in good)
        # a request whose plan alone exceeds the budget is refused at submit
        huge = S.System(N=1000, M=1024, P=16, L=1.0, xi=8.0, mode="force")
        x, q = np.zeros(3000), np.zeros(1000)
        with pytest.raises(_lib.SEError):
            srv.submit(huge, torch.tensor(x), torch.tensor(q), torch.empty(3000, dtype=torch.float64))
        # sizes that do not match N
        s, x, q = reqs[1]
        with pytest.raises(ValueError):
            srv.submit(s, torch.tensor(x[:-1]), torch.tensor(q), torch.empty(s.N))
        st = srv.stats()
        assert st["failed"] == 1 and st["completed"] == 3
    with pytest.raises(_lib.SEError):
        serve.Server(slots=0)


def test_queue_limit(env):
    import torch
    from se_fast_gridding_b200 import _lib
    serve, S = env
    s, x, q = mixed_requests(S, 1, seed=15, n_max=1000)[0]
    xt, qt = torch.tensor(x).pin_memory(), torch.tensor(q).pin_memory()
    pool = [torch.empty(s.out_width * s.N, dtype=torch.float64).pin_memory() for _ in range(64)]
    with serve.Server(slots=1, precision="fp32", hbm_budget=8 << 30, max_queue=2) as srv:
        outs, refused = [], 0
        for o in pool:
            try:
                srv.submit(s, xt, qt, o)
                outs.append(o)
            except _lib.SEError as e:
                assert "queue full" in str(e)
                refused += 1
        srv.drain(timeout=60)
        assert refused > 0
        assert srv.stats()["completed"] == len(outs)
        for o in outs[1:]:
            np.testing.assert_array_equal(o.numpy(), outs[0].numpy())
