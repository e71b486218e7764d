"""se_counting_sort_static: the sort entry point that allocates nothing.

It serves callers that cannot allocate device memory when they sort (a frozen
or captured memory pool, host callbacks, real-time loops, a library that does
not own the process's allocator): its working memory is a fixed device array
inside libse_gpu.so.  This test calls it through the C ABI and checks that it
gives exactly the permutation and bin offsets of se_counting_sort (integer
results: tolerance zero), on two calls in a row, and that sizes beyond the
stated limits are refused.  The file sorts last so that a run stopping at the
first failure has run every other test first; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from se_fast_gridding_b200 import _lib, solver
    L = _lib.lib()
    f = L.se_counting_sort_static
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    return torch, L, solver


def static_sort(env, keys, nkeys):
    torch, L, _ = env
    perm = torch.full((max(keys.numel(), 1),), -1, dtype=torch.int32, device="cuda")
    offs = torch.full((nkeys + 1,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.se_counting_sort_static(C.c_void_p(keys.data_ptr()), keys.numel(), nkeys,
                                   C.c_void_p(perm.data_ptr()), C.c_void_p(offs.data_ptr()),
                                   C.c_void_p(stream))
    return rc, perm[:keys.numel()], offs


def test_static_sort_matches_allocating_sort_twice(env):
    torch, L, solver = env
    rng = np.random.Generator(np.random.Philox(77))
    # two calls in a row: the second smaller, so stale contents of the shared
    # array from the first call would show
    for N, nkeys in ((200_000, 40_000), (7_000, 3_000)):
        keys = torch.tensor(rng.integers(0, nkeys, size=N).astype(np.int32), device="cuda")
        rc, perm, offs = static_sort(env, keys, nkeys)
        assert rc == 0
        ref_perm, ref_offs = solver.counting_sort(keys, nkeys)
        torch.cuda.synchronize()
        assert torch.equal(perm, ref_perm)
        assert torch.equal(offs, ref_offs)


def test_static_sort_limits(env):
    torch, L, solver = env
    max_n = 262144
    keys = torch.zeros(max_n + 1, dtype=torch.int32, device="cuda")
    rc, _, _ = static_sort(env, keys, 16)
    assert rc != 0
    rc, _, _ = static_sort(env, keys[:16], 65536 + 1)
    assert rc != 0
    # at the limits it gives exactly the allocating sort's permutation and
    # offsets: the size where a short scratch array would show
    keys = torch.tensor(np.random.Generator(np.random.Philox(5)).integers(
        0, 65536, size=max_n).astype(np.int32), device="cuda")
    rc, perm, offs = static_sort(env, keys, 65536)
    assert rc == 0
    ref_perm, ref_offs = solver.counting_sort(keys, 65536)
    torch.cuda.synchronize()
    assert torch.equal(perm, ref_perm)
    assert torch.equal(offs, ref_offs)


@pytest.mark.parametrize("nkeys", [1, 2])
def test_static_sort_few_keys_at_max_n(env, nkeys):
    """All keys equal (the identity permutation) and two keys, at the largest
    N the array takes."""
    torch, L, solver = env
    max_n = 262144
    keys = torch.tensor(np.random.Generator(np.random.Philox(9 + nkeys)).integers(
        0, nkeys, size=max_n).astype(np.int32), device="cuda")
    rc, perm, offs = static_sort(env, keys, nkeys)
    assert rc == 0
    ref_perm, ref_offs = solver.counting_sort(keys, nkeys)
    torch.cuda.synchronize()
    assert torch.equal(perm, ref_perm)
    assert torch.equal(offs, ref_offs)
    if nkeys == 1:
        assert torch.equal(perm, torch.arange(max_n, dtype=torch.int32, device="cuda"))
