"""The allocation-free PAR3 solve entry point against the regular one.

pp_gf64_solve_and_reconstruct_noalloc is for callers that cannot allocate
device memory at the point where they need the repair solve (a device pool
owned by another allocator, latency-bound loops, services that must not run
out of memory after start-up).  It keeps its working storage in a fixed array
inside the library instead of allocating.

These checks call it through the C ABI on device buffers and compare it with
pp_gf64_solve_and_reconstruct (which allocates its scratch through a context)
on two calls in a row, so the second call also shows that what the first call
left in the shared array does not leak into its result.  Results are integer
GF(2^64) words: the comparison is bit-exact.  This file is collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def _system(oracle, seed, n, b):
    rng = np.random.default_rng(seed)
    cols = rng.choice(4 * n, n, replace=False)
    A = np.ascontiguousarray(oracle.gf64_build_cauchy(4 * n, n, 0, 4 * n)[:, cols])
    A[0, 0] = 0  # forces a row exchange in the first pivot step
    rhs = rng.integers(0, 2**64, (n, b), dtype=np.uint64)
    return A, rhs


def test_noalloc_solve_matches_regular_entry_point(ctx, oracle):
    import torch
    import parparpar_b200._lib as L

    for seed, n, b in [(101, 37, 64), (202, 120, 33)]:  # two calls in a row
        A, rhs = _system(oracle, seed, n, b)

        ref_A, ref_rhs = _dev(A), _dev(rhs)
        st = L.lib.pp_gf64_solve_and_reconstruct(ctx.h, ref_A.data_ptr(), ref_rhs.data_ptr(), n, b)
        ctx.synchronize()
        assert st == L.PP_OK

        new_A, new_rhs = _dev(A), _dev(rhs)
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream().cuda_stream
        st = L.lib.pp_gf64_solve_and_reconstruct_noalloc(new_A.data_ptr(), new_rhs.data_ptr(), n, b, stream)
        assert st == L.PP_OK

        assert np.array_equal(_host(new_rhs), _host(ref_rhs))
        assert np.array_equal(_host(new_A), _host(ref_A))
        # and both equal the oracle's solution
        oA, orhs = A.copy(), rhs.copy()
        assert oracle.gf64_solve_and_reconstruct(oA, orhs) == 0
        assert np.array_equal(_host(new_rhs), orhs)


def test_noalloc_solve_on_a_side_stream_and_singular(ctx, oracle):
    import torch
    import parparpar_b200._lib as L

    A, rhs = _system(oracle, 303, 50, 17)
    dA, dR = _dev(A), _dev(rhs)
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    assert L.lib.pp_gf64_solve_and_reconstruct_noalloc(dA.data_ptr(), dR.data_ptr(), 50, 17, side.cuda_stream) \
        == L.PP_OK
    oA, orhs = A.copy(), rhs.copy()
    oracle.gf64_solve_and_reconstruct(oA, orhs)
    assert np.array_equal(_host(dR), orhs)

    sing = np.zeros((3, 3), dtype=np.uint64)
    sing[0] = [1, 2, 3]
    sing[1] = [5, 7, 11]
    sing[2] = sing[0] ^ sing[1]
    srhs = np.arange(12, dtype=np.uint64).reshape(3, 4)
    a1, r1 = _dev(sing), _dev(srhs)
    a2, r2 = _dev(sing), _dev(srhs)
    torch.cuda.synchronize()
    st_ref = L.lib.pp_gf64_solve_and_reconstruct(ctx.h, a1.data_ptr(), r1.data_ptr(), 3, 4)
    st_new = L.lib.pp_gf64_solve_and_reconstruct_noalloc(a2.data_ptr(), r2.data_ptr(), 3, 4, None)
    assert st_ref == st_new == L.PP_ERR_SINGULAR


def test_noalloc_solve_rejects_sizes_above_the_limit(ctx):
    import parparpar_b200._lib as L
    import torch

    big = L.PP_NOALLOC_SOLVE_MAX_N + 1
    t = torch.zeros(16, dtype=torch.int64, device="cuda")
    assert L.lib.pp_gf64_solve_and_reconstruct_noalloc(t.data_ptr(), t.data_ptr(), big, 1, None) == \
        L.PP_ERR_TOO_LARGE
    # host buffers are refused (the entry point never stages through allocations)
    h = np.zeros(16, dtype=np.uint64)
    assert L.lib.pp_gf64_solve_and_reconstruct_noalloc(h.ctypes.data, h.ctypes.data, 2, 1, None) == \
        L.PP_ERR_INVALID_ARG
    # so is a device matrix beside a host right-hand side
    assert L.lib.pp_gf64_solve_and_reconstruct_noalloc(t.data_ptr(), h.ctypes.data, 2, 1, None) == \
        L.PP_ERR_INVALID_ARG
    # buffers on the current device are accepted (a 2 x 2 identity solves to itself)
    eye = torch.tensor([1, 0, 0, 1], dtype=torch.int64, device="cuda")
    r = torch.tensor([7, 9], dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    assert L.lib.pp_gf64_solve_and_reconstruct_noalloc(eye.data_ptr(), r.data_ptr(), 2, 1, None) == L.PP_OK
    assert r.cpu().tolist() == [7, 9]
    # buffers on another GPU are refused the same way
    if torch.cuda.device_count() > 1:
        other = torch.zeros(16, dtype=torch.int64, device="cuda:1")
        torch.cuda.synchronize(1)
        assert L.lib.pp_gf64_solve_and_reconstruct_noalloc(other.data_ptr(), other.data_ptr(), 2, 1, None) == \
            L.PP_ERR_INVALID_ARG
