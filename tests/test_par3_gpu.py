"""PAR3 / GF(2^64) parity on the GPU: the CUDA kernels through the C ABI
against the golden fixtures and the oracle, bit-exact."""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["lut", "tensor"])
def kctx(ctx, request):
    """The default context with the GF(2^64) region kernel forced to one
    implementation (the tensor kernel applies where rows are 16-byte aligned
    and the word count is even; other shapes use the lookup kernel)."""
    import parparpar_b200._lib as L
    ctx.set_gf64_kernel(L.PP_GF16_KERNEL_LUT if request.param == "lut" else L.PP_GF16_KERNEL_TENSOR)
    yield ctx
    ctx.set_gf64_kernel(L.PP_GF16_KERNEL_AUTO)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def test_par3_golden_all_kernels(kctx, golden):
    from parparpar_b200 import par3
    g = golden("par3_golden.npz")
    inp = g["inputs"]
    for fn in (par3.compute_recovery, par3.compute_recovery_full, par3.compute_recovery_barycentric,
               par3.compute_recovery_fenger):
        out = np.zeros((2, 128), dtype=np.uint64)
        fn(inp, out, 5, 2, 1024, 0, 5)
        assert zlib.crc32(out.tobytes()) == 0x6A941C15, fn.__name__


def test_gf64_ops_golden(kctx, golden):
    from parparpar_b200 import par3
    g = golden("gf64_ops.npz")
    a, b = g["a"], g["b"]
    out = np.zeros_like(a)
    for i in range(0, 64):
        par3.gf64_region_mul(out[i:i + 1], a[i:i + 1], 1, int(b[i]), kctx)
    assert np.array_equal(out[:64], g["prod"][:64])
    par3.gf64_region_mul_arr(out, a, b, a.size, 1)  # n_coeff=1: all by b[0]
    inv = np.zeros_like(a)
    par3.gf64_inverse_batch(inv, a, a.size, kctx)
    assert np.array_equal(inv, g["inv"])
    assert np.array_equal(par3.GF64Controller.BuildCauchyMatrixAlloc(37, 9, 3, 40), g["cauchy"])
    assert np.array_equal(par3.GF64Controller.BuildCauchyMatrixAlloc(8, 4, 0, 2), g["cauchy_clash"])
    out = np.zeros((7, 96), dtype=np.uint64)
    par3.GF64Controller.ComputeRecoveryBlocks(g["inp"], 33, out, 7, 96, 0, 33)
    assert np.array_equal(out, g["matvec"])
    out = g["acc0"].copy()
    par3.GF64Controller.ComputeRecoveryBlocks(g["inp"], 33, out, 7, 96, 0, 33, accumulate=True)
    assert np.array_equal(out, g["matvec_acc"])
    A, rhs = g["A"].copy(), g["rhs"].copy()
    assert par3.GF64Controller.SolveAndReconstruct(A, rhs, A.shape[0], rhs.shape[1]) == 0
    assert np.array_equal(rhs, g["solved"])
    assert par3.GF64Controller.SolveAndReconstruct(g["sing"].copy(), g["sing_rhs"].copy(), 3, 4) == -1


def test_region_elementwise_vs_oracle(ctx, oracle):
    from parparpar_b200 import par3
    rng = np.random.default_rng(40)
    for n in (1, 7, 1000, 4097):
        x = rng.integers(0, 2**64, n, dtype=np.uint64)
        for nc in (1, 3, 8):
            c = rng.integers(0, 2**64, nc, dtype=np.uint64)
            out = np.zeros(n, dtype=np.uint64)
            par3.gf64_region_mul_arr(out, x, c, n, nc)
            assert np.array_equal(out, oracle.gf64_region("mul_arr", x, c, np.zeros(n, dtype=np.uint64)))
            base = rng.integers(0, 2**64, n, dtype=np.uint64)
            out = base.copy()
            par3.gf64_region_muladd_arr(out, x, c, n, nc)
            assert np.array_equal(out, oracle.gf64_region("muladd_arr", x, c, base.copy()))
        out = np.zeros(n, dtype=np.uint64)
        par3.gf64_region_mul(out, x, n, 0xDEADBEEFCAFEBABE)
        assert np.array_equal(out, oracle.gf64_region("mul", x, 0xDEADBEEFCAFEBABE, np.zeros(n, dtype=np.uint64)))


@pytest.mark.parametrize("n,r,b,fi,fr", [
    (1, 1, 1, 0, 1), (2, 7, 3, 0, 2), (5, 8, 128, 0, 5), (64, 9, 1000, 0, 64), (257, 33, 1025, 0, 257),
    (300, 8, 1024, 0, 300), (40, 17, 64, 5, 3), (1024, 1, 2048, 0, 1024), (3000, 8, 16, 0, 3000),
    (3, 5, 514, 0, 3), (4001, 3, 1026, 7, 9000),
])
def test_compute_recovery_vs_oracle(kctx, oracle, n, r, b, fi, fr):
    from parparpar_b200 import par3
    rng = np.random.default_rng(n + r * 7 + b * 13)
    inp = rng.integers(0, 2**64, (n, b), dtype=np.uint64)
    exp = oracle.gf64_compute_recovery(inp, r, fi, fr)
    out = np.zeros((r, b), dtype=np.uint64)
    par3.GF64Controller.ComputeRecoveryBlocks(inp, n, out, r, b, fi, fr)
    assert np.array_equal(out, exp)
    base = rng.integers(0, 2**64, (r, b), dtype=np.uint64)
    out = base.copy()
    par3.GF64Controller.ComputeRecoveryBlocks(inp, n, out, r, b, fi, fr, accumulate=True)
    assert np.array_equal(out, exp ^ base)
    # device-resident buffers
    dout = _dev(np.zeros((r, b), dtype=np.uint64))
    par3.GF64Controller.ComputeRecoveryBlocks(_dev(inp), n, dout, r, b, fi, fr)
    kctx.synchronize()
    assert np.array_equal(_host(dout), exp)


def test_with_coeff_and_build(kctx, oracle):
    from parparpar_b200 import par3
    rng = np.random.default_rng(41)
    n, r, b = 70, 11, 300
    coeff = rng.integers(0, 2**64, (r, n), dtype=np.uint64)
    inp = rng.integers(0, 2**64, (n, b), dtype=np.uint64)
    out = np.zeros((r, b), dtype=np.uint64)
    par3.GF64Controller.ComputeRecoveryBlocksWithCoeff(inp, n, out, r, b, coeff)
    assert np.array_equal(out, oracle.gf64_matvec(inp, coeff))
    m = np.zeros((r, n), dtype=np.uint64)
    par3.GF64Controller.BuildCauchyMatrix(m, n, r, 2**40 + 3, 2**41 + 5)
    assert np.array_equal(m, oracle.gf64_build_cauchy(n, r, 2**40 + 3, 2**41 + 5))
    dm = _dev(np.zeros((r, n), dtype=np.uint64))
    par3.GF64Controller.BuildCauchyMatrix(dm, n, r, 7, 1000)
    kctx.synchronize()
    assert np.array_equal(_host(dm), oracle.gf64_build_cauchy(n, r, 7, 1000))


def test_pointer_table_region_ops(kctx, oracle):
    from parparpar_b200 import par3
    rng = np.random.default_rng(42)
    L, K, G = 777, 5, 9
    ins = [rng.integers(0, 2**64, L, dtype=np.uint64) for _ in range(G)]
    C = rng.integers(0, 2**64, (K, 12), dtype=np.uint64)  # K_stride 12 > G
    outs = [rng.integers(0, 2**64, L, dtype=np.uint64) for _ in range(K)]
    exp = [o.copy() for o in outs]
    for k in range(K):
        for g in range(G):
            oracle.gf64_region("muladd_arr", ins[g], C[k, g], exp[k])
    par3.gf64_region_2d_muladd_arr(outs, K, ins, G, C, 12, L)
    for k in range(K):
        assert np.array_equal(outs[k], exp[k])
    # coupled: G inputs -> 1 output
    out = rng.integers(0, 2**64, L, dtype=np.uint64)
    e = out.copy()
    cb = C[0, :G].copy()
    for g in range(G):
        oracle.gf64_region("muladd_arr", ins[g], cb[g], e)
    par3.gf64_region_coupled_muladd_arr(out, ins, cb, L, G)
    assert np.array_equal(out, e)
    # fused output: 1 input -> K outputs, device buffers
    douts = [_dev(o) for o in outs]
    starts = [C[k, 3:4].copy() for k in range(K)]
    e = [o.copy() for o in outs]
    for k in range(K):
        oracle.gf64_region("muladd_arr", ins[0], starts[k][0], e[k])
    par3.gf64_region_fused_output_muladd_arr(douts, _dev(ins[0]), starts, L, K)
    for k in range(K):
        assert np.array_equal(_host(douts[k]), e[k])


def test_solve_vs_oracle(ctx, oracle):
    from parparpar_b200 import par3
    rng = np.random.default_rng(43)
    for n, b in [(1, 5), (2, 1), (17, 33), (120, 64)]:
        # a Cauchy submatrix with one zero forcing a row swap
        A = oracle.gf64_build_cauchy(400, n, 0, 400)[:, rng.choice(400, n, replace=False)].copy()
        if n > 1:
            A[0, 0] = 0
        rhs = rng.integers(0, 2**64, (n, b), dtype=np.uint64)
        A1, r1 = A.copy(), rhs.copy()
        rc = oracle.gf64_solve_and_reconstruct(A1, r1)
        A2, r2 = A.copy(), rhs.copy()
        assert par3.GF64Controller.SolveAndReconstruct(A2, r2, n, b) == rc
        if rc == 0:
            assert np.array_equal(r2, r1)
            assert np.array_equal(A2, A1)


def test_par3_repair_roundtrip(kctx):
    """create -> erase -> (RHS via with_coeff) -> solve restores the blocks."""
    from parparpar_b200 import par3
    rng = np.random.default_rng(44)
    N, R, B = 400, 16, 256
    data = rng.integers(0, 2**64, (N, B), dtype=np.uint64)
    rec = np.zeros((R, B), dtype=np.uint64)
    par3.GF64Controller.ComputeRecoveryBlocks(data, N, rec, R, B, 0, N)
    lost = np.sort(rng.choice(N, 10, replace=False))
    n = lost.size
    M = par3.GF64Controller.BuildCauchyMatrixAlloc(N, n, 0, N)
    known = np.setdiff1d(np.arange(N), lost)
    A = np.ascontiguousarray(M[:, lost])
    rhs = rec[:n].copy()
    par3.GF64Controller.ComputeRecoveryBlocksWithCoeff(np.ascontiguousarray(data[known]), known.size, rhs, n, B,
                                                       np.ascontiguousarray(M[:, known]), accumulate=True)
    assert par3.GF64Controller.SolveAndReconstruct(A, rhs, n, B) == 0
    assert np.array_equal(rhs, data[lost])


def test_par3_repair_fused_vs_oracle(kctx, oracle):
    """pp_gf64_repair (the decode of lib/par3gen.js:3840-4010 on the device):
    restores the lost blocks; with an absent recovery block (its rhs row
    zero-filled, as the reference does) it matches the oracle's solution of
    the same system bit for bit."""
    from parparpar_b200 import par3
    rng = np.random.default_rng(45)
    N, R, B = 300, 12, 96
    data = rng.integers(0, 2**64, (N, B), dtype=np.uint64)
    rec = oracle.gf64_compute_recovery(data, R, 0, N)
    lost = np.sort(rng.choice(N, 7, replace=False))
    n = lost.size
    damaged = data.copy()
    damaged[lost] = rng.integers(0, 2**64, (n, B), dtype=np.uint64)  # lost rows must not be read
    restored = par3.repair(damaged, lost, rec[:n].copy(), B, 0, N, ctx=kctx)
    assert np.array_equal(restored, data[lost])
    # device buffers
    d_out = _dev(np.zeros((n, B), dtype=np.uint64))
    par3.repair(_dev(damaged), lost, _dev(rec[:n]), B, 0, N, restored=d_out, ctx=kctx)
    kctx.synchronize()
    assert np.array_equal(_host(d_out), data[lost])
    # recovery block 3 absent: rhs row 3 zero
    present = np.ones(n, dtype=np.uint8)
    present[3] = 0
    got = par3.repair(damaged, lost, rec[:n].copy(), B, 0, N, recovery_present=present, ctx=kctx)
    M = oracle.gf64_build_cauchy(N, n, 0, N)
    known = np.setdiff1d(np.arange(N), lost)
    rhs = rec[:n].copy()
    rhs[3] = 0
    oracle.gf64_matvec(np.ascontiguousarray(data[known]), np.ascontiguousarray(M[:, known]), out=rhs,
                       accumulate=True)
    A = np.ascontiguousarray(M[:, lost])
    assert oracle.gf64_solve_and_reconstruct(A, rhs) == 0
    assert np.array_equal(got, rhs)


@pytest.mark.parametrize("N,n,B,fI,fR", [
    (2000, 150, 64, 0, 2000),     # closed-form Cauchy inverse, tensor-core n x n product
    (50, 1, 8, 0, 50),            # one lost block
    (64, 6, 16, 0, 10),           # lost ids meet row ids fR + j: entries mapped to 1, Gauss-Jordan
    (64, 5, 16, 7, 2**64 - 3),    # row ids wrap around 2^64
])
def test_par3_repair_inverse_paths_vs_oracle(kctx, oracle, N, n, B, fI, fR):
    """Both solve paths of pp_gf64_repair (closed-form Cauchy inverse when the
    system is a true Cauchy matrix, Gauss-Jordan when a lost column id equals
    a row id) give the oracle's Gauss-Jordan solution bit for bit."""
    from parparpar_b200 import par3
    rng = np.random.default_rng(N + n)
    data = rng.integers(0, 2**64, (N, B), dtype=np.uint64)
    lost = np.sort(rng.choice(N, n, replace=False))
    if fR == 10:
        lost[0] = 12  # fI + 12 == fR + 2
        lost = np.unique(lost)
        n = lost.size
    rec = rng.integers(0, 2**64, (n, B), dtype=np.uint64)  # any right-hand side
    got = par3.repair(data, lost, rec.copy(), B, fI, fR, ctx=kctx)
    M = oracle.gf64_build_cauchy(N, n, fI, fR)
    known = np.setdiff1d(np.arange(N), lost)
    rhs = rec.copy()
    oracle.gf64_matvec(np.ascontiguousarray(data[known]), np.ascontiguousarray(M[:, known]), out=rhs,
                       accumulate=True)
    A = np.ascontiguousarray(M[:, lost])
    assert oracle.gf64_solve_and_reconstruct(A, rhs) == 0
    assert np.array_equal(got, rhs)


@pytest.mark.parametrize("N,R", [(16385, 3), (20003, 5)])
def test_compute_recovery_host_inputs_in_overlapped_chunks(kctx, oracle, N, R):
    """Host inputs of >= two 64 MiB chunks are copied chunk by chunk on a copy
    stream while the previous chunk's product runs (products accumulate from
    the second chunk on); the last chunk goes in halving pieces.  16,385
    blocks of 8 KiB leave a one-block last chunk; 20,003 blocks give 8,192,
    8,192, 1,810, 904, 512 and 393 (R=5: the SM-pair kernel).  Sampled word
    ranges of every block against the oracle, plus accumulate."""
    from parparpar_b200 import par3
    rng = np.random.default_rng(81 + N)
    B, fI, fR = 1024, 5, 20000 + N
    data = rng.integers(0, 2**64, (N, B), dtype=np.uint64)
    out = np.zeros((R, B), dtype=np.uint64)
    par3.GF64Controller.ComputeRecoveryBlocks(data, N, out, R, B, fI, fR)
    for w in (0, 1000):
        want = oracle.gf64_compute_recovery(np.ascontiguousarray(data[:, w:w + 2]), R, fI, fR)
        assert np.array_equal(out[:, w:w + 2], want), w
    acc = out.copy()
    par3.GF64Controller.ComputeRecoveryBlocks(data, N, acc, R, B, fI, fR, accumulate=True)
    assert not acc.any()  # x ^ x
