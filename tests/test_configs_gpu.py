"""Parity at the benchmark configurations, on the GPU.

Each configuration the benchmarks quote runs at its full size through the
product (the C ABI behind the Python binding) and is checked bit for bit:

* PAR2 create 256 x 64 KiB, R=8 (input numbers 0..255, exponents 0..7):
  whole output against the oracle and against the SHA-256 digest of the
  reference controller's output (PAR2Proc + PAR2ProcCPU, test-ctrl.cpp
  semantics, generated by tests/golden/make_golden.py), through
  pp_par2_create (host and device buffers) and the processor.
* PAR2 create 1,024 x 1 MiB, R=8 and PAR3 create 131,072 x 8 KiB, R=1,024:
  windows of every slice that include its first and last 32 bytes and the
  word-tile boundaries of the tensor-core kernels, against the oracle /
  the reference build (each output byte depends only on the same position
  of the inputs, so a window is an independent product).
* PAR2 repair 32,768 x 32 KiB with 64 seeded lost slices: the factors
  against the digest of the reference's Galois16RecMatrix::GetFactor
  matrix, and the restored slices against the erased originals.
* The memory checksum's `valid` flag goes false when an output row is
  changed between the product and getOutput (lib/par2.js:307-310 treats
  that as "Memory checksum error").

Results are integer GF words: every comparison is exact.
"""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sha(a) -> bytes:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest()


def _par2_windows(s):
    """32-byte windows: a slice's first and last 32 bytes and the 256- and
    512-word tile boundaries of the GF(2^16) tensor-core kernel."""
    starts = {0, s - 32}
    for b in (512, 1024, s // 2):
        if 16 <= b <= s - 16:
            starts.add(b - 16)
    return sorted(x for x in starts if 0 <= x <= s - 32)


def _check_par2_windows(oracle, inputs, out, coeffs, s):
    for st in _par2_windows(s):
        cols = np.ascontiguousarray(inputs[:, st:st + 32].cpu().numpy())
        want = oracle.par2_muladd(list(cols), 32, coeffs)
        assert np.array_equal(out[:, st:st + 32].cpu().numpy(), want), f"window at byte {st}"


def _gf64_expect(oracle, cols, n_rec, first_in, first_rec):
    """(rows, expected rows) of a GF(2^64) create restricted to the columns
    `cols`: every row from the reference build when it is present, else two
    rows at each end from the oracle (whose scalar inverse is slow)."""
    import oracle as orc
    if orc.Reference.available():
        return np.arange(n_rec), orc.Reference().gf64_compute_recovery(0, cols, n_rec, first_in, first_rec)
    rows = np.array(sorted({0, 1, n_rec - 2, n_rec - 1} & set(range(n_rec))))
    want = np.stack([oracle.gf64_compute_recovery(cols, 1, first_in, first_rec + int(r))[0] for r in rows])
    return rows, want


# ---------------------------------------------------------------- PAR2 create
@pytest.mark.parametrize("kernel", ["tensor", "lut"])
def test_par2_create_256x64KiB_R8_against_the_reference(ctx, oracle, golden, kernel):
    import torch
    import oracle as orc
    import parparpar_b200._lib as L
    from parparpar_b200 import par2
    g = golden("configs.npz")
    n, s, r = 256, 65536, 8
    data = orc.pattern_bytes(n * s, int(g["cfg1_seed"])).reshape(n, s)
    want = oracle.par2_muladd(list(data), s, oracle.par2_coeff_matrix(np.arange(n), list(range(r))))
    assert _sha(want) == g["cfg1_sha256"].tobytes(), "oracle differs from the reference controller"
    ctx.set_gf16_kernel(L.PP_GF16_KERNEL_TENSOR if kernel == "tensor" else L.PP_GF16_KERNEL_LUT)
    try:
        # pp_par2_create, host buffers
        got = par2.par2_create(data, np.arange(n), list(range(r)), ctx=ctx)
        assert _sha(got) == g["cfg1_sha256"].tobytes()
        # device buffers
        d_out = torch.zeros((r, s), dtype=torch.uint8, device="cuda")
        par2.par2_create(torch.from_numpy(data).cuda(), np.arange(n), list(range(r)), out=d_out, ctx=ctx)
        ctx.synchronize()
        assert np.array_equal(d_out.cpu().numpy(), want)
        # the processor, one addInput per slice (the controller's call pattern)
        proc = par2.PAR2ProcCUDA(s, ctx=ctx)
        assert proc.setRecoverySlices(r, list(range(r)))
        for i in range(n):
            proc.waitForAdd()
            proc.addInput(data[i], s, i)
        proc.endInput()
        buf = np.zeros((r, s), dtype=np.uint8)
        for o in range(r):
            assert proc.getOutput(o, buf[o])
        proc.deinit()
        assert _sha(buf) == g["cfg1_sha256"].tobytes()
    finally:
        ctx.set_gf16_kernel(L.PP_GF16_KERNEL_AUTO)


def test_par2_create_1024x1MiB_R8_windows(ctx, oracle):
    """Full-size device run; every slice's first/last 32 bytes and the tile
    boundaries against the oracle; the host-buffer path (banded copies
    overlapped with the products) equal to the device result."""
    import torch
    from parparpar_b200 import par2
    n, s, r = 1024, 1 << 20, 8
    gen = torch.Generator(device="cuda")
    gen.manual_seed(81)
    d_in = torch.randint(0, 256, (n, s), dtype=torch.uint8, device="cuda", generator=gen)
    out = torch.zeros((r, s), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    exps = list(range(r))
    par2.par2_create(d_in, np.arange(n), exps, out=out, ctx=ctx)
    ctx.synchronize()
    _check_par2_windows(oracle, d_in, out, oracle.par2_coeff_matrix(np.arange(n), exps), s)
    h_in = torch.empty((n, s), dtype=torch.uint8).pin_memory()
    h_in.copy_(d_in)
    h_out = torch.zeros((r, s), dtype=torch.uint8).pin_memory()
    par2.par2_create(h_in, np.arange(n), exps, out=h_out, ctx=ctx)
    assert torch.equal(h_out.cuda(), out)


# ---------------------------------------------------------------- PAR3 create
def test_par3_create_131072x8KiB_R1024_windows(ctx, oracle):
    """R=1,024 with fR = N (the create's own first recovery index): a 1 GiB
    Cauchy matrix resident on the device.  Words [0, 4), [252, 260),
    [508, 516) and [1020, 1024) of every block (each block's first and last
    32 bytes, the 256- and 512-word tile edges of the SM-pair kernel)."""
    import torch
    from parparpar_b200 import par3
    N, words, R = 131072, 1024, 1024
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1024)
    d_in = torch.randint(-2**63, 2**63 - 1, (N, words), dtype=torch.int64, device="cuda", generator=gen)
    out = torch.zeros((R, words), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    par3.GF64Controller.ctx = ctx
    par3.GF64Controller.ComputeRecoveryBlocks(d_in, N, out, R, words, 0, N)
    ctx.synchronize()
    sel = np.r_[0:4, 252:260, 508:516, 1020:1024]
    cols = np.ascontiguousarray(d_in[:, torch.from_numpy(sel).cuda()].cpu().numpy().view(np.uint64))
    rows, want = _gf64_expect(oracle, cols, R, 0, N)
    got = out[:, torch.from_numpy(sel).cuda()].cpu().numpy().view(np.uint64)
    assert np.array_equal(got[rows], want)
    del d_in, out
    torch.cuda.empty_cache()


def test_par3_create_131072x8KiB_R8_host_buffers(ctx):
    """The host-buffer path (chunked copies overlapped with accumulating
    products, tapered last chunk) equals the device-resident result."""
    import torch
    from parparpar_b200 import par3
    N, words, R = 131072, 1024, 8
    gen = torch.Generator(device="cuda")
    gen.manual_seed(88)
    d_in = torch.randint(-2**63, 2**63 - 1, (N, words), dtype=torch.int64, device="cuda", generator=gen)
    out = torch.zeros((R, words), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    par3.GF64Controller.ctx = ctx
    par3.GF64Controller.ComputeRecoveryBlocks(d_in, N, out, R, words, 0, N)
    ctx.synchronize()
    h_in = torch.empty((N, words), dtype=torch.int64).pin_memory()
    h_in.copy_(d_in)
    h_out = torch.zeros((R, words), dtype=torch.int64).pin_memory()
    par3.GF64Controller.ComputeRecoveryBlocks(h_in, N, h_out, R, words, 0, N)
    assert torch.equal(h_out.cuda(), out)


# ---------------------------------------------------------------- PAR2 repair
def test_par2_repair_32768x32KiB_lost64_against_the_reference(ctx, oracle, golden):
    """Create 64 recovery slices (exponents 0..63) of 32,768 x 32 KiB, erase
    the 64 seeded slices, invert: the factor matrix hashes to the reference
    Galois16RecMatrix's, and the decode restores the erased slices."""
    import torch
    from parparpar_b200 import par2
    g = golden("configs.npz")
    n, s, m = 32768, 32768, 64
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3264)
    data = torch.randint(0, 256, (n, s), dtype=torch.uint8, device="cuda", generator=gen)
    rec = torch.zeros((m, s), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    par2.par2_create(data, np.arange(n), list(range(m)), out=rec, ctx=ctx)
    ctx.synchronize()
    lost = g["repair_lost"]
    valid = np.ones(n, dtype=bool)
    valid[lost] = False
    mat = par2.Galois16RecMatrix(ctx=ctx)
    used = list(range(m))
    assert mat.Compute(valid, n - m, used)
    assert used == [int(x) for x in g["repair_used"]]
    assert _sha(mat.factors) == g["repair_factors_sha256"].tobytes(), "factors differ from the reference"
    ok, f, used_o = oracle.par2_invert(valid.astype(np.uint8), list(range(m)))
    assert ok and used_o == used and np.array_equal(mat.factors, f)
    keep = torch.from_numpy(valid).cuda()
    srcs = torch.cat([data[keep], rec[torch.tensor(used, device="cuda")]], dim=0)
    restored = torch.zeros((m, s), dtype=torch.uint8, device="cuda")
    par2.gf16_muladd(srcs, torch.from_numpy(mat.factors.view(np.int16)).cuda(), out=restored, ctx=ctx)
    ctx.synchronize()
    assert torch.equal(restored, data[torch.from_numpy(lost).cuda()])


# ------------------------------------------------------ memory checksum flag
@pytest.mark.parametrize("slice_size", [4096, 4094, 4001, 300000])
def test_proc_valid_is_false_for_a_changed_output_row(ctx, oracle, slice_size):
    """Between the product and the first getOutput one byte of output row 2
    is flipped on the device: getOutput reports that row invalid (and only
    that row), its data differs from the oracle in that byte alone; the next
    job on the same processor verifies again."""
    import torch
    import parparpar_b200._lib as L
    from parparpar_b200 import par2
    rng = np.random.default_rng(slice_size)
    n, r = 20, 4
    data = rng.integers(0, 256, (n, slice_size), dtype=np.uint8)
    want = oracle.par2_muladd(list(data), slice_size, oracle.par2_coeff_matrix(np.arange(n), list(range(r))))
    proc = par2.PAR2ProcCUDA(slice_size, ctx=ctx)
    assert proc.setRecoverySlices(r, list(range(r)))
    for job in range(2):
        for i in range(n):
            proc.waitForAdd()
            proc.addInput(data[i], slice_size, i)
        proc.endInput()
        pos = slice_size - 7 if job == 0 else 0
        if job == 0:
            mask = torch.tensor([0x40], dtype=torch.uint8, device="cuda")
            torch.cuda.synchronize()
            ctx.check(L.lib.pp_xor_buffers(ctx.h, proc.outputDevicePtr(2) + pos, mask.data_ptr(), 1))
            ctx.synchronize()
        for o in range(r):
            buf = np.zeros(slice_size, dtype=np.uint8)
            ok = proc.getOutput(o, buf)
            if job == 0 and o == 2:
                assert not ok
                diff = np.flatnonzero(buf != want[o])
                assert diff.tolist() == [pos] and buf[pos] == want[o][pos] ^ 0x40
            else:
                assert ok and np.array_equal(buf, want[o])
        proc.discardOutput()
    proc.deinit()
