"""PAR2 / GF(2^16) parity on the GPU: the CUDA kernels through the C ABI
against the golden fixtures and the oracle, bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["lut", "tensor"])
def kctx(ctx, request):
    """The default context with the GF(2^16) region kernel forced to one
    implementation; every parity test below runs against both."""
    import parparpar_b200._lib as L
    ctx.set_gf16_kernel(L.PP_GF16_KERNEL_LUT if request.param == "lut" else L.PP_GF16_KERNEL_TENSOR)
    yield ctx
    ctx.set_gf16_kernel(L.PP_GF16_KERNEL_AUTO)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(t):
    return t.cpu().numpy()


def test_par2_create_golden(kctx, golden):
    from parparpar_b200 import par2
    g = golden("par2_create.npz")
    for k in range(int(g["ncases"])):
        inp, idx, exps, out = g[f"c{k}_inputs"], g[f"c{k}_idx"], g[f"c{k}_exps"], g[f"c{k}_out"]
        got = par2.par2_create(inp, idx, exps, ctx=kctx)
        assert np.array_equal(got, out), f"case {k}"
        # same through device buffers
        dout = _dev(np.zeros_like(out))
        par2.par2_create(_dev(inp), idx, exps, out=dout, ctx=kctx)
        kctx.synchronize()
        assert np.array_equal(_host(dout), out), f"case {k} (device)"
    got = par2.gf16_muladd(g["coef_inputs"], g["coef_coeffs"], ctx=kctx)
    assert np.array_equal(got, g["coef_out"])


@pytest.mark.parametrize("n,r,s", [
    (1, 1, 2), (1, 3, 3), (7, 1, 16), (8, 4, 17), (9, 5, 1000), (33, 8, 8192), (33, 9, 8193),
    (300, 17, 40000), (16, 16, 20000), (15, 15, 19998), (64, 2, 64 * 1024 + 6),
])
def test_gf16_muladd_vs_oracle(kctx, oracle, n, r, s):
    from parparpar_b200 import par2
    rng = np.random.default_rng(n * 1000 + r * 10 + s)
    inp = rng.integers(0, 256, (n, s), dtype=np.uint8)
    co = rng.integers(0, 65536, (r, n)).astype(np.uint16)
    co[:, 0] = 1  # exponent-0 style columns
    if r > 1:
        co[1, :] = 0
    exp = oracle.par2_muladd(list(inp), s, co)
    assert np.array_equal(par2.gf16_muladd(inp, co, ctx=kctx), exp)
    # accumulate into existing contents
    base = rng.integers(0, 256, (r, s), dtype=np.uint8)
    out = base.copy()
    par2.gf16_muladd(inp, co, out=out, accumulate=True, ctx=kctx)
    assert np.array_equal(out, exp ^ base)


def test_gf16_muladd_device_strided(kctx, oracle):
    """Device rows with padding between them; bytes outside the slices are
    neither read as data nor written."""
    from parparpar_b200 import par2
    rng = np.random.default_rng(9)
    n, r, s, stride = 20, 6, 1001, 1040
    big = rng.integers(0, 256, (n, stride), dtype=np.uint8)
    co = rng.integers(0, 65536, (r, n)).astype(np.uint16)
    exp = oracle.par2_muladd([big[i, :s] for i in range(n)], s, co)
    dout_np = rng.integers(0, 256, (r, stride), dtype=np.uint8)
    dout = _dev(dout_np)
    par2.gf16_muladd(_dev(big)[:, :s], co, out=dout[:, :s], slice_bytes=s, ctx=kctx)
    kctx.synchronize()
    got = _host(dout)
    assert np.array_equal(got[:, :s], exp)
    assert np.array_equal(got[:, s:], dout_np[:, s:]), "wrote past the slice"


def test_gf16_muladd_split_inputs(kctx, oracle):
    """Many inputs and a small slice: the launcher splits the input range
    across blocks and combines with atomic XOR."""
    from parparpar_b200 import par2
    rng = np.random.default_rng(10)
    n, r, s = 2000, 8, 4096
    inp = rng.integers(0, 256, (n, s), dtype=np.uint8)
    co = rng.integers(0, 65536, (r, n)).astype(np.uint16)
    exp = oracle.par2_muladd(list(inp), s, co)
    assert np.array_equal(par2.gf16_muladd(inp, co, ctx=kctx), exp)
    out = _dev(np.zeros((r, s), dtype=np.uint8))
    par2.gf16_muladd(_dev(inp), _dev(co), out=out, ctx=kctx)
    kctx.synchronize()
    assert np.array_equal(_host(out), exp)


def _ctrl_case(ctx, oracle, slice_size, last, n_in, n_out, seed, batch=0, areas=2):
    from parparpar_b200 import par2
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, 0x8000, n_in).astype(np.uint16)
    exps = rng.integers(0, 0xFFFF, n_out).astype(np.uint16)
    exps[0] = 0
    src = [rng.integers(0, 256, slice_size if i < n_in - 1 else last, dtype=np.uint8) for i in range(n_in)]
    proc = par2.PAR2ProcCUDA(slice_size, areas, batch, ctx=ctx)
    assert proc.setRecoverySlices(n_out, exps)
    for i in range(n_in):
        proc.waitForAdd()
        proc.addInput(src[i], src[i].size, int(idx[i]))
    proc.endInput()
    exp = oracle.par2_muladd(src, slice_size, oracle.par2_coeff_matrix(idx, exps))
    for o in range(n_out):
        buf = np.zeros(slice_size, dtype=np.uint8)
        assert proc.getOutput(o, buf)
        assert np.array_equal(buf, exp[o]), (slice_size, last, n_in, n_out, o)
    proc.deinit()


def test_proc_test_ctrl_grid(kctx, oracle):
    """The grid of test/gf16/test-ctrl.cpp:281-306: slice sizes {2, 19998,
    20000}, last-slice sizes {1, 2, S-1, S}, 1/15/16 inputs x 1/15/16 outputs."""
    seed = 0x01020304
    for s in (2, 19998, 20000):
        lasts = [1, 2] + ([s - 1, s] if s > 2 else [])
        for last in lasts:
            for n_out in (1, 15, 16):
                for n_in in (1, 15, 16):
                    if n_in == 1 and last != s:
                        continue
                    if last != s and last != 1 and (n_in > 15 or n_out > 2):
                        continue
                    seed += 1
                    _ctrl_case(kctx, oracle, s, last, n_in, n_out, seed)


def test_proc_batches_and_reuse(kctx, oracle):
    from parparpar_b200 import par2
    # small batch to exercise several staging areas, flush, and a second pass
    _ctrl_case(kctx, oracle, 4096, 4096, 50, 5, 77, batch=4, areas=3)
    rng = np.random.default_rng(78)
    proc = par2.PAR2ProcCUDA(2048, 2, 3, ctx=kctx)
    proc.setRecoverySlices(3, [0, 1, 2])
    data = rng.integers(0, 256, (7, 2048), dtype=np.uint8)
    for rnd in range(2):
        for i in range(7):
            proc.waitForAdd()
            proc.addInput(data[i], 2048, i, flush=(i == 3))
        proc.endInput()
        exp = oracle.par2_muladd(list(data), 2048, oracle.par2_coeff_matrix(range(7), [0, 1, 2]))
        for o in range(3):
            buf = np.zeros(2048, dtype=np.uint8)
            proc.getOutput(o, buf)
            assert np.array_equal(buf, exp[o])
        proc.discardOutput()
    # decode overload: explicit coefficients per input
    co = rng.integers(0, 65536, (7, 3)).astype(np.uint16)
    for i in range(7):
        proc.waitForAdd()
        proc.addInput(data[i], 2048, co[i])
    proc.endInput()
    exp = oracle.par2_muladd(list(data), 2048, co.T.copy())
    for o in range(3):
        buf = np.zeros(2048, dtype=np.uint8)
        proc.getOutput(o, buf)
        assert np.array_equal(buf, exp[o])
    proc.deinit()


def test_proc_input_hashes_in_its_own_pass(kctx, oracle):
    """setInputHashes: the processor hashes every slice it stages (IFSC entry:
    MD5 || CRC32le of the slice zero-padded to the slice size) at its input
    number -- full host slices over 256 KiB (copied straight to the device),
    short host slices (staged through pinned rows, zero-padded), a CUDA
    input, inputs added out of order, several batches, decode inputs left
    unhashed, and entries of numbers never added reading zero."""
    import torch
    from parparpar_b200 import par2
    from oracle import par2_block_hashes
    rng = np.random.default_rng(91)
    S, n, R = 300_000, 23, 3
    sizes = [S if i % 3 else int(rng.integers(1, S)) for i in range(n)]
    data = np.zeros((n, S), dtype=np.uint8)
    for i, sz in enumerate(sizes):
        data[i, :sz] = rng.integers(0, 256, sz, dtype=np.uint8)
    proc = par2.PAR2ProcCUDA(S, 2, 4, ctx=kctx)
    proc.setRecoverySlices(R, [0, 1, 2])
    proc.setInputHashes(n + 5)
    order = list(rng.permutation(n))
    for k, i in enumerate(order):
        proc.waitForAdd()
        buf = torch.from_numpy(data[i, :sizes[i]].copy()).cuda() if i == 5 else data[i, :sizes[i]]
        proc.addInput(buf, sizes[i], int(i), flush=(k == 10))
    proc.endInput()
    got = proc.getInputHashes(n + 5)
    assert np.array_equal(got[:n], par2_block_hashes(data, S))
    assert not got[n:].any()
    exp = oracle.par2_muladd(list(data), S, oracle.par2_coeff_matrix(range(n), [0, 1, 2]))
    for o in range(R):
        out = np.zeros(S, dtype=np.uint8)
        assert proc.getOutput(o, out)
        assert np.array_equal(out, exp[o])
    # decode inputs (explicit coefficients) add no entries
    proc.discardOutput()
    proc.setInputHashes(4)
    co = rng.integers(1, 65536, (2, R)).astype(np.uint16)
    for i in range(2):
        proc.waitForAdd()
        proc.addInput(data[i], S, co[i])
    proc.endInput()
    assert not proc.getInputHashes(4).any()
    # hashing switched on with a batch half staged: only the later inputs get entries
    proc.discardOutput()
    proc.setInputHashes(0)
    for i in range(2):
        proc.waitForAdd()
        proc.addInput(data[i], S, i)
    proc.setInputHashes(10)
    for i in range(2, 4):
        proc.waitForAdd()
        proc.addInput(data[i], S, i)
    proc.endInput()
    got = proc.getInputHashes(10)
    assert not got[:2].any() and not got[4:].any()
    assert np.array_equal(got[2:4], par2_block_hashes(data[2:4], S))
    proc.deinit()


def test_proc_mixed_host_device_inputs_reused_on_return(kctx, oracle):
    """Host inputs are staged in pinned rows and copied per batch, device
    inputs are copied at once; mixed in one batch, each buffer overwritten as
    soon as addInput returns (the caller may reuse it), the outputs are the
    oracle's."""
    import torch
    from parparpar_b200 import par2
    rng = np.random.default_rng(79)
    n, sb, exps = 37, 3000, [0, 5, 9, 11]
    data = rng.integers(0, 256, (n, sb), dtype=np.uint8)
    proc = par2.PAR2ProcCUDA(sb, ctx=kctx)
    assert proc.setRecoverySlices(len(exps), exps)
    host_buf = np.zeros(sb, dtype=np.uint8)
    dev_buf = torch.zeros(sb, dtype=torch.uint8, device="cuda")
    for i in range(n):
        proc.waitForAdd()
        if i % 3 == 1:
            dev_buf.copy_(torch.from_numpy(data[i]))
            torch.cuda.synchronize()
            proc.addInput(dev_buf, sb, i)
            dev_buf.fill_(0xAB)
        else:
            host_buf[:] = data[i]
            proc.addInput(host_buf, sb, i)
            host_buf[:] = 0xCD
    proc.endInput()
    exp = oracle.par2_muladd(list(data), sb, oracle.par2_coeff_matrix(range(n), exps))
    for o in range(len(exps)):
        buf = np.zeros(sb, dtype=np.uint8)
        assert proc.getOutput(o, buf)
        assert np.array_equal(buf, exp[o]), o
    proc.deinit()


@pytest.mark.parametrize("n,r,s", [
    (8, 32, 512), (13, 32, 1000), (9, 29, 200), (40, 64, 333), (17, 64, 8193), (3000, 32, 4096),
])
def test_gf16_wide_outputs_vs_oracle(ctx, oracle, n, r, s):
    """Output counts of 25-64 on the tensor-core kernel (two output groups per
    CTA): ragged last word tiles, a slice shorter than one tile (200 bytes),
    odd slices, input counts that are not a multiple of 8, a job split over
    CTAs (3000 inputs: atomic XOR of partial products) and accumulation."""
    import parparpar_b200._lib as L
    from parparpar_b200 import par2
    rng = np.random.default_rng(n * 7 + r * 11 + s)
    inp = rng.integers(0, 256, (n, s), dtype=np.uint8)
    co = rng.integers(0, 65536, (r, n)).astype(np.uint16)
    exp = oracle.par2_muladd(list(inp), s, co)
    ctx.set_gf16_kernel(L.PP_GF16_KERNEL_TENSOR)
    try:
        assert np.array_equal(par2.gf16_muladd(inp, co, ctx=ctx), exp)
        base = rng.integers(0, 256, (r, s), dtype=np.uint8)
        out = base.copy()
        par2.gf16_muladd(inp, co, out=out, accumulate=True, ctx=ctx)
        assert np.array_equal(out, exp ^ base)
    finally:
        ctx.set_gf16_kernel(L.PP_GF16_KERNEL_AUTO)


def test_par2_invert_golden(ctx, golden):
    from parparpar_b200 import par2
    g = golden("par2_invert.npz")
    for k in range(int(g["ncases"])):
        valid = [bool(x) for x in g[f"c{k}_valid"]]
        rec = [int(x) for x in g[f"c{k}_rec"]]
        m = par2.Galois16RecMatrix(ctx=ctx)
        ok = m.Compute(valid, sum(valid), rec)
        assert ok == bool(g[f"c{k}_ok"]), f"case {k}"
        if ok:
            assert rec == [int(x) for x in g[f"c{k}_used"]]
            assert np.array_equal(m.factors, g[f"c{k}_factors"]), f"case {k}"


def test_par2_invert_vs_oracle(ctx, oracle):
    from parparpar_b200 import par2
    rng = np.random.default_rng(21)
    # lost blocks of 3..200 rows: one-CTA elimination (<= 128) and the
    # multi-launch form (> 128), lookup (< 8) and tensor-core products
    for n, miss, extra in [(1000, 40, 3), (32768, 8, 0), (257, 257, 1), (50, 3, 0), (3000, 200, 2), (600, 129, 0)]:
        v = np.ones(n, dtype=np.uint8)
        v[rng.choice(n, miss, replace=False)] = 0
        rec = sorted(rng.choice(65535, miss + extra, replace=False).tolist())
        ok, f, used = oracle.par2_invert(v, rec)
        m = par2.Galois16RecMatrix(ctx=ctx)
        r2 = list(rec)
        assert m.Compute([bool(x) for x in v], int(v.sum()), r2) == ok
        assert r2 == used and np.array_equal(m.factors, f)
        # the same flags as a numpy array (converted without a Python loop)
        m2, r3 = par2.Galois16RecMatrix(ctx=ctx), list(rec)
        assert m2.Compute(v.astype(bool), int(v.sum()), r3) == ok
        assert r3 == used and (not ok or np.array_equal(m2.factors, f))


def test_par2_repair_roundtrip(kctx):
    """create -> erase -> invert -> decode restores the erased slices."""
    from parparpar_b200 import par2
    rng = np.random.default_rng(31)
    n, s, r = 500, 8192, 12
    data = rng.integers(0, 256, (n, s), dtype=np.uint8)
    exps = list(range(r))
    rec = par2.par2_create(data, np.arange(n), exps, ctx=kctx)
    lost = sorted(rng.choice(n, 10, replace=False).tolist())
    valid = np.ones(n, dtype=bool)
    valid[lost] = False
    m = par2.Galois16RecMatrix(ctx=kctx)
    used = list(exps)
    assert m.Compute(list(valid), int(valid.sum()), used)
    srcs = np.concatenate([data[valid], rec[[exps.index(e) for e in used]]], axis=0)
    restored = par2.gf16_muladd(srcs, m.factors, ctx=kctx)
    assert np.array_equal(restored, data[lost])


def test_par2_create_resident_tables_across_calls(kctx, oracle):
    """pp_par2_create keeps the coefficient table of (input numbers,
    exponents) on the device between calls: repeated keys with new data,
    more distinct keys than the cache holds (eviction), and the same key
    again afterwards all give the oracle's result."""
    from parparpar_b200 import par2
    rng = np.random.default_rng(77)
    keys = []
    for k in range(6):
        n, r = int(rng.integers(9, 60)), int(rng.integers(1, 12))
        keys.append((rng.choice(32768, n, replace=False).astype(np.uint16),
                     rng.choice(65535, r, replace=False).astype(np.uint16)))
    for ids, exps in keys + keys + keys[:2]:  # first sightings, tables (6 > 4: evictions), hits
        data = rng.integers(0, 256, (ids.size, 640), dtype=np.uint8)
        got = par2.par2_create(data, ids, exps, ctx=kctx)
        co = oracle.par2_coeff_matrix(ids, list(exps))
        assert np.array_equal(got, oracle.par2_muladd(list(data), 640, co))


def test_par2_create_host_inputs_in_overlapped_chunks(kctx, oracle):
    """Host inputs of >= 8192 slices go to the device in chunks of 4096 whose
    copies overlap the products of the previous chunk (each chunk's kernel
    accumulates), the last 4096 in halving pieces; 10,003 slices give chunks
    of 4096, 4096, 912, 456, 256 and a ragged 187.  Checked against the
    oracle for create (first call: scratch tiles; second: resident table) and
    for an accumulating region product."""
    from parparpar_b200 import par2
    rng = np.random.default_rng(80)
    n, sb, exps = 10003, 66, [0, 1, 7, 300, 65000]
    data = rng.integers(0, 256, (n, sb), dtype=np.uint8)
    co = oracle.par2_coeff_matrix(np.arange(n), exps)
    want = oracle.par2_muladd(list(data), sb, co)
    for _ in range(2):
        assert np.array_equal(par2.par2_create(data, np.arange(n), exps, ctx=kctx), want)
    base = rng.integers(0, 256, (len(exps), sb), dtype=np.uint8)
    out = base.copy()
    par2.gf16_muladd(data, co, out=out, accumulate=True, ctx=kctx)
    assert np.array_equal(out, base ^ want)
