"""Device block hashes against the oracle (and, through the oracle's pins,
the reference's hasher):

* PAR2 IFSC entries -- MD5 + CRC32 of zero-padded slices
  (HasherInput::getBlock, hasher/hasher_input_base.h:104-117);
* PAR3 data-block BLAKE3 checksums (lib/par3gen.js:1001-1017);
* PAR3 recovery packets (src/gf64_addon.cc:2784-2936).

Bit-exact comparisons throughout: every byte of every digest.
"""
import numpy as np
import pytest

from oracle import par2_block_hashes as par2_oracle
from oracle import pattern_bytes

gpu = pytest.mark.gpu


def _torch():
    import torch
    return torch


# ------------------------------------------------------------------- PAR2
@gpu
@pytest.mark.parametrize("slice_size", [4, 8, 60, 64, 100, 1000, 1028, 4096, 32768, 65540])
def test_par2_block_hashes_full_rows(ctx, rng, slice_size):
    from parparpar_b200 import par2
    n = 37
    blocks = rng.integers(0, 256, (n, slice_size), dtype=np.uint8)
    got = par2.block_hashes(blocks, ctx=ctx)
    assert (got == par2_oracle(blocks, slice_size)).all()


@gpu
def test_par2_block_hashes_ragged_lengths_and_zero_pad(ctx, rng):
    from parparpar_b200 import par2
    sl = 4096
    lens = np.array([0, 1, 3, 4, 63, 64, 65, 127, 128, 1000, 4095, 4096, 2048, 17], dtype=np.uint64)
    blocks = rng.integers(0, 256, (lens.size, sl), dtype=np.uint8)  # bytes past each length are NOT zero
    got = par2.block_hashes(blocks, sl, lengths=lens, ctx=ctx)
    assert (got == par2_oracle(blocks, sl, lens)).all()


@gpu
def test_par2_block_hashes_device_rows_in_place_and_misaligned(ctx, rng):
    torch = _torch()
    from parparpar_b200 import par2
    sl, n = 3000, 65
    host = rng.integers(0, 256, (n, sl + 40), dtype=np.uint8)
    dev = torch.from_numpy(host).cuda()
    want = par2_oracle(host[:, :sl], sl)
    # 16-aligned rows used in place, outputs on the device
    d_al = torch.zeros((n, 3008), dtype=torch.uint8, device="cuda")
    d_al[:, :sl] = dev[:, :sl]
    out = torch.zeros((n, 20), dtype=torch.uint8, device="cuda")
    par2.block_hashes(d_al[:, :sl], sl, out=out, ctx=ctx)
    ctx.synchronize()  # device buffers only: the call is asynchronous
    assert (out.cpu().numpy() == want).all()
    # a misaligned view (offset 3 bytes, stride 3040) is staged
    view = dev[:, 3:3 + sl]
    want2 = par2_oracle(host[:, 3:3 + sl], sl)
    assert (par2.block_hashes(view, sl, ctx=ctx) == want2).all()


@gpu
def test_par2_block_hashes_length_above_slice_is_an_error(ctx):
    from parparpar_b200 import PPError, par2
    blocks = np.zeros((2, 64), dtype=np.uint8)
    with pytest.raises(PPError):
        par2.block_hashes(blocks, 64, lengths=[64, 65], ctx=ctx)


@gpu
def test_hasher_input_matches_reference_stream(ctx, golden):
    """HasherInput fed in odd pieces reproduces the reference hasher's IFSC
    entries and file MD5 (fixture from the reference build)."""
    from parparpar_b200 import par2
    g = golden("hashes.npz")
    for k, (sl, ln, seed) in enumerate(g["par2_cases"]):
        sl, ln = int(sl), int(ln)
        data = pattern_bytes(ln, int(seed)).tobytes()
        n = (ln + sl - 1) // sl
        ifsc = bytearray(20 * n)
        h = par2.HasherInput(sl, ifsc, batch=3, ctx=ctx)
        pos, step = 0, 1
        while pos < ln:
            h.update(data[pos:pos + step])
            pos += step
            step = step * 3 + 1
        md5 = bytearray(16)
        h.end(md5)
        assert bytes(ifsc) == g[f"par2_ifsc{k}"].tobytes(), (sl, ln)
        assert bytes(md5) == g[f"par2_md5_{k}"].tobytes()


# ------------------------------------------------------------------- PAR3
@gpu
@pytest.mark.parametrize("block_size", [8, 24, 992, 1000, 1024, 2016, 2048, 4096, 8192, 24 * 1024 + 8])
def test_par3_block_hashes(ctx, oracle, rng, block_size):
    from parparpar_b200 import par3
    n = 23
    blocks = rng.integers(0, 256, (n, block_size), dtype=np.uint8)
    after = rng.integers(0, 256, 24, dtype=np.uint8).tobytes()
    first = (1 << 40) + 12345
    got = par3.block_hashes(blocks, block_size, first, after, num_blocks=n, ctx=ctx)
    assert (got == oracle.par3_block_hashes(blocks, first, after)).all()


@gpu
def test_par3_block_hashes_golden(ctx, golden):
    from parparpar_b200 import par3
    g = golden("hashes.npz")
    after = g["par3_after"].tobytes()
    for k, (n, bs, first, seed) in enumerate(g["par3_cases"]):
        blocks = pattern_bytes(int(n) * int(bs), int(seed))
        got = par3.block_hashes(blocks, int(bs), int(first), after, ctx=ctx)
        assert (got == g[f"par3_hash{k}"]).all(), (n, bs)


@gpu
def test_par3_block_hashes_unaligned_layouts_on_device(ctx, oracle, rng):
    torch = _torch()
    from parparpar_b200 import par3
    # odd block size and stride (byte-granular path); device rows and outputs
    bs, stride, n = 1001, 1013, 19
    host = rng.integers(0, 256, n * stride + 16, dtype=np.uint8)
    dev = torch.from_numpy(host).cuda()
    rows = np.stack([host[5 + i * stride: 5 + i * stride + bs] for i in range(n)])
    after = rng.integers(0, 256, 24, dtype=np.uint8).tobytes()
    out = torch.zeros((n, 16), dtype=torch.uint8, device="cuda")
    par3.block_hashes(dev[5:], bs, 9, after, num_blocks=n, block_stride=stride, out=out, ctx=ctx)
    ctx.synchronize()
    assert (out.cpu().numpy() == oracle.par3_block_hashes(rows, 9, after)).all()


@gpu
@pytest.mark.parametrize("block_size", [8, 984, 1000, 4096, 8192, 65536 + 8])
def test_par3_recovery_packets(ctx, oracle, rng, block_size):
    from parparpar_b200 import par3
    n = 7
    rec = rng.integers(0, 256, (n, block_size), dtype=np.uint8)
    sid = rng.integers(0, 256, 8, dtype=np.uint8).tobytes()
    first = 2**35 + 3
    got = par3.assemble_recovery_packets(rec.reshape(-1), sid, first, n, block_size, ctx=ctx)
    assert (got == oracle.par3_recovery_packets(rec, sid, first)).all()


@gpu
def test_par3_recovery_packets_golden_device_buffers(ctx, golden):
    torch = _torch()
    from parparpar_b200 import par3
    g = golden("hashes.npz")
    sid = g["pkt_set_id"].tobytes()
    for k, (n, bs, first, seed) in enumerate(g["pkt_cases"]):
        n, bs = int(n), int(bs)
        rec = torch.from_numpy(pattern_bytes(n * bs, int(seed))).cuda()
        out = torch.zeros(n * (64 + bs), dtype=torch.uint8, device="cuda")
        par3.assemble_recovery_packets(rec, sid, int(first), n, bs, out=out, ctx=ctx)
        ctx.synchronize()
        assert (out.cpu().numpy() == g[f"pkt{k}"]).all(), (n, bs)


# ------------------------------------------------------------- full size
@gpu
def test_par2_block_hashes_full_size_sampled(ctx):
    """1 GiB of slices (32768 x 32 KiB) resident on the device; every digest
    of a sample of rows against the oracle, and the digests of all rows
    distinct (a checksum-of-checksums property at full size)."""
    torch = _torch()
    from parparpar_b200 import par2
    n, sl = 32768, 32768
    g = torch.Generator(device="cuda").manual_seed(5)
    d = torch.randint(0, 256, (n, sl), dtype=torch.uint8, device="cuda", generator=g)
    out = torch.zeros((n, 20), dtype=torch.uint8, device="cuda")
    par2.block_hashes(d, sl, out=out, ctx=ctx)
    ctx.synchronize()
    got = out.cpu().numpy()
    idx = np.linspace(0, n - 1, 256).astype(np.int64)
    rows = d[torch.from_numpy(idx).cuda()].cpu().numpy()
    assert (got[idx] == par2_oracle(rows, sl)).all()
    assert len({r.tobytes() for r in got}) == n
    del d


@gpu
def test_par3_block_hashes_full_size_sampled(ctx, oracle):
    """131072 x 8 KiB blocks resident on the device (1 GiB)."""
    torch = _torch()
    from parparpar_b200 import par3
    n, bs = 131072, 8192
    g = torch.Generator(device="cuda").manual_seed(6)
    d = torch.randint(0, 256, (n, bs), dtype=torch.uint8, device="cuda", generator=g)
    after = bytes(range(24))
    out = torch.zeros((n, 16), dtype=torch.uint8, device="cuda")
    par3.block_hashes(d, bs, 1000, after, num_blocks=n, out=out, ctx=ctx)
    ctx.synchronize()
    got = out.cpu().numpy()
    idx = np.linspace(0, n - 1, 512).astype(np.int64)
    rows = d[torch.from_numpy(idx).cuda()].cpu().numpy()
    want = np.stack([oracle.par3_block_hashes(rows[j:j + 1], 1000 + int(i), after)[0] for j, i in enumerate(idx)])
    assert (got[idx] == want).all()
    assert len({r.tobytes() for r in got}) == n
    del d


# ------------------------------------------------------------- fused pass
@gpu
@pytest.mark.parametrize("n", [5, 300, 10003])
def test_par2_create_hashed_host_inputs(ctx, oracle, rng, n):
    """Recovery slices and the inputs' IFSC entries from one pass over host
    inputs (10003 slices takes the chunked copy path)."""
    from parparpar_b200 import par2
    sl = 1024
    data = rng.integers(0, 256, (n, sl), dtype=np.uint8)
    exps = [0, 1, 7, 300]
    hashes = np.zeros((n, 20), dtype=np.uint8)
    out = par2.par2_create(data, np.arange(n), exps, hashes=hashes, ctx=ctx)
    assert (hashes == par2_oracle(data, sl)).all()
    # the recovery slices are those of the plain create (itself pinned to the oracle elsewhere)
    assert (out == par2.par2_create(data, np.arange(n), exps, ctx=ctx)).all()
    if n <= 300:
        co = oracle.par2_coeff_matrix(np.arange(n), exps)
        assert (out == oracle.par2_muladd(list(data), sl, co)).all()


@gpu
@pytest.mark.parametrize("n,sl,exps", [(300, 450002, [0, 1, 7, 300] + list(range(9, 21))),
                                       (64, 2 * 1024 * 1024 + 6, [2, 5, 9, 11, 13, 17, 19, 23])])
def test_par2_create_hashed_column_bands(ctx, rng, n, sl, exps):
    """Host inputs of few large slices (>= 128 MiB staged) go to the device as
    column bands of every slice, each band's product and MD5 / CRC32 blocks
    running as it lands (the hash state carried from band to band): 300 x
    450,002 B makes three bands, the last one 2,642 B (odd: a partial final
    word); 64 x (2 MiB + 6 B) makes bands of 1 MiB, 1 MiB and 6 B (a band
    with no whole 64-byte block).  The IFSC entries match
    hashlib / zlib, the recovery slices the create from device-resident inputs
    (a path without bands, pinned to the oracle elsewhere)."""
    torch = _torch()
    from parparpar_b200 import par2
    data = rng.integers(0, 256, (n, sl), dtype=np.uint8)
    want = par2_oracle(data, sl)
    d_out = torch.zeros((len(exps), sl), dtype=torch.uint8, device="cuda")
    par2.par2_create(torch.from_numpy(data).cuda(), np.arange(n), exps, out=d_out, ctx=ctx)
    ctx.synchronize()
    ref = d_out.cpu().numpy()
    # three calls: the key's later uses run on its resident coefficient tiles
    for _ in range(3):
        hashes = np.zeros((n, 20), dtype=np.uint8)
        out = par2.par2_create(data, np.arange(n), exps, hashes=hashes, ctx=ctx)
        assert (hashes == want).all()
        assert (out == ref).all()


@gpu
def test_par2_create_hashed_device_inputs(ctx, rng):
    torch = _torch()
    from parparpar_b200 import par2
    n, sl = 77, 4096
    data = rng.integers(0, 256, (n, sl), dtype=np.uint8)
    d_in = torch.from_numpy(data).cuda()
    d_out = torch.zeros((3, sl), dtype=torch.uint8, device="cuda")
    d_h = torch.zeros((n, 20), dtype=torch.uint8, device="cuda")
    par2.par2_create(d_in, np.arange(n), [1, 2, 3], out=d_out, hashes=d_h, ctx=ctx)
    ctx.synchronize()
    assert (d_h.cpu().numpy() == par2_oracle(data, sl)).all()
    ref = par2.par2_create(data, np.arange(n), [1, 2, 3], ctx=ctx)
    assert (d_out.cpu().numpy() == ref).all()


@gpu
@pytest.mark.parametrize("n_in,words", [(40, 128), (20000, 512)])
def test_par3_create_packets_matches_separate_steps(ctx, oracle, rng, n_in, words):
    """Fused create: packets == assemble(compute_recovery(inputs)) and data
    hashes == block hashes of the inputs; 20000 x 4 KiB host inputs take the
    chunked copy path."""
    from parparpar_b200 import par3
    R, fI, fR = 6, 3, n_in + 3
    x = rng.integers(0, 2**64, (n_in, words), dtype=np.uint64)
    after = rng.integers(0, 256, 24, dtype=np.uint8).tobytes()
    sid = b"setid-01"
    pk, dh = par3.create_packets(x, n_in, words, fI, R, fR, sid, data_after_checksum=after, ctx=ctx)
    rec = np.zeros((R, words), dtype=np.uint64)
    par3.GF64Controller.ComputeRecoveryBlocks(x, n_in, rec, R, words, fI, fR)
    want_pk = oracle.par3_recovery_packets(rec.view(np.uint8).reshape(R, words * 8), sid, fR)
    assert (pk == want_pk).all()
    rows = np.linspace(0, n_in - 1, min(n_in, 200)).astype(np.int64)
    blocks = x.view(np.uint8).reshape(n_in, words * 8)
    want_h = np.stack([oracle.par3_block_hashes(blocks[i:i + 1], fI + int(i), after)[0] for i in rows])
    assert (dh[rows] == want_h).all()
    if n_in <= 64:
        assert (rec == oracle.gf64_compute_recovery(x, R, fI, fR)).all()


@gpu
def test_par3_create_packets_device_buffers(ctx, oracle, rng):
    torch = _torch()
    from parparpar_b200 import par3
    n_in, words, R = 300, 256, 4
    x = rng.integers(0, 2**64, (n_in, words), dtype=np.uint64)
    d_x = torch.from_numpy(x.view(np.int64)).cuda()
    d_pk = torch.zeros(R * (64 + words * 8), dtype=torch.uint8, device="cuda")
    d_h = torch.zeros((n_in, 16), dtype=torch.uint8, device="cuda")
    after = bytes(range(100, 124))
    par3.create_packets(d_x, n_in, words, 0, R, n_in, b"ABCDEFGH", data_after_checksum=after, data_hashes=d_h,
                        packets=d_pk, ctx=ctx)
    ctx.synchronize()
    rec = oracle.gf64_compute_recovery(x, R, 0, n_in)
    assert (d_pk.cpu().numpy() == oracle.par3_recovery_packets(rec.view(np.uint8).reshape(R, -1), b"ABCDEFGH",
                                                               n_in)).all()
    assert (d_h.cpu().numpy() == oracle.par3_block_hashes(x.view(np.uint8).reshape(n_in, -1), 0, after)).all()


# ---------------------------------------------------- PAR2 memory checksum
@gpu
@pytest.mark.parametrize("sl", [2, 16, 30, 512, 4100, 32768, 100000])
def test_par2_memory_checksums(ctx, oracle, rng, sl):
    from parparpar_b200 import par2
    rows = rng.integers(0, 256, (45, sl + 7), dtype=np.uint8)
    got = par2.memory_checksums(rows, sl, ctx=ctx)
    assert (got == oracle.par2_memory_checksums(rows[:, :sl], sl)).all()


@gpu
@pytest.mark.parametrize("sl,shrink", [(4096, 4096), (4096, 1002), (1 << 20, (1 << 20) - 6)])
def test_proc_outputs_pass_the_memory_checksum(ctx, oracle, rng, sl, shrink):
    """Every processor output reports valid: the checksum blocks attached at
    staging, multiplied with the data, equal the checksums of the outputs."""
    from parparpar_b200 import par2
    n, exps = 20, [0, 3, 9]
    data = rng.integers(0, 256, (n, shrink), dtype=np.uint8)
    proc = par2.PAR2ProcCUDA(sl, ctx=ctx)
    proc.setCurrentSliceSize(shrink)
    proc.setRecoverySlices(len(exps), exps)
    for i in range(n):
        proc.addInput(data[i], shrink, i, flush=(i == 7))
    proc.endInput()
    want = oracle.par2_muladd(list(data), shrink, oracle.par2_coeff_matrix(np.arange(n), exps))
    for o in range(len(exps)):
        buf = np.zeros(shrink, dtype=np.uint8)
        assert proc.getOutput(o, buf) is True
        assert (buf == want[o]).all()
    proc.deinit()


# ------------------------------------------------------- streaming create
def _file(tmp_path, name, data):
    p = tmp_path / name
    p.write_bytes(bytes(data))
    return str(p)


@gpu
@pytest.mark.parametrize("size,bs", [(1, 8), (8 * 1000 + 3, 64), (200 * 1024 * 1024 + 13, 8192)])
def test_par3_create_streaming_matches_in_memory_create(ctx, oracle, rng, tmp_path, size, bs):
    """Recovery from a file, read in pipelined chunks (the 200 MiB case spans
    four 64 MiB chunks), equals the create over the zero-padded blocks; the
    data-block hashes come from the same pass."""
    from parparpar_b200 import par3
    data = rng.integers(0, 256, size, dtype=np.uint8)
    path = _file(tmp_path, "src.bin", data)
    n = (size + bs - 1) // bs
    blocks = np.zeros(n * bs, dtype=np.uint8)
    blocks[:size] = data
    R, fI, fR = 5, 2, n + 9
    after = bytes(range(7, 31))
    hashes = np.zeros((n, 16), dtype=np.uint8)
    res = par3.par3_create_streaming(path, {"recoverySlices": R, "blockSize": bs, "firstInput": fI,
                                            "firstRecovery": fR}, data_hashes=hashes, data_after_checksum=after,
                                     ctx=ctx)
    assert res["recoveryBytes"] == R * bs and res["numInputs"] == n and res["bytesRead"] == size
    x = blocks.view(np.uint64).reshape(n, bs // 8)
    want = np.zeros((R, bs // 8), dtype=np.uint64)
    par3.GF64Controller.ComputeRecoveryBlocks(x, n, want, R, bs // 8, fI, fR)
    assert (res["recoveryBuffer"].view(np.uint64).reshape(R, -1) == want).all()
    if n <= 2000:
        assert (want == oracle.gf64_compute_recovery(x, R, fI, fR)).all()
    rows = np.linspace(0, n - 1, min(n, 100)).astype(np.int64)
    b8 = blocks.reshape(n, bs)
    want_h = np.stack([oracle.par3_block_hashes(b8[i:i + 1], fI + int(i), after)[0] for i in rows])
    assert (hashes[rows] == want_h).all()


@gpu
def test_par3_create_streaming_errors(ctx, tmp_path):
    import parparpar_b200 as pp
    from parparpar_b200 import par3
    with pytest.raises(pp.PPError) as e:
        par3.par3_create_streaming(str(tmp_path / "missing.bin"), {"recoverySlices": 2, "blockSize": 64}, ctx=ctx)
    assert e.value.status == pp.PP_ERR_IO and "open failed for sourcePath" in str(e.value)
    empty = _file(tmp_path, "empty.bin", b"")
    got = []
    par3.par3_create_streaming(empty, {"recoverySlices": 2, "blockSize": 64}, callback=lambda err, r: got.append((err, r)),
                               ctx=ctx)
    assert got[0][1] is None and got[0][0].status == pp.PP_ERR_IO and "sourcePath is empty" in str(got[0][0])


@gpu
@pytest.mark.parametrize("sl", [4, 28, 32, 60, 1000, 32768, 1 << 20])
def test_par2_recovery_packet_headers(ctx, rng, sl):
    from oracle import par2_recovery_packet_headers as want_hdr
    from parparpar_b200 import par2
    n = 9
    slices = rng.integers(0, 256, (n, sl), dtype=np.uint8)
    exps = [0, 1, 2, 100, 65534, 7, 8, 9, 31000]
    sid = rng.integers(0, 256, 16, dtype=np.uint8).tobytes()
    got = par2.recovery_packet_headers(slices, exps, sid, ctx=ctx)
    assert (got == want_hdr(slices, exps, sid, sl)).all()
