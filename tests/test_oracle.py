"""Pin the oracle (the C restatement in oracle/) to the reference.

1. Golden fixtures generated from the reference's own build
   (tests/golden/make_golden.py) and the reference's frozen PAR3 golden
   vector (test/par3-golden.js: CRC32 6A941C15).
2. Where the reference build (oracle/_ref) is present, direct randomized
   cross-checks against it.
"""
import zlib

import numpy as np
import pytest


def test_par3_golden_crc(oracle, golden):
    g = golden("par3_golden.npz")
    assert int(g["crc32"]) == 0x6A941C15
    out = oracle.gf64_compute_recovery(g["inputs"], 2, int(g["first_input"]), int(g["first_recovery"]))
    assert np.array_equal(out, g["recovery"])
    assert zlib.crc32(out.tobytes()) == 0x6A941C15


def test_gf64_mul_inv(oracle, golden):
    g = golden("gf64_ops.npz")
    for a, b, p, i in zip(g["a"], g["b"], g["prod"], g["inv"]):
        assert oracle.gf64_mul(int(a), int(b)) == int(p)
        assert oracle.gf64_inv(int(a)) == int(i)


def test_gf64_cauchy_matvec_solve(oracle, golden):
    g = golden("gf64_ops.npz")
    assert np.array_equal(oracle.gf64_build_cauchy(37, 9, 3, 40), g["cauchy"])
    assert np.array_equal(oracle.gf64_build_cauchy(8, 4, 0, 2), g["cauchy_clash"])
    assert np.array_equal(oracle.gf64_compute_recovery(g["inp"], 7, 0, 33), g["matvec"])
    out = g["acc0"].copy()
    oracle.gf64_compute_recovery(g["inp"], 7, 0, 33, out=out, accumulate=True)
    assert np.array_equal(out, g["matvec_acc"])
    A, rhs = g["A"].copy(), g["rhs"].copy()
    assert oracle.gf64_solve_and_reconstruct(A, rhs) == int(g["rc"]) == 0
    assert np.array_equal(rhs, g["solved"])
    assert oracle.gf64_solve_and_reconstruct(g["sing"].copy(), g["sing_rhs"].copy()) == int(g["sing_rc"]) == -1


def test_par2_create_golden(oracle, golden):
    g = golden("par2_create.npz")
    for k in range(int(g["ncases"])):
        inp, idx, exps, last, out = (g[f"c{k}_inputs"], g[f"c{k}_idx"], g[f"c{k}_exps"], int(g[f"c{k}_last"]),
                                     g[f"c{k}_out"])
        n, s = inp.shape
        srcs = [inp[i] if i < n - 1 else inp[i][:last] for i in range(n)]
        c = oracle.par2_coeff_matrix(idx, exps)
        assert np.array_equal(oracle.par2_muladd(srcs, s, c), out), f"case {k}"
    got = oracle.par2_muladd(list(g["coef_inputs"]), g["coef_inputs"].shape[1], g["coef_coeffs"])
    assert np.array_equal(got, g["coef_out"])


def test_par2_invert_golden(oracle, golden):
    g = golden("par2_invert.npz")
    for k in range(int(g["ncases"])):
        ok, f, used = oracle.par2_invert(g[f"c{k}_valid"], g[f"c{k}_rec"])
        assert ok == bool(g[f"c{k}_ok"]), f"case {k}"
        if ok:
            assert used == [int(x) for x in g[f"c{k}_used"]], f"case {k}"
            assert np.array_equal(f, g[f"c{k}_factors"]), f"case {k}"


def test_par2_invert_flaw_drops_a_row(oracle):
    # test/gf16/test-inv.cpp:115-139: recovery {0,5,6} over the flawed input set
    valid = np.ones(6555, dtype=np.uint8)
    valid[0] = valid[6554] = 0
    ok, _, used = oracle.par2_invert(valid, [0, 5, 6])
    assert ok and len(used) == 2 and used[1] == 6 and used[0] in (0, 5)
    ok, _, _ = oracle.par2_invert(valid, [0, 5])
    assert not ok


def test_gf16_field_axioms(oracle):
    rng = np.random.default_rng(3)
    for a, b, c in rng.integers(1, 65536, (200, 3)):
        a, b, c = int(a), int(b), int(c)
        assert oracle.gf16_mul(a, b) == oracle.gf16_mul(b, a)
        assert oracle.gf16_mul(a, b ^ c) == oracle.gf16_mul(a, b) ^ oracle.gf16_mul(a, c)
        assert oracle.gf16_mul(a, oracle.L.or_gf16_inv(a)) == 1


# ---------------------------------------------------------------- vs _ref
def test_oracle_vs_reference_par2(oracle, reference):
    rng = np.random.default_rng(11)
    for n, s, r in [(13, 1000, 5), (40, 4096, 16), (1, 2, 1), (7, 998, 3)]:
        idx = rng.integers(0, 32768, n)
        exps = rng.integers(0, 65535, r)
        inp = rng.integers(0, 256, (n, s), dtype=np.uint8)
        ref, _ = reference.par2_create(inp, s, idx, exps)
        got = oracle.par2_muladd(list(inp), s, oracle.par2_coeff_matrix(idx, exps))
        assert np.array_equal(got, ref)


def test_oracle_vs_reference_par3(oracle, reference):
    rng = np.random.default_rng(12)
    for n, r, b, fi, fr in [(64, 8, 64, 0, 64), (17, 33, 40, 5, 100), (100, 1, 8, 0, 100), (16, 40, 24, 3, 7)]:
        inp = rng.integers(0, 2**64, (n, b), dtype=np.uint64)
        for kind in (0, 1, 2):
            ref = reference.gf64_compute_recovery(kind, inp, r, fi, fr)
            assert np.array_equal(oracle.gf64_compute_recovery(inp, r, fi, fr), ref), (n, r, kind)


def test_oracle_vs_reference_par2_invert(oracle, reference):
    rng = np.random.default_rng(13)
    for n, miss, extra in [(50, 5, 2), (300, 30, 0), (12, 12, 3)]:
        v = np.ones(n, dtype=np.uint8)
        v[rng.choice(n, miss, replace=False)] = 0
        rec = rng.choice(65535, miss + extra, replace=False).tolist()
        a = oracle.par2_invert(v, rec)
        b = reference.par2_invert(v, rec)
        assert a[0] == b[0] and a[2] == b[2] and np.array_equal(a[1], b[1])


def test_gf64_fft_golden(oracle, golden):
    """Additive FFT forward/inverse vs the reference's
    gf64_addfft64_{fwd,inv}_recursive_scratch outputs."""
    g = golden("gf64_fft.npz")
    for n in g["sizes"]:
        n = int(n)
        assert np.array_equal(oracle.gf64_fft(g[f"x{n}"]), g[f"fwd{n}"]), n
        assert np.array_equal(oracle.gf64_fft(g[f"x{n}"], inverse=True), g[f"inv{n}"]), n


def test_gf64_fft_cantor_basis(oracle):
    # v_0 = 1 and v_{i+1}^2 + v_{i+1} = v_i (gf64/gf64_cantor_basis.h:8-13)
    import ctypes
    oracle.L.or_gf64_cantor.restype = ctypes.c_uint64
    v = [oracle.L.or_gf64_cantor(i) for i in range(20)]
    assert v[0] == 1 and v[19] == 0x4A8DCF8BD7EDE826
    for i in range(19):
        assert oracle.gf64_mul(v[i + 1], v[i + 1]) ^ v[i + 1] == v[i]


def test_oracle_vs_reference_fft(oracle, reference):
    rng = np.random.default_rng(14)
    for n in (2, 32, 512, 8192, 65536):
        x = rng.integers(0, 2**64, n, dtype=np.uint64)
        assert np.array_equal(oracle.gf64_fft(x), reference.gf64_fft_fwd(x)), n
        assert np.array_equal(oracle.gf64_fft(x, True), reference.gf64_fft_inv(x)), n


# ---------------------------------------------------------------- block hashes
def test_blake3_published_empty_digest(oracle):
    # the BLAKE3 specification's digest of the empty input
    assert oracle.blake3(b"").hex() == "af1349b9f5f9a1a6a0404dea36dcc9499bcb25c9adc112b7cc9a93cae41f3262"


def test_blake3_golden(oracle, golden):
    from oracle import pattern_bytes
    g = golden("hashes.npz")
    for n, dig in zip(g["b3_lens"], g["b3_digests"]):
        assert oracle.blake3(pattern_bytes(int(n), 1000 + int(n))) == dig.tobytes(), int(n)


def test_par2_block_hash_golden(golden):
    import hashlib

    from oracle import par2_block_hashes, pattern_bytes
    g = golden("hashes.npz")
    for k, (sl, ln, seed) in enumerate(g["par2_cases"]):
        sl, ln = int(sl), int(ln)
        data = pattern_bytes(ln, int(seed))
        n = (ln + sl - 1) // sl
        rows = np.zeros((n, sl), dtype=np.uint8)
        lens = []
        for i in range(n):
            c = data[i * sl:(i + 1) * sl]
            rows[i, :c.size] = c
            lens.append(c.size)
        assert (par2_block_hashes(rows, sl, lens) == g[f"par2_ifsc{k}"]).all(), (sl, ln)
        assert hashlib.md5(data.tobytes()).digest() == g[f"par2_md5_{k}"].tobytes()


def test_par3_block_hash_golden(oracle, golden):
    from oracle import pattern_bytes
    g = golden("hashes.npz")
    after = g["par3_after"].tobytes()
    for k, (n, bs, first, seed) in enumerate(g["par3_cases"]):
        blocks = pattern_bytes(int(n) * int(bs), int(seed)).reshape(int(n), int(bs))
        assert (oracle.par3_block_hashes(blocks, int(first), after) == g[f"par3_hash{k}"]).all(), (n, bs)


def test_par3_recovery_packets_golden(oracle, golden):
    from oracle import pattern_bytes
    g = golden("hashes.npz")
    sid = g["pkt_set_id"].tobytes()
    for k, (n, bs, first, seed) in enumerate(g["pkt_cases"]):
        rec = pattern_bytes(int(n) * int(bs), int(seed)).reshape(int(n), int(bs))
        assert (oracle.par3_recovery_packets(rec, sid, int(first)) == g[f"pkt{k}"]).all(), (n, bs)


def test_hash_oracle_vs_reference(oracle, reference, rng):
    from oracle import par2_block_hashes
    for n in list(rng.integers(0, 9000, 40)) + [1024 * 33 + 7]:
        d = rng.integers(0, 256, int(n), dtype=np.uint8)
        assert oracle.blake3(d.tobytes()) == reference.blake3(d.tobytes())
    for sl in (4, 12, 64, 1000, 4096):
        ln = int(rng.integers(0, 5 * sl))
        d = rng.integers(0, 256, ln, dtype=np.uint8)
        ifsc, _ = reference.par2_hash_file(d, sl)
        n = ifsc.shape[0]
        rows = np.zeros((n, sl), dtype=np.uint8)
        lens = []
        for i in range(n):
            c = d[i * sl:(i + 1) * sl]
            rows[i, :c.size] = c
            lens.append(c.size)
        assert (par2_block_hashes(rows, sl, lens) == ifsc).all()


def test_par3_hash_oracle_vs_reference(oracle, reference, rng):
    from oracle import pattern_bytes
    for n, bs in [(3, 8), (2, 1000), (2, 4096), (1, 65536 + 8)]:
        b = pattern_bytes(n * bs, bs).reshape(n, bs)
        after = rng.integers(0, 256, 24, dtype=np.uint8).tobytes()
        assert (oracle.par3_block_hashes(b, 2**40, after) == reference.par3_block_hashes(b, 2**40, after)).all()
        assert (oracle.par3_recovery_packets(b, b"idid-idi", 77) ==
                reference.par3_recovery_packets(b, b"idid-idi", 77)).all()


# ------------------------------------------------------- PAR2 memory checksum
def test_memory_checksum_is_carried_by_the_region_product(oracle, rng):
    """The staging checksum is GF(2^16)-linear: the region product of the
    inputs' checksum blocks equals the checksum of the product (what lets the
    processor carry it as one more block per row)."""
    n, sl = 9, 100
    data = rng.integers(0, 256, (n, sl), dtype=np.uint8)
    ck = oracle.par2_memory_checksums(data, sl)
    co = oracle.par2_coeff_matrix(np.arange(n), [0, 1, 5, 65534])
    prod = oracle.par2_muladd(list(data), sl, co)
    carried = oracle.par2_muladd(list(ck), 16, co)
    assert (oracle.par2_memory_checksums(prod, sl) == carried).all()


def test_memory_checksum_detects_single_bit_errors(oracle, rng):
    sl = 72
    row = rng.integers(0, 256, (1, sl), dtype=np.uint8)
    base = oracle.par2_memory_checksums(row, sl)
    for byte in range(sl):
        for bit in range(8):
            bad = row.copy()
            bad[0, byte] ^= 1 << bit
            assert (oracle.par2_memory_checksums(bad, sl) != base).any(), (byte, bit)
