"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a checkout where the reference sources are available and
``make -C oracle ref`` has built ``oracle/_ref/libppref.so`` (the reference's
own C/C++ hot-path code compiled from its sources).  The fixtures it writes
are small ``.npz`` files that the tests read; the tests never need the
reference at run time.

    python tests/golden/make_golden.py [fixture ...]   (default: all of them)

Fixtures:
  par3_golden.npz  the reference's frozen golden case (test/par3-golden.js:27-98):
                   5 blocks x 1024 B, every u64 word = its global byte offset,
                   R=2, firstInput=0, firstRecovery=5; CRC32 6A941C15.
  par2_create.npz  PAR2 controller output (PAR2Proc + PAR2ProcCPU) on seeded
                   inputs: even/odd slice sizes and a short last slice.
  par2_invert.npz  Galois16RecMatrix factors for the cases of
                   test/gf16/test-inv.cpp:100-140 (incl. the PAR2 flaw).
  gf64_ops.npz     gf64 mul/inverse pairs, a Cauchy matrix, a matvec, a solve.
  gf64_fft.npz     additive FFT forward/inverse (recursive, Cantor basis).
  hashes.npz       block hashes from the reference's hasher: PAR2 IFSC entries
                   and file MD5s (the HasherInput variant setup_hasher selects,
                   driven like src/gf.cc:928-1037),
                   BLAKE3 digests (hasher/hasher_blake3.c), the PAR3 data-block
                   checksum layout of lib/par3gen.js:1001-1017 and recovery
                   packets laid out as src/gf64_addon.cc:2884-2934, checksummed
                   with the reference's BLAKE3.  Inputs are oracle.pattern_bytes
                   streams, regenerated by the tests from (length, seed).
  configs.npz      SHA-256 digests of the reference's outputs at benchmark
                   sizes: PAR2 create 256 x 64 KiB, R=8, and the factors of a
                   32,768-input PAR2 repair with 64 seeded lost slices.
"""
from __future__ import annotations

import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from oracle import Reference, pattern_bytes  # noqa: E402


def par3_golden(R: Reference):
    inputs = np.arange(0, 5 * 1024, 8, dtype=np.uint64).reshape(5, 128)
    out = R.gf64_compute_recovery(0, inputs, 2, 0, 5)
    crc = zlib.crc32(out.tobytes())
    assert crc == 0x6A941C15, hex(crc)
    np.savez_compressed(os.path.join(HERE, "par3_golden.npz"), inputs=inputs, recovery=out,
                        first_input=0, first_recovery=5, crc32=np.uint32(crc))


def par2_create(R: Reference):
    rng = np.random.default_rng(0x01020304)
    cases = {}
    # (numInputs, sliceSize, lastSize, exps)
    specs = [
        (16, 4000, 4000, [0, 1, 2, 3, 4, 5, 6, 7]),
        (15, 3998, 1, [0, 65534, 1, 300]),
        (16, 4000, 3999, [5, 0]),
        (1, 2, 2, [0, 1, 2]),
        (16, 2, 1, [0, 9, 100]),
        (40, 1024, 1024, list(range(16))),
    ]
    for k, (n, s, last, exps) in enumerate(specs):
        idx = rng.integers(0, 0x8000, n).astype(np.uint16)
        inp = rng.integers(0, 256, (n, s), dtype=np.uint8)
        out, _ = R.par2_create(inp, s, idx, exps, last_size=last, threads=2)
        inp_clean = inp.copy()
        inp_clean[-1, last:] = 0  # bytes past the short last slice are not part of the input
        cases[f"c{k}_inputs"] = inp_clean
        cases[f"c{k}_idx"] = idx
        cases[f"c{k}_exps"] = np.asarray(exps, dtype=np.uint16)
        cases[f"c{k}_last"] = np.int64(last)
        cases[f"c{k}_out"] = out
    # explicit coefficient overload (decode path)
    inp = rng.integers(0, 256, (12, 2048), dtype=np.uint8)
    coeffs = rng.integers(0, 65536, (5, 12)).astype(np.uint16)
    out, _ = R.par2_create_coeffs(inp, 2048, coeffs, threads=2)
    cases["coef_inputs"] = inp
    cases["coef_coeffs"] = coeffs
    cases["coef_out"] = out
    cases["ncases"] = np.int64(len(specs))
    np.savez_compressed(os.path.join(HERE, "par2_create.npz"), **cases)


def par2_invert(R: Reference):
    flawed = [True] * 6555
    flawed[0] = False
    flawed[6554] = False
    specs = [
        ([False], [0]),
        ([False], [1]),
        ([False], [65534]),
        ([False, True], [0]),
        ([False, False, True, False], [0, 1, 2]),
        ([False, False, False, False], [0, 1, 5]),
        ([False, False, False, False], [1, 5, 8, 100]),
        (flawed, [0, 5]),
        (flawed, [0, 6]),
        (flawed, [0, 5, 6]),
        ([False] * 5, [0, 3, 5, 17, 65534]),
    ]
    rng = np.random.default_rng(7)
    for n, miss, extra in [(200, 20, 5), (1000, 3, 0), (64, 64, 2)]:
        v = np.ones(n, dtype=bool)
        v[rng.choice(n, miss, replace=False)] = False
        rec = sorted(rng.choice(65535, miss + extra, replace=False).tolist())
        specs.append((v.tolist(), rec))
    d = {"ncases": np.int64(len(specs))}
    for k, (valid, rec) in enumerate(specs):
        ok, f, used = R.par2_invert(np.asarray(valid, dtype=np.uint8), rec, threads=1)
        d[f"c{k}_valid"] = np.asarray(valid, dtype=np.uint8)
        d[f"c{k}_rec"] = np.asarray(rec, dtype=np.uint16)
        d[f"c{k}_ok"] = np.int64(ok)
        d[f"c{k}_factors"] = f if ok else np.zeros((0, len(valid)), dtype=np.uint16)
        d[f"c{k}_used"] = np.asarray(used if ok else [], dtype=np.uint16)
    np.savez_compressed(os.path.join(HERE, "par2_invert.npz"), **d)


def gf64_ops(R: Reference):
    rng = np.random.default_rng(64)
    a = rng.integers(0, 2**64, 2000, dtype=np.uint64)
    b = rng.integers(0, 2**64, 2000, dtype=np.uint64)
    a[:8] = [0, 1, 2, 3, 2**63, 2**64 - 1, 0x1B, 0x8000000000000000]
    b[:8] = [5, 0, 2**63, 2**64 - 1, 2, 7, 1, 0x8000000000000000]
    prod = np.array([R.L.ref_gf64_mul(int(x), int(y)) for x, y in zip(a, b)], dtype=np.uint64)
    inv = np.array([R.L.ref_gf64_inverse(int(x)) for x in a], dtype=np.uint64)
    cauchy = R.gf64_build_cauchy(37, 9, 3, 40)
    cauchy_clash = R.gf64_build_cauchy(8, 4, 0, 2)  # fR inside the input range: denom 0 -> 1
    inp = rng.integers(0, 2**64, (33, 96), dtype=np.uint64)
    acc0 = rng.integers(0, 2**64, (7, 96), dtype=np.uint64)
    matvec = R.gf64_compute_recovery(0, inp, 7, 0, 33)
    matvec_acc = R.gf64_compute_recovery(0, inp, 7, 0, 33, out=acc0.copy(), accumulate=True)
    # repair solve: n x n Cauchy submatrix, RHS blocks
    n, B = 11, 40
    A = R.gf64_build_cauchy(60, n, 0, 60)[:, rng.choice(60, n, replace=False)].copy()
    rhs = rng.integers(0, 2**64, (n, B), dtype=np.uint64)
    A0, rhs0 = A.copy(), rhs.copy()
    rc = R.gf64_solve_and_reconstruct(A, rhs)
    sing = np.zeros((3, 3), dtype=np.uint64)
    sing[0] = [1, 2, 3]
    sing[1] = [2, 4, 6]  # not a multiple in GF(2^64) in general, make row 2 = row0 ^ row1
    sing[2] = sing[0] ^ sing[1]
    srhs = rng.integers(0, 2**64, (3, 4), dtype=np.uint64)
    src = R.gf64_solve_and_reconstruct(sing.copy(), srhs.copy())
    np.savez_compressed(os.path.join(HERE, "gf64_ops.npz"), a=a, b=b, prod=prod, inv=inv,
                        cauchy=cauchy, cauchy_clash=cauchy_clash, inp=inp, acc0=acc0,
                        matvec=matvec, matvec_acc=matvec_acc, A=A0, rhs=rhs0, solved=rhs, rc=np.int64(rc),
                        sing=sing, sing_rhs=srhs, sing_rc=np.int64(src))


def gf64_fft(R: Reference):
    rng = np.random.default_rng(2026)
    d = {}
    sizes = [2, 4, 8, 16, 64, 256, 1024, 4096]
    for n in sizes:
        x = rng.integers(0, 2**64, n, dtype=np.uint64)
        d[f"x{n}"] = x
        d[f"fwd{n}"] = R.gf64_fft_fwd(x)
        d[f"inv{n}"] = R.gf64_fft_inv(x)
    d["sizes"] = np.asarray(sizes, dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "gf64_fft.npz"), **d)


def hashes(R: Reference):
    d = {}
    # BLAKE3 over lengths around the 64-byte block and 1 KiB chunk boundaries
    b3_lens = [0, 1, 63, 64, 65, 1023, 1024, 1025, 2048, 2049, 3072, 3073, 4096, 4097, 5121, 8192, 8193, 8224,
               16384, 31744, 102400]
    d["b3_lens"] = np.asarray(b3_lens, dtype=np.int64)
    d["b3_digests"] = np.stack([np.frombuffer(R.blake3(pattern_bytes(n, 1000 + n)), dtype=np.uint8)
                                for n in b3_lens])
    # PAR2: whole files through the reference hasher (slice, file length, seed)
    par2 = [(4, 10, 1), (64, 64 * 7, 2), (100, 1000, 3), (1024, 5000, 4), (4096, 4096 * 3 + 17, 5),
            (32768, 32768 * 4, 6), (65536, 65536 + 1, 7), (1028, 1027, 8)]
    d["par2_cases"] = np.asarray(par2, dtype=np.int64)
    for k, (sl, ln, seed) in enumerate(par2):
        ifsc, md5 = R.par2_hash_file(pattern_bytes(ln, seed), sl)
        d[f"par2_ifsc{k}"] = ifsc
        d[f"par2_md5_{k}"] = np.frombuffer(md5, dtype=np.uint8)
    # PAR3 data-block checksums: (n, block_size, first_index, seed)
    par3 = [(5, 8, 0, 11), (3, 992, 5, 12), (4, 1000, 2**40 + 3, 13), (3, 4096, 7, 14), (2, 8192, 1, 15),
            (2, 65536, 123456789, 16)]
    d["par3_cases"] = np.asarray(par3, dtype=np.uint64)
    after = pattern_bytes(24, 99)
    d["par3_after"] = after
    for k, (n, bs, first, seed) in enumerate(par3):
        blocks = pattern_bytes(int(n) * int(bs), int(seed)).reshape(int(n), int(bs))
        hs = []
        for i in range(int(n)):
            msg = after.tobytes() + int(first + i).to_bytes(8, "little") + blocks[i].tobytes()
            hs.append(np.frombuffer(R.blake3(msg, 16), dtype=np.uint8))
        d[f"par3_hash{k}"] = np.stack(hs)
    # PAR3 recovery packets: (n, block_size, first_index, seed)
    pk = [(3, 1000, 5, 21), (2, 4096, 2**33, 22), (1, 8, 0, 23)]
    d["pkt_cases"] = np.asarray(pk, dtype=np.uint64)
    sid = pattern_bytes(8, 77)
    d["pkt_set_id"] = sid
    for k, (n, bs, first, seed) in enumerate(pk):
        n, bs = int(n), int(bs)
        rec = pattern_bytes(n * bs, int(seed)).reshape(n, bs)
        out = bytearray()
        for i in range(n):
            p = bytearray(64 + bs)
            p[0:8] = b"PAR3\x00PKT"
            p[24:32] = (64 + bs).to_bytes(8, "little")
            p[32:40] = sid.tobytes()
            p[40:48] = b"PAR REC\x00"
            p[48:56] = int(first + i).to_bytes(8, "little")
            p[56:64] = (1).to_bytes(8, "little")
            p[64:] = rec[i].tobytes()
            p[8:24] = R.blake3(bytes(p[24:]), 16)
            out += p
        d[f"pkt{k}"] = np.frombuffer(bytes(out), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "hashes.npz"), **d)


def configs(R: Reference):
    """Digests of the reference's outputs at two benchmark configurations:
    PAR2 create 256 x 64 KiB, R=8 (input numbers 0..255, exponents 0..7) on
    pattern_bytes data, and the Galois16RecMatrix factors of a PAR2 repair of
    32,768 inputs with 64 seeded lost slices and recovery exponents 0..63.
    The outputs themselves (512 KiB, 4 MiB) are not stored: the tests hash
    what the device computes and compare digests."""
    import hashlib
    n, s, r = 256, 65536, 8
    data = pattern_bytes(n * s, CFG1_SEED).reshape(n, s)
    out, ok = R.par2_create(data, s, np.arange(n, dtype=np.uint16), list(range(r)), threads=0)
    d = {"cfg1_seed": np.int64(CFG1_SEED), "cfg1_sha256": np.frombuffer(hashlib.sha256(out.tobytes()).digest(),
                                                                         dtype=np.uint8),
         "cfg1_valid": np.int64(ok)}
    N, m = 32768, 64
    lost = np.sort(np.random.default_rng(REPAIR_SEED).choice(N, m, replace=False)).astype(np.int64)
    valid = np.ones(N, dtype=np.uint8)
    valid[lost] = 0
    ok, f, used = R.par2_invert(valid, list(range(m)), threads=0)
    assert ok
    d.update(repair_lost=lost, repair_used=np.asarray(used, dtype=np.uint16),
             repair_factors_sha256=np.frombuffer(hashlib.sha256(np.ascontiguousarray(f).tobytes()).digest(),
                                                 dtype=np.uint8))
    np.savez_compressed(os.path.join(HERE, "configs.npz"), **d)


CFG1_SEED = 0xC0F1
REPAIR_SEED = 0x5EED


GENERATORS = {"hashes": hashes, "par3_golden": par3_golden, "par2_create": par2_create,
              "par2_invert": par2_invert, "gf64_ops": gf64_ops, "gf64_fft": gf64_fft, "configs": configs}


def main():
    R = Reference()
    for name in (sys.argv[1:] or GENERATORS):
        GENERATORS[name](R)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
