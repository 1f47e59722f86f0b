"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a checkout where the reference sources are available and
``make -C oracle ref`` has built ``oracle/_ref/libppref.so`` (the reference's
own C/C++ hot-path code compiled from its sources).  The fixtures it writes
are small ``.npz`` files that the tests read; the tests never need the
reference at run time.

    python tests/golden/make_golden.py

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
"""
from __future__ import annotations

import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from oracle import Reference  # noqa: E402


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


def main():
    R = Reference()
    par3_golden(R)
    par2_create(R)
    par2_invert(R)
    gf64_ops(R)
    gf64_fft(R)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
