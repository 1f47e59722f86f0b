"""The reference's PAR3 parity grids restated: the parameter sets and
deterministic data of test/par3-barycentric-parity.js (27 cases),
test/par3-full-recovery-parity.js (16 cases) and test/par3-repair-parity.js
(5 scenarios), plus the argument edge cases of test/par3-native-edge.js.
The data come from the same mulberry32 generator the reference's tests use
(restated below); the expected outputs come from the oracle (whose own pin
to the reference build is in test_oracle.py).
"""
import numpy as np
import pytest

gpu = pytest.mark.gpu


def mulberry32(seed):
    """The mulberry32 PRNG as the reference's JS tests define it (32-bit
    wraparound at every step); returns floats in [0, 1)."""
    s = seed & 0xFFFFFFFF

    def imul(a, b):
        return (a * b) & 0xFFFFFFFF

    def rnd():
        nonlocal s
        s = (s + 0x6D2B79F5) & 0xFFFFFFFF
        t = imul(s ^ (s >> 15), 1 | s)
        t = ((t + imul(t ^ (t >> 7), 61 | t)) & 0xFFFFFFFF) ^ t
        return ((t ^ (t >> 14)) & 0xFFFFFFFF) / 4294967296.0

    return rnd


def random_words(rng, n):
    """n u64 words, each (hi << 32) | lo from two draws, as the JS fillRandom."""
    out = np.empty(n, dtype=np.uint64)
    for w in range(n):
        hi = int(rng() * 4294967296) & 0xFFFFFFFF
        lo = int(rng() * 4294967296) & 0xFFFFFFFF
        out[w] = (hi << 32) | lo
    return out


BARY_N, BARY_R, BARY_BS = [16, 64, 256], [1, 4, 8], [8, 64, 1024]
BARY_CASES = [(n, r, b) for n in BARY_N for r in BARY_R for b in BARY_BS]


@gpu
@pytest.mark.parametrize("ci", range(len(BARY_CASES)))
def test_barycentric_grid(ctx, oracle, ci):
    """test/par3-barycentric-parity.js: fI = 0, fR = N + 1, per-case seed
    SEED ^ ((ci + 1) * 0x9E3779B1)."""
    from parparpar_b200 import par3
    n, r, bs = BARY_CASES[ci]
    seed = (0xDEADBEEF ^ (((ci + 1) * 0x9E3779B1) & 0xFFFFFFFF)) & 0xFFFFFFFF
    x = random_words(mulberry32(seed), n * bs // 8).reshape(n, bs // 8)
    out = np.zeros((r, bs // 8), dtype=np.uint64)
    par3.compute_recovery_barycentric(x, out, n, r, bs, 0, n + 1, 0)
    assert (out == oracle.gf64_compute_recovery(x, r, 0, n + 1)).all()


def full_recovery_configs():
    """The 16 draws of test/par3-full-recovery-parity.js (seed 0xC0FFEE42),
    each with its input data."""
    rng = mulberry32(0xC0FFEE42)
    cfgs = []
    for _ in range(16):
        ni = [4, 16, 64][int(rng() * 3)]
        nr = [2, 8, 16][int(rng() * 3)]
        bs = [4096, 16384][int(rng() * 2)]
        fi = int(rng() * 100)
        fr = int(rng() * 100) + 200
        x = random_words(rng, ni * bs // 8).reshape(ni, bs // 8)
        cfgs.append((ni, nr, bs, fi, fr, x))
    return cfgs


@gpu
def test_full_recovery_grid(ctx, oracle):
    from parparpar_b200 import par3
    for ni, nr, bs, fi, fr, x in full_recovery_configs():
        out = np.zeros((nr, bs // 8), dtype=np.uint64)
        par3.compute_recovery_full(x, out, ni, nr, bs, fi, fr, 0)
        assert (out == oracle.gf64_compute_recovery(x, nr, fi, fr)).all(), (ni, nr, bs, fi, fr)
        # the streaming export over the same inputs cut into two batches
        out2 = np.zeros_like(out)
        cut = ni // 2
        par3.compute_recovery_streaming([x[:cut].copy(), x[cut:].copy()], out2, ni, nr, bs, fi, fr)
        assert (out2 == out).all()


REPAIR_SCENARIOS = [(8, 3, 64, [1, 2, 3]), (16, 4, 128, [1, 2, 3, 4]), (8, 2, 1024, [1, 2]),
                    (32, 5, 256, [1, 2, 3, 4, 5]), (10, 3, 512, [1, 2, 3])]


@gpu
def test_repair_grid(ctx, oracle):
    """test/par3-repair-parity.js (seed 0xCAFEF00D): per scenario fI in
    [0, 100], fR in [200, 300]; per lost count the lost blocks and the data
    are drawn, the recovery blocks encoded, the lost blocks restored."""
    from parparpar_b200 import par3
    rng = mulberry32(0xCAFEF00D)
    for total, rcount, bs, counts in REPAIR_SCENARIOS:
        fi = int(rng() * 101)
        fr = int(rng() * 101) + 200
        for m in counts:
            if m > rcount:
                continue
            used, lost = set(), []
            for _ in range(m):
                while True:
                    idx = int(rng() * total)
                    if idx not in used:
                        break
                used.add(idx)
                lost.append(idx)
            lost.sort()
            words = bs // 8
            x = np.stack([random_words(rng, words) for _ in range(total)])
            rec = oracle.gf64_compute_recovery(x, rcount, fi, fr)
            damaged = x.copy()
            damaged[lost] = 0
            restored = par3.repair(damaged, np.array(lost, dtype=np.uint64), rec[:m], words, fi, fr, ctx=ctx)
            assert (np.asarray(restored).reshape(m, words) == x[lost]).all(), (total, rcount, bs, m)


@gpu
def test_native_edge_cases(ctx, oracle):
    """test/par3-native-edge.js scenarios that produce output: one input and
    one recovery block (output non-zero and not the input), blockSize 8,
    large blocks; deterministic across calls."""
    from parparpar_b200 import par3
    x = np.array([[0xDEADBEEFCAFEBABE]], dtype=np.uint64)
    out = np.zeros((1, 1), dtype=np.uint64)
    par3.compute_recovery(x, out, 1, 1, 8, 0, 2, 1)  # fR = 2: coefficient 1/(0 + 2) != 1
    assert out[0, 0] != 0 and out[0, 0] != x[0, 0]
    assert (out == oracle.gf64_compute_recovery(x, 1, 0, 2)).all()
    x2 = np.arange(1, 3, dtype=np.uint64).reshape(2, 1)
    a = np.zeros((1, 1), dtype=np.uint64)
    b = np.zeros((1, 1), dtype=np.uint64)
    par3.compute_recovery(x2, a, 2, 1, 8, 0, 2, 0)
    par3.compute_recovery(x2, b, 2, 1, 8, 0, 2, 64)
    assert a[0, 0] != 0 and (a == b).all()
    big = np.random.default_rng(3).integers(0, 2**63, (3, 128 * 1024), dtype=np.uint64)
    o3 = np.zeros((2, 128 * 1024), dtype=np.uint64)
    par3.compute_recovery(big, o3, 3, 2, 8 * 128 * 1024, 0, 3)
    assert o3.any() and (o3 == oracle.gf64_compute_recovery(big, 2, 0, 3)).all()


@gpu
def test_small_exports(ctx, oracle, rng):
    """mul_arr, xor_buffers and gf64_solve exports."""
    from parparpar_b200 import par3
    x = rng.integers(0, 2**63, 37, dtype=np.uint64)
    co = rng.integers(1, 2**63, 3, dtype=np.uint64)
    out = np.zeros(37, dtype=np.uint64)
    par3.mul_arr(out, x, co, 37, 3)
    assert all(int(out[i]) == oracle.gf64_mul(int(x[i]), int(co[i % 3])) for i in range(37))
    d = rng.integers(0, 256, 1003, dtype=np.uint8)
    s = rng.integers(0, 256, 1003, dtype=np.uint8)
    want = d ^ s
    par3.xor_buffers(d, s)
    assert (d == want).all()
    with pytest.raises(ValueError):
        par3.xor_buffers(np.zeros(8, np.uint8), np.zeros(9, np.uint8))
    n = 9
    A = oracle.gf64_build_cauchy(n, n, 0, 100).copy()
    b = rng.integers(0, 2**63, n, dtype=np.uint64)
    A0, b0 = A.copy(), b.copy()
    xs = par3.gf64_solve(A, b, n)
    assert (A == A0).all() and (b == b0).all()
    # A x == b
    for row in range(n):
        acc = 0
        for col in range(n):
            acc ^= oracle.gf64_mul(int(A0[row, col]), int(xs[col]))
        assert acc == int(b0[row])
    assert par3.gf64_solve(np.zeros((2, 2), np.uint64), np.ones(2, np.uint64), 2) is None
