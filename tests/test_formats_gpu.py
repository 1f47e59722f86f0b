"""Both operand formats of the tensor-core region kernels against the oracle.

Each tensor-core product has two operand formats, block-scaled FP4
(tcgen05 kind::mxf4) and int8 (kind::i8), chosen per process
(PARPAR_B200_GF16_TC, PARPAR_B200_GF64_TC = f4 | i8; resident GF(2^16)
coefficient tiles are laid out for one format).  The defaults are FP4 for
GF(2^16) and, for GF(2^64), FP4 on SM pairs (launches whose jobs all have at
least 4 outputs) and int8 on one CTA; the rest of the suite exercises them;
this file runs the same parity cases in a child process with both fields on
each format, so every kernel stays bit-exact.  Integer GF
words: exact comparisons.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import sys
import numpy as np
sys.path.insert(0, ROOT)
sys.path.insert(0, ROOT + "/oracle")
import oracle as orc
import parparpar_b200 as pp
import parparpar_b200._lib as L
from parparpar_b200 import par2, par3
O = orc.Oracle()
ctx = pp.Context(0)
ctx.set_gf16_kernel(L.PP_GF16_KERNEL_TENSOR)
ctx.set_gf64_kernel(L.PP_GF16_KERNEL_TENSOR)
par3.GF64Controller.ctx = ctx
rng = np.random.default_rng(2027)
# GF(2^16): one-group and two-group tiles, odd slices, ragged stages, an
# accumulating product, tile edges of both formats (240/256/480/512 words)
for n, s, r in [(16, 480, 8), (17, 961, 16), (40, 4001, 8), (33, 20000, 16), (300, 8192, 24), (9, 1026, 40)]:
    data = rng.integers(0, 256, (n, s), dtype=np.uint8)
    exps = list(range(r))
    want = O.par2_muladd(list(data), s, O.par2_coeff_matrix(np.arange(n), exps))
    assert np.array_equal(par2.par2_create(data, np.arange(n), exps, ctx=ctx), want), ("gf16", n, s, r)
    co = rng.integers(0, 65536, (r, n)).astype(np.uint16)
    base = rng.integers(0, 256, (r, s), dtype=np.uint8)
    out = base.copy()
    par2.gf16_muladd(data, co, out=out, accumulate=True, ctx=ctx)
    assert np.array_equal(out, base ^ O.par2_muladd(list(data), s, co)), ("gf16 acc", n, s, r)
# GF(2^64): tile edges (480/512 words), ragged stages, accumulate, and the
# SM pair's per-job MMA width (2 words: N = 16; 16: 16; 512: 128; 1024: 176)
for N, W, R in [(4, 480, 2), (5, 482, 3), (33, 1000, 8), (64, 96, 5), (200, 2048, 16),
                (9, 2, 4), (20, 16, 6), (40, 512, 4), (70, 1024, 8)]:
    x = rng.integers(0, 2**64, (N, W), dtype=np.uint64)
    want = O.gf64_compute_recovery(x, R, 0, N)
    got = np.zeros((R, W), dtype=np.uint64)
    par3.GF64Controller.ComputeRecoveryBlocks(x, N, got, R, W, 0, N)
    assert np.array_equal(got, want), ("gf64", N, W, R)
    acc = rng.integers(0, 2**64, (R, W), dtype=np.uint64)
    got = acc.copy()
    par3.GF64Controller.ComputeRecoveryBlocks(x, N, got, R, W, 0, N, accumulate=True)
    assert np.array_equal(got, acc ^ want), ("gf64 acc", N, W, R)
print("formats ok")
'''


@pytest.mark.parametrize("fmt", ["f4", "i8"])
def test_tensor_core_formats_against_the_oracle(fmt):
    env = dict(os.environ, PARPAR_B200_GF16_TC=fmt, PARPAR_B200_GF64_TC=fmt)
    code = f"ROOT = {ROOT!r}\n" + CHILD
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "formats ok" in r.stdout, (r.stdout[-2000:], r.stderr[-2000:])
