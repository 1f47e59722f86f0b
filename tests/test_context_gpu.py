"""Context-level machinery on the GPU: the Cauchy-matrix cache under
eviction, kernel-timing brackets and host tracing.

* More PAR3 shapes than the cache holds (8, as the reference's
  GetOrBuildCoeffMatrix), cycled twice: evicted matrices' buffers are reused
  in stream order for the next matrices, and every result must still equal
  the oracle's.
* pp_ctx_set_kernel_timing / pp_ctx_kernel_time: one bracket per region
  product, positive device time, none when switched off.
* PARPAR_B200_TRACE=1 in a child process: the entry point's span is printed.
Integer GF words: exact comparisons.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cauchy_cache_evicts_and_reuses_buffers(oracle):
    import parparpar_b200 as pp
    from parparpar_b200 import par3
    ctx = pp.Context(0)  # a fresh cache
    par3.GF64Controller.ctx = ctx
    rng = np.random.default_rng(99)
    shapes = [(int(rng.integers(3, 70)), int(rng.integers(1, 9)), int(rng.integers(0, 1000))) for _ in range(12)]
    for rnd in range(2):
        for N, R, fI in shapes:
            W = 34
            x = rng.integers(0, 2**64, (N, W), dtype=np.uint64)
            got = np.zeros((R, W), dtype=np.uint64)
            par3.GF64Controller.ComputeRecoveryBlocks(x, N, got, R, W, fI, fI + N)
            assert np.array_equal(got, oracle.gf64_compute_recovery(x, R, fI, fI + N)), (rnd, N, R, fI)


def test_kernel_timing_brackets_region_products(ctx):
    import torch
    from parparpar_b200 import par2
    d = torch.randint(0, 256, (64, 65536), dtype=torch.uint8, device="cuda")
    o = torch.zeros((16, 65536), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ctx.kernel_time()
    ctx.set_kernel_timing(True)
    for _ in range(3):
        par2.par2_create(d, np.arange(64), list(range(16)), out=o, ctx=ctx)
    ctx.set_kernel_timing(False)
    ms, n = ctx.kernel_time()
    assert n == 3 and ms > 0
    par2.par2_create(d, np.arange(64), list(range(16)), out=o, ctx=ctx)
    ms, n = ctx.kernel_time()
    assert n == 0 and ms == 0


def test_trace_spans_on_stderr():
    code = (f"import sys; sys.path.insert(0, {ROOT!r})\n"
            "import numpy as np, torch\n"
            "import parparpar_b200 as pp\n"
            "from parparpar_b200 import par2\n"
            "ctx = pp.Context(0)\n"
            "d = np.random.default_rng(1).integers(0, 256, (4096, 32768), dtype=np.uint8)\n"
            "par2.par2_create(d, np.arange(4096), list(range(16)), ctx=ctx)\n")
    r = subprocess.run([sys.executable, "-c", code], env=dict(os.environ, PARPAR_B200_TRACE="1"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "pp-trace call-par2_create" in r.stderr
    r = subprocess.run([sys.executable, "-c", code], env=dict(os.environ, PARPAR_B200_TRACE="0"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "pp-trace" not in r.stderr
