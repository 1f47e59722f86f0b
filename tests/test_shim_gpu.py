"""The reference's PAR2 front controller driving the CUDA backend shim.

PAR2Proc (gf16/controller.cpp, the reference's own code, non-libuv build as
test/gf16/test-ctrl.cpp uses it) drives PAR2ProcCUDA
(parparpar_b200/shim/controller_cuda.cpp, compiled against the reference's
controller.h) (a) alone and (b) beside the reference's PAR2ProcCPU, each
slice split by byte range: [0, k) on the CPU, [k, S) on the GPU
(controller.cpp:42-84).  Outputs must equal the reference CPU backend's
alone, byte for byte, and the memory-checksum flags must hold.  The shim
library is built by `make -C oracle shim` (oracle/_ref/libppshim.so).
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shim():
    if not orc.Shim.available():
        pytest.skip("oracle/_ref/libppshim.so not built (needs the reference sources)")
    return orc.Shim()


def _want(oracle, data, s, idx, exps, last):
    d = data.copy()
    d[-1, last:] = 0  # bytes past a short last slice are not input
    return oracle.par2_muladd(list(d), s, oracle.par2_coeff_matrix(idx, exps))


@pytest.mark.parametrize("s,last,n,r", [
    (2, 2, 1, 1), (2, 1, 16, 3), (19998, 19998, 15, 16), (20000, 1, 16, 15), (20000, 19999, 16, 2),
    (65536, 65536, 40, 8), (4001, 4001, 9, 5), (300000, 123457, 5, 4),
])
def test_par2proc_over_the_cuda_backend_alone_and_split(ctx, oracle, shim, s, last, n, r):
    rng = np.random.default_rng(s * 31 + n * 7 + r)
    data = rng.integers(0, 256, (n, s), dtype=np.uint8)
    idx = rng.choice(32768, n, replace=False).astype(np.uint16)
    exps = rng.choice(65535, r, replace=False).astype(np.uint16)
    want = _want(oracle, data, s, idx, exps, last)
    cpu, st_cpu = shim.par2_create(data, s, idx, exps, split=s, last_size=last)
    assert np.array_equal(cpu, want)
    # (a) the CUDA backend alone
    gpu, st = shim.par2_create(data, s, idx, exps, split=0, last_size=last)
    assert st == 1 and np.array_equal(gpu, want)
    # (b) CPU on [0, k), CUDA on [k, S): k a word boundary
    for k in sorted({2, (s // 2) & ~1, (s - 2) & ~1} - {0, s}):
        if k >= s:
            continue
        got, st = shim.par2_create(data, s, idx, exps, split=k, last_size=last)
        assert np.array_equal(got, want), k
        # the reference CPU backend flags odd slice sizes invalid; here its part [0, k) is even
        assert st == 1, k
    if s % 2 == 0:
        assert st_cpu == 1


def test_par2proc_decode_overload_split(ctx, oracle, shim):
    rng = np.random.default_rng(44)
    n, s, r = 30, 8192, 6
    data = rng.integers(0, 256, (n, s), dtype=np.uint8)
    co = rng.integers(0, 65536, (r, n)).astype(np.uint16)
    want = oracle.par2_muladd(list(data), s, co)
    for split in (0, 4096, 8190):
        got, st = shim.par2_create_coeffs(data, s, co, split=split)
        assert st == 1 and np.array_equal(got, want), split


def test_second_set_slice_size_reallocates(ctx, oracle, shim):
    rng = np.random.default_rng(45)
    n, s, exps = 10, 6000, [0, 3]
    data = rng.integers(0, 256, (n, s), dtype=np.uint8)
    got, st = shim.par2_resize_then_create(data, 1000, s, np.arange(n), exps)
    assert st == 1
    assert np.array_equal(got, _want(oracle, data, s, np.arange(n), exps, s))


def test_par2proc_config_256x64KiB_R8_split_between_cpu_and_gpu(ctx, oracle, shim, golden):
    """The plain-create configuration through the reference controller with
    half of every slice on each backend: the output hashes to the digest of
    the reference controller's own output."""
    import hashlib
    g = golden("configs.npz")
    n, s, r = 256, 65536, 8
    data = orc.pattern_bytes(n * s, int(g["cfg1_seed"])).reshape(n, s)
    got, st = shim.par2_create(data, s, np.arange(n), list(range(r)), split=32768)
    assert st == 1
    assert hashlib.sha256(got.tobytes()).digest() == g["cfg1_sha256"].tobytes()


def test_batches_done_counts_finished_staging_areas(ctx):
    """pp_par2_proc_batches_done / wait_batches: every started batch is
    counted once its device work has finished (what the libuv build of the
    shim reports to PAR2Proc::onBackendProcess)."""
    import parparpar_b200._lib as L
    from parparpar_b200 import par2
    proc = par2.PAR2ProcCUDA(4096, 2, 4, ctx=ctx)
    assert proc.setRecoverySlices(3, [0, 1, 2])
    data = np.random.default_rng(9).integers(0, 256, (11, 4096), dtype=np.uint8)
    for i in range(11):
        proc.waitForAdd()
        proc.addInput(data[i], 4096, i)
    started = proc.getBatchesStarted()
    assert started == 2  # two full areas of 4
    assert L.lib.pp_par2_proc_wait_batches(proc.h, started) == L.PP_OK
    assert L.lib.pp_par2_proc_batches_done(proc.h) == started
    proc.endInput()
    assert proc.getBatchesStarted() == 3
    assert L.lib.pp_par2_proc_wait_batches(proc.h, 3) == L.PP_OK
    assert L.lib.pp_par2_proc_batches_done(proc.h) == 3
    proc.deinit()
