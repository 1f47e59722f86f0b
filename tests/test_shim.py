"""The reference's PAR2 front controller over the CUDA backend shim, on CPU.

parparpar_b200/shim/controller_cuda.cpp implements the reference's
IPAR2ProcBackend (gf16/controller.h:77-217) over the C ABI; oracle/Makefile
compiles it against the reference's own controller sources into
oracle/_ref/libppshim.so.  Without a GPU: the library loads, the CPU-only
split of PAR2Proc gives the reference controller's output, and a CUDA
backend that cannot open a device reports it at init (the controller's
caller then leaves the backend out).  The GPU side is tests/test_shim_gpu.py.
"""
import numpy as np
import pytest

import oracle as orc


@pytest.fixture(scope="module")
def shim():
    if not orc.Shim.available():
        pytest.skip("oracle/_ref/libppshim.so not built (needs the reference sources)")
    return orc.Shim()


def test_cpu_alone_through_the_shim_library(shim, oracle):
    rng = np.random.default_rng(5)
    n, s, exps = 12, 4000, [0, 1, 5]
    data = rng.integers(0, 256, (n, s), dtype=np.uint8)
    out, st = shim.par2_create(data, s, np.arange(n), exps, split=s)
    assert st == 1
    assert np.array_equal(out, oracle.par2_muladd(list(data), s, oracle.par2_coeff_matrix(np.arange(n), exps)))


def test_cuda_backend_without_a_device_fails_at_init(shim):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    data = np.zeros((2, 64), dtype=np.uint8)
    _, st = shim.par2_create(data, 64, [0, 1], [0], split=0)
    assert st == -3
