"""Parity at the benchmark configurations' full sizes.

The oracle cannot run a whole 1 GiB job in seconds, so these tests use what
the domain offers: each output byte depends only on the same byte position
of the inputs, so sampled byte (word) ranges of every slice are recomputed
by the oracle; and a create -> erase -> repair round trip must give back the
original blocks exactly.  Integer GF words: all comparisons are exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sync():
    from parparpar_b200 import default_context
    default_context().synchronize()


def test_par2_create_32768x32KiB_R64_sampled(oracle):
    import torch
    from parparpar_b200 import par2
    n, sb, r = 32768, 32 * 1024, 64
    g = torch.Generator(device="cuda")
    g.manual_seed(2024)
    d_in = torch.randint(0, 256, (n, sb), dtype=torch.uint8, device="cuda", generator=g)
    out = torch.zeros((r, sb), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    exps = np.arange(r, dtype=np.uint16)
    par2.par2_create(d_in, np.arange(n), exps, out=out)
    _sync()
    co = oracle.par2_coeff_matrix(np.arange(n), list(exps))
    for s in (0, 20000):  # two 32-byte windows of every slice
        cols = d_in[:, s:s + 32].cpu().numpy()
        want = oracle.par2_muladd(list(cols), 32, co)
        assert np.array_equal(out[:, s:s + 32].cpu().numpy(), want), s


def test_par3_create_131072x8KiB_R8_sampled(oracle):
    import torch
    from parparpar_b200 import par3
    N, words, R = 131072, 1024, 8
    g = torch.Generator(device="cuda")
    g.manual_seed(2025)
    d_in = torch.randint(-2**63, 2**63 - 1, (N, words), dtype=torch.int64, device="cuda", generator=g)
    out = torch.zeros((R, words), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    par3.GF64Controller.ComputeRecoveryBlocks(d_in, N, out, R, words, 0, N)
    _sync()
    for w in (0, 777):  # two 2-word windows of every block
        cols = np.ascontiguousarray(d_in[:, w:w + 2].cpu().numpy().view(np.uint64))
        want = oracle.gf64_compute_recovery(cols, R, 0, N)
        assert np.array_equal(out[:, w:w + 2].cpu().numpy().view(np.uint64), want), w


def test_par3_repair_262144x4KiB_1pct_roundtrip():
    import torch
    from parparpar_b200 import par3
    N, words = 262144, 512
    n = round(0.01 * N)
    g = torch.Generator(device="cuda")
    g.manual_seed(2026)
    data = torch.randint(-2**63, 2**63 - 1, (N, words), dtype=torch.int64, device="cuda", generator=g)
    rec = torch.zeros((n, words), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    par3.GF64Controller.ComputeRecoveryBlocks(data, N, rec, n, words, 0, N)
    _sync()
    lost = np.sort(np.random.default_rng(7).choice(N, n, replace=False)).astype(np.uint64)
    idx = torch.from_numpy(lost.astype(np.int64)).cuda()
    keep = data[idx].clone()
    data[idx] = 0  # erased blocks are never read
    torch.cuda.synchronize()
    restored = torch.zeros((n, words), dtype=torch.int64, device="cuda")
    par3.repair(data, lost, rec, words, 0, N, restored=restored)
    _sync()
    assert torch.equal(restored, keep)
