"""Batched additive FFT on the GPU vs the oracle and the reference fixtures."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fft_golden_single(ctx, golden):
    from parparpar_b200 import par3
    g = golden("gf64_fft.npz")
    for n in g["sizes"]:
        n = int(n)
        x = g[f"x{n}"].copy()
        par3.gf64_addfft64_fwd(x, ctx=ctx)
        assert np.array_equal(x, g[f"fwd{n}"]), n
        y = g[f"x{n}"].copy()
        par3.gf64_addfft64_inv(y, ctx=ctx)
        assert np.array_equal(y, g[f"inv{n}"]), n


@pytest.mark.parametrize("n,batch", [(2, 7), (64, 33), (1024, 256), (16384, 3), (131072, 4)])
def test_fft_batched_vs_oracle(ctx, oracle, n, batch):
    import torch
    from parparpar_b200 import par3
    rng = np.random.default_rng(n + batch)
    x = rng.integers(0, 2**64, (n, batch), dtype=np.uint64)
    exp_f = np.stack([oracle.gf64_fft(x[:, b]) for b in range(batch)], axis=1)
    exp_i = np.stack([oracle.gf64_fft(x[:, b], inverse=True) for b in range(batch)], axis=1)
    h = x.copy()
    par3.gf64_addfft64_fwd(h, ctx=ctx)
    assert np.array_equal(h, exp_f)
    d = torch.from_numpy(x.view(np.int64).copy()).cuda()
    par3.gf64_addfft64_inv(d, ctx=ctx)
    ctx.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint64), exp_i)


def test_fft_roundtrip_identity(ctx):
    """For the novel-polynomial transform pair, inverse(forward(p)) == p
    (checked on the oracle too); a size-independent property."""
    from parparpar_b200 import par3
    rng = np.random.default_rng(5)
    for n in (4, 256, 4096):
        x = rng.integers(0, 2**64, (n, 16), dtype=np.uint64)
        y = x.copy()
        par3.gf64_addfft64_fwd(y, ctx=ctx)
        par3.gf64_addfft64_inv(y, ctx=ctx)
        assert np.array_equal(y, x)
