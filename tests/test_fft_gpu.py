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


@pytest.mark.parametrize("n,batch", [(2, 7), (64, 33), (512, 9), (1024, 256), (2048, 17), (8192, 12), (16384, 3),
                                     (65536, 9), (131072, 4), (2**18, 3), (2**19, 5), (2**20, 2)])
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


def test_fft_full_size_1GiB(ctx, oracle):
    """The bench's transform: 1,024 polynomials of 131,072 coefficients
    (the 1 GiB PAR3 data, 8 KiB slices) on the device.  Sampled columns
    (first, second, a middle and the last polynomial) against the oracle,
    then the inverse must give back the whole input."""
    import torch
    from parparpar_b200 import par3
    n, batch = 131072, 1024
    g = torch.Generator(device="cuda").manual_seed(17)
    d = torch.randint(0, 256, (n * batch * 8,), dtype=torch.uint8, device="cuda", generator=g).view(torch.int64)
    d = d.view(n, batch)
    orig = d.clone()
    par3.gf64_addfft64_fwd(d, ctx=ctx)
    ctx.synchronize()
    cols = [0, 1, 511, 1023]
    x = orig[:, cols].cpu().numpy().view(np.uint64)
    y = d[:, cols].cpu().numpy().view(np.uint64)
    for k in range(len(cols)):
        assert np.array_equal(y[:, k], oracle.gf64_fft(x[:, k].copy())), cols[k]
    par3.gf64_addfft64_inv(d, ctx=ctx)
    ctx.synchronize()
    assert torch.equal(d, orig)
