"""Batches (pp_batch_*): many jobs of mixed kinds and sizes fused into a few
tensor-core launches and replayed from a CUDA graph.

Each job's output must equal, bit for bit, the same job run alone through the
single-job entry points (which the other GPU tests pin to the oracle), and a
small job of each kind is also checked against the oracle directly.  Results
are integer GF words: every comparison is exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _u64(t):
    return t.cpu().numpy().view(np.uint64)


def _par2_rows(rng, n, slice_bytes, stride):
    import torch
    buf = torch.zeros((n, stride), dtype=torch.uint8, device="cuda")
    buf[:, :slice_bytes] = _t(rng.integers(0, 256, (n, slice_bytes), dtype=np.uint8))
    return buf


def _mixed_jobs(rng):
    """(kind, job tuple, single-job reference function) for a mix of shapes."""
    import torch
    from parparpar_b200 import batch as B
    from parparpar_b200 import default_context, par2, par3

    jobs, checks = [], []

    # PAR2 create: odd slice length (rows padded to 16 bytes), arbitrary ids
    for n, sb, stride, r in [(40, 1001, 1008, 5), (300, 4096, 4096, 16), (9, 64, 64, 1)]:
        inp = _par2_rows(rng, n, sb, stride)
        ids = rng.choice(32768, n, replace=False).astype(np.uint16)
        exps = rng.choice(65535, r, replace=False).astype(np.uint16)
        out = torch.zeros((r, stride), dtype=torch.uint8, device="cuda")
        jobs.append(B.par2_create_job(inp[:, :sb], exps, out, input_ids=ids, slice_bytes=sb))

        def ref(inp=inp, ids=ids, exps=exps, sb=sb, r=r):
            o = torch.zeros((r, sb), dtype=torch.uint8, device="cuda")
            par2.par2_create(inp[:, :sb].contiguous(), ids, exps, out=o)
            default_context().synchronize()  # device buffers: the call is asynchronous on the context's stream
            return o.cpu().numpy()
        checks.append(("par2", lambda out=out, sb=sb: out[:, :sb].cpu().numpy(), ref))

    # PAR3 create
    for N, words, R, fI, fR in [(50, 64, 3, 0, 50), (1000, 16, 20, 5, 2000), (7, 2, 9, 0, 7)]:
        inp = _t(rng.integers(0, 2**64, (N, words), dtype=np.uint64).view(np.int64))
        out = torch.zeros((R, words), dtype=torch.int64, device="cuda")
        jobs.append(B.par3_create_job(inp, out, fI, fR))

        def ref(inp=inp, N=N, words=words, R=R, fI=fI, fR=fR):
            o = torch.zeros((R, words), dtype=torch.int64, device="cuda")
            par3.GF64Controller.ComputeRecoveryBlocks(inp, N, o, R, words, fI, fR)
            default_context().synchronize()
            return _u64(o)
        checks.append(("par3", lambda out=out: _u64(out), ref))

    # PAR3 repair: closed-form inverse, and the Gauss-Jordan case (a lost id
    # equals a recovery row id) with one absent recovery row
    for N, words, n, fI, fR, collide, absent in [(400, 32, 12, 0, 400, False, None), (64, 8, 6, 0, 10, True, 2)]:
        data = rng.integers(0, 2**64, (N, words), dtype=np.uint64)
        lost = np.sort(rng.choice(N, n, replace=False))
        if collide:
            lost[0] = 12
            lost = np.unique(lost)
            n = lost.size
        rec = rng.integers(0, 2**64, (n, words), dtype=np.uint64)
        present = None
        if absent is not None:
            present = np.ones(n, dtype=np.uint8)
            present[absent] = 0
        d_in = _t(data.view(np.int64))
        d_rec = _t(rec.view(np.int64))
        restored = torch.zeros((n, words), dtype=torch.int64, device="cuda")
        jobs.append(B.par3_repair_job(d_in, lost, d_rec, restored, fI, fR, recovery_present=present))

        def ref(data=data, lost=lost, rec=rec, words=words, fI=fI, fR=fR, present=present):
            return par3.repair(data, lost, rec.copy(), words, fI, fR, recovery_present=present)
        checks.append(("repair", lambda restored=restored: _u64(restored), ref))
    return jobs, checks


@pytest.mark.parametrize("graph", [True, False])
def test_mixed_batch_matches_single_jobs(graph):
    """Replayed from its CUDA graph, or (graph=False, jobs seen once) built
    without the eager run and capture and issued directly at run()."""
    from parparpar_b200 import batch as B
    import torch
    rng = np.random.default_rng(7)
    jobs, checks = _mixed_jobs(rng)
    torch.cuda.synchronize()  # inputs were written on torch's stream; the library uses its own
    b = B.Batch(jobs, graph=graph)
    if graph:
        assert b.launches >= 3
    for rep in range(2):  # graph replays
        b.run()
        b.ctx.synchronize()
        for kind, got, ref in checks:
            assert np.array_equal(got(), ref()), (kind, rep)
    b.close()


def test_batch_replay_reads_current_inputs_and_tuning_keeps_results():
    import torch
    from parparpar_b200 import batch as B
    from parparpar_b200 import par3
    rng = np.random.default_rng(8)
    N, words, R = 3000, 64, 12
    inp = _t(rng.integers(0, 2**64, (N, words), dtype=np.uint64).view(np.int64))
    out = torch.zeros((R, words), dtype=torch.int64, device="cuda")
    b = B.Batch([B.par3_create_job(inp, out)], tune=True)
    b.run()
    b.ctx.synchronize()
    first = _u64(out).copy()
    ref = torch.zeros_like(out)
    par3.GF64Controller.ComputeRecoveryBlocks(inp, N, ref, R, words, 0, N)
    b.ctx.synchronize()
    assert np.array_equal(first, _u64(ref))
    inp[5].fill_(0x1234)  # new input data, same plan
    torch.cuda.synchronize()
    b.run()
    b.ctx.synchronize()
    par3.GF64Controller.ComputeRecoveryBlocks(inp, N, ref, R, words, 0, N)
    b.ctx.synchronize()
    assert np.array_equal(_u64(out), _u64(ref))
    assert not np.array_equal(_u64(out), first)
    b.close()


def test_batch_with_more_jobs_than_one_table(oracle):
    import torch
    from parparpar_b200 import batch as B
    rng = np.random.default_rng(9)
    jobs, expect, outs = [], [], []
    for k in range(30):
        N, words, R = int(rng.integers(2, 40)), 2 * int(rng.integers(1, 20)), int(rng.integers(1, 6))
        data = rng.integers(0, 2**64, (N, words), dtype=np.uint64)
        out = torch.zeros((R, words), dtype=torch.int64, device="cuda")
        jobs.append(B.par3_create_job(_t(data.view(np.int64)), out, k, 1000 + k))
        expect.append(oracle.gf64_compute_recovery(data, R, k, 1000 + k))
        outs.append(out)
    b = B.Batch(jobs)
    b.run()
    b.ctx.synchronize()
    for e, o in zip(expect, outs):
        assert np.array_equal(_u64(o), e)
    b.close()


def test_batch_small_jobs_vs_oracle(oracle):
    import torch
    from parparpar_b200 import batch as B
    rng = np.random.default_rng(10)
    n, sb, r = 20, 512, 4
    data = rng.integers(0, 256, (n, sb), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint16)
    out = torch.zeros((r, sb), dtype=torch.uint8, device="cuda")
    N, words, n_lost = 100, 8, 5
    d64 = rng.integers(0, 2**64, (N, words), dtype=np.uint64)
    rec = oracle.gf64_compute_recovery(d64, n_lost, 0, N)
    lost = np.sort(rng.choice(N, n_lost, replace=False))
    restored = torch.zeros((n_lost, words), dtype=torch.int64, device="cuda")
    b = B.Batch([B.par2_create_job(_t(data), exps, out),
                 B.par3_repair_job(_t(d64.view(np.int64)), lost, _t(rec.view(np.int64)), restored)])
    b.run()
    b.ctx.synchronize()
    co = oracle.par2_coeff_matrix(np.arange(n), list(exps))
    assert np.array_equal(out.cpu().numpy(), oracle.par2_muladd(list(data), sb, co))
    assert np.array_equal(_u64(restored), d64[lost])
    b.close()


def test_batch_rejects_misaligned_rows():
    import torch
    from parparpar_b200 import PPError
    from parparpar_b200 import batch as B
    buf = torch.zeros((4, 80), dtype=torch.uint8, device="cuda")
    out = torch.zeros((2, 64), dtype=torch.uint8, device="cuda")
    with pytest.raises(PPError):
        B.Batch([B.par2_create_job(buf[:, 8:72], [0, 1], out)])  # rows start 8 bytes off 16
