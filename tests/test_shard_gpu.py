"""One job split by byte range over several contexts, through the product.

pp_par2_create_split / pp_gf64_compute_recovery_split give each context (one
per GPU in production) a contiguous byte range of every slice, as PAR2Proc
splits a slice over its backends (gf16/controller.cpp:42-84).  One GPU is
available here, so the contexts share device 0; the ranges still run on
separate contexts, streams and host threads, and nothing waits across them.
Also: two `gloo` ranks (processes) on the one GPU, each computing its own
range through the CUDA library, gathered on rank 0 and compared with the
single-call result and the oracle.
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctxs(k):
    import parparpar_b200 as pp
    return [pp.Context(0) for _ in range(k)]


@pytest.mark.parametrize("n,s,k", [(40, 4096, 2), (33, 10001, 3), (300, 65536, 4), (5, 2, 2)])
def test_par2_create_split_equals_one_call(ctx, oracle, n, s, k):
    import torch
    from parparpar_b200 import par2
    from parparpar_b200.shard import byte_ranges, par2_create_split
    rng = np.random.default_rng(n + s + k)
    data = rng.integers(0, 256, (n, s), dtype=np.uint8)
    exps = [0, 1, 17, 300, 65000]
    want = oracle.par2_muladd(list(data), s, oracle.par2_coeff_matrix(np.arange(n), exps))
    cs = _ctxs(k)
    assert np.array_equal(par2_create_split(data, np.arange(n), exps, cs), want)
    # device buffers on the contexts' own GPU, uneven word-aligned ranges
    d_in = torch.from_numpy(data).cuda()
    d_out = torch.zeros((len(exps), s), dtype=torch.uint8, device="cuda")
    cut = [0] + sorted({(s * j // (k + 1)) & ~1 for j in range(1, k)}) + [s]
    ranges = list(zip(cut[:-1], cut[1:]))
    par2_create_split(d_in, np.arange(n), exps, cs[:len(ranges)], ranges=ranges, out=d_out)
    assert np.array_equal(d_out.cpu().numpy(), want)
    assert np.array_equal(par2.par2_create(data, np.arange(n), exps, ctx=ctx), want)
    assert byte_ranges(s, k, 2)  # the default split is the one checked above


def test_par3_create_split_equals_one_call(ctx, oracle):
    from parparpar_b200 import par3
    from parparpar_b200.shard import par3_create_split
    rng = np.random.default_rng(3)
    N, W, R = 64, 200, 5
    x = rng.integers(0, 2**64, (N, W), dtype=np.uint64)
    want = oracle.gf64_compute_recovery(x, R, 0, N)
    for k in (2, 3, 5):
        assert np.array_equal(par3_create_split(x, R, 0, N, _ctxs(k)), want), k
    one = np.zeros((R, W), dtype=np.uint64)
    par3.GF64Controller.ctx = ctx
    par3.GF64Controller.ComputeRecoveryBlocks(x, N, one, R, W, 0, N)
    assert np.array_equal(one, want)


def test_split_rejects_a_bad_cover(ctx):
    import parparpar_b200 as pp
    from parparpar_b200.shard import par2_create_split, par3_create_split
    cs = _ctxs(2)
    data = np.zeros((4, 100), dtype=np.uint8)
    for bad in ([(0, 51), (51, 100)], [(0, 40), (50, 100)], [(0, 60), (50, 100)]):
        with pytest.raises(pp.PPError) as ei:
            par2_create_split(data, np.arange(4), [0], cs, ranges=bad)
        assert ei.value.status == pp.PP_ERR_INVALID_ARG
    x = np.zeros((4, 10), dtype=np.uint64)
    with pytest.raises(pp.PPError):
        par3_create_split(x, 2, 0, 4, cs, ranges=[(0, 36), (36, 80)])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, result_path):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    sys.path.insert(0, root)
    import oracle as orc
    import parparpar_b200 as pp
    from parparpar_b200 import par2, par3
    from parparpar_b200.shard import byte_ranges

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ctx = pp.Context(0)  # every rank on the one GPU here; on a node, rank r on GPU r
    rng = np.random.default_rng(5)  # the same data on every rank
    n, sb, exps = 23, 1001, [0, 3, 9]
    data2 = rng.integers(0, 256, (n, sb), dtype=np.uint8)
    N, words, R = 17, 24, 3
    data3 = rng.integers(0, 2**64, (N, words), dtype=np.uint64)
    s, e = byte_ranges(sb, world, 2)[rank]
    part2 = par2.par2_create(np.ascontiguousarray(data2[:, s:e]), np.arange(n), exps, ctx=ctx) if e > s else None
    s3, e3 = byte_ranges(words * 8, world, 16)[rank]
    part3 = None
    if e3 > s3:
        part3 = np.zeros((R, (e3 - s3) // 8), dtype=np.uint64)
        par3.GF64Controller.ctx = ctx
        par3.GF64Controller.ComputeRecoveryBlocks(np.ascontiguousarray(data3[:, s3 // 8:e3 // 8]), N, part3, R,
                                                  (e3 - s3) // 8, 0, N)
    parts = [None] * world
    dist.all_gather_object(parts, (part2, part3))
    if rank == 0:
        O = orc.Oracle()
        full2 = O.par2_muladd(list(data2), sb, O.par2_coeff_matrix(np.arange(n), exps))
        full3 = O.gf64_compute_recovery(data3, R, 0, N)
        got2 = np.concatenate([p[0] for p in parts if p[0] is not None], axis=1)
        got3 = np.concatenate([p[1] for p in parts if p[1] is not None], axis=1)
        ok = np.array_equal(got2, full2) and np.array_equal(got3, full3)
        with open(result_path, "w") as f:
            f.write("ok" if ok else "mismatch")
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_run_the_product_on_their_ranges(tmp_path):
    import torch.multiprocessing as mp
    out = tmp_path / "result.txt"
    mp.spawn(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True)
    assert out.read_text() == "ok"
