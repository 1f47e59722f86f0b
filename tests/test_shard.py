"""Byte-range sharding (parparpar_b200/shard.py) across ranks, on CPU.

The split must satisfy the reference's own acceptance rule for a backend
split (gf16/controller.cpp:42-84), and the per-rank results must concatenate
to the single-rank result.  Here, without a GPU, the multi-rank case runs as
world-size-2 `gloo` processes that compute their byte ranges with the oracle:
it checks the split arithmetic and the gather.  The same ranks running the
CUDA library, and the split entry points, are in tests/test_shard_gpu.py.
"""
import os
import socket

import numpy as np
import pytest


def test_ranges_follow_the_reference_rule():
    from parparpar_b200.shard import byte_ranges, check_ranges
    for sb in (0, 1, 2, 7, 1000, 1001, 65536, 65537):
        for world in (1, 2, 3, 8):
            r = byte_ranges(sb, world, 2)
            assert len(r) == world and check_ranges(r, sb), (sb, world, r)
    for sb, world in ((8192, 3), (4096, 8), (48, 4)):
        r = byte_ranges(sb, world, 16)
        assert check_ranges(r, sb) and all(s % 16 == 0 for s, _ in r)
    assert not check_ranges([(0, 3), (3, 8)], 8)       # odd start
    assert not check_ranges([(0, 4), (5, 8)], 8)       # gap
    assert not check_ranges([(0, 6), (4, 8)], 8)       # overlap
    assert check_ranges([(0, 4), (4, 7)], 7)           # odd size only at the end


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
    from parparpar_b200.shard import byte_ranges

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    O = orc.Oracle()
    rng = np.random.default_rng(5)  # the same data on every rank
    n, sb, exps = 23, 1001, [0, 3, 9]
    data2 = rng.integers(0, 256, (n, sb), dtype=np.uint8)
    N, words, R = 17, 24, 3
    data3 = rng.integers(0, 2**64, (N, words), dtype=np.uint64)
    s, e = byte_ranges(sb, world, 2)[rank]
    co = O.par2_coeff_matrix(np.arange(n), exps)
    part2 = O.par2_muladd([np.ascontiguousarray(row[s:e]) for row in data2], e - s, co) if e > s else None
    s3, e3 = byte_ranges(words * 8, world, 16)[rank]
    part3 = O.gf64_compute_recovery(np.ascontiguousarray(data3[:, s3 // 8:e3 // 8]), R, 0, N) if e3 > s3 else None
    parts = [None] * world
    dist.all_gather_object(parts, (s, e, part2, s3, e3, part3))
    if rank == 0:
        full2 = O.par2_muladd(list(data2), sb, co)
        full3 = O.gf64_compute_recovery(data3, R, 0, N)
        got2 = np.concatenate([p[2] for p in parts if p[2] is not None], axis=1)
        got3 = np.concatenate([p[5] for p in parts if p[5] is not None], axis=1)
        ok = np.array_equal(got2, full2) and np.array_equal(got3, full3)
        with open(result_path, "w") as f:
            f.write("ok" if ok else "mismatch")
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_concatenate_to_the_full_result(tmp_path, oracle):
    import torch.multiprocessing as mp
    out = tmp_path / "result.txt"
    mp.spawn(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True)
    assert out.read_text() == "ok"
