"""The benchmark's job mixes, checked against the oracle.

* The 16 uneven PAR3 repair jobs of the batched comparison (64 MiB-1 GiB,
  4-64 KiB blocks, 1 % lost; bench.batched_repair_jobs): the recovery rows
  are made consistent with the inputs (the create's first n rows), sampled
  rows and windows of them are checked against the reference build / the
  oracle, and then the batch plan and the single-job call must both give
  back the erased blocks exactly.
* The 32-job serving mix (PAR2/PAR3 create and repair, 1 MiB-1 GiB,
  4 KiB-1 MiB slices, R 4-512; bench.serving_jobs) submitted at once to the
  serving loop: every create / decode output on windows of every slice
  (first and last bytes) against the oracle, every PAR3 repair restores its
  erased blocks, and the single-job calls give the same bytes.

Integer GF words: exact comparisons.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gf64_rows(oracle, cols, n_rec, first_in, first_rec, rows):
    """Rows `rows` of a GF(2^64) create restricted to the columns `cols`,
    from the reference build when present, else from the oracle."""
    import oracle as orc
    src = orc.Reference() if orc.Reference.available() else None
    out = []
    for r in rows:
        if src is not None:
            out.append(src.gf64_compute_recovery(0, cols, 1, first_in, first_rec + int(r))[0])
        else:
            out.append(oracle.gf64_compute_recovery(cols, 1, first_in, first_rec + int(r))[0])
    return np.stack(out)


def _edge_rows(n):
    return sorted({0, n // 2, n - 1})


def _word_windows(words):
    """Each block's first and last 32 bytes (4 words each)."""
    return sorted(set(range(min(4, words))) | set(range(max(0, words - 4), words)))


def test_batch16_uneven_repairs_restore_the_erased_blocks(ctx, oracle):
    import torch
    import bench
    from parparpar_b200 import batch as B
    from parparpar_b200 import par3
    par3.GF64Controller.ctx = ctx
    jobs = bench.batched_repair_jobs(0)
    keep = []
    for j in jobs:
        N, n, words = j["N"], j["n"], j["words"]
        par3.GF64Controller.ComputeRecoveryBlocks(j["d_in"], N, j["d_rec"], n, words, 0, N)
        ctx.synchronize()
        sel = torch.tensor(_word_windows(words), device="cuda")
        cols = np.ascontiguousarray(j["d_in"][:, sel].cpu().numpy().view(np.uint64))
        rows = _edge_rows(n)
        want = _gf64_rows(oracle, cols, n, 0, N, rows)
        got = j["d_rec"][:, sel].cpu().numpy().view(np.uint64)[rows]
        assert np.array_equal(got, want), (N, n, words)
        idx = torch.from_numpy(j["lost"].astype(np.int64)).cuda()
        keep.append(j["d_in"][idx].clone())
        j["d_in"][idx] = 0  # erased blocks are never read
    torch.cuda.synchronize()
    outs = [torch.zeros((j["n"], j["words"]), dtype=torch.int64, device="cuda") for j in jobs]
    b = B.Batch([B.par3_repair_job(j["d_in"], j["lost"], j["d_rec"], o) for j, o in zip(jobs, outs)], ctx=ctx)
    b.run()
    ctx.synchronize()
    b.close()
    for k, (o, want) in enumerate(zip(outs, keep)):
        assert torch.equal(o, want), f"batched job {k}"
        o.zero_()
    for k, (j, o, want) in enumerate(zip(jobs, outs, keep)):
        par3.repair(j["d_in"], j["lost"], j["d_rec"], j["words"], 0, j["N"], restored=o, ctx=ctx)
        ctx.synchronize()
        assert torch.equal(o, want), f"single-job call, job {k}"
    del jobs, outs, keep
    torch.cuda.empty_cache()


def test_serving_mix_32_jobs_against_the_oracle(ctx, oracle):
    import torch
    import bench
    from parparpar_b200 import batch as B
    from parparpar_b200 import par2, par3
    from parparpar_b200.server import Server
    par3.GF64Controller.ctx = ctx
    jobs = bench.serving_jobs(0)
    # PAR3 repairs: recovery rows consistent with the inputs, erased blocks kept aside
    for j in jobs:
        if j["kind"] == "par3_repair":
            N, n, w = j["N"], j["R"], j["sl"] // 8
            par3.GF64Controller.ComputeRecoveryBlocks(j["inp"], N, j["rec"], n, w, 0, N)
            idx = torch.from_numpy(j["lost"].astype(np.int64))
            j["keep"] = j["inp"][idx].clone()
            j["inp"][idx] = 0

    def out_of(j):
        w = j["sl"] if j["kind"].startswith("par2") else j["sl"] // 8
        dt = torch.uint8 if j["kind"].startswith("par2") else torch.int64
        return torch.zeros((j["R"], w), dtype=dt).pin_memory()

    def job_of(j, o):
        k = j["kind"]
        if k == "par2_create":
            return B.par2_create_job(j["inp"], j["exps"], o)
        if k == "par2_repair":
            return B.gf16_muladd_job(j["inp"], j["coeffs"], o)
        if k == "par3_create":
            return B.par3_create_job(j["inp"], o, 0, j["N"])
        return B.par3_repair_job(j["inp"], j["lost"], j["rec"], o, 0, j["N"])

    srv = Server(0, hbm_budget_bytes=120 * 10**9, lanes=2)
    outs = [out_of(j) for j in jobs]
    tickets = [srv.submit(job_of(j, o)) for j, o in zip(jobs, outs)]
    assert [srv.wait(t) for t in tickets] == [0] * len(jobs)
    srv.close()

    for k, (j, o) in enumerate(zip(jobs, outs)):
        kind, N, sl, R = j["kind"], j["N"], j["sl"], j["R"]
        if kind == "par3_repair":
            assert torch.equal(o, j["keep"]), f"job {k}: {kind}"
            continue
        if kind.startswith("par2"):
            co = (oracle.par2_coeff_matrix(np.arange(N), list(j["exps"])) if kind == "par2_create"
                  else j["coeffs"])
            for st in sorted({0, max(0, sl - 32)}):
                wd = min(32, sl - st)
                cols = np.ascontiguousarray(j["inp"][:, st:st + wd].numpy())
                want = oracle.par2_muladd(list(cols), wd, co)
                assert np.array_equal(o[:, st:st + wd].numpy(), want), f"job {k}: {kind} at byte {st}"
        else:
            w = sl // 8
            sel = _word_windows(w)
            cols = np.ascontiguousarray(j["inp"][:, sel].numpy().view(np.uint64))
            rows = _edge_rows(R)
            want = _gf64_rows(oracle, cols, R, 0, N, rows)
            assert np.array_equal(o[:, sel].numpy().view(np.uint64)[rows], want), f"job {k}: {kind}"

    # the single-job entry points give the same bytes
    for k, (j, o) in enumerate(zip(jobs, outs)):
        p = out_of(j)
        kind = j["kind"]
        if kind == "par2_create":
            par2.par2_create(j["inp"], np.arange(j["N"]), j["exps"], out=p, ctx=ctx)
        elif kind == "par2_repair":
            par2.gf16_muladd(j["inp"], j["coeffs"], out=p, ctx=ctx)
        elif kind == "par3_create":
            par3.GF64Controller.ComputeRecoveryBlocks(j["inp"], j["N"], p, j["R"], j["sl"] // 8, 0, j["N"])
        else:
            par3.repair(j["inp"], j["lost"], j["rec"], j["sl"] // 8, 0, j["N"], restored=p, ctx=ctx)
        ctx.synchronize()
        assert torch.equal(p, o), f"job {k}: {kind}"
