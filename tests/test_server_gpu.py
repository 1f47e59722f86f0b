"""Serving loop (pp_server_*): continuous batching under a device-memory budget.

The property the serving loop must keep is that a job's result does not
depend on what else is in flight: every job is run once alone (submitted and
waited for before the next) and once in a mix submitted all at once from
several threads, and the outputs are compared bit for bit; each alone result
is also checked against the single-job entry points or the oracle.  Results
are integer GF words, so the tolerance is zero.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _np(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


class _Spec:
    """Inputs of one job plus a factory for fresh outputs."""

    def __init__(self, make, check):
        self.make = make    # () -> (job tuple, output buffer)
        self.check = check  # (output as numpy) -> None


def _specs(rng, oracle):
    import torch
    from parparpar_b200 import batch as B
    specs = []
    # PAR2 create, host (pinned) buffers, odd slice length
    for n, sb, r in [(64, 3001, 6), (300, 8192, 20)]:
        data = rng.integers(0, 256, (n, sb), dtype=np.uint8)
        exps = rng.choice(65535, r, replace=False).astype(np.uint16)
        h_in = _pinned(data)

        def make(h_in=h_in, exps=exps, r=r, sb=sb):
            out = _pinned(np.zeros((r, sb), dtype=np.uint8))
            return B.par2_create_job(h_in, exps, out), out

        def check(got, data=data, exps=exps, n=n, sb=sb, small=(n * sb < 300000)):
            if small:
                co = oracle.par2_coeff_matrix(np.arange(n), list(exps))
                assert np.array_equal(got, oracle.par2_muladd(list(data), sb, co))
        specs.append(_Spec(make, check))
    # PAR3 create, device buffers; and one with an odd word count (lookup path), host buffers
    for N, words, R, fI, fR, dev in [(2000, 64, 16, 0, 2000, True), (500, 7, 5, 3, 900, False)]:
        data = rng.integers(0, 2**64, (N, words), dtype=np.uint64)
        src = _dev(data.view(np.int64)) if dev else _pinned(data.view(np.int64))

        def make(src=src, R=R, words=words, fI=fI, fR=fR, dev=dev):
            z = np.zeros((R, words), dtype=np.int64)
            out = _dev(z) if dev else _pinned(z)
            return B.par3_create_job(src, out, fI, fR), out

        def check(got, data=data, R=R, fI=fI, fR=fR, N=N):
            if N * R <= 20000:
                assert np.array_equal(got.view(np.uint64), oracle.gf64_compute_recovery(data, R, fI, fR))
        specs.append(_Spec(make, check))
    # PAR3 repair: host buffers; device buffers with an absent recovery row; odd words
    for N, words, n, dev, absent in [(1500, 32, 15, False, None), (800, 16, 8, True, 3), (300, 5, 3, False, None)]:
        data = rng.integers(0, 2**64, (N, words), dtype=np.uint64)
        rec = oracle.gf64_compute_recovery(data, n, 0, N)
        lost = np.sort(rng.choice(N, n, replace=False))
        present = None
        if absent is not None:
            present = np.ones(n, dtype=np.uint8)
            present[absent] = 0
        damaged = data.copy()
        damaged[lost] = 0
        src = _dev(damaged.view(np.int64)) if dev else _pinned(damaged.view(np.int64))
        rsrc = _dev(rec.view(np.int64)) if dev else _pinned(rec.view(np.int64))

        def make(src=src, rsrc=rsrc, lost=lost, n=n, words=words, dev=dev, present=present):
            z = np.zeros((n, words), dtype=np.int64)
            out = _dev(z) if dev else _pinned(z)
            return B.par3_repair_job(src, lost, rsrc, out, recovery_present=present), out

        def check(got, data=data, lost=lost, present=present):
            if present is None:
                assert np.array_equal(got.view(np.uint64), data[lost])
        specs.append(_Spec(make, check))
    return specs


def _run_alone(srv, specs):
    outs = []
    for sp in specs:
        job, out = sp.make()
        assert srv.wait(srv.submit(job)) == 0
        outs.append(_np(out).copy())
    return outs


def test_each_result_identical_alone_and_in_the_mix(oracle):
    from parparpar_b200.server import Server
    rng = np.random.default_rng(31)
    specs = _specs(rng, oracle)
    srv = Server(hbm_budget_bytes=8 << 30, lanes=2)
    alone = _run_alone(srv, specs)
    for sp, a in zip(specs, alone):
        sp.check(a)
    # the mix: every job three times, submitted from four threads at once
    order = [i for i in range(len(specs)) for _ in range(3)]
    rng.shuffle(order)
    made = [specs[i].make() for i in order]
    tickets = [None] * len(made)

    def submit(lo):
        for k in range(lo, len(made), 4):
            tickets[k] = srv.submit(made[k][0])

    ths = [threading.Thread(target=submit, args=(t,)) for t in range(4)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for k, i in enumerate(order):
        assert srv.wait(tickets[k]) == 0
        assert np.array_equal(_np(made[k][1]), alone[i]), (k, i)
    st = srv.stats()
    assert st["completed"] == len(specs) + len(made) and st["failed"] == 0
    assert st["waves"] < st["completed"]  # jobs shared waves
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["hbm_peak_bytes"] <= 8 << 30
    srv.close()


def test_budget_admission_and_too_large_jobs():
    from parparpar_b200 import PP_ERR_TOO_LARGE
    from parparpar_b200 import batch as B
    from parparpar_b200.server import Server
    rng = np.random.default_rng(32)
    budget = 48 << 20
    srv = Server(hbm_budget_bytes=budget, lanes=2)
    small = []
    for k in range(12):  # each needs ~6-10 MiB of staging: several waves under the budget
        data = _pinned(rng.integers(0, 2**63, (1024, 512), dtype=np.int64))
        out = _pinned(np.zeros((8, 512), dtype=np.int64))
        small.append((srv.submit(B.par3_create_job(data, out, 0, 1024)), data, out))
    big_in = _pinned(np.zeros((8192, 1024), dtype=np.int64))  # 64 MiB of staging alone
    big_out = _pinned(np.zeros((4, 1024), dtype=np.int64))
    t_big = srv.submit(B.par3_create_job(big_in, big_out, 0, 8192))
    for t, _, _ in small:
        assert srv.wait(t) == 0
    assert srv.wait(t_big) == PP_ERR_TOO_LARGE
    st = srv.stats()
    assert st["hbm_peak_bytes"] <= budget
    assert st["failed"] == 1 and st["completed"] == 12
    # identical inputs and shapes: one resident Cauchy table served all of them
    assert st["tables_resident"] == 1
    srv.close()


def test_par2_repair_through_the_server():
    """PAR2 repair: pp_par2_invert factors, then the decode as a GF(2^16) job."""
    from parparpar_b200 import batch as B
    from parparpar_b200 import par2
    from parparpar_b200.server import Server
    rng = np.random.default_rng(33)
    n, sb = 50, 2048
    data = rng.integers(0, 256, (n, sb), dtype=np.uint8)
    exps = list(range(10))
    rec = par2.par2_create(data, np.arange(n), exps)
    lost = [3, 7, 20, 33, 49]
    valid = [i not in lost for i in range(n)]
    m = par2.Galois16RecMatrix()
    used = list(exps)
    assert m.Compute(valid, n - len(lost), used)
    inputs = np.concatenate([data[[i for i in range(n) if valid[i]]], rec[[exps.index(e) for e in used]]])
    srv = Server(hbm_budget_bytes=1 << 30)
    out = _pinned(np.zeros((len(lost), sb), dtype=np.uint8))
    assert srv.wait(srv.submit(B.gf16_muladd_job(_pinned(inputs), m.factors, out))) == 0
    assert np.array_equal(_np(out), data[lost])
    srv.close()


def test_large_par3_create_among_concurrent_lanes():
    """A 283 MB PAR3 create (3,975 blocks of 71,344 bytes, R=413: the last
    word tile is partial) submitted with 20 other jobs to 8 lanes: every
    result equals the single-job entry points.  Each wave's staging buffers
    must stay reserved until the wave has completed; returned to the pool in
    stream order right after the issue, the large job's last tiles read bytes
    another lane had staged meanwhile."""
    import torch
    from parparpar_b200 import batch as B
    from parparpar_b200 import par2, par3
    from parparpar_b200.server import Server
    rng = np.random.default_rng(34)
    g = torch.Generator(device="cuda").manual_seed(34)

    def pinned_random(shape, dtype):
        t = torch.empty(shape, dtype=dtype).pin_memory()
        n = int(np.prod(shape)) * t.element_size()
        t.view(-1).view(torch.uint8).copy_(torch.randint(0, 256, (n,), dtype=torch.uint8, device="cuda",
                                                         generator=g))
        return t

    jobs = [("par3", pinned_random((3975, 71344 // 8), torch.int64), 413)]
    for k in range(20):
        if k % 2:
            n, sb, r = int(rng.integers(200, 2000)), int(rng.integers(4, 64)) * 1024, int(rng.integers(4, 200))
            jobs.append(("par2", pinned_random((n, sb), torch.uint8), r))
        else:
            n, words, r = int(rng.integers(100, 2000)), int(rng.integers(64, 4096)), int(rng.integers(4, 300))
            jobs.append(("par3", pinned_random((n, words), torch.int64), r))
    ctx = par3._ctx(None)

    def out_of(kind, inp, r):
        return torch.zeros((r, inp.shape[1]), dtype=inp.dtype).pin_memory()

    plain = []
    for kind, inp, r in jobs:
        o = out_of(kind, inp, r)
        if kind == "par2":
            par2.par2_create(inp, np.arange(inp.shape[0]), np.arange(r, dtype=np.uint16), out=o, ctx=ctx)
        else:
            par3.GF64Controller.ctx = ctx
            par3.GF64Controller.ComputeRecoveryBlocks(inp, inp.shape[0], o, r, inp.shape[1], 0, inp.shape[0])
        ctx.synchronize()
        plain.append(o)
    for rep in range(2):
        srv = Server(hbm_budget_bytes=120 * 10**9, max_jobs_per_wave=2, lanes=8)
        outs = [out_of(*j) for j in jobs]
        tickets = []
        for (kind, inp, r), o in zip(jobs, outs):
            job = (B.par2_create_job(inp, np.arange(r, dtype=np.uint16), o) if kind == "par2"
                   else B.par3_create_job(inp, o, 0, inp.shape[0]))
            tickets.append(srv.submit(job))
        assert [srv.wait(t) for t in tickets] == [0] * len(jobs)
        srv.close()
        bad = [i for i in range(len(jobs)) if not torch.equal(plain[i], outs[i])]
        assert not bad, (rep, bad)
