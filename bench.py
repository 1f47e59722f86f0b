"""Benchmark: create/repair input GB/s on one B200, with the HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Default workload (one step = one pass of the hot path over one job):
  PAR2 create at scale, 32,768 input slices x 32 KiB (1 GiB) of seeded random
  bytes, GF(2^16), 64 recovery slices with exponents 0..63.  Inputs are larger
  than L2 (126 MB), so no L2 flush is needed between steps.
Secondary lines (rank 0, a few steps each): PAR2 1,024 x 1 MiB R=8, PAR2
plain 256 x 64 KiB R=8, PAR3 create 131,072 x 8 KiB R=8.

JSON fields (one line on rank 0):
  value          input GB/s with inputs resident in HBM (device-timed, CUDA
                 events on the launching stream, max over ranks)
  e2e            the same metric through the public API with pinned HOST
                 buffers: H2D of the inputs and D2H of the recovery slices
                 inside the timed region
  roofline       the dominant kernel (region multiply-accumulate): algorithmic
                 bytes (inputs read once + outputs written once) per launch /
                 average launch time, against MEASURED_PEAKS.json hbm_gbs
  cpu_baseline   the reference's own CPU code (oracle/_ref, compiled from its
                 sources) on a bounded sample of the same workload
Multi-GPU (torchrun): every rank runs its own job on its own GPU (weak
scaling, no data-path collective); value = all ranks' input bytes / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GIB = 1 << 30


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def int8_peak_tops(dev):
    """Dense int8 tensor throughput measured here: cuBLASLt int8 GEMM
    (torch._int_mm, 8192^3, 2 ops per MAC), best of 10 after warm-up."""
    import torch
    try:
        a = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device=f"cuda:{dev}")
        b = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device=f"cuda:{dev}")
        for _ in range(3):
            torch._int_mm(a, b)
        best = 1e30
        for _ in range(10):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2 * 8192**3 / (best * 1e-3) / 1e12
    except Exception:
        return None


def bit_macs(w):
    """GF(2) multiply-accumulates of a create: every (input word, output)
    pair is a 16x16 (GF(2^16)) or 64x64 (GF(2^64)) bit-matrix product; the
    tensor-core kernels run exactly these as int8 MACs."""
    if w["field"] in ("gf16", "gf16_repair"):  # PAR2 repair: the decode product over all N sources
        return (w["n"] * w["s"] // 2) * w["r"] * 256
    if w["field"] == "gf64":
        return (w["n"] * w["s"] // 8) * w["r"] * 4096
    n_known = w["n"] - w["r"]  # repair: the known-input sum dominates
    return (n_known * w["s"] // 8) * w["r"] * 4096


def roofline(w, args, hbm_achieved, hbm_peak, peak_kind, kms, int8_tops):
    """Roofline of the dominant kernel.  The tensor-core kernels compute each
    GF product as a dense GF(2) bit-matrix contraction in FP4 or int8 MMAs,
    so their binding unit is the tensor pipe: achieved = 2 x bit-MACs /
    kernel time against the FP4 or int8 dense rate (tensor_peak); the HBM
    view of the same launch (algorithmic bytes / time against
    MEASURED_PEAKS.json) is given beside it."""
    kern = dominant_kernel(w, args)
    hbm = {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_achieved / hbm_peak,
           "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
           else "fallback 6.65 TB/s"}
    r = {"kernel": kern, "kernel_ms": kms, "traffic": load_traffic(f"{kern}.{args.workload}")}
    if kern.endswith(("_tc", "_tc_pair", "_f4", "_f4_pair")):
        tops = 2 * bit_macs(w) / (kms * 1e-3) / 1e12
        peak, kind, nominal, nominal_kind = tensor_peak(kern, int8_tops)
        fmt = "FP4 (e2m1 with block scales, exact counts)" if "_f4" in kern else "int8"
        r.update({"bound": "tensor", "achieved": tops, "peak": peak, "unit": "TFLOP/s", "frac": tops / peak,
                  "peak_kind": kind, "ops": f"{fmt} tensor ops (2 per MAC), one MAC per GF(2) bit product",
                  "nominal_peak": nominal, "frac_of_nominal": tops / nominal, "nominal_kind": nominal_kind,
                  "hbm": hbm})
    else:
        r.update({"bound": "hbm", "achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                  "frac": hbm_achieved / hbm_peak, "peak_kind": hbm["peak_kind"]})
    return r


def load_bf16_peak():
    """(dense bf16 TFLOP/s, source): the measured burst figure of
    MEASURED_PEAKS.json, else the fallback 1,590 TFLOP/s."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = json.load(f).get("bf16_tflops")
        if v:
            return float(v), "MEASURED_PEAKS.json bf16_tflops"
    except Exception:
        pass
    return 1590.0, "fallback bf16 1,590 TFLOP/s"


# DRAM bytes (read + write) per launch of the dominant kernel, from the ncu
# captures summarised in profiles/ (the file named after kernel and workload)
TRAFFIC = {
    # the 8,192-slice capture (543.1 + 9.5 MB) scaled to the 32,768-slice launch
    "k_gf16_muladd_tc.par2_create_32768x32KiB_R64": 4 * (543139328 + 9490176),
    "k_gf16_muladd_tc.par2_create_1024x1MiB_R8": 1087907000 + 10907904,
    "k_gf64_matvec_tc.par3_create_131072x8KiB_R8": 1083011000 + 3985664,
    # FP4 GF(2^16) kernel (input rows by tensor-map boxes): the 8,192-slice R=64
    # capture (404.9 + 4.8 MB) and the 256 x 1 MiB R=8 capture (268.8 + 8.8 MB),
    # each scaled by 4 to the 1 GiB launch
    "k_gf16_muladd_f4.par2_create_32768x32KiB_R64": 4 * (404915712 + 4844544),
    "k_gf16_muladd_f4.par2_create_1024x1MiB_R8": 4 * (268810240 + 8846336),
    # the SM-pair kernels' 32,768-block captures scaled to 131,072 blocks: int8
    # (270.8 + 4.3 MB), FP4 (270.8 + 5.4 MB; the input read once, as for int8)
    "k_gf64_matvec_tc_pair.par3_create_131072x8KiB_R8": 4 * (270800000 + 4300000),
    "k_gf64_matvec_f4_pair.par3_create_131072x8KiB_R8": 4 * (270786304 + 5406464),
}


def load_traffic(name):
    return TRAFFIC.get(name)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.lines = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={gpu_id}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t_end = time.time() + 3.0
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


def gpu_uuid(dev: int) -> str:
    import torch
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev)


# ------------------------------------------------------------------ workloads
WORKLOADS = {
    "par2_create_32768x32KiB_R64": dict(field="gf16", n=32768, s=32 * 1024, r=64),
    "par2_create_1024x1MiB_R8": dict(field="gf16", n=1024, s=1 << 20, r=8),
    "par2_create_256x64KiB_R8": dict(field="gf16", n=256, s=64 * 1024, r=8),
    "par3_create_131072x8KiB_R8": dict(field="gf64", n=131072, s=8 * 1024, r=8),
    "par3_create_131072x8KiB_R1024": dict(field="gf64", n=131072, s=8 * 1024, r=1024),
    # 1 % of 262,144 blocks lost, solved from the first 2,621 of R=4,096 recovery blocks
    "par3_repair_262144x4KiB_R4096_1pct": dict(field="gf64_repair", n=262144, s=4 * 1024, r=2621),
    # forward additive FFT of the same 1 GiB: 1,024 word columns of 131,072 coefficients
    "par3_fft_fwd_131072x8KiB": dict(field="fft", n=131072, s=8 * 1024, r=0),
    # PAR2 repair: 64 of 32,768 slices lost, restored from the R=64 recovery slices
    "par2_repair_32768x32KiB_R64_lost64": dict(field="gf16_repair", n=32768, s=32 * 1024, r=64),
    # block hashes over 1 GiB of resident slices / blocks
    "par2_hash_32768x32KiB": dict(field="hash2", n=32768, s=32 * 1024, r=0),
    "par3_hash_131072x8KiB": dict(field="hash3", n=131072, s=8 * 1024, r=0),
    "par3_packets_131072x8KiB": dict(field="pkt3", n=131072, s=8 * 1024, r=0),
}
HASH_FIELDS = ("hash2", "hash3", "pkt3")
PAR3_AFTER = bytes(range(24))      # a data packet's post-checksum header bytes (synthetic)
PAR3_SET_ID = b"\x5a" * 8           # input-set id (synthetic)
PRIMARY = "par2_create_32768x32KiB_R64"


class Timer:
    """CUDA-event timing on the stream the library launches on."""

    def __init__(self, stream):
        import torch
        self.torch = torch
        self.stream = stream

    def run(self, fn, steps):
        torch = self.torch
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(self.stream)
        for _ in range(steps):
            fn()
        b.record(self.stream)
        b.synchronize()
        return a.elapsed_time(b) / steps  # ms


def setup_job(name, dev, seed, ctx):
    import torch
    from parparpar_b200 import par2
    w = WORKLOADS[name]
    g = torch.Generator(device=f"cuda:{dev}")
    g.manual_seed(seed)
    job = dict(w)
    if w["field"] == "gf16_repair":
        # the decode's sources: the valid inputs then the recovery slices (the
        # recovery contents do not change the work); the lost set is seeded
        n, m = w["n"], w["r"]
        lost = np.sort(np.random.default_rng(seed).choice(n, m, replace=False))
        valid = np.ones(n, dtype=bool)
        valid[lost] = False
        srcs = torch.randint(0, 256, (n, w["s"]), dtype=torch.uint8, device=f"cuda:{dev}", generator=g)
        job.update(d_in=srcs, valid=valid, exps=list(range(m)),
                   d_fac=torch.zeros((m, n), dtype=torch.int16, device=f"cuda:{dev}"),
                   d_out=torch.zeros((m, w["s"]), dtype=torch.uint8, device=f"cuda:{dev}"))
        return job
    if w["field"] in HASH_FIELDS:
        d_in = torch.randint(0, 256, (w["n"], w["s"]), dtype=torch.uint8, device=f"cuda:{dev}", generator=g)
        out_bytes = {"hash2": 20, "hash3": 16, "pkt3": 64 + w["s"]}[w["field"]]
        d_out = torch.zeros((w["n"], out_bytes), dtype=torch.uint8, device=f"cuda:{dev}")
        job.update(d_in=d_in, d_out=d_out)
    elif w["field"] == "gf16":
        d_in = torch.randint(0, 256, (w["n"], w["s"]), dtype=torch.uint8, device=f"cuda:{dev}", generator=g)
        d_out = torch.zeros((w["r"], w["s"]), dtype=torch.uint8, device=f"cuda:{dev}")
        idx = np.arange(w["n"], dtype=np.uint16)
        exps = np.arange(w["r"], dtype=np.uint16)
        coeffs = torch.from_numpy(par2.coeff_matrix(idx, exps, ctx=ctx)).to(f"cuda:{dev}")
        job.update(d_in=d_in, d_out=d_out, idx=idx, exps=exps, coeffs=coeffs)
    else:
        words = w["s"] // 8
        d_in = torch.randint(-2**63, 2**63 - 1, (w["n"], words), dtype=torch.int64, device=f"cuda:{dev}",
                             generator=g)
        d_out = torch.zeros((w["r"], words), dtype=torch.int64, device=f"cuda:{dev}")
        job.update(d_in=d_in, d_out=d_out, words=words)
        if w["field"] == "gf64_repair":
            # seeded erasure pattern; the recovery rows' content does not change the work
            lost = np.sort(np.random.default_rng(seed).choice(w["n"], w["r"], replace=False)).astype(np.uint64)
            d_rec = torch.randint(-2**63, 2**63 - 1, (w["r"], words), dtype=torch.int64, device=f"cuda:{dev}",
                                  generator=g)
            job.update(lost=lost, d_rec=d_rec)
    return job


def step_fn(job, ctx):
    from parparpar_b200 import par2, par3
    if job["field"] == "gf16":
        return lambda: par2.par2_create(job["d_in"], job["idx"], job["exps"], out=job["d_out"], ctx=ctx)
    if job["field"] == "gf16_repair":
        return lambda: par2_repair_step(job, ctx)
    if job["field"] in HASH_FIELDS:
        return hash_fn(job, job["d_in"], job["d_out"], ctx)
    par3.GF64Controller.ctx = ctx
    if job["field"] == "fft":  # in place; each step transforms the previous result
        return lambda: par3.gf64_addfft64_fwd(job["d_in"], job["n"], job["words"], job["words"], ctx=ctx)
    if job["field"] == "gf64_repair":
        return lambda: par3.repair(job["d_in"], job["lost"], job["d_rec"], job["words"], 0, job["n"],
                                   restored=job["d_out"], ctx=ctx)
    return lambda: par3.GF64Controller.ComputeRecoveryBlocks(job["d_in"], job["n"], job["d_out"], job["r"],
                                                             job["words"], 0, job["n"])


def par2_repair_step(job, ctx):
    """Galois16RecMatrix inversion (factors on the device) + the decode product."""
    from parparpar_b200 import par2
    m = par2.Galois16RecMatrix(ctx=ctx)
    used = list(job["exps"])
    if not m.Compute(job["valid"], int(job["valid"].sum()), used, out=job["d_fac"]):
        raise RuntimeError("PAR2 repair matrix not invertible")
    par2.gf16_muladd(job["d_in"], job["d_fac"], out=job["d_out"], ctx=ctx)


def dtype_of(w):
    """Arithmetic type of the path: GF(2^16) symbols, GF(2^64) words, or the
    32-bit words of MD5 / CRC32 / BLAKE3."""
    return {"gf16": "u16", "gf16_repair": "u16"}.get(w["field"], "u32" if w["field"] in HASH_FIELDS else "u64")


def hash_fn(job, src, dst, ctx):
    from parparpar_b200 import par2, par3
    n, s = job["n"], job["s"]
    if job["field"] == "hash2":
        return lambda: par2.block_hashes(src, s, out=dst, ctx=ctx)
    if job["field"] == "hash3":
        return lambda: par3.block_hashes(src, s, 0, PAR3_AFTER, num_blocks=n, out=dst, ctx=ctx)
    return lambda: par3.assemble_recovery_packets(src.reshape(-1), PAR3_SET_ID, n, n, s, out=dst.reshape(-1),
                                                  ctx=ctx)


def kernel_fn(job, ctx):
    """The dominant kernel alone: after the first call the coefficient table
    (PAR2 tiles / PAR3 Cauchy matrix) is resident, so a step is the region
    kernel (plus, when the job is split over CTAs, a memset of the outputs).
    PAR2 repair: the decode product with the factors of one inversion."""
    if job["field"] == "gf16_repair":
        from parparpar_b200 import par2
        par2_repair_step(job, ctx)
        return lambda: par2.gf16_muladd(job["d_in"], job["d_fac"], out=job["d_out"], ctx=ctx)
    return step_fn(job, ctx)


def dominant_kernel(w, args):
    """Name of the region kernel the library's dispatch picks for this workload
    (AUTO: tensor cores for >= 8 GF(2^16) inputs, and for 16-byte aligned
    GF(2^64) rows of an even word count)."""
    gf16_tc = "k_gf16_muladd_tc" if os.environ.get("PARPAR_B200_GF16_TC") == "i8" else "k_gf16_muladd_f4"
    if w["field"] == "gf16":
        return "k_gf16_muladd_lut" if args.gf16_kernel == "lut" else gf16_tc
    if w["field"] == "fft":
        return "k_fft_*"
    if w["field"] == "gf16_repair":
        return gf16_tc
    if w["field"] == "hash2":
        return "k_par2_block_hash"
    if w["field"] in ("hash3", "pkt3"):
        return "k_b3_chunks"
    if args.gf64_kernel == "lut":
        return "k_gf64_matvec_lut"
    # the SM-pair kernel runs when every job of the launch has >= 4 outputs;
    # FP4 on SM pairs, int8 on one CTA, unless PARPAR_B200_GF64_TC fixes one
    pair = w["r"] >= 4
    fmt = os.environ.get("PARPAR_B200_GF64_TC")
    f4 = fmt == "f4" or (fmt != "i8" and pair)
    if f4:
        return "k_gf64_matvec_f4_pair" if pair else "k_gf64_matvec_f4"
    return "k_gf64_matvec_tc_pair" if pair else "k_gf64_matvec_tc"


def tensor_peak(kern, int8_tops):
    """(peak TOP/s, how it was obtained, nominal, nominal's source) for a
    tensor-core region kernel: the FP4 kernels against 4 x the measured dense
    bf16 GEMM rate (B200's dense FP4 rate is 4x its bf16 rate), the int8
    kernels against the cuBLASLt int8 GEMM measured in this run (else 2 x
    bf16)."""
    bf16, src = load_bf16_peak()
    if "_f4" in kern:
        return (4 * bf16, f"4 x {src} (dense FP4 rate = 4x bf16)", 9000.0,
                "B200 dense FP4 tensor rate (NVIDIA's 9 PFLOP/s dense figure)")
    if int8_tops:
        peak, kind = int8_tops, "measured here: cuBLASLt dense int8 GEMM 8192^3 (torch._int_mm), best of 10"
    else:
        peak, kind = 2 * bf16, f"2 x {src} (int8 dense rate = 2x bf16)"
    return peak, kind, 4500.0, "B200 dense int8 tensor rate (NVIDIA's 4.5 POP/s dense figure)"


def algo_bytes(job):
    if job["field"] == "fft":  # the data read and written once
        return 2 * job["n"] * job["s"]
    if job["field"] == "hash2":  # slices read, 20-byte entries written
        return job["n"] * (job["s"] + 20)
    if job["field"] == "hash3":
        return job["n"] * (job["s"] + 16)
    if job["field"] == "pkt3":  # blocks read, packets written
        return job["n"] * (2 * job["s"] + 64)
    if job["field"] in ("gf64_repair", "gf16_repair"):  # (N - n) known + n recovery read, n written
        return (job["n"] + job["r"]) * job["s"]
    return (job["n"] + job["r"]) * job["s"]


def input_bytes_of(name):
    w = WORKLOADS[name]
    return w["n"] * w["s"]  # create: the input slices; repair: known blocks + recovery blocks (N*S)


def timed_steps(ctx, timer, f, steps):
    """Time `steps` calls of f with CUDA events on the launching stream and,
    in the same calls, the device time of the region products the library
    brackets with its own events (pp_ctx_set_kernel_timing).  Returns
    (ms per step, region ms per launch or None, region launches, library
    launches)."""
    import parparpar_b200 as pp
    ctx.kernel_time()  # drop earlier brackets
    ctx.set_kernel_timing(True)
    l0 = pp.launch_count()
    ms = timer.run(f, steps)
    launches = pp.launch_count() - l0
    ctx.set_kernel_timing(False)
    kt, kn = ctx.kernel_time()
    return ms, (kt / kn if kn else None), kn, launches


def kernel_ms_of(job, ctx, timer, steps, kms):
    """The dominant kernel's time per launch: the library's own brackets in
    the timed steps when it made any, else (block hashes, FFT) the step's
    kernel timed alone."""
    if kms is not None:
        return kms, "CUDA events around each region product inside the timed steps"
    kf = kernel_fn(job, ctx)
    kf()
    return timer.run(kf, max(3, min(steps, 20))), "the kernel's call timed alone after the timed steps"


def measure(job, ctx, timer, steps, warmup, peak):
    f = step_fn(job, ctx)
    for _ in range(warmup):
        f()
    ctx.synchronize()
    ms, kms, _, launches = timed_steps(ctx, timer, f, steps)
    kms, _ = kernel_ms_of(job, ctx, timer, steps, kms)
    achieved = algo_bytes(job) / (kms * 1e-3) / 1e9
    return dict(ms=ms, launches=launches, kernel_ms=kms, achieved=achieved, frac=achieved / peak)


def host_isa():
    """CPU model and the SIMD extensions the reference's kernels pick from."""
    model, flags = "", set()
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name") and not model:
                    model = ln.split(":", 1)[1].strip()
                elif ln.startswith("flags") and not flags:
                    flags = set(ln.split(":", 1)[1].split())
    except OSError:
        pass
    ext = [x for x in ("avx2", "avx512f", "avx512bw", "avx512vl", "avx512vbmi", "gfni", "vpclmulqdq", "pclmulqdq")
           if x in flags]
    return f"{model}; {' '.join(ext)}".strip("; ")


_SAMPLE_INPUTS = {}


def cpu_baseline_sample(name, budget_s=12.0, threads=0, full=False):
    """Reference CPU code on a bounded sample of the workload: every slice,
    a contiguous byte sub-range of each (cost is linear in the slice length),
    or with full=True (PAR2 create) the whole job once."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    w = WORKLOADS[name]
    rng = np.random.default_rng(99)
    cores = os.cpu_count() or 1
    if w["field"] in HASH_FIELDS:
        # one thread: the reference hashes each file / packet batch on one thread
        sub_n = {"hash2": 256, "hash3": 1024, "pkt3": 1024}[w["field"]]
        inp = rng.integers(0, 256, (sub_n, w["s"]), dtype=np.uint8)
        nbytes = inp.nbytes
        if orc.Reference.available():
            R, kind = orc.Reference(), "reference"
        else:
            orc.build()
            R, kind = orc.Oracle(), "port"
        if w["field"] == "hash2":
            if kind == "reference":
                run = lambda: R.par2_hash_file(inp.reshape(-1), w["s"])
                what = (f"HasherInput_{R.par2_hasher_method()} (the variant the reference selects on this CPU; "
                        "block MD5+CRC32 and the file MD5 lane)")
            else:
                run = lambda: orc.par2_block_hashes(inp, w["s"])
                what = "hashlib MD5 + zlib CRC32"
        elif w["field"] == "hash3":
            run = lambda: R.par3_block_hashes(inp, 0, bytes(range(24)))
            what = "BLAKE3 per block (hasher/hasher_blake3.c)" if kind == "reference" else "oracle BLAKE3"
        else:
            run = lambda: R.par3_recovery_packets(inp, b"\x5a" * 8, 0)
            what = ("assemble_recovery_packets loop around the reference BLAKE3" if kind == "reference"
                    else "oracle packet assembly")
        sample = f"{sub_n} x {w['s']} B of the workload's {w['n']} blocks; {what}; 1 thread"
        cores = 1
    elif w["field"] == "gf16_repair" and orc.Reference.available():
        # the reference's Galois16RecMatrix inversion + its coefficient-driven
        # PAR2 controller decode over a 2,048-byte sub-range of every source
        R, kind, cores = orc.Reference(), "reference", os.cpu_count() or 1
        sub = 2048
        inp = rng.integers(0, 256, (w["n"], sub), dtype=np.uint8)
        lost = np.sort(rng.choice(w["n"], w["r"], replace=False))
        valid = np.ones(w["n"], dtype=np.uint8)
        valid[lost] = 0

        # the inversion's cost does not depend on the slice length, the
        # decode's is linear in it: time both, scale the decode to full slices
        t0 = time.perf_counter()
        ok, f, used = R.par2_invert(valid, list(range(w["r"])), threads=threads)
        t_inv = time.perf_counter() - t0
        t0 = time.perf_counter()
        R.par2_create_coeffs(inp, sub, f, threads=threads)
        t_dec = time.perf_counter() - t0
        t_full = t_inv + t_dec * (w["s"] / sub)
        sample = (f"inversion ({w['r']} lost of {w['n']}, {t_inv:.2f} s) + decode of {w['n']} sources x {sub} B "
                  f"(a {sub}-byte sub-range of every slice, {t_dec:.3f} s, scaled x{w['s'] // sub} to the slices)")
        return dict(value=w["n"] * w["s"] / t_full / 1e9, unit="GB/s", cores=cores, kind=kind, sample=sample,
                    seconds_per_run=t_full, runs=1)
    elif orc.Reference.available():
        R = orc.Reference()
        kind = "reference"
        if w["field"] == "gf16":
            sub = w["s"] if full else min(2048, w["s"])
            key = (w["n"], sub)
            if key not in _SAMPLE_INPUTS:  # generated once per process (1 GiB for the whole job)
                _SAMPLE_INPUTS.clear()
                _SAMPLE_INPUTS[key] = rng.integers(0, 256, (w["n"], sub), dtype=np.uint8)
            inp = _SAMPLE_INPUTS[key]
            run = lambda: R.par2_create(inp, sub, np.arange(w["n"]), list(range(w["r"])), threads=threads)
            sample = (f"the whole job: {w['n']} slices x {sub} B, R={w['r']}" if sub == w["s"] else
                      f"{w['n']} slices x {sub} B (a {sub}-byte sub-range of every slice), R={w['r']}")
            if full:
                budget_s = 0.0  # one run of the whole job
            nbytes = inp.nbytes
        else:
            # the whole job where it takes seconds (R <= 64); a sub-range of
            # every block otherwise (cost is linear in the block length)
            sub = w["s"] if (full and w["r"] <= 64) else 256
            key = ("gf64", w["n"], sub)
            if key not in _SAMPLE_INPUTS:
                _SAMPLE_INPUTS.clear()
                _SAMPLE_INPUTS[key] = rng.integers(0, 2**64, (w["n"], sub // 8), dtype=np.uint64)
            inp = _SAMPLE_INPUTS[key]
            run = lambda: R.gf64_compute_recovery(0, inp, w["r"], 0, w["n"], threads=threads)
            sample = (f"the whole job: {w['n']} blocks x {sub} B, R={w['r']}" if sub == w["s"] else
                      f"{w['n']} blocks x {sub} B (a {sub}-byte sub-range of every block), R={w['r']}")
            if sub == w["s"]:
                budget_s = 0.0
            nbytes = inp.nbytes
    else:
        orc.build()
        O = orc.Oracle()
        kind = "port"
        cores = 1
        sub = 64
        n = min(w["n"], 4096)
        if w["field"] == "gf16":
            inp = rng.integers(0, 256, (n, sub), dtype=np.uint8)
            co = O.par2_coeff_matrix(np.arange(n), list(range(w["r"])))
            run = lambda: O.par2_muladd(list(inp), sub, co)
        else:
            inp = rng.integers(0, 2**64, (n, sub // 8), dtype=np.uint64)
            run = lambda: O.gf64_compute_recovery(inp, w["r"], 0, n)
        sample = f"{n} slices x {sub} B, R={w['r']} (oracle C port, 1 thread)"
        nbytes = inp.nbytes
    times = []
    t_end = time.time() + budget_s
    while True:
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
        if time.time() > t_end or len(times) >= 5:
            break
    t = statistics.median(times)
    out = dict(value=nbytes / t / 1e9, unit="GB/s", cores=cores, kind=kind, sample=sample,
               seconds_per_run=t, runs=len(times), host=host_isa())
    if kind == "reference" and w["field"] == "gf16":
        out["method"] = R.par2_method()  # PAR2ProcCPU::getMethodName() of the GF16_AUTO choice
    return out


def batched_repair_jobs(dev, seed=2024, count=16):
    """16 PAR3 repair jobs of uneven sizes: input 64 MiB-1 GiB and block size
    4-64 KiB, both log-uniform (seeded), 1 % of the blocks lost, recovery
    rows fR = N onwards.  Inputs and recovery rows are seeded random device
    data (the work does not depend on their values)."""
    import torch
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=f"cuda:{dev}")
    g.manual_seed(seed)
    jobs = []
    for _ in range(count):
        size = int(2 ** rng.uniform(26, 30))
        sl = int(2 ** rng.uniform(12, 16)) // 16 * 16
        N = size // sl
        n = max(1, round(0.01 * N))
        words = sl // 8
        d_in = torch.randint(-2**63, 2**63 - 1, (N, words), dtype=torch.int64, device=f"cuda:{dev}", generator=g)
        d_rec = torch.randint(-2**63, 2**63 - 1, (n, words), dtype=torch.int64, device=f"cuda:{dev}", generator=g)
        lost = np.sort(rng.choice(N, n, replace=False)).astype(np.uint64)
        jobs.append(dict(N=N, n=n, words=words, d_in=d_in, d_rec=d_rec, lost=lost))
    return jobs


def measure_batched_vs_plain(ctx, timer, steps, warmup, dev):
    """The same 16 repair jobs run (a) one after another through the
    single-job call par3.repair and (b) as one batch plan replayed from its
    CUDA graph; both timed with CUDA events on the library's stream, outputs
    compared bit for bit."""
    import torch
    from parparpar_b200 import batch as B
    from parparpar_b200 import par3
    jobs = batched_repair_jobs(dev)
    in_bytes = sum(j["N"] * j["words"] * 8 for j in jobs)
    plain_out = [torch.zeros((j["n"], j["words"]), dtype=torch.int64, device=f"cuda:{dev}") for j in jobs]
    batch_out = [torch.zeros_like(o) for o in plain_out]

    def plain():
        for j, o in zip(jobs, plain_out):
            par3.repair(j["d_in"], j["lost"], j["d_rec"], j["words"], 0, j["N"], restored=o, ctx=ctx)

    for _ in range(max(1, warmup - 1)):
        plain()
    plain_ms = timer.run(plain, steps)

    def jobs_of(outs):
        return [B.par3_repair_job(j["d_in"], j["lost"], j["d_rec"], o) for j, o in zip(jobs, outs)]

    # jobs seen once: a fresh plan for this set of erasures (every repair
    # system's inverse and tables, no graph) plus its one run, wall clock
    # around synchronised calls -- the same work as one plain pass
    once = []
    for _ in range(max(1, steps)):
        ctx.synchronize()
        t0 = time.perf_counter()
        bo = B.Batch(jobs_of(batch_out), graph=False, ctx=ctx)
        bo.run()
        ctx.synchronize()
        once.append((time.perf_counter() - t0) * 1e3)
        bo.close()
    incl_create_ms = statistics.median(once)
    # a resident plan (tuned once, replayed from its CUDA graph)
    t0 = time.perf_counter()
    b = B.Batch(jobs_of(batch_out), tune=True, ctx=ctx)
    ctx.synchronize()
    create_s = time.perf_counter() - t0
    for _ in range(warmup):
        b.run()
    batch_ms = timer.run(b.run, steps)
    ctx.synchronize()
    same = all(torch.equal(a, c) for a, c in zip(plain_out, batch_out))
    launches = b.launches
    b.close()
    del jobs, plain_out, batch_out
    torch.cuda.empty_cache()
    return {"workload": "par3_repair_batch16_uneven_64MiB-1GiB_4-64KiB_1pct", "unit": "GB/s",
            "input_bytes": in_bytes,
            "plain_value": in_bytes / (plain_ms * 1e-3) / 1e9, "plain_ms": plain_ms,
            # equal work: plan creation (inverses, tables, capture) + one run, for jobs seen once
            "batched_incl_create_value": in_bytes / (incl_create_ms * 1e-3) / 1e9,
            "batched_incl_create_ms": incl_create_ms,
            "batched_incl_create_over_plain": plain_ms / incl_create_ms,
            # resident plan: graph replay of a plan built (and tuned) beforehand
            "resident_plan_value": in_bytes / (batch_ms * 1e-3) / 1e9, "resident_plan_ms": batch_ms,
            "resident_plan_over_plain": plain_ms / batch_ms, "resident_plan_create_s_tuned": create_s,
            "batch_graph_launches": launches, "outputs_identical": bool(same)}


def serving_jobs(dev, seed=5, count=32):
    """Mixed stream: PAR2 / PAR3 create and repair, input size log-uniform
    1 MiB-1 GiB, slice size log-uniform 4 KiB-1 MiB, R uniform 4-512 for
    creates, 1 % of the slices lost for repairs (at least one).  PAR2 slices
    are raised so that N <= 32768 and rounded to even bytes, PAR3 blocks to
    16 bytes.  Data is seeded random bytes in pinned host memory (the PAR2
    repair decode coefficients and the recovery rows are random: the work
    does not depend on their values)."""
    import torch
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=f"cuda:{dev}")
    g.manual_seed(seed)

    def pinned(shape, dtype):
        t = torch.empty(shape, dtype=dtype).pin_memory()
        lo, hi = (0, 256) if dtype == torch.uint8 else (-2**63, 2**63 - 1)
        rows = max(1, (256 << 20) // max(1, t[0].numel() * t.element_size()))
        for r0 in range(0, shape[0], rows):  # generate on the device in chunks
            r1 = min(shape[0], r0 + rows)
            t[r0:r1].copy_(torch.randint(lo, hi, (r1 - r0,) + tuple(shape[1:]), dtype=dtype,
                                         device=f"cuda:{dev}", generator=g))
        return t

    jobs = []
    for _ in range(count):
        kind = str(rng.choice(["par2_create", "par2_repair", "par3_create", "par3_repair"]))
        size = int(2 ** rng.uniform(20, 30))
        sl = int(2 ** rng.uniform(12, 20))
        R = int(rng.integers(4, 513))
        if kind.startswith("par2"):
            sl = max(sl, -(-size // 32768))
            sl = (sl + 1) // 2 * 2
            N = max(1, size // sl)
            inp = pinned((N, sl), torch.uint8)
            if kind == "par2_create":
                jobs.append(dict(kind=kind, N=N, sl=sl, R=R, inp=inp, exps=np.arange(R, dtype=np.uint16)))
            else:
                m = max(1, round(0.01 * N))
                co = rng.integers(1, 65536, (m, N), dtype=np.uint16)
                jobs.append(dict(kind=kind, N=N, sl=sl, R=m, inp=inp, coeffs=co))
        else:
            sl = max(16, sl // 16 * 16)
            N = max(1, size // sl)
            inp = pinned((N, sl // 8), torch.int64)
            if kind == "par3_create":
                jobs.append(dict(kind=kind, N=N, sl=sl, R=R, inp=inp))
            else:
                n = max(1, round(0.01 * N))
                lost = np.sort(rng.choice(N, n, replace=False)).astype(np.uint64)
                jobs.append(dict(kind=kind, N=N, sl=sl, R=n, inp=inp, lost=lost, rec=pinned((n, sl // 8), torch.int64)))
    return jobs


def measure_serving(ctx, dev, count=32, seed=5, budget=120 * 10**9):
    """The mixed job stream (a) run one job at a time through the single-job
    calls with the same host buffers, wall clock, and (b) submitted to the
    serving loop with Poisson arrivals at twice the plain service rate;
    outputs compared bit for bit."""
    import torch
    from parparpar_b200 import batch as B
    from parparpar_b200 import par2, par3
    from parparpar_b200.server import Server
    jobs = serving_jobs(dev, seed, count)
    in_bytes = sum(j["N"] * j["sl"] for j in jobs)

    def out_of(j):
        w = j["sl"] if j["kind"].startswith("par2") else j["sl"] // 8
        dt = torch.uint8 if j["kind"].startswith("par2") else torch.int64
        return torch.zeros((j["R"], w), dtype=dt).pin_memory()

    plain_out = [out_of(j) for j in jobs]

    def run_plain(j, o):
        k = j["kind"]
        if k == "par2_create":
            par2.par2_create(j["inp"], np.arange(j["N"]), j["exps"], out=o, ctx=ctx)
        elif k == "par2_repair":
            par2.gf16_muladd(j["inp"], j["coeffs"], out=o, ctx=ctx)
        elif k == "par3_create":
            par3.GF64Controller.ctx = ctx
            par3.GF64Controller.ComputeRecoveryBlocks(j["inp"], j["N"], o, j["R"], j["sl"] // 8, 0, j["N"])
        else:
            par3.repair(j["inp"], j["lost"], j["rec"], j["sl"] // 8, 0, j["N"], restored=o, ctx=ctx)

    run_plain(jobs[0], plain_out[0])  # warm-up (kernels, tables)
    ctx.synchronize()
    t0 = time.perf_counter()
    plain_lat = []
    for j, o in zip(jobs, plain_out):
        a = time.perf_counter()
        run_plain(j, o)
        ctx.synchronize()
        plain_lat.append((time.perf_counter() - a) * 1e3)
    plain_s = time.perf_counter() - t0

    def job_of(j, o):
        k = j["kind"]
        if k == "par2_create":
            return B.par2_create_job(j["inp"], j["exps"], o)
        if k == "par2_repair":
            return B.gf16_muladd_job(j["inp"], j["coeffs"], o)
        if k == "par3_create":
            return B.par3_create_job(j["inp"], o, 0, j["N"])
        return B.par3_repair_job(j["inp"], j["lost"], j["rec"], o, 0, j["N"])

    # small waves on many lanes: one wave's copies overlap other waves' kernels
    # (a sweep of the 32-job mix: 2 lanes x 24 jobs 18 GB/s, 4 x 4 22 GB/s,
    # 8 x 2 29 GB/s)
    srv = Server(dev, hbm_budget_bytes=budget, max_jobs_per_wave=2, lanes=8)
    srv_out = [out_of(j) for j in jobs]
    srv.wait(srv.submit(job_of(jobs[0], srv_out[0])))  # warm-up
    srv.reset_stats()
    rate = 2.0 * len(jobs) / plain_s  # arrivals per second: twice the plain service rate
    arr = np.cumsum(np.random.default_rng(seed + 1).exponential(1.0 / rate, len(jobs)))
    tickets = []
    t0 = time.perf_counter()
    for j, o, at in zip(jobs, srv_out, arr):
        d = at - (time.perf_counter() - t0)
        if d > 0:
            time.sleep(d)
        tickets.append(srv.submit(job_of(j, o)))
    statuses = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    same = all(torch.equal(a, b) for a, b in zip(plain_out, srv_out)) and all(x == 0 for x in statuses)
    pl = sorted(plain_lat)
    kinds = {}
    for j in jobs:
        kinds[j["kind"]] = kinds.get(j["kind"], 0) + 1
    del jobs, plain_out, srv_out
    return {"workload": f"serving_{count}jobs_mixed_1MiB-1GiB_4KiB-1MiB_R4-512_1pct", "jobs": count,
            "kinds": kinds, "input_bytes": in_bytes, "host_buffers": "pinned", "hbm_budget_bytes": budget,
            "arrivals": f"Poisson, {rate:.1f}/s (twice the plain service rate)",
            "served_gbps": st["gbps"], "served_p50_ms": st["p50_ms"], "served_p99_ms": st["p99_ms"],
            "served_max_ms": st["max_ms"], "served_elapsed_s": st["elapsed_s"], "waves": st["waves"],
            "hbm_peak_bytes": st["hbm_peak_bytes"], "tables_resident": st["tables_resident"],
            "plain_gbps": in_bytes / plain_s / 1e9, "plain_elapsed_s": plain_s,
            "plain_job_p50_ms": pl[len(pl) // 2], "plain_job_p99_ms": pl[min(len(pl) - 1, int(0.99 * len(pl)))],
            "served_over_plain": (in_bytes / max(st["elapsed_s"], 1e-9)) / (in_bytes / plain_s),
            "outputs_identical": bool(same)}


def measure_fenger_estimate(ctx, timer, dev, dense_ms):
    """The Fenger route for PAR3 R=1,024 (131,072 inputs) costed from
    measured device pieces.  Per block word, the reference's interpolation
    (gf64/gf64_fenger.c:524-590) walks the 17 levels of the subproduct tree;
    at level l its 2^l nodes each multiply two polynomial pairs of output
    size n = N / 2^l (the tree polynomials' transforms can be kept, so a
    product is one forward transform, one pointwise product and one inverse
    transform of size n).  Measured here on 1,024 words at once: the additive
    FFT of the 1 GiB array (n = N) and the pointwise GF(2^64) product; a level
    is charged 2 x (2 FFT x log2(n) / log2(N) + pointwise).  The evaluation
    on the 1,024-point tree and the final division are left out, so the
    estimate is a lower bound of the route's device time."""
    import math

    import torch
    from parparpar_b200 import par3
    N, batch = 131072, 1024
    g = torch.Generator(device=f"cuda:{dev}")
    g.manual_seed(17)
    a = torch.randint(-2**63, 2**63 - 1, (N, batch), dtype=torch.int64, device=f"cuda:{dev}", generator=g)
    b = torch.randint(-2**63, 2**63 - 1, (N, batch), dtype=torch.int64, device=f"cuda:{dev}", generator=g)
    torch.cuda.synchronize()
    fft = lambda: par3.gf64_addfft64_fwd(a, N, batch, batch, ctx=ctx)
    pw = lambda: par3.mul_arr(a, a, b, N * batch, N * batch, ctx=ctx)
    fft()
    pw()
    t_fft = timer.run(fft, 3)
    t_pw = timer.run(pw, 3)
    L = int(math.log2(N))
    est = sum(2 * (2 * t_fft * math.log2(N >> lev) / L + t_pw) for lev in range(L))
    del a, b
    torch.cuda.empty_cache()
    return {"workload": "par3_create_131072x8KiB_R1024 via Fenger (estimate)", "fft_ms_1GiB": t_fft,
            "pointwise_ms_1GiB": t_pw, "fenger_interp_lower_bound_ms": est, "dense_tensor_core_ms": dense_ms,
            "fenger_over_dense": est / dense_ms if dense_ms else None}


def measure_fused(ctx, dev):
    """End to end with pinned host inputs (1 GiB): each create with and
    without the hashes of its inputs computed in the same pass, and the PAR3
    streaming create from a 1 GiB file (page cache warm).  Median of 3."""
    import tempfile

    import torch
    from parparpar_b200 import par2, par3

    def med(f, reps=3):
        f()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            f()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts)

    out = {"unit": "GB/s", "host_buffers": "pinned"}
    g = torch.Generator(device=f"cuda:{dev}")
    g.manual_seed(3)
    n, sl, r = 32768, 32768, 64
    h_in = torch.empty((n, sl), dtype=torch.uint8).pin_memory()
    h_in.copy_(torch.randint(0, 256, (n, sl), dtype=torch.uint8, device=f"cuda:{dev}", generator=g))
    h_out = torch.empty((r, sl), dtype=torch.uint8).pin_memory()
    h_hash = torch.empty((n, 20), dtype=torch.uint8).pin_memory()
    idx, exps = np.arange(n), list(range(r))
    t_plain = med(lambda: par2.par2_create(h_in, idx, exps, out=h_out, ctx=ctx))
    t_hash = med(lambda: par2.par2_create(h_in, idx, exps, out=h_out, hashes=h_hash, ctx=ctx))
    out["par2_create_32768x32KiB_R64"] = {"plain": n * sl / t_plain / 1e9, "with_ifsc_hashes": n * sl / t_hash / 1e9}
    # few large slices: the hashed create copies column bands of every slice
    n1, sl1, r1 = 1024, 1 << 20, 8
    x1 = h_in.view(n1, sl1)
    o1 = torch.empty((r1, sl1), dtype=torch.uint8).pin_memory()
    h1 = torch.empty((n1, 20), dtype=torch.uint8).pin_memory()
    t_plain = med(lambda: par2.par2_create(x1, np.arange(n1), list(range(r1)), out=o1, ctx=ctx))
    t_hash = med(lambda: par2.par2_create(x1, np.arange(n1), list(range(r1)), out=o1, hashes=h1, ctx=ctx))
    out["par2_create_1024x1MiB_R8"] = {"plain": n1 * sl1 / t_plain / 1e9, "with_ifsc_hashes": n1 * sl1 / t_hash / 1e9}
    # the PAR3 inputs reuse the same pinned bytes as 131,072 x 8 KiB blocks
    nb, words, R = 131072, 1024, 8
    x = h_in.view(torch.int64).view(nb, words)
    rec = torch.empty((R, words), dtype=torch.int64).pin_memory()
    pk = torch.empty(R * (64 + 8 * words), dtype=torch.uint8).pin_memory()
    dh = torch.empty((nb, 16), dtype=torch.uint8).pin_memory()
    par3.GF64Controller.ctx = ctx
    t_plain = med(lambda: par3.GF64Controller.ComputeRecoveryBlocks(x, nb, rec, R, words, 0, nb))
    t_pk = med(lambda: par3.create_packets(x, nb, words, 0, R, nb, b"\x5a" * 8, data_after_checksum=PAR3_AFTER,
                                           data_hashes=dh, packets=pk, ctx=ctx))
    out["par3_create_131072x8KiB_R8"] = {"plain": nb * 8 * words / t_plain / 1e9,
                                         "with_block_hashes_and_packets": nb * 8 * words / t_pk / 1e9}
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "src.bin")
        with open(path, "wb") as f:
            f.write(h_in.numpy().tobytes())
        opts = {"recoverySlices": R, "blockSize": 8 * words, "firstInput": 0, "firstRecovery": nb}
        t_st = med(lambda: par3.par3_create_streaming(path, opts, ctx=ctx))
        t_sth = med(lambda: par3.par3_create_streaming(path, opts, data_hashes=dh.numpy(),
                                                       data_after_checksum=PAR3_AFTER, ctx=ctx))
        res = par3.par3_create_streaming(path, opts, ctx=ctx)
        same = bool(np.array_equal(res["recoveryBuffer"].view(np.int64).reshape(R, words), rec.numpy()))
    out["par3_create_streaming_1GiB_8KiB_R8"] = {"from_file": nb * 8 * words / t_st / 1e9,
                                                 "with_block_hashes": nb * 8 * words / t_sth / 1e9,
                                                 "read_share": res["readMs"] / res["durationMs"],
                                                 "matches_in_memory_create": same}
    del h_in, h_out, h_hash, rec, pk, dh
    return out


def profile_tc(ctx, dev):
    """The small ncu case of the tensor-core region kernels, 256 MiB of
    seeded device input each (larger than L2): PAR2 create 8,192 x 32 KiB,
    R=64, three calls (the third runs with the coefficient tiles resident, so
    it is the region kernel alone), then PAR3 create 32,768 x 8 KiB, R=8,
    then PAR2 create 256 x 1 MiB, R=8, three calls."""
    import torch
    from parparpar_b200 import par2, par3
    g = torch.Generator(device=f"cuda:{dev}")
    g.manual_seed(1)
    d = torch.randint(0, 256, (8192, 32768), dtype=torch.uint8, device=f"cuda:{dev}", generator=g)
    o = torch.zeros((64, 32768), dtype=torch.uint8, device=f"cuda:{dev}")
    for _ in range(3):
        par2.par2_create(d, np.arange(8192), list(range(64)), out=o, ctx=ctx)
        ctx.synchronize()
    x = d.view(torch.int64).view(32768, 1024)
    r = torch.zeros((8, 1024), dtype=torch.int64, device=f"cuda:{dev}")
    par3.GF64Controller.ctx = ctx
    par3.GF64Controller.ComputeRecoveryBlocks(x, 32768, r, 8, 1024, 0, 32768)
    ctx.synchronize()
    # PAR2 create 256 x 1 MiB, R=8 (one output group: the one-group tile), three calls
    d8 = d.view(256, 1 << 20)
    o8 = torch.zeros((8, 1 << 20), dtype=torch.uint8, device=f"cuda:{dev}")
    for _ in range(3):
        par2.par2_create(d8, np.arange(256), list(range(8)), out=o8, ctx=ctx)
        ctx.synchronize()
    print(json.dumps({"profile_tc": "ok"}), flush=True)


def profile_hashes(ctx, dev):
    """The small ncu case of the hash kernels: 256 MiB of seeded device data
    (larger than L2) hashed once each way -- PAR2 MD5 + CRC32 of 8,192 x
    32 KiB slices, PAR3 BLAKE3 of 32,768 x 8 KiB blocks, PAR2 memory checksums
    of the 8,192 slices."""
    import torch
    from parparpar_b200 import par2, par3
    g = torch.Generator(device=f"cuda:{dev}")
    g.manual_seed(1)
    d = torch.randint(0, 256, (8192, 32768), dtype=torch.uint8, device=f"cuda:{dev}", generator=g)
    o = torch.zeros((8192, 20), dtype=torch.uint8, device=f"cuda:{dev}")
    par2.block_hashes(d, 32768, out=o, ctx=ctx)
    ctx.synchronize()
    o2 = torch.zeros((32768, 16), dtype=torch.uint8, device=f"cuda:{dev}")
    par3.block_hashes(d.view(32768, 8192), 8192, 0, PAR3_AFTER, num_blocks=32768, out=o2, ctx=ctx)
    ctx.synchronize()
    o3 = torch.zeros((8192, 16), dtype=torch.uint8, device=f"cuda:{dev}")
    par2.memory_checksums(d, 32768, out=o3, ctx=ctx)
    ctx.synchronize()
    print(json.dumps({"profile_hashes": "ok"}), flush=True)


def run_reference(args, rank):
    """--impl reference: the reference's own CPU implementation on the host
    cores, on the same workload/metric (bounded sample per step)."""
    if rank != 0:
        return
    name = args.workload
    w = WORKLOADS[name]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    times = []
    for i in range(args.warmup + args.steps):
        # warm-ups: the sub-range sample (threads, tables, code); timed steps:
        # the whole job where it runs in seconds (PAR2 create), else the sample
        r = cpu_baseline_sample(name, budget_s=0.0, full=i >= args.warmup)
        if i >= args.warmup:
            times.append(r)
    val = statistics.median([t["value"] for t in times])
    spr = statistics.median([t["seconds_per_run"] for t in times])
    line = {
        "impl": "reference", "metric": f"{name} input GB/s", "value": val, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": spr * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(w),
        "data": "synthetic (seeded uniform random bytes)",
        "config": {"workload": name, "num_inputs": w["n"], "slice_bytes": w["s"], "num_recovery": w["r"]},
        "cpu_baseline": {"value": val, "unit": "GB/s", "cores": times[0]["cores"], "kind": times[0]["kind"],
                         "sample": times[0]["sample"], "host": times[0].get("host"),
                         "method": times[0].get("method")},
        "e2e": {"value": val, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=PRIMARY, choices=sorted(WORKLOADS))
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--batched-only", action="store_true", help="print only the batched-vs-plain comparison")
    ap.add_argument("--serving-only", action="store_true", help="print only the serving-loop comparison")
    ap.add_argument("--fused-only", action="store_true", help="print only the fused-pass (hashes, packets, "
                    "streaming) end-to-end comparison")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-hashes", action="store_true",
                    help="one launch of each block-hash kernel on 256 MiB (a small case for ncu), then exit")
    ap.add_argument("--profile-tc", action="store_true",
                    help="the small ncu case of the tensor-core region kernels (256 MiB), then exit")
    ap.add_argument("--gf16-kernel", default="auto", choices=["auto", "lut", "tensor"])
    ap.add_argument("--gf64-kernel", default="auto", choices=["auto", "lut", "tensor"])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import parparpar_b200 as pp
    ctx = pp.Context(local)
    # a dedicated (non-default) stream shared by the library's launches and
    # the timing events
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_gf16_kernel({"auto": 0, "lut": 1, "tensor": 2}[args.gf16_kernel])
    ctx.set_gf64_kernel({"auto": 0, "lut": 1, "tensor": 2}[args.gf64_kernel])
    timer = Timer(stream)
    peak, peak_kind = load_peaks()

    if args.profile_hashes:
        profile_hashes(ctx, local)
        return
    if args.profile_tc:
        profile_tc(ctx, local)
        return
    if args.batched_only:
        print(json.dumps(measure_batched_vs_plain(ctx, timer, args.steps, args.warmup, local)), flush=True)
        return
    if args.serving_only:
        print(json.dumps(measure_serving(ctx, local)), flush=True)
        return
    if args.fused_only:
        print(json.dumps(measure_fused(ctx, local)), flush=True)
        return

    job = setup_job(args.workload, local, 1234 + rank, ctx)
    f = step_fn(job, ctx)
    sampler = ClockSampler(gpu_uuid(local))
    for _ in range(args.warmup):
        f()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms, kms, _, launches = timed_steps(ctx, timer, f, args.steps)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    if dist:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    int8_tops = int8_peak_tops(local)

    # the dominant kernel's launches inside the timed steps, for the roofline
    kms, kms_how = kernel_ms_of(job, ctx, timer, args.steps, kms)
    achieved = algo_bytes(job) / (kms * 1e-3) / 1e9

    # end to end through the public API with pinned host buffers
    w = WORKLOADS[args.workload]
    from parparpar_b200 import par2, par3
    if w["field"] in HASH_FIELDS:
        h_in = torch.empty((w["n"], w["s"]), dtype=torch.uint8).pin_memory()
        h_in.copy_(job["d_in"])
        h_out = torch.empty(tuple(job["d_out"].shape), dtype=torch.uint8).pin_memory()
        e2e_f = hash_fn(job, h_in, h_out, ctx)
    elif w["field"] == "gf16_repair":
        h_in = torch.empty((w["n"], w["s"]), dtype=torch.uint8).pin_memory()
        h_in.copy_(job["d_in"])
        h_out = torch.empty((w["r"], w["s"]), dtype=torch.uint8).pin_memory()
        # host slices in, restored slices out; the factors stay on the device
        # between the inversion and the decode, as a GPU caller keeps them
        hjob = dict(job, d_in=h_in, d_out=h_out)
        e2e_f = lambda: par2_repair_step(hjob, ctx)
    elif w["field"] == "gf16":
        h_in = torch.empty((w["n"], w["s"]), dtype=torch.uint8).pin_memory()
        h_in.copy_(job["d_in"])
        h_out = torch.empty((w["r"], w["s"]), dtype=torch.uint8).pin_memory()
        e2e_f = lambda: par2.par2_create(h_in, job["idx"], job["exps"], out=h_out, ctx=ctx)
    else:
        h_in = torch.empty((w["n"], w["s"] // 8), dtype=torch.int64).pin_memory()
        h_in.copy_(job["d_in"])
        h_out = torch.empty((w["r"], w["s"] // 8), dtype=torch.int64).pin_memory()
        if w["field"] == "gf64_repair":
            h_rec = torch.empty_like(h_out).pin_memory()
            h_rec.copy_(job["d_rec"])
            e2e_f = lambda: par3.repair(h_in, job["lost"], h_rec, w["s"] // 8, 0, w["n"], restored=h_out, ctx=ctx)
        else:
            e2e_f = lambda: par3.GF64Controller.ComputeRecoveryBlocks(h_in, w["n"], h_out, w["r"], w["s"] // 8, 0,
                                                                      w["n"])
    e2e_f()
    torch.cuda.synchronize()
    e2e_steps = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_f()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    ok = torch.equal(h_out.to(f"cuda:{local}"), job["d_out"])
    del h_in, h_out

    input_bytes = w["n"] * w["s"]
    h2d = input_bytes + (w["r"] * w["s"] if w["field"] == "gf64_repair" else 0)
    d2h = job["d_out"].numel() * job["d_out"].element_size()
    line = {
        "metric": f"{args.workload} input GB/s", "value": input_bytes * world / (ms * 1e-3) / 1e9, "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(w),
        "data": "synthetic (seeded uniform random bytes, generated on the device)",
        "config": {"workload": args.workload, "num_inputs": w["n"], "slice_bytes": w["s"], "num_recovery": w["r"],
                   "exponents": f"0..{w['r'] - 1}", "parallelism": f"replicas x{world} (one job per GPU)",
                   "l2": "inputs (1 GiB) larger than L2; no flush needed"},
        "roofline": dict(roofline(w, args, achieved, peak, peak_kind, kms, int8_tops), kernel_timing=kms_how),
        "e2e": {"value": input_bytes / e2e_s / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "host_buffers": "pinned", "matches_device_result": bool(ok)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }

    if rank == 0 and world == 1 and not args.no_secondary:
        sec = []
        for name in WORKLOADS:
            if name == args.workload:
                continue
            try:
                j = setup_job(name, local, 77, ctx)
                heavy = WORKLOADS[name]["field"] == "gf64_repair" or WORKLOADS[name]["r"] >= 1024
                m = measure(j, ctx, timer, 2 if heavy else 5, 1 if heavy else 3, peak)
                ent = {"workload": name, "value": input_bytes_of(name) / (m["ms"] * 1e-3) / 1e9,
                       "unit": "GB/s", "ms_per_step": m["ms"], "kernel_ms": m["kernel_ms"], "hbm_frac": m["frac"]}
                kern = dominant_kernel(WORKLOADS[name], args)
                if kern.endswith(("_tc", "_tc_pair", "_f4", "_f4_pair")):
                    ent["kernel"] = kern
                    ent["tensor_frac"] = (2 * bit_macs(WORKLOADS[name]) / (m["kernel_ms"] * 1e-3) / 1e12 /
                                          tensor_peak(kern, int8_tops)[0])
                sec.append(ent)
                del j
                torch.cuda.empty_cache()
            except Exception as e:  # report, keep the primary line
                sec.append({"workload": name, "error": str(e)[:200]})
        line["secondary"] = sec
        # the 1 GiB R=8 shapes at the top level of the line
        r8 = {}
        for e in sec:
            if e.get("workload") in ("par2_create_1024x1MiB_R8", "par3_create_131072x8KiB_R8") and "value" in e:
                r8[e["workload"]] = {"gbps": round(e["value"], 1), "hbm_frac_of_measured": round(e["hbm_frac"], 4),
                                     "kernel_ms": round(e["kernel_ms"], 4)}
        line["r8"] = r8
        dense = next((e.get("kernel_ms") for e in sec if e.get("workload") == "par3_create_131072x8KiB_R1024"), None)
        try:
            line["fenger_estimate"] = measure_fenger_estimate(ctx, timer, local, dense)
        except Exception as e:  # report, keep the primary line
            line["fenger_estimate"] = {"error": str(e)[:200]}

    if rank == 0 and world == 1 and not args.no_secondary:
        try:
            line["batched_vs_plain"] = measure_batched_vs_plain(ctx, timer, 3, 3, local)
        except Exception as e:  # report, keep the primary line
            line["batched_vs_plain"] = {"error": str(e)[:200]}
        try:
            line["serving"] = measure_serving(ctx, local)
        except Exception as e:
            line["serving"] = {"error": str(e)[:200]}
        try:
            line["fused"] = measure_fused(ctx, local)
        except Exception as e:
            line["fused"] = {"error": str(e)[:200]}

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_sample(args.workload, full=True)
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}

    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
