// Batch plans (pp_batch_*): many create / repair jobs of mixed kinds and
// sizes run as a few fused tensor-core launches, captured once in a CUDA
// graph and replayed.  No counterpart in the reference, which runs one job at
// a time on its CPU threads; each job computes exactly what the single-job
// entry points compute (PAR2: gf16/controller_cpu.cpp muladd over the
// coefficients of gf16/gfmat_coeff.c; PAR3 create: par3_engine.cc
// ComputeRecoveryBlocks; PAR3 repair: the known-input sum of
// lib/par3gen.js:3892-3960 followed by SolveAndReconstruct, par3_engine.cc:980).
//
// A run of the graph is:
//   1. repair right-hand sides <- recovery rows (copies; absent rows zeroed)
//   2. one GF(2^16) launch: every PAR2 create job
//   3. one GF(2^64) launch: every PAR3 create job and every repair's
//      known-input sum (pointer rows, the lost rows point at a zero row)
//   4. one GF(2^64) launch: restored = A^-1 * rhs for every repair job
// (a phase with more jobs than one job table holds takes several launches).
// Everything the launches read besides the jobs' own buffers is built at
// creation and stays on the device: the expanded PAR2 coefficient tiles, the
// PAR3 Cauchy matrices, the pointer tables and the inverse of each repair
// system (closed-form Cauchy inverse, or Gauss-Jordan against the identity
// when a lost column id meets a recovery row id and the system is not a true
// Cauchy matrix).
#include "../../include/parpar_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pp_internal.h"

using namespace pp;

namespace {

// shape signature of a fused launch -> best q found by tuning
std::mutex g_tune_mu;
std::map<std::string, uint32_t> g_tuned;

template <class Job>
std::string signature(const TcBatch<Job>& b, int field) {
  std::string s = std::to_string(field);
  for (uint32_t j = 0; j < b.n_jobs; j++) {
    const Job& J = b.job[j];
    s += "|" + std::to_string(J.n_in) + "," + std::to_string(J.n_out) + "," + std::to_string(J.wt);
  }
  return s;
}

bool aligned(const void* p, size_t a) { return ((uintptr_t)p % a) == 0; }

}  // namespace

struct pp_batch {
  pp_ctx* ctx = nullptr;
  int device = 0;
  std::vector<void*> allocs;
  std::vector<Gf16TcBatch> t16;
  std::vector<Gf64TcBatch> t64a, t64b;
  struct RhsInit {
    uint64_t* rhs;
    const void* rec;
    size_t rec_stride;
    size_t n, words;
    std::vector<uint8_t> present;
  };
  std::vector<RhsInit> rhs_init;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;

  ~pp_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void* p : allocs) cudaFree(p);
  }
  void* alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    allocs.push_back(p);
    return p;
  }
};

// Issue one run of the batch on stream s (used eagerly while tuning and
// under stream capture for the graph).  Returns the number of launches.
static cudaError_t issue(pp_batch* b, cudaStream_t s, int* n_launch) {
  const int sms = ctx_sms(b->ctx);
  int* st = ctx_status_word(b->ctx);
  const uint64_t l0 = launches();
  for (auto& r : b->rhs_init) {
    cudaError_t e = cudaMemcpy2DAsync(r.rhs, r.words * 8, r.rec, r.rec_stride, r.words * 8, r.n,
                                      cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    note_launch();
    for (size_t k = 0; k < r.present.size(); k++) {
      if (r.present[k]) continue;
      e = cudaMemsetAsync(r.rhs + k * r.words, 0, r.words * 8, s);
      if (e != cudaSuccess) return e;
      note_launch();
    }
  }
  for (auto t : b->t16) {  // copies: the launchers fill in derived fields
    cudaError_t e = launch_gf16_tc_batch(t, sms, st, s);
    if (e != cudaSuccess) return e;
  }
  for (auto t : b->t64a) {
    cudaError_t e = launch_gf64_tc_batch(t, sms, st, s);
    if (e != cudaSuccess) return e;
  }
  for (auto t : b->t64b) {
    cudaError_t e = launch_gf64_tc_batch(t, sms, st, s);
    if (e != cudaSuccess) return e;
  }
  if (n_launch) *n_launch = (int)(launches() - l0);
  return cudaSuccess;
}

// Time candidate target item lengths for one fused launch on the jobs' own
// buffers and keep the fastest (remembered per shape).
template <class Job>
static cudaError_t tune_table(TcBatch<Job>& t, int field, cudaError_t (*launch)(TcBatch<Job>&, int, int*, cudaStream_t),
                              int sms, int* st, cudaStream_t s) {
  const std::string sig = signature(t, field);
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tuned.find(sig);
    if (it != g_tuned.end()) {
      t.q_hint = it->second;
      return cudaSuccess;
    }
  }
  cudaEvent_t a, z;
  cudaEventCreate(&a);
  cudaEventCreate(&z);
  auto timed = [&](uint32_t q, float* ms, uint32_t* used) -> cudaError_t {
    TcBatch<Job> c = t;
    c.q_hint = q;
    cudaEventRecord(a, s);
    cudaError_t err = launch(c, sms, st, s);
    cudaEventRecord(z, s);
    if (err != cudaSuccess) return err;
    cudaEventSynchronize(z);
    cudaEventElapsedTime(ms, a, z);
    if (used) *used = c.q_hint;
    return cudaSuccess;
  };
  // the analytic choice first; launches longer than kTuneMaxMs are left to
  // it (the wave model is accurate when items are long), shorter ones try
  // half and double the item length, one timed run each
  constexpr float kTuneMaxMs = 50.f;
  float best = 0;
  uint32_t q0 = 0;
  cudaError_t e = timed(0, &best, &q0);
  uint32_t best_q = q0;
  if (e == cudaSuccess && best < kTuneMaxMs) {
    for (uint32_t q : {std::max(1u, q0 / 2), q0 * 2}) {
      float ms = 0;
      if ((e = timed(q, &ms, nullptr)) != cudaSuccess) break;
      if (ms < best) {
        best = ms;
        best_q = q;
      }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(z);
  if (e != cudaSuccess) return e;
  t.q_hint = best_q;
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tuned[sig] = best_q;
  return cudaSuccess;
}

#define BTRY(expr, msg)                                                  \
  do {                                                                   \
    cudaError_t _e = (expr);                                             \
    if (_e != cudaSuccess) {                                             \
      std::string m = std::string(msg) + ": " + cudaGetErrorString(_e); \
      delete b;                                                          \
      return ctx_fail(ctx, PP_ERR_CUDA, m.c_str());                      \
    }                                                                    \
  } while (0)
#define BFAIL(code, msg)             \
  do {                               \
    delete b;                        \
    return ctx_fail(ctx, code, msg); \
  } while (0)

extern "C" {

PP_API int pp_batch_create(pp_ctx* ctx, const pp_job* jobs, size_t n_jobs, int flags, pp_batch** out) {
  if (!ctx || !out || (!jobs && n_jobs)) return PP_ERR_INVALID_ARG;
  *out = nullptr;
  std::lock_guard<std::mutex> g(ctx_mutex(ctx));
  if (cudaSetDevice(ctx_device(ctx)) != cudaSuccess) return ctx_fail(ctx, PP_ERR_CUDA, "cudaSetDevice failed");
  const cudaStream_t s = ctx_stream(ctx);
  pp_batch* b = new pp_batch();
  b->ctx = ctx;
  b->device = ctx_device(ctx);

  std::vector<Gf16TcJob> j16;
  std::vector<Gf64TcJob> j64a, j64b;
  for (size_t k = 0; k < n_jobs; k++) {
    const pp_job& J = jobs[k];
    if (J.kind == PP_JOB_PAR2_CREATE || J.kind == PP_JOB_GF16_MULADD) {
      const bool custom = J.kind == PP_JOB_GF16_MULADD;
      const size_t n = J.num_inputs, r = J.num_recovery, sb = J.slice_bytes;
      if (!r || !sb) continue;
      if (n > 32768 || r > 65535 || (custom ? !J.coeffs : !J.exponents))
        BFAIL(PP_ERR_INVALID_ARG, "GF16 job: bad counts, or no exponents / coefficients");
      if (!J.inputs || !J.outputs || !aligned(J.inputs, 16) || J.input_stride % 16 ||
          J.input_stride < ((sb + 15) & ~(size_t)15) || !aligned(J.outputs, 4) || J.output_stride % 4 ||
          J.output_stride < sb)
        BFAIL(PP_ERR_INVALID_ARG, "GF16 job: inputs need 16-byte aligned rows of >= slice bytes rounded to 16, "
                                  "outputs 4-byte aligned rows");
      // coefficient matrix -> expanded tensor-core tiles, resident
      uint16_t* d_coef = (uint16_t*)b->alloc(n * r * 2);
      uint8_t* d_aexp = (uint8_t*)b->alloc(gf16_tc_coeff_bytes((unsigned)n, (unsigned)r));
      if (!d_coef || !d_aexp) BFAIL(PP_ERR_NO_MEMORY, "GF16 coefficient tables");
      if (n && custom) {
        BTRY(cudaMemcpyAsync(d_coef, J.coeffs, n * r * 2, cudaMemcpyHostToDevice, s), "copy coefficients");
      } else if (n) {
        std::vector<uint16_t> logs(n), exps(J.exponents, J.exponents + r);
        for (size_t i = 0; i < n; i++) logs[i] = pp_par2_input_log(J.input_ids ? J.input_ids[i] : (uint16_t)i);
        uint16_t* d_logs = (uint16_t*)b->alloc(n * 2);
        uint16_t* d_exps = (uint16_t*)b->alloc(r * 2);
        if (!d_logs || !d_exps) BFAIL(PP_ERR_NO_MEMORY, "PAR2 coefficient tables");
        BTRY(cudaMemcpyAsync(d_logs, logs.data(), n * 2, cudaMemcpyHostToDevice, s), "copy input logs");
        BTRY(cudaMemcpyAsync(d_exps, exps.data(), r * 2, cudaMemcpyHostToDevice, s), "copy exponents");
        BTRY(launch_gf16_coeff_matrix(d_logs, (unsigned)n, d_exps, (unsigned)r, d_coef, s), "coefficients");
      }
      if (n) BTRY(launch_gf16_tc_expand(d_coef, n, (unsigned)n, (unsigned)r, d_aexp, s), "coefficient tiles");
      Gf16TcJob t{};
      t.in = (const uint8_t*)J.inputs;
      t.in_stride = J.input_stride;
      t.a_exp = d_aexp;
      t.out = (uint8_t*)J.outputs;
      t.out_stride = J.output_stride;
      t.slice_bytes = sb;
      t.n_in = (uint32_t)n;
      t.n_out = (uint32_t)r;
      j16.push_back(t);
    } else if (J.kind == PP_JOB_PAR3_CREATE || J.kind == PP_JOB_PAR3_REPAIR) {
      const size_t N = J.num_inputs, words = J.slice_bytes / 8;
      if (J.slice_bytes % 16) BFAIL(PP_ERR_UNSUPPORTED, "PAR3 job: block bytes must be a multiple of 16 in a batch");
      if (!J.inputs || !aligned(J.inputs, 16) || J.input_stride % 16 || J.input_stride < J.slice_bytes || !J.outputs ||
          !aligned(J.outputs, 8) || J.output_stride % 8 || J.output_stride < J.slice_bytes)
        BFAIL(PP_ERR_INVALID_ARG, "PAR3 job: inputs need 16-byte aligned rows, outputs 8-byte aligned rows");
      if (!words) continue;
      if (N > 0xFFFFFFFFull) BFAIL(PP_ERR_INVALID_ARG, "PAR3 job: too many inputs");
      if (J.kind == PP_JOB_PAR3_CREATE) {
        const size_t R = J.num_recovery;
        if (!R) continue;
        uint64_t* d_m = (uint64_t*)b->alloc(R * N * 8);
        if (!d_m) BFAIL(PP_ERR_NO_MEMORY, "PAR3 Cauchy matrix");
        BTRY(launch_gf64_cauchy(d_m, N, R, J.first_input, J.first_recovery, N, s), "Cauchy matrix");
        Gf64TcJob t{};
        t.in = (const uint64_t*)J.inputs;
        t.in_stride = J.input_stride / 8;
        t.coeff = d_m;
        t.ldc = N;
        t.out = (uint64_t*)J.outputs;
        t.out_stride = J.output_stride / 8;
        t.words = words;
        t.n_in = (uint32_t)N;
        t.n_out = (uint32_t)R;
        j64a.push_back(t);
      } else {
        const size_t n = J.num_missing;
        if (!n) continue;
        if (!J.missing || !J.recovery || !aligned(J.recovery, 8) || J.recovery_stride % 8 ||
            J.recovery_stride < J.slice_bytes || n > N)
          BFAIL(PP_ERR_INVALID_ARG, "PAR3 repair job: bad missing list or recovery rows");
        std::vector<uint8_t> lost(N, 0);
        bool cauchy = true;
        for (size_t c = 0; c < n; c++) {
          const uint64_t m = J.missing[c];
          if (m >= N || lost[m]) BFAIL(PP_ERR_INVALID_ARG, "PAR3 repair job: bad missing index list");
          lost[m] = 1;
          if (J.first_input + m - J.first_recovery < n) cauchy = false;
        }
        // known-input sum: rhs (plan-owned) += M * (inputs, lost rows -> zero row)
        uint64_t* d_m = (uint64_t*)b->alloc(n * N * 8);
        uint64_t* rhs = (uint64_t*)b->alloc(n * words * 8);
        uint64_t* zero = (uint64_t*)b->alloc(words * 8);
        const uint64_t** d_ptrs = (const uint64_t**)b->alloc(N * sizeof(void*));
        uint64_t* dA = (uint64_t*)b->alloc(n * n * 8);
        uint64_t* dinv = (uint64_t*)b->alloc(n * n * 8);
        uint64_t* dcols = (uint64_t*)b->alloc(n * 8);
        uint64_t* dw = (uint64_t*)b->alloc((2 * n + 64) * 8);
        if (!d_m || !rhs || !zero || !d_ptrs || !dA || !dinv || !dcols || !dw)
          BFAIL(PP_ERR_NO_MEMORY, "PAR3 repair tables");
        std::vector<const uint64_t*> ptrs(N);
        for (size_t i = 0; i < N; i++)
          ptrs[i] = lost[i] ? zero : (const uint64_t*)((const uint8_t*)J.inputs + i * J.input_stride);
        BTRY(cudaMemsetAsync(zero, 0, words * 8, s), "zero row");
        BTRY(cudaMemcpyAsync(d_ptrs, ptrs.data(), N * sizeof(void*), cudaMemcpyHostToDevice, s), "pointer table");
        BTRY(launch_gf64_cauchy(d_m, N, n, J.first_input, J.first_recovery, N, s), "Cauchy matrix");
        BTRY(cudaMemcpyAsync(dcols, J.missing, n * 8, cudaMemcpyHostToDevice, s), "lost columns");
        BTRY(launch_gf64_cauchy_cols(dA, n, dcols, n, J.first_input, J.first_recovery, s), "repair system");
        if (cauchy) {
          BTRY(launch_gf64_cauchy_inverse(dA, dcols, n, J.first_input, J.first_recovery, dw, dinv, s),
               "closed-form inverse");
        } else {
          // Gauss-Jordan against the identity: dinv <- A^-1
          std::vector<uint64_t> ones(n, 1);
          BTRY(cudaMemsetAsync(dinv, 0, n * n * 8, s), "identity");
          BTRY(cudaMemcpy2DAsync(dinv, (n + 1) * 8, ones.data(), 8, 8, n, cudaMemcpyHostToDevice, s), "identity");
          int* dS = (int*)(dw + n + 2);
          BTRY(cudaMemsetAsync(dS, 0, sizeof(int), s), "status");
          BTRY(launch_gf64_solve(dA, dinv, n, n, dw, dS, s), "repair system inverse");
          int hs = 0;
          BTRY(cudaMemcpyAsync(&hs, dS, sizeof(int), cudaMemcpyDeviceToHost, s), "status");
          BTRY(cudaStreamSynchronize(s), "inverse");
          if (hs) BFAIL(PP_ERR_SINGULAR, "repair matrix is singular");
        }
        pp_batch::RhsInit ri;
        ri.rhs = rhs;
        ri.rec = J.recovery;
        ri.rec_stride = J.recovery_stride;
        ri.n = n;
        ri.words = words;
        if (J.recovery_present) ri.present.assign(J.recovery_present, J.recovery_present + n);
        b->rhs_init.push_back(std::move(ri));
        Gf64TcJob t{};
        t.in_ptrs = d_ptrs;
        t.coeff = d_m;
        t.ldc = N;
        t.out = rhs;
        t.out_stride = words;
        t.words = words;
        t.n_in = (uint32_t)N;
        t.n_out = (uint32_t)n;
        t.accumulate = 1;
        j64a.push_back(t);
        Gf64TcJob u{};
        u.in = rhs;
        u.in_stride = words;
        u.coeff = dinv;
        u.ldc = n;
        u.out = (uint64_t*)J.outputs;
        u.out_stride = J.output_stride / 8;
        u.words = words;
        u.n_in = (uint32_t)n;
        u.n_out = (uint32_t)n;
        j64b.push_back(u);
      }
    } else {
      BFAIL(PP_ERR_INVALID_ARG, "unknown job kind");
    }
  }
  // job tables of at most kTcMaxJobs each
  auto split16 = [&](const std::vector<Gf16TcJob>& v, std::vector<Gf16TcBatch>& out) {
    for (size_t i = 0; i < v.size(); i += kTcMaxJobs) {
      Gf16TcBatch t{};
      t.n_jobs = (uint32_t)std::min<size_t>(kTcMaxJobs, v.size() - i);
      for (uint32_t j = 0; j < t.n_jobs; j++) t.job[j] = v[i + j];
      out.push_back(t);
    }
  };
  auto split64 = [&](const std::vector<Gf64TcJob>& v, std::vector<Gf64TcBatch>& out) {
    for (size_t i = 0; i < v.size(); i += kTcMaxJobs) {
      Gf64TcBatch t{};
      t.n_jobs = (uint32_t)std::min<size_t>(kTcMaxJobs, v.size() - i);
      for (uint32_t j = 0; j < t.n_jobs; j++) t.job[j] = v[i + j];
      out.push_back(t);
    }
  };
  split16(j16, b->t16);
  split64(j64a, b->t64a);
  split64(j64b, b->t64b);

  const int sms = ctx_sms(ctx);
  int* st = ctx_status_word(ctx);
  if (flags & PP_BATCH_NO_GRAPH) {  // tables only; runs are issued eagerly
    *out = b;
    return PP_OK;
  }
  // one eager run before capture: sets the kernels' attributes and checks
  // every launch of the plan (the outputs are written)
  BTRY(issue(b, s, nullptr), "batch first run");
  if (flags & PP_BATCH_TUNE) {
    for (auto& t : b->t16) BTRY(tune_table(t, 16, launch_gf16_tc_batch, sms, st, s), "tuning");
    for (auto& t : b->t64a) BTRY(tune_table(t, 64, launch_gf64_tc_batch, sms, st, s), "tuning");
    for (auto& t : b->t64b) BTRY(tune_table(t, 65, launch_gf64_tc_batch, sms, st, s), "tuning");
  }
  BTRY(cudaStreamSynchronize(s), "batch set-up");

  // capture one run into a graph
  cudaStream_t cap;
  BTRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream");
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t ei = issue(b, cap, &b->launches);
    e = cudaStreamEndCapture(cap, &b->graph);
    if (ei != cudaSuccess) e = ei;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  cudaStreamDestroy(cap);
  BTRY(e, "graph capture");
  *out = b;
  return PP_OK;
}

PP_API int pp_batch_run(pp_batch* b) {
  if (!b) return PP_ERR_INVALID_ARG;
  pp_ctx* ctx = b->ctx;
  std::lock_guard<std::mutex> g(ctx_mutex(ctx));
  if (cudaSetDevice(b->device) != cudaSuccess) return ctx_fail(ctx, PP_ERR_CUDA, "cudaSetDevice failed");
  if (!b->exec) {  // PP_BATCH_NO_GRAPH: issue the fused launches directly
    int n = 0;
    cudaError_t e = issue(b, ctx_stream(ctx), &n);
    if (e != cudaSuccess) return ctx_fail(ctx, PP_ERR_CUDA, cudaGetErrorString(e));
    b->launches = n;
    return PP_OK;
  }
  cudaError_t e = cudaGraphLaunch(b->exec, ctx_stream(ctx));
  if (e != cudaSuccess) return ctx_fail(ctx, PP_ERR_CUDA, cudaGetErrorString(e));
  note_launch(b->launches);
  return PP_OK;
}

PP_API int pp_batch_launches(const pp_batch* b) { return b ? b->launches : 0; }

PP_API void pp_batch_destroy(pp_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(ctx_stream(b->ctx));
  delete b;
}

}  // extern "C"
