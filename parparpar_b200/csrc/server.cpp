// Serving loop (pp_server_*): continuous batching of create / repair jobs of
// mixed kinds and sizes under a device-memory budget.  No counterpart in the
// reference; each job computes what the single-job entry points compute
// (PAR2: gf16/controller_cpu.cpp over gf16/gfmat_coeff.c coefficients; PAR3
// create: par3_engine.cc ComputeRecoveryBlocks; PAR3 repair: the known-input
// sum of lib/par3gen.js:3892-3960 and SolveAndReconstruct, par3_engine.cc:980).
//
// One scheduler thread owns all device work.  Its loop:
//   1. reap: waves whose completion event has fired return their buffers to
//      the pool and release their memory reservations and table references;
//      their jobs complete.
//   2. admit + launch: while a lane (stream) is free and jobs are queued,
//      take jobs from the head of the queue while their device memory fits
//      the budget (evicting unused resident tables first) and issue them as
//      one wave on that lane:
//        staging copies of host buffers -> coefficient tables (resident,
//        built once) -> repair systems and their inverses -> one fused
//        GF(2^16) launch -> one fused GF(2^64) launch (creates and repair
//        known-input sums) -> one fused GF(2^64) launch (repair restores)
//        -> copies back to host buffers -> completion event.
//   3. sleep until a submit, or poll the in-flight events.
// Waves on different lanes overlap on the device; a job arriving while
// others run joins the next wave (continuous batching, not a queue that
// drains one job at a time).
#include "../../include/parpar_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pp_internal.h"

using namespace pp;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
size_t r16(size_t x) { return (x + 15) & ~(size_t)15; }
bool aligned(const void* p, size_t a) { return ((uintptr_t)p % a) == 0; }
bool is_dev(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Resident coefficient table: PAR3 Cauchy rows fR..fR+rows-1 over N columns
// (a repair with n lost blocks uses the first n rows of the same table as a
// create with >= n recovery rows), or PAR2 expanded coefficient tiles.
struct Table {
  int kind = 0;  // 2: PAR3 Cauchy, 1: PAR2 tiles
  uint64_t N = 0, rows = 0, fI = 0, fR = 0;
  std::string par2_key;
  void* d = nullptr;
  size_t bytes = 0;
  int refs = 0;
  uint64_t last_use = 0;
  cudaEvent_t ready = nullptr;  // recorded after the kernels that fill it
};

struct Req {
  uint64_t ticket = 0;
  pp_job job{};
  std::vector<uint16_t> ids, exps, coeffs;
  std::vector<uint64_t> missing;
  std::vector<uint8_t> present;
  bool in_dev = false, out_dev = false, rec_dev = false;
  uint64_t in_bytes = 0;
  size_t need = 0;  // device bytes reserved while admitted (tables apart)
  double t_submit = 0, t_done = 0;
  int status = PP_OK;
  bool done = false;
};

struct Wave {
  int lane = 0;
  cudaEvent_t ev = nullptr;
  std::vector<Req*> jobs;
  std::vector<Table*> tables;
  std::vector<int> singular_slot;  // per job: index into h_words of its solve status, or -1
  int* h_words = nullptr;          // pinned: [0] kernel status, then solve statuses
  int* d_words = nullptr;          // device copy
  size_t reserved = 0;
  bool failed = false;             // an API call of the wave's issue failed
  // staging buffers and temporaries of the wave: returned to the pool only
  // after the host has seen the wave complete, so no other lane's
  // allocation can take them while this lane's kernels may still read them
  // (the budget already counts them until then)
  std::vector<void*> frees;
};

constexpr int kMaxWords = 64;

}  // namespace

struct pp_server {
  pp_ctx* ctx = nullptr;
  int device = 0, sms = 148;
  size_t budget = 0;
  int max_wave = kTcMaxJobs;
  std::vector<cudaStream_t> lanes;
  std::vector<bool> lane_busy;
  std::vector<int*> lane_words_d, lane_words_h;
  cudaMemPool_t pool = nullptr;
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<Req*> queue;
  std::map<uint64_t, Req*> reqs;
  std::list<Wave*> inflight;
  std::list<Table*> tables;
  size_t used = 0, peak = 0, table_bytes = 0;
  uint64_t next_ticket = 1, use_clock = 0;
  bool stop = false;
  std::thread th;
  uint64_t submitted = 0, completed = 0, failed = 0, waves = 0, in_bytes = 0;
  double t_first = 0, t_last = 0;
  std::vector<double> lat_ms;
  std::string err;

  void* dalloc(size_t bytes, cudaStream_t s) {
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, pool, s) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return p;
  }
};

namespace {

// ---------------------------------------------------------------- sizing
struct Need {
  size_t job = 0;        // staging + temporaries of the job
  Table* table = nullptr;  // resident table to reuse, if any
  size_t table_new = 0;  // bytes of a table to build
};

bool par3_tc(const pp_job& J) { return J.slice_bytes % 16 == 0; }

Table* find_table(pp_server* S, const Req* r) {
  const pp_job& J = r->job;
  for (Table* t : S->tables) {
    if (J.kind == PP_JOB_PAR3_CREATE || J.kind == PP_JOB_PAR3_REPAIR) {
      const uint64_t rows = J.kind == PP_JOB_PAR3_CREATE ? J.num_recovery : J.num_missing;
      if (t->kind == 2 && t->N == J.num_inputs && t->fI == J.first_input && t->fR == J.first_recovery &&
          t->rows >= rows)
        return t;
    } else if (J.kind == PP_JOB_PAR2_CREATE) {
      if (t->kind == 1 && t->N == J.num_inputs && t->rows == J.num_recovery) {
        std::string key((const char*)r->ids.data(), r->ids.size() * 2);
        key.append((const char*)r->exps.data(), r->exps.size() * 2);
        if (t->par2_key == key) return t;
      }
    }
  }
  return nullptr;
}

Need need_of(pp_server* S, Req* r) {
  const pp_job& J = r->job;
  Need n;
  const size_t N = J.num_inputs, sb = J.slice_bytes;
  if (J.kind == PP_JOB_PAR2_CREATE || J.kind == PP_JOB_GF16_MULADD) {
    const size_t R = J.num_recovery;
    if (!r->in_dev || !aligned(J.inputs, 16) || J.input_stride % 16 || J.input_stride < r16(sb)) n.job += N * r16(sb);
    if (!r->out_dev || !aligned(J.outputs, 4) || J.output_stride % 4) n.job += R * r16(sb);
    const size_t tiles = gf16_tc_coeff_bytes((unsigned)N, (unsigned)R);
    n.job += N * R * 2 + N * 2 + R * 2 + 256;  // coefficient matrix (temporary)
    if (J.kind == PP_JOB_GF16_MULADD) {
      n.job += tiles;
    } else if (!(n.table = find_table(S, r))) {
      n.table_new = tiles;
    }
  } else {
    const size_t rows = J.kind == PP_JOB_PAR3_CREATE ? J.num_recovery : J.num_missing;
    const bool tc = par3_tc(J);
    if (!r->in_dev || !aligned(J.inputs, 16) || J.input_stride % 16) n.job += N * sb;
    if (!r->out_dev || !aligned(J.outputs, 8) || J.output_stride % 8) n.job += rows * sb;
    if (J.kind == PP_JOB_PAR3_REPAIR) {
      const size_t m = J.num_missing;
      if (!r->rec_dev || !aligned(J.recovery, 8) || J.recovery_stride % 8) n.job += m * sb;
      n.job += m * sb + sb + N * 8 + 2 * m * m * 8 + (3 * m + 64) * 8 + (tc ? 0 : m * 8);
    }
    if (!(n.table = find_table(S, r))) n.table_new = rows * N * 8;
  }
  n.job += 4096;  // alignment slack
  return n;
}

void note_peak(pp_server* S) { S->peak = std::max(S->peak, S->used); }

// Evict unreferenced tables (least recently used first) until `bytes` more fit.
bool make_room(pp_server* S, size_t bytes) {
  while (S->used + bytes > S->budget) {
    Table* victim = nullptr;
    for (Table* t : S->tables)
      if (!t->refs && (!victim || t->last_use < victim->last_use)) victim = t;
    if (!victim) return false;
    cudaFreeAsync(victim->d, S->lanes[0]);
    if (victim->ready) cudaEventDestroy(victim->ready);
    S->used -= victim->bytes;
    S->table_bytes -= victim->bytes;
    S->tables.remove(victim);
    delete victim;
  }
  return true;
}

void finish(pp_server* S, Req* r, int status) {
  r->status = status;
  r->done = true;
  r->t_done = now_s();
  S->t_last = r->t_done;
  if (status == PP_OK) {
    S->completed++;
    S->in_bytes += r->in_bytes;
    S->lat_ms.push_back((r->t_done - r->t_submit) * 1e3);
  } else {
    S->failed++;
  }
}

// ---------------------------------------------------------------- wave issue
struct Staged {
  const uint8_t* in = nullptr;
  size_t in_stride = 0;
  uint8_t* out = nullptr;
  size_t out_stride = 0;
  const uint8_t* rec = nullptr;
  size_t rec_stride = 0;
};

#define WTRY(expr)                          \
  do {                                      \
    cudaError_t _e = (expr);                \
    if (_e != cudaSuccess) return _e;       \
  } while (0)

// Issue one wave on its lane.  Errors leave the wave to complete with an
// error status for all of its jobs.
cudaError_t issue_wave(pp_server* S, Wave* w, std::vector<Need>& needs, std::vector<void*>& frees) {
  const cudaStream_t s = S->lanes[w->lane];
  auto alloc = [&](size_t bytes) -> void* {
    void* p = S->dalloc(bytes, s);
    if (p) frees.push_back(p);
    return p;
  };
  WTRY(cudaMemsetAsync(w->d_words, 0, kMaxWords * sizeof(int), s));
  std::vector<Gf16TcJob> j16;
  std::vector<Gf64TcJob> j64a, j64b;
  struct RhsInit {
    uint64_t* rhs;
    const uint8_t* rec;
    size_t rec_stride, n, words;
    const std::vector<uint8_t>* present;
  };
  std::vector<RhsInit> rhs_init;
  struct Lut {
    int kind;  // 0 create matvec, 1 repair
    Req* r;
    Staged st;
    const uint64_t* coeff;
    const uint64_t** ptrs;
    uint64_t** out_ptrs;
    uint64_t* rhs;
    uint64_t* inv;
  };
  std::vector<Lut> luts;
  std::vector<Staged> staged(w->jobs.size());
  std::vector<std::vector<const uint64_t*>> host_ptrs;
  std::vector<std::vector<uint64_t*>> host_optrs;
  int next_word = 1;

  for (size_t k = 0; k < w->jobs.size(); k++) {
    Req* r = w->jobs[k];
    const pp_job& J = r->job;
    Staged& st = staged[k];
    const size_t N = J.num_inputs, sb = J.slice_bytes;
    Table* tab = needs[k].table;
    if (!tab && needs[k].table_new && J.kind != PP_JOB_GF16_MULADD) {
      // an earlier job of this wave may have built the same table
      if ((tab = find_table(S, r))) {
        S->used -= needs[k].table_new;
        needs[k].table_new = 0;
        needs[k].table = tab;
      }
    }
    if (tab && tab->ready) WTRY(cudaStreamWaitEvent(s, tab->ready, 0));
    if (J.kind == PP_JOB_PAR2_CREATE || J.kind == PP_JOB_GF16_MULADD) {
      const size_t R = J.num_recovery;
      // inputs: 16-byte aligned rows readable to r16(slice)
      if (r->in_dev && aligned(J.inputs, 16) && J.input_stride % 16 == 0 && J.input_stride >= r16(sb)) {
        st.in = (const uint8_t*)J.inputs;
        st.in_stride = J.input_stride;
      } else if (N) {
        uint8_t* d = (uint8_t*)alloc(N * r16(sb));
        if (!d) return cudaErrorMemoryAllocation;
        WTRY(cudaMemcpy2DAsync(d, r16(sb), J.inputs, J.input_stride, sb, N, cudaMemcpyDefault, s));
        st.in = d;
        st.in_stride = r16(sb);
      }
      if (r->out_dev && aligned(J.outputs, 4) && J.output_stride % 4 == 0) {
        st.out = (uint8_t*)J.outputs;
        st.out_stride = J.output_stride;
      } else {
        st.out = (uint8_t*)alloc(R * r16(sb));
        if (!st.out) return cudaErrorMemoryAllocation;
        st.out_stride = r16(sb);
      }
      const uint8_t* aexp = nullptr;
      if (tab) {
        aexp = (const uint8_t*)tab->d;
      } else {
        uint16_t* d_coef = (uint16_t*)alloc(N * R * 2 + 16);
        if (!d_coef) return cudaErrorMemoryAllocation;
        uint8_t* d_aexp = nullptr;
        if (J.kind == PP_JOB_GF16_MULADD) {
          d_aexp = (uint8_t*)alloc(gf16_tc_coeff_bytes((unsigned)N, (unsigned)R));
          if (!d_aexp) return cudaErrorMemoryAllocation;
          if (N) WTRY(cudaMemcpyAsync(d_coef, r->coeffs.data(), N * R * 2, cudaMemcpyHostToDevice, s));
        } else {
          Table* t = new Table();
          t->kind = 1;
          t->N = N;
          t->rows = R;
          t->par2_key.assign((const char*)r->ids.data(), r->ids.size() * 2);
          t->par2_key.append((const char*)r->exps.data(), r->exps.size() * 2);
          t->bytes = needs[k].table_new;
          t->d = S->dalloc(t->bytes, s);
          if (!t->d) {
            S->used -= t->bytes;
            delete t;
            return cudaErrorMemoryAllocation;
          }
          cudaEventCreateWithFlags(&t->ready, cudaEventDisableTiming);
          S->tables.push_back(t);
          S->table_bytes += t->bytes;
          d_aexp = (uint8_t*)t->d;
          tab = needs[k].table = t;
          std::vector<uint16_t> logs(N);
          for (size_t i = 0; i < N; i++) logs[i] = pp_par2_input_log(r->ids.empty() ? (uint16_t)i : r->ids[i]);
          uint16_t* d_le = (uint16_t*)alloc(N * 2 + R * 2 + 16);
          if (!d_le) return cudaErrorMemoryAllocation;
          if (N) WTRY(cudaMemcpyAsync(d_le, logs.data(), N * 2, cudaMemcpyHostToDevice, s));
          WTRY(cudaMemcpyAsync(d_le + N, r->exps.data(), R * 2, cudaMemcpyHostToDevice, s));
          if (N) WTRY(launch_gf16_coeff_matrix(d_le, (unsigned)N, d_le + N, (unsigned)R, d_coef, s));
        }
        if (N) WTRY(launch_gf16_tc_expand(d_coef, N, (unsigned)N, (unsigned)R, d_aexp, s));
        if (tab) WTRY(cudaEventRecord(tab->ready, s));
        aexp = d_aexp;
      }
      if (tab) {
        tab->refs++;
        tab->last_use = ++S->use_clock;
        w->tables.push_back(tab);
      }
      Gf16TcJob t{};
      t.in = st.in;
      t.in_stride = st.in_stride;
      t.a_exp = aexp;
      t.out = st.out;
      t.out_stride = st.out_stride;
      t.slice_bytes = sb;
      t.n_in = (uint32_t)N;
      t.n_out = (uint32_t)R;
      j16.push_back(t);
      continue;
    }
    // PAR3
    const size_t words = sb / 8;
    const bool tc = par3_tc(J);
    const size_t rows = J.kind == PP_JOB_PAR3_CREATE ? J.num_recovery : J.num_missing;
    if (r->in_dev && aligned(J.inputs, 16) && J.input_stride % 16 == 0) {
      st.in = (const uint8_t*)J.inputs;
      st.in_stride = J.input_stride;
    } else {
      uint8_t* d = (uint8_t*)alloc(N * sb);
      if (!d) return cudaErrorMemoryAllocation;
      WTRY(cudaMemcpy2DAsync(d, sb, J.inputs, J.input_stride, sb, N, cudaMemcpyDefault, s));
      st.in = d;
      st.in_stride = sb;
    }
    if (r->out_dev && aligned(J.outputs, 8) && J.output_stride % 8 == 0) {
      st.out = (uint8_t*)J.outputs;
      st.out_stride = J.output_stride;
    } else {
      st.out = (uint8_t*)alloc(rows * sb);
      if (!st.out) return cudaErrorMemoryAllocation;
      st.out_stride = sb;
    }
    if (!tab) {
      Table* t = new Table();
      t->kind = 2;
      t->N = N;
      t->rows = rows;
      t->fI = J.first_input;
      t->fR = J.first_recovery;
      t->bytes = needs[k].table_new;
      t->d = S->dalloc(t->bytes, s);
      if (!t->d) {
        S->used -= t->bytes;
        delete t;
        return cudaErrorMemoryAllocation;
      }
      cudaEventCreateWithFlags(&t->ready, cudaEventDisableTiming);
      S->tables.push_back(t);
      S->table_bytes += t->bytes;
      WTRY(launch_gf64_cauchy((uint64_t*)t->d, N, rows, J.first_input, J.first_recovery, N, s));
      WTRY(cudaEventRecord(t->ready, s));
      tab = needs[k].table = t;
    }
    tab->refs++;
    tab->last_use = ++S->use_clock;
    w->tables.push_back(tab);
    const uint64_t* M = (const uint64_t*)tab->d;
    if (J.kind == PP_JOB_PAR3_CREATE) {
      if (tc) {
        Gf64TcJob t{};
        t.in = (const uint64_t*)st.in;
        t.in_stride = st.in_stride / 8;
        t.coeff = M;
        t.ldc = N;
        t.out = (uint64_t*)st.out;
        t.out_stride = st.out_stride / 8;
        t.words = words;
        t.n_in = (uint32_t)N;
        t.n_out = (uint32_t)rows;
        j64a.push_back(t);
      } else {
        luts.push_back(Lut{0, r, st, M, nullptr, nullptr, nullptr, nullptr});
      }
      continue;
    }
    // repair
    const size_t n = J.num_missing;
    if (r->rec_dev && aligned(J.recovery, 8) && J.recovery_stride % 8 == 0) {
      st.rec = (const uint8_t*)J.recovery;
      st.rec_stride = J.recovery_stride;
    } else {
      uint8_t* d = (uint8_t*)alloc(n * sb);
      if (!d) return cudaErrorMemoryAllocation;
      WTRY(cudaMemcpy2DAsync(d, sb, J.recovery, J.recovery_stride, sb, n, cudaMemcpyDefault, s));
      st.rec = d;
      st.rec_stride = sb;
    }
    uint64_t* rhs = (uint64_t*)alloc(n * sb);
    uint64_t* zero = (uint64_t*)alloc(sb);
    const uint64_t** d_ptrs = (const uint64_t**)alloc(N * 8);
    uint64_t* dA = (uint64_t*)alloc(n * n * 8);
    uint64_t* dinv = (uint64_t*)alloc(n * n * 8);
    uint64_t* dcols = (uint64_t*)alloc(n * 8);
    uint64_t* dw = (uint64_t*)alloc((2 * n + 64) * 8);
    if (!rhs || !zero || !d_ptrs || !dA || !dinv || !dcols || !dw) return cudaErrorMemoryAllocation;
    std::vector<uint8_t> lost(N, 0);
    bool cauchy = true;
    for (size_t c = 0; c < n; c++) {
      lost[r->missing[c]] = 1;
      if (J.first_input + r->missing[c] - J.first_recovery < n) cauchy = false;
    }
    host_ptrs.emplace_back(N);
    auto& hp = host_ptrs.back();
    for (size_t i = 0; i < N; i++)
      hp[i] = lost[i] ? zero : (const uint64_t*)(st.in + i * st.in_stride);
    WTRY(cudaMemsetAsync(zero, 0, sb, s));
    WTRY(cudaMemcpyAsync(d_ptrs, hp.data(), N * 8, cudaMemcpyHostToDevice, s));
    WTRY(cudaMemcpyAsync(dcols, r->missing.data(), n * 8, cudaMemcpyHostToDevice, s));
    WTRY(launch_gf64_cauchy_cols(dA, n, dcols, n, J.first_input, J.first_recovery, s));
    if (cauchy) {
      WTRY(launch_gf64_cauchy_inverse(dA, dcols, n, J.first_input, J.first_recovery, dw, dinv, s));
    } else {
      const std::vector<uint64_t> ones(n, 1);  // pageable source: staged before the call returns
      WTRY(cudaMemsetAsync(dinv, 0, n * n * 8, s));
      WTRY(cudaMemcpy2DAsync(dinv, (n + 1) * 8, ones.data(), 8, 8, n, cudaMemcpyHostToDevice, s));
      if (next_word >= kMaxWords) return cudaErrorInvalidValue;
      const int slot = next_word++;
      w->singular_slot[k] = slot;
      WTRY(launch_gf64_solve(dA, dinv, n, n, dw, w->d_words + slot, s));
    }
    rhs_init.push_back(RhsInit{rhs, st.rec, st.rec_stride, n, words, &r->present});
    if (tc) {
      Gf64TcJob t{};
      t.in_ptrs = d_ptrs;
      t.coeff = M;
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
      u.out = (uint64_t*)st.out;
      u.out_stride = st.out_stride / 8;
      u.words = words;
      u.n_in = (uint32_t)n;
      u.n_out = (uint32_t)n;
      j64b.push_back(u);
    } else {
      uint64_t** d_optrs = (uint64_t**)alloc(n * 8);
      if (!d_optrs) return cudaErrorMemoryAllocation;
      host_optrs.emplace_back(n);
      for (size_t e = 0; e < n; e++) host_optrs.back()[e] = rhs + e * words;
      WTRY(cudaMemcpyAsync(d_optrs, host_optrs.back().data(), n * 8, cudaMemcpyHostToDevice, s));
      luts.push_back(Lut{1, r, st, M, d_ptrs, d_optrs, rhs, dinv});
    }
  }
  // right-hand sides <- recovery rows (absent rows zero)
  for (auto& ri : rhs_init) {
    WTRY(cudaMemcpy2DAsync(ri.rhs, ri.words * 8, ri.rec, ri.rec_stride, ri.words * 8, ri.n, cudaMemcpyDeviceToDevice,
                           s));
    for (size_t e = 0; e < ri.present->size(); e++)
      if (!(*ri.present)[e]) WTRY(cudaMemsetAsync(ri.rhs + e * ri.words, 0, ri.words * 8, s));
  }
  // fused launches
  int* kst = w->d_words;
  for (size_t i = 0; i < j16.size(); i += kTcMaxJobs) {
    Gf16TcBatch t{};
    t.n_jobs = (uint32_t)std::min<size_t>(kTcMaxJobs, j16.size() - i);
    for (uint32_t j = 0; j < t.n_jobs; j++) t.job[j] = j16[i + j];
    WTRY(launch_gf16_tc_batch(t, S->sms, kst, s));
  }
  for (auto* v : {&j64a, &j64b}) {
    for (size_t i = 0; i < v->size(); i += kTcMaxJobs) {
      Gf64TcBatch t{};
      t.n_jobs = (uint32_t)std::min<size_t>(kTcMaxJobs, v->size() - i);
      for (uint32_t j = 0; j < t.n_jobs; j++) t.job[j] = (*v)[i + j];
      // one-CTA kernels: the lanes overlap on the device
      WTRY(launch_gf64_tc_batch_one_cta(t, S->sms, kst, s));
    }
    if (v == &j64a) {
      // lookup-kernel jobs (block bytes not a multiple of 16), between the phases
      for (auto& L : luts) {
        const pp_job& J = L.r->job;
        const size_t N = J.num_inputs, words = J.slice_bytes / 8;
        if (L.kind == 0) {
          WTRY(launch_gf64_matvec((const uint64_t*)L.st.in, L.st.in_stride / 8, N, words, L.coeff, N,
                                  J.num_recovery, (uint64_t*)L.st.out, L.st.out_stride / 8, false, S->sms, s));
        } else {
          const size_t n = J.num_missing;
          WTRY(launch_gf64_2d_gather(L.out_ptrs, n, L.ptrs, N, L.coeff, N, words, S->sms, s));
          WTRY(launch_gf64_matvec(L.rhs, words, n, words, L.inv, n, n, (uint64_t*)L.st.out, L.st.out_stride / 8,
                                  false, S->sms, s));
        }
      }
    }
  }
  // results to host buffers
  for (size_t k = 0; k < w->jobs.size(); k++) {
    Req* r = w->jobs[k];
    const pp_job& J = r->job;
    const Staged& st = staged[k];
    const size_t rows = J.kind == PP_JOB_PAR3_REPAIR ? J.num_missing : J.num_recovery;
    if ((uint8_t*)J.outputs != st.out)
      WTRY(cudaMemcpy2DAsync(J.outputs, J.output_stride, st.out, st.out_stride, J.slice_bytes, rows,
                             cudaMemcpyDefault, s));
  }
  WTRY(cudaMemcpyAsync(w->h_words, w->d_words, kMaxWords * sizeof(int), cudaMemcpyDeviceToHost, s));
  return cudaSuccess;
}

// Admit queued jobs (FIFO, within the budget) into a wave on a free lane.
bool launch_one(pp_server* S) {
  int lane = -1;
  for (size_t l = 0; l < S->lanes.size(); l++)
    if (!S->lane_busy[l]) {
      lane = (int)l;
      break;
    }
  if (lane < 0 || S->queue.empty()) return false;
  Wave* w = new Wave();
  w->lane = lane;
  w->d_words = S->lane_words_d[lane];
  w->h_words = S->lane_words_h[lane];
  std::vector<Need> needs;
  size_t solves = 0;
  while (!S->queue.empty() && (int)w->jobs.size() < S->max_wave) {
    Req* r = S->queue.front();
    Need n = need_of(S, r);
    const size_t want = n.job + n.table_new;
    if (want > S->budget) {  // can never fit, whatever else is resident
      S->queue.pop_front();
      finish(S, r, PP_ERR_TOO_LARGE);
      S->cv_done.notify_all();
      continue;
    }
    if (n.table) n.table->refs++;  // keep it from eviction while making room
    const bool fits = make_room(S, want);
    if (n.table) n.table->refs--;
    if (!fits) {
      if (S->inflight.empty() && w->jobs.empty() && S->tables.empty()) {
        S->queue.pop_front();
        finish(S, r, PP_ERR_TOO_LARGE);  // can never fit
        S->cv_done.notify_all();
        continue;
      }
      break;
    }
    if (r->job.kind == PP_JOB_PAR3_REPAIR && solves + 2 > (size_t)kMaxWords) break;
    if (r->job.kind == PP_JOB_PAR3_REPAIR) solves++;
    S->queue.pop_front();
    S->used += want;
    w->reserved += n.job;
    w->jobs.push_back(r);
    needs.push_back(n);
  }
  if (w->jobs.empty()) {
    delete w;
    return false;
  }
  note_peak(S);
  w->singular_slot.assign(w->jobs.size(), -1);
  const cudaStream_t s = S->lanes[lane];
  cudaError_t e = issue_wave(S, w, needs, w->frees);
  if (e != cudaSuccess) {
    cudaGetLastError();
    S->err = cudaGetErrorString(e);
    w->failed = true;  // every job of the wave reports PP_ERR_CUDA
  }
  cudaEventCreateWithFlags(&w->ev, cudaEventDisableTiming);
  cudaEventRecord(w->ev, s);
  S->lane_busy[lane] = true;
  S->inflight.push_back(w);
  S->waves++;
  return true;
}

bool reap(pp_server* S) {
  bool any = false;
  for (auto it = S->inflight.begin(); it != S->inflight.end();) {
    Wave* w = *it;
    if (cudaEventQuery(w->ev) != cudaSuccess) {
      cudaGetLastError();
      ++it;
      continue;
    }
    const int kst = w->h_words[0];
    for (size_t k = 0; k < w->jobs.size(); k++) {
      int st = PP_OK;
      if (w->failed) st = PP_ERR_CUDA;
      else if (kst) st = PP_ERR_TIMEOUT;
      else if (w->singular_slot[k] >= 0 && w->h_words[w->singular_slot[k]]) st = PP_ERR_SINGULAR;
      finish(S, w->jobs[k], st);
    }
    for (Table* t : w->tables) t->refs--;
    for (void* p : w->frees) cudaFreeAsync(p, S->lanes[w->lane]);  // the wave's work has completed
    S->used -= w->reserved;
    S->lane_busy[w->lane] = false;
    cudaEventDestroy(w->ev);
    it = S->inflight.erase(it);
    delete w;
    any = true;
  }
  if (any) S->cv_done.notify_all();
  return any;
}

void scheduler(pp_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    bool progressed = reap(S);
    while (launch_one(S)) progressed = true;
    if (S->stop && S->queue.empty() && S->inflight.empty()) break;
    if (progressed) continue;
    if (!S->inflight.empty())
      S->cv_sched.wait_for(lk, std::chrono::microseconds(50));
    else
      S->cv_sched.wait(lk);
  }
}

}  // namespace

extern "C" {

PP_API int pp_server_create(int device, size_t hbm_budget_bytes, int max_jobs_per_wave, int lanes,
                            pp_server** out) {
  if (!out || !hbm_budget_bytes) return PP_ERR_INVALID_ARG;
  *out = nullptr;
  pp_server* S = new pp_server();
  int r = pp_ctx_create(device, &S->ctx);
  if (r != PP_OK) {
    delete S;
    return r;
  }
  S->device = device;
  S->sms = ctx_sms(S->ctx);
  S->budget = hbm_budget_bytes;
  S->max_wave = std::max(1, std::min(max_jobs_per_wave > 0 ? max_jobs_per_wave : kTcMaxJobs, kTcMaxJobs));
  const int nl = std::max(1, std::min(lanes > 0 ? lanes : 2, 8));
  cudaSetDevice(device);
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  if (cudaMemPoolCreate(&S->pool, &props) != cudaSuccess) {
    cudaGetLastError();
    pp_ctx_destroy(S->ctx);
    delete S;
    return PP_ERR_CUDA;
  }
  uint64_t keep = ~0ull;  // freed blocks stay in the pool for the next waves
  cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  for (int l = 0; l < nl; l++) {
    cudaStream_t s;
    int* d = nullptr;
    int* h = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&d, kMaxWords * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&h, kMaxWords * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      pp_server_destroy(S);
      return PP_ERR_CUDA;
    }
    memset(h, 0, kMaxWords * sizeof(int));
    S->lanes.push_back(s);
    S->lane_busy.push_back(false);
    S->lane_words_d.push_back(d);
    S->lane_words_h.push_back(h);
  }
  S->th = std::thread(scheduler, S);
  *out = S;
  return PP_OK;
}

PP_API int pp_server_submit(pp_server* S, const pp_job* job, uint64_t* ticket) {
  if (!S || !job || !ticket) return PP_ERR_INVALID_ARG;
  const pp_job& J = *job;
  Req* r = new Req();
  r->job = J;
  // argument checks (the same as the batch plan's)
  auto bad = [&](const char* m) {
    std::lock_guard<std::mutex> g(S->mu);
    S->err = m;
    delete r;
    return PP_ERR_INVALID_ARG;
  };
  if (!J.inputs && J.num_inputs) return bad("null inputs");
  if (!J.outputs) return bad("null outputs");
  if (J.kind == PP_JOB_PAR2_CREATE || J.kind == PP_JOB_GF16_MULADD) {
    if (J.num_inputs > 32768 || !J.num_recovery || J.num_recovery > 65535 || !J.slice_bytes)
      return bad("GF16 job: bad counts");
    if (J.input_stride < J.slice_bytes || J.output_stride < J.slice_bytes) return bad("GF16 job: strides");
    if (J.kind == PP_JOB_PAR2_CREATE) {
      if (!J.exponents) return bad("PAR2 job: no exponents");
      r->exps.assign(J.exponents, J.exponents + J.num_recovery);
      if (J.input_ids) r->ids.assign(J.input_ids, J.input_ids + J.num_inputs);
      else
        for (size_t i = 0; i < J.num_inputs; i++) r->ids.push_back((uint16_t)i);
    } else {
      if (!J.coeffs) return bad("GF16 job: no coefficients");
      r->coeffs.assign(J.coeffs, J.coeffs + J.num_recovery * J.num_inputs);
    }
    r->in_bytes = J.num_inputs * J.slice_bytes;
  } else if (J.kind == PP_JOB_PAR3_CREATE || J.kind == PP_JOB_PAR3_REPAIR) {
    if (!J.slice_bytes || J.slice_bytes % 8) return bad("PAR3 job: block bytes must be a positive multiple of 8");
    if (J.input_stride < J.slice_bytes || J.output_stride < J.slice_bytes || J.input_stride % 8 ||
        J.output_stride % 8)
      return bad("PAR3 job: strides");
    if (!J.num_inputs || J.num_inputs > 0xFFFFFFFFull) return bad("PAR3 job: bad input count");
    if (J.kind == PP_JOB_PAR3_CREATE) {
      if (!J.num_recovery) return bad("PAR3 job: no recovery rows");
    } else {
      if (!J.num_missing || !J.missing || !J.recovery || J.num_missing > J.num_inputs ||
          J.recovery_stride < J.slice_bytes || J.recovery_stride % 8)
        return bad("PAR3 repair job: bad missing list or recovery rows");
      r->missing.assign(J.missing, J.missing + J.num_missing);
      std::vector<uint8_t> seen(J.num_inputs, 0);
      for (uint64_t m : r->missing) {
        if (m >= J.num_inputs || seen[m]) return bad("PAR3 repair job: bad missing index list");
        seen[m] = 1;
      }
      if (J.recovery_present) r->present.assign(J.recovery_present, J.recovery_present + J.num_missing);
      r->rec_dev = is_dev(J.recovery);
    }
    r->in_bytes = J.num_inputs * J.slice_bytes;
  } else {
    return bad("unknown job kind");
  }
  // pointers into the copies above (the caller's arrays may go away)
  r->job.input_ids = nullptr;
  r->job.exponents = nullptr;
  r->job.missing = nullptr;
  r->job.recovery_present = nullptr;
  r->job.coeffs = nullptr;
  r->in_dev = J.num_inputs ? is_dev(J.inputs) : true;
  r->out_dev = is_dev(J.outputs);
  std::lock_guard<std::mutex> g(S->mu);
  if (S->stop) {
    delete r;
    return PP_ERR_BUSY;
  }
  r->ticket = S->next_ticket++;
  r->t_submit = now_s();
  if (!S->submitted || S->t_first == 0) S->t_first = r->t_submit;
  S->submitted++;
  S->reqs[r->ticket] = r;
  S->queue.push_back(r);
  *ticket = r->ticket;
  S->cv_sched.notify_one();
  return PP_OK;
}

PP_API int pp_server_wait(pp_server* S, uint64_t ticket, int timeout_ms) {
  if (!S) return PP_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return PP_ERR_INVALID_ARG;
  Req* r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0) {
    S->cv_done.wait(lk, ready);
  } else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return PP_ERR_TIMEOUT;
  }
  const int st = r->status;
  S->reqs.erase(it);
  delete r;
  return st;
}

PP_API int pp_server_get_stats(pp_server* S, pp_server_stats* o) {
  if (!S || !o) return PP_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(S->mu);
  memset(o, 0, sizeof *o);
  o->submitted = S->submitted;
  o->completed = S->completed;
  o->failed = S->failed;
  o->waves = S->waves;
  o->input_bytes = S->in_bytes;
  o->elapsed_s = S->t_last > S->t_first ? S->t_last - S->t_first : 0;
  o->gbps = o->elapsed_s > 0 ? (double)S->in_bytes / o->elapsed_s / 1e9 : 0;
  if (!S->lat_ms.empty()) {
    std::vector<double> v = S->lat_ms;
    std::sort(v.begin(), v.end());
    auto q = [&](double p) { return v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))]; };
    o->p50_ms = q(0.50);
    o->p99_ms = q(0.99);
    o->max_ms = v.back();
  }
  o->hbm_peak_bytes = S->peak;
  o->tables_resident = S->tables.size();
  o->table_bytes = S->table_bytes;
  return PP_OK;
}

PP_API void pp_server_reset_stats(pp_server* S) {
  if (!S) return;
  std::lock_guard<std::mutex> g(S->mu);
  S->submitted = S->completed = S->failed = S->waves = S->in_bytes = 0;
  S->t_first = S->t_last = 0;
  S->lat_ms.clear();
  S->peak = S->used;
}

PP_API const char* pp_server_last_error(pp_server* S) { return S ? S->err.c_str() : "no server"; }

PP_API void pp_server_destroy(pp_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
    S->cv_sched.notify_all();
  }
  if (S->th.joinable()) S->th.join();
  cudaSetDevice(S->device);
  for (cudaStream_t s : S->lanes) cudaStreamSynchronize(s);
  for (Table* t : S->tables) {
    cudaFreeAsync(t->d, S->lanes.empty() ? nullptr : S->lanes[0]);
    if (t->ready) cudaEventDestroy(t->ready);
    delete t;
  }
  for (cudaStream_t s : S->lanes) cudaStreamSynchronize(s);
  for (auto& kv : S->reqs) delete kv.second;
  for (int* d : S->lane_words_d) cudaFree(d);
  for (int* h : S->lane_words_h) cudaFreeHost(h);
  for (cudaStream_t s : S->lanes) cudaStreamDestroy(s);
  if (S->pool) cudaMemPoolDestroy(S->pool);
  pp_ctx_destroy(S->ctx);
  delete S;
}

}  // extern "C"
