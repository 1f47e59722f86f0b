// Job tables of the tensor-core region kernels (gf16_tc.cu,
// gf64_tc.cu).  One launch runs up to kTcMaxJobs independent region products
// out[o][w] (^)= XOR_i c[o][i] * in_i[w] of different shapes.
//
// Work decomposition: a job is tiles (CTA output tile x word tile) times
// stages (input groups).  Each job's stage range is cut into `splits` equal
// parts, giving items (split, word tile, output group), output group fastest.
// Item k runs as CTA k.  The block scheduler starts CTAs in index order, so
// the CTAs resident at one time work on the same stage range of neighbouring
// tiles: the output groups of a word tile share its input rows, and the
// word tiles of a group share its coefficient tiles, through L2.  The split
// counts are chosen on the host so that the items fill whole waves of SMs.  A job cut into more
// than one split XORs its partial results atomically, so its outputs must be
// zero before the launch unless it accumulates.
//
// The table is a kernel parameter (__grid_constant__, < 4 KiB), so a launch
// needs no device-side descriptor memory and is captured as-is in CUDA graphs.
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace pp {

constexpr int kTcMaxJobs = 24;

struct Gf16TcJob {
  const uint8_t* in;      // input row i at in + i * in_stride (bytes)
  size_t in_stride;
  const uint8_t* a_exp;   // expanded coefficient tiles (launch_gf16_tc_expand)
  uint8_t* out;           // output row o at out + o * out_stride
  size_t out_stride;
  size_t slice_bytes;
  uint32_t n_in, n_out;
  uint32_t n_stages;      // ceil(n_in / 8)
  uint32_t groups;        // ceil(n_out / 8)
  uint32_t wt;            // word tiles: ceil(words / 512)
  uint32_t accumulate;
  uint32_t splits, per;   // stage range cut into `splits` parts of `per` stages
  uint32_t a_stride;      // stages per output group in a_exp (0: n_stages); a job over a
                          // column range of a larger coefficient matrix points a_exp at its
                          // first stage and keeps the whole matrix's stride
  uint32_t reserved;
};

struct Gf64TcJob {
  const uint64_t* in;                 // row i: in_ptrs ? in_ptrs[i] : in + i * in_stride (words)
  const uint64_t* const* in_ptrs;
  size_t in_stride;
  const uint64_t* coeff;              // c[o][i] = coeff[o * ldc + i]
  size_t ldc;
  uint64_t* out;                      // row o: out_ptrs ? out_ptrs[o] : out + o * out_stride
  uint64_t* const* out_ptrs;
  size_t out_stride;
  size_t words;
  uint32_t n_in, n_out;
  uint32_t n_stages;                  // ceil(n_in / 2)
  uint32_t pairs;                     // output groups of a tile: ceil(n_out / 2), or
                                      // ceil(n_out / 4) for the CTA-pair kernel
  uint32_t wt;                        // ceil(words / 512)
  uint32_t accumulate;
  uint32_t splits, per;               // stage range cut into `splits` parts of `per` stages
  uint32_t n_mma;                     // FP4 pair kernel: the MMA's N (words per CTA; a tile is 2 n_mma words)
  uint32_t reserved;
};

template <class Job>
struct TcBatch {
  uint32_t n_jobs;
  uint32_t q_hint;                    // host: target stages per item, 0 = chosen by the estimate;
                                      // tc_batch_plan leaves the value it used here
  uint64_t total;                     // items of all jobs
  uint64_t prefix[kTcMaxJobs + 1];    // items before job j
  Job job[kTcMaxJobs];
};
using Gf16TcBatch = TcBatch<Gf16TcJob>;
using Gf64TcBatch = TcBatch<Gf64TcJob>;
static_assert(sizeof(Gf16TcBatch) < 4000 && sizeof(Gf64TcBatch) < 4000, "job table must stay a small kernel parameter");

// Host side.  Estimated time of a plan in stage units: items dealt to the SMs
// in order (round robin, the steady state of the block scheduler with one
// resident CTA per SM), each item its stages plus a fixed epilogue /
// pipeline-fill cost.
constexpr uint64_t kTcItemOverhead = 8;

// max_per: at most this many stages per item (0: no limit) -- an fp32
// accumulator counts exactly only up to 2^24, so the FP4 kernels bound the
// inputs one item sums
template <class Job>
inline void tc_set_splits(Job& J, uint32_t splits, uint32_t max_per = 0) {
  if (max_per && splits < (J.n_stages + max_per - 1) / max_per) splits = (J.n_stages + max_per - 1) / max_per;
  if (splits < 1) splits = 1;
  if (splits > J.n_stages) splits = J.n_stages;
  J.per = (J.n_stages + splits - 1) / splits;
  J.splits = (J.n_stages + J.per - 1) / J.per;
}

template <class Job>
inline uint64_t tc_batch_estimate(TcBatch<Job>& b, uint64_t tiles_of(const Job&), unsigned ctas,
                                  std::vector<int64_t>& diff) {
  // load of CTA c = base + prefix sum of diff (cyclic ranges of the round robin)
  diff.assign(ctas + 1, 0);
  uint64_t base = 0, k = 0;
  for (uint32_t j = 0; j < b.n_jobs; j++) {
    const Job& J = b.job[j];
    const uint64_t t = tiles_of(J);
    for (uint32_t sp = 0; sp < J.splits; sp++) {
      const int64_t len = (int64_t)std::min<uint64_t>(J.per, J.n_stages - (uint64_t)sp * J.per) + kTcItemOverhead;
      // t consecutive items of this length from CTA k mod ctas on
      base += (t / ctas) * (uint64_t)len;
      const uint64_t rem = t % ctas, end = k + rem;
      if (rem) {
        diff[k] += len;
        if (end <= ctas) {
          diff[end] -= len;
        } else {
          diff[ctas] -= len;
          diff[0] += len;
          diff[end - ctas] -= len;
        }
      }
      k = (k + t) % ctas;
    }
  }
  int64_t run = 0, mx = 0;
  for (unsigned c = 0; c < ctas; c++) {
    run += diff[c];
    mx = std::max(mx, run);
  }
  return base + (uint64_t)mx;
}

// Choose every job's split count (one target item length for the whole
// table), fill prefix/total and return the grid size (one CTA per item).
template <class Job>
inline uint64_t tc_batch_plan(TcBatch<Job>& b, uint64_t tiles_of(const Job&), int sms, uint32_t max_per = 0) {
  const unsigned ctas = (unsigned)(sms > 0 ? sms : 148);
  uint32_t smax = 1;
  for (uint32_t j = 0; j < b.n_jobs; j++) smax = std::max(smax, b.job[j].n_stages);
  std::vector<int64_t> load;
  uint64_t best = ~0ull;
  uint32_t best_q = smax;
  for (uint32_t d = 1; d <= 256 && !b.q_hint; d++) {
    const uint32_t q = (smax + d - 1) / d;  // target stages per item
    if (d > 1 && q == (smax + d - 2) / (d - 1)) continue;
    for (uint32_t j = 0; j < b.n_jobs; j++) tc_set_splits(b.job[j], (b.job[j].n_stages + q - 1) / q, max_per);
    const uint64_t est = tc_batch_estimate(b, tiles_of, ctas, load);
    if (est < best) {
      best = est;
      best_q = q;
    }
    if (q <= 1) break;
  }
  if (b.q_hint) best_q = b.q_hint;
  b.q_hint = best_q;
  for (uint32_t j = 0; j < b.n_jobs; j++)
    tc_set_splits(b.job[j], (b.job[j].n_stages + best_q - 1) / best_q, max_per);
  b.total = 0;
  for (uint32_t j = 0; j < b.n_jobs; j++) {
    b.prefix[j] = b.total;
    b.total += tiles_of(b.job[j]) * b.job[j].splits;
  }
  b.prefix[b.n_jobs] = b.total;
  return b.total;
}

}  // namespace pp

#ifdef __CUDACC__
namespace pp {

// One item: stages [st0, st1) of tile `tile` of job `job`; mode 0 store,
// 1 xor into the output, 2 atomic xor (the job is split over CTAs).
struct TcSeg {
  uint32_t job;
  uint32_t st0, st1;
  int mode;
  uint64_t tile;
};

// Copy of a job descriptor held in registers.  The table lives in the
// read-only parameter space; indexed at run time, a plain copy may be
// re-loaded from there at every use inside the stage loops, so each word is
// passed through an empty asm that the compiler cannot re-derive.
template <class Job>
__device__ __forceinline__ Job pinned_job(const Job& src) {
  static_assert(sizeof(Job) % 4 == 0, "job descriptors are whole 32-bit words");
  Job j;
  const uint32_t* s = reinterpret_cast<const uint32_t*>(&src);
  uint32_t* d = reinterpret_cast<uint32_t*>(&j);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(Job) / 4); i++) {
    uint32_t v = s[i];
    asm volatile("" : "+r"(v));
    d[i] = v;
  }
  return j;
}

// Decode item k of the table.
template <class Job>
__device__ __forceinline__ TcSeg tc_item(const TcBatch<Job>* b, uint64_t k) {
  uint32_t j = 0;
  while (j + 1 < b->n_jobs && b->prefix[j + 1] <= k) j++;
  const uint64_t local = k - b->prefix[j];
  const uint32_t splits = b->job[j].splits, per = b->job[j].per, n_stages = b->job[j].n_stages;
  const uint64_t tiles = (b->prefix[j + 1] - b->prefix[j]) / splits;
  const uint32_t sp = (uint32_t)(local / tiles);
  TcSeg s;
  s.job = j;
  s.tile = local % tiles;
  s.st0 = sp * per;
  s.st1 = min(n_stages, s.st0 + per);
  s.mode = splits == 1 ? (b->job[j].accumulate ? 1 : 0) : 2;
  return s;
}

}  // namespace pp
#endif
