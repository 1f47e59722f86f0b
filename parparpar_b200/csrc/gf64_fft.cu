// Additive FFT over GF(2^64) in the novel-polynomial basis on the Cantor
// basis (sm_100a), batched.
//
// Semantics: gf64_addfft64_{fwd,inv}_recursive_scratch
// (reference gf64/gf64_additive_fft_hqc2026.c:1656-1705):
//   forward = monomial -> novel-polynomial basis conversion (hqc_cvt, an
//             XOR-only network, :1011-1017) followed by radix-2 butterflies
//             (butterfly_fwd, :1068-1086) with affine shift v_{n/2};
//   inverse = inverse butterflies (:1088-1108), then the inverse conversion.
//
// Layout: `batch` polynomials of n = 2^L coefficients, coefficient c of
// polynomial b at data[c * ld + b] (the batch index is the fast axis: one
// polynomial per word position of a block set).
//
// The operations, on row indices r in [0, n):
//   * conversion phase (polylen, sh, sl), dd = sh - sl, inside every aligned
//     block of polylen rows, rows r in [sl, polylen - dd):
//       forward (the reference's descending in-place loop)
//         d[r] ^= d[r + dd], r descending
//       inverse (ascending)  d[r] ^= d[r + dd]
//   * butterfly depth d, on bit k = L-1-d, block t = r >> (k+1), twiddle
//     w = v_{2^d XOR 2t} (v_j = XOR of the Cantor basis vectors at the set
//     bits of j); forward lo = f[r] ^ w*f[r+h], f[r+h] ^= lo, f[r] = lo;
//     inverse fh = f[r] ^ f[r+h], f[r] ^= w*fh, f[r+h] = fh   (h = 2^k).
//
// Pass plan (host).  The conversion recursion sched(lb, pl) (hqc_cvt's call
// tree) emits its top phases, then recurses into sched(lb, si) and
// sched(lb+si, pl-si).  Every phase of sched(lb, pl) XORs rows that differ
// only in bits [lb, lb+pl) and its condition depends only on those bits, so
// a subtree acts identically along all other bits, and the two children act
// on disjoint bit ranges and commute.  Hence:
//   * a subtree of at most kTileBits bits runs as one tile pass: a CTA loads
//     the 2^p rows that vary in those bits (stride 2^lb) for 8 polynomials
//     into shared memory and applies all its phases there;
//   * the top phases of wider nodes run as global passes, in place, one
//     thread per chain {r, r+dd, r+2dd, ...} of a column, so every element
//     is read and written once;
//   * the butterflies of kTileBits consecutive bits run as one tile pass
//     (high bits first for the forward transform).
// For n = 2^17: 9 global conversion passes + 2 conversion tiles + 2
// butterfly tiles, in place (13 passes over the data).
#include <algorithm>
#include <mutex>
#include <vector>

#include "pp_common.cuh"
#include "pp_internal.h"

namespace pp {
namespace fft {

// Cantor basis of GF(2^64) for x^64+x^4+x^3+x+1: v_0 = 1,
// v_{i+1}^2 + v_{i+1} = v_i (the reference's table, gf64/gf64_cantor_basis.h:23-44).
static const uint64_t kCantor[20] = {
    0x0000000000000001ULL, 0x19c9369f278adc02ULL, 0xa181e7d66f5ff794ULL, 0x5db84357ce785d08ULL,
    0xb973d466f5c9d0caULL, 0x521ac889831a075eULL, 0x033ce8beddc8a656ULL, 0xb5846c4e07b91010ULL,
    0x4087b8cbb37a32ecULL, 0x00d0d3888c0ae17cULL, 0xafd5ac70237f2222ULL, 0xe3f5af99cc3aaaf8ULL,
    0x5a1db3b16a0b58b8ULL, 0x09947c54fe7ee248ULL, 0x0e8eaf0e0068f544ULL, 0xa2a113500b4b4f5aULL,
    0xe96f9805d6ce0bb0ULL, 0x53496f8b5c9edd4cULL, 0xad325cb6f4ac2a9eULL, 0x4a8dcf8bd7ede826ULL,
};

// v_j for j < 2^20 = tw[j & 1023] ^ tw[1024 + (j >> 10)]: two tables of the
// XOR combinations of kCantor[0..9] and kCantor[10..19], written once per
// device by the host (upload_twiddles)
__device__ uint64_t g_tw[2048];

PP_D uint64_t cantor_v(uint32_t j) { return __ldg(&g_tw[j & 1023]) ^ __ldg(&g_tw[1024 + (j >> 10)]); }

constexpr int kTileBits = 9;   // at most 512 rows per tile
constexpr int kTileCols = 8;   // polynomials per tile (64-byte row segments)
constexpr int kTileThreads = 256;
constexpr int kMaxChain = 8;   // dd >= polylen / 4: chains have at most 4 rows
constexpr int kMaxOps = 32;

struct TileOp {
  int32_t kind;  // 0: conversion phase, 1: butterfly
  uint32_t a, b, c;  // phase: local polylen, dd, sl;  butterfly: local bit, global bit, depth
};
struct TilePlan {
  uint32_t lo, p, L, n_ops;
  int32_t inverse;
  uint32_t col_tiles;  // kTileCols-wide column chunks per row
  TileOp op[kMaxOps];
};

// One conversion phase over the whole array, in place: one thread per
// (chain, polynomial); a chain is {base + rho + k*dd} inside one aligned
// block of polylen rows (n <= 2^20, so chain indices fit 32 bits).
__global__ void __launch_bounds__(256) k_fft_cvt_chain(uint64_t* __restrict__ d, size_t n, size_t batch, size_t ld,
                                                       uint32_t polylen, uint32_t dd, uint32_t sl, int inverse,
                                                       uint32_t col_blocks) {
  const uint32_t chain = blockIdx.x / col_blocks;
  const size_t col = (size_t)(blockIdx.x - chain * col_blocks) * blockDim.x + threadIdx.x;
  if (col >= batch) return;
  const uint32_t blk = chain / dd;
  const uint32_t rho = chain - blk * dd;
  const size_t base = (size_t)blk * polylen + rho;
  const uint32_t hi = polylen - dd;  // rows [sl, hi) of the block change
  uint64_t v[kMaxChain];
  uint32_t K = 0;
#pragma unroll
  for (int k = 0; k < kMaxChain; k++)
    if (rho + (uint32_t)k * dd < polylen) {
      v[k] = d[(base + (size_t)k * dd) * ld + col];
      K = k + 1;
    }
  if (!inverse) {
    // descending: d[r] ^= d[r + dd] with d[r + dd] already updated
#pragma unroll
    for (int k = kMaxChain - 2; k >= 0; k--) {
      const uint32_t r = rho + (uint32_t)k * dd;
      if ((uint32_t)k + 1 < K && r >= sl && r < hi) {
        v[k] ^= v[k + 1];
        d[(base + (size_t)k * dd) * ld + col] = v[k];
      }
    }
  } else {
    // ascending: d[r] ^= d[r + dd] with d[r + dd] not yet updated
#pragma unroll
    for (int k = 0; k < kMaxChain - 1; k++) {
      const uint32_t r = rho + (uint32_t)k * dd;
      if ((uint32_t)k + 1 < K && r >= sl && r < hi) d[(base + (size_t)k * dd) * ld + col] = v[k] ^ v[k + 1];
    }
  }
}

// A tile pass: 2^p rows varying in bits [lo, lo+p) (the other bits fixed
// by the tile index) x kTileCols polynomials (the column chunk), in shared
// memory, column-major with a padded column stride.
__global__ void __launch_bounds__(kTileThreads) k_fft_tile(uint64_t* __restrict__ d, size_t n, size_t batch,
                                                           size_t ld, const __grid_constant__ TilePlan P) {
  constexpr uint32_t kStride = (1u << kTileBits) + 1;
  constexpr int kPerThread = (1 << kTileBits) * kTileCols / kTileThreads;  // 16
  __shared__ uint64_t s[kStride * kTileCols];
  const uint32_t p = P.p, T = 1u << p;
  // column chunk fastest: the CTAs resident together cover whole rows
  const uint64_t t = blockIdx.x / P.col_tiles;
  const size_t col0 = (size_t)(blockIdx.x - t * P.col_tiles) * kTileCols;
  const uint64_t low = t & ((1ull << P.lo) - 1), high = t >> P.lo;
  auto row_of = [&](uint32_t u) -> size_t { return low + ((size_t)u << P.lo) + (high << (P.lo + p)); };
  // load: consecutive threads read consecutive polynomials of a row
  for (uint32_t e = threadIdx.x; e < T * kTileCols; e += kTileThreads) {
    const uint32_t u = e >> 3, c = e & 7;
    s[c * kStride + u] = col0 + c < batch ? d[row_of(u) * ld + col0 + c] : 0;
  }
  __syncthreads();
  for (uint32_t oi = 0; oi < P.n_ops; oi++) {
    const TileOp op = P.op[oi];
    if (op.kind == 0) {
      // conversion phase from the old values (at most two links: dd >= polylen / 4)
      const uint32_t PL = op.a, DD = op.b, SL = op.c, HI = PL - DD;
      uint64_t nv[kPerThread];
#pragma unroll
      for (int q = 0; q < kPerThread; q++) {
        const uint32_t e = threadIdx.x + q * kTileThreads;
        nv[q] = 0;
        if (e >= T * kTileCols) continue;
        const uint32_t u = e & (T - 1), c = e >> p;
        const uint32_t r = u & (PL - 1);
        const uint64_t* col = s + c * kStride;
        uint64_t v = col[u];
        if (r >= SL && r < HI) {
          v ^= col[u + DD];
          if (!P.inverse && r + 2 * DD < PL) v ^= col[u + 2 * DD];
        }
        nv[q] = v;
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kPerThread; q++) {
        const uint32_t e = threadIdx.x + q * kTileThreads;
        if (e < T * kTileCols) s[(e >> p) * kStride + (e & (T - 1))] = nv[q];
      }
    } else {
      const uint32_t kl = op.a, kg = op.b, depth = op.c, h = 1u << kl;
      for (uint32_t e = threadIdx.x; e < (T / 2) * kTileCols; e += kTileThreads) {
        const uint32_t pr = e & (T / 2 - 1), c = e >> (p - 1);
        const uint32_t u = ((pr >> kl) << (kl + 1)) | (pr & (h - 1));  // bit kl of u is 0
        const uint64_t tb = row_of(u) >> (kg + 1);                        // block index of the global row
        const uint64_t w = cantor_v((1u << depth) ^ (uint32_t)(2 * tb));
        uint64_t* col = s + c * kStride;
        const uint64_t a = col[u], b = col[u + h];
        if (!P.inverse) {
          const uint64_t lo = a ^ gf64_mul(w, b);
          col[u] = lo;
          col[u + h] = b ^ lo;
        } else {
          const uint64_t fh = a ^ b;
          col[u] = a ^ gf64_mul(w, fh);
          col[u + h] = fh;
        }
      }
    }
    __syncthreads();
  }
  for (uint32_t e = threadIdx.x; e < T * kTileCols; e += kTileThreads) {
    const uint32_t u = e >> 3, c = e & 7;
    if (col0 + c < batch) d[row_of(u) * ld + col0 + c] = s[c * kStride + u];
  }
}

// ------------------------------------------------------------------- plan
struct Phase {
  uint32_t polylen, sh, sl;
};
struct Pass {
  bool tile;
  Phase g;        // global conversion phase
  TilePlan plan;  // tile pass
};

static int choose_si(int pl) {
  int si = 1;
  for (int i = 1; (1 << i) < pl; i++) si = 1 << i;
  return si;
}
// hqc_cvt / hqc_icvt call trees (reference :1011-1026)
static void sched_fwd(int lb, int pl, std::vector<Phase>& out) {
  if (pl <= 1) return;
  const int si = choose_si(pl);
  for (int i = pl - 1; i >= si; i--) out.push_back({1u << (i + lb + 1), 1u << (i + lb), 1u << (i + lb - si)});
  sched_fwd(lb, si, out);
  sched_fwd(lb + si, pl - si, out);
}
static void sched_inv(int lb, int pl, std::vector<Phase>& out) {
  if (pl <= 1) return;
  const int si = choose_si(pl);
  sched_inv(lb, si, out);
  sched_inv(lb + si, pl - si, out);
  for (int i = si; i < pl; i++) out.push_back({1u << (i + lb + 1), 1u << (i + lb), 1u << (i + lb - si)});
}

static Pass tile_pass(uint32_t lo, uint32_t p, uint32_t L, bool inverse) {
  Pass ps{};
  ps.tile = true;
  ps.plan.lo = lo;
  ps.plan.p = p;
  ps.plan.L = L;
  ps.plan.inverse = inverse ? 1 : 0;
  return ps;
}
static void add_cvt_ops(Pass& ps, const std::vector<Phase>& ph, uint32_t lo) {
  for (const Phase& f : ph) {  // every value of the subtree is a multiple of 2^lo
    TileOp& o = ps.plan.op[ps.plan.n_ops++];
    o.kind = 0;
    o.a = f.polylen >> lo;
    o.b = (f.sh - f.sl) >> lo;
    o.c = f.sl >> lo;
  }
}

// conversion: global top phases of wide nodes, one tile per narrow subtree
static void plan_cvt(int lb, int pl, uint32_t L, bool inverse, std::vector<Pass>& out) {
  if (pl <= 1) return;
  if (pl <= kTileBits) {
    std::vector<Phase> ph;
    if (!inverse) sched_fwd(lb, pl, ph);
    else sched_inv(lb, pl, ph);
    Pass ps = tile_pass(lb, pl, L, inverse);
    add_cvt_ops(ps, ph, lb);
    out.push_back(ps);
    return;
  }
  const int si = choose_si(pl);
  std::vector<Phase> top;
  if (!inverse)
    for (int i = pl - 1; i >= si; i--) top.push_back({1u << (i + lb + 1), 1u << (i + lb), 1u << (i + lb - si)});
  else
    for (int i = si; i < pl; i++) top.push_back({1u << (i + lb + 1), 1u << (i + lb), 1u << (i + lb - si)});
  if (!inverse)
    for (const Phase& f : top) out.push_back(Pass{false, f, {}});
  plan_cvt(lb, si, L, inverse, out);
  plan_cvt(lb + si, pl - si, L, inverse, out);
  if (inverse)
    for (const Phase& f : top) out.push_back(Pass{false, f, {}});
}

// butterflies in groups of kTileBits bits: forward from the top bit down
static void plan_bfly(uint32_t L, bool inverse, std::vector<Pass>& out) {
  std::vector<Pass> groups;
  for (int top = (int)L; top > 0; top -= kTileBits) {
    const uint32_t lo = (uint32_t)std::max(0, top - kTileBits), p = (uint32_t)top - lo;
    Pass ps = tile_pass(lo, p, L, inverse);
    if (!inverse) {
      for (int k = top - 1; k >= (int)lo; k--) {  // depth d = L-1-k, ascending
        TileOp& o = ps.plan.op[ps.plan.n_ops++];
        o.kind = 1;
        o.a = (uint32_t)k - lo;
        o.b = (uint32_t)k;
        o.c = L - 1 - (uint32_t)k;
      }
    } else {
      for (int k = (int)lo; k < top; k++) {  // depth descending
        TileOp& o = ps.plan.op[ps.plan.n_ops++];
        o.kind = 1;
        o.a = (uint32_t)k - lo;
        o.b = (uint32_t)k;
        o.c = L - 1 - (uint32_t)k;
      }
    }
    groups.push_back(ps);
  }
  if (inverse) std::reverse(groups.begin(), groups.end());  // low bits first
  for (auto& g : groups) out.push_back(g);
}

// the twiddle tables of the current device (synchronous copy, once per device)
static cudaError_t upload_twiddles() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  std::vector<uint64_t> tw(2048, 0);
  for (uint32_t j = 0; j < 1024; j++)
    for (int k = 0; k < 10; k++)
      if ((j >> k) & 1) {
        tw[j] ^= kCantor[k];
        tw[1024 + j] ^= kCantor[10 + k];
      }
  e = cudaMemcpyToSymbol(g_tw, tw.data(), 2048 * sizeof(uint64_t));
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
  return e;
}

}  // namespace fft

// In place: every pass reads and writes d_data only.
cudaError_t launch_gf64_fft(uint64_t* d_data, size_t n, size_t batch, size_t ld, bool inverse, cudaStream_t s) {
  using namespace fft;
  if (n <= 1 || !batch) return cudaSuccess;
  if (n > ((size_t)1 << 20)) return cudaErrorInvalidValue;  // twiddle indices < 2^20
  cudaError_t te = upload_twiddles();
  if (te != cudaSuccess) return te;
  uint32_t L = 0;
  while (((size_t)1 << L) < n) L++;
  std::vector<Pass> passes;
  if (!inverse) {
    plan_cvt(0, (int)L, L, false, passes);
    plan_bfly(L, false, passes);
  } else {
    plan_bfly(L, true, passes);
    plan_cvt(0, (int)L, L, true, passes);
  }
  const unsigned col_tiles = (unsigned)ceil_div(batch, (size_t)kTileCols);
  const uint32_t col_blocks = (uint32_t)ceil_div(batch, (size_t)256);
  for (Pass& ps : passes) {
    if (ps.tile) {
      const size_t blocks = (n >> ps.plan.p) * col_tiles;
      if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
      ps.plan.col_tiles = col_tiles;
      k_fft_tile<<<(unsigned)blocks, kTileThreads, 0, s>>>(d_data, n, batch, ld, ps.plan);
    } else {
      const uint32_t dd = ps.g.sh - ps.g.sl;
      const size_t chains = (n / ps.g.polylen) * dd;
      if (chains * col_blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
      k_fft_cvt_chain<<<(unsigned)(chains * col_blocks), 256, 0, s>>>(d_data, n, batch, ld, ps.g.polylen, dd,
                                                                     ps.g.sl, inverse ? 1 : 0, col_blocks);
    }
    note_launch();
  }
  return cudaGetLastError();
}

}  // namespace pp
