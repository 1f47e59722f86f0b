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
//     dd >= polylen / 4, so a forward row takes at most two links:
//     new d[r] = d[r] ^ d[r + dd] ^ (d[r + 2 dd] if r + 2 dd < polylen).
//   * butterfly depth d, on bit k = L-1-d, block t = r >> (k+1), twiddle
//     w = v_{2^d XOR 2t} (v_j = XOR of the Cantor basis vectors at the set
//     bits of j); forward lo = f[r] ^ w*f[r+h], f[r+h] ^= lo, f[r] = lo;
//     inverse fh = f[r] ^ f[r+h], f[r] ^= w*fh, f[r+h] = fh   (h = 2^k).
//
// Pass plan (host).  The conversion recursion sched(lb, pl) (hqc_cvt's call
// tree) emits its top phases, then recurses into sched(lb, si) and
// sched(lb+si, pl-si).  Every phase of sched(lb, pl) XORs rows that differ
// only in bits [lb, lb+pl) and its condition depends only on those bits, so
// a subtree acts identically along all other bits (a Kronecker factor), and
// the two children act on disjoint bit ranges and commute.  A butterfly on
// bit k acts identically along the bits below k.  Hence, all in place:
//   * class pass: the top phases of the nodes wider than kTileBits bits
//     (for n <= 2^20: of the root and of its 16-bit child) come first.  They
//     move data by dd = (2^si - 1) 2^j with si a multiple of 8, all
//     multiples of m = 255, so the rows congruent to rho mod m are closed
//     under all of them: one CTA per class and column chunk holds the class
//     (n / 255 rows) in shared memory and applies every such phase (the
//     subtrees below are on disjoint bits and commute with them);
//   * fused tiles: the butterflies run in groups of at most kTileBits
//     consecutive bits, from the top (no group boundary inside a conversion
//     subtree); a conversion subtree on bits X commutes with the butterflies
//     on bits above X, so it runs inside the tile of the group holding X,
//     before that group's butterflies.  A CTA loads the 2^p rows that vary
//     in the group's bits (stride 2^lo) for 8 polynomials into shared memory.
//   The inverse transform runs the same passes in reverse order, each
//   inverted.  n = 2^17: 1 class pass + 2 fused tiles (3 passes over the data).
#include <algorithm>
#include <mutex>
#include <numeric>
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

// w * b for one twiddle w and many b: the masked quarters of w's three
// Karatsuba operands are formed once.  Same products as gf64_mul (32 x 32
// carry-less products by integer multiplies on every 4th bit, Karatsuba over
// the halves, then the reduction).
struct MulByW {
  uint32_t q[3][4];
  PP_D static void split(uint32_t* o, uint32_t a) {
    o[0] = a & 0x11111111u;
    o[1] = a & 0x22222222u;
    o[2] = a & 0x44444444u;
    o[3] = a & 0x88888888u;
  }
  PP_D explicit MulByW(uint64_t w) {
    const uint32_t lo = (uint32_t)w, hi = (uint32_t)(w >> 32);
    split(q[0], lo);
    split(q[1], hi);
    split(q[2], lo ^ hi);
  }
  PP_D static uint64_t wide(uint32_t x, uint32_t y) { return (uint64_t)x * y; }
  PP_D static uint64_t clmul(const uint32_t* a, uint32_t b) {
    const uint32_t b0 = b & 0x11111111u, b1 = b & 0x22222222u, b2 = b & 0x44444444u, b3 = b & 0x88888888u;
    const uint64_t z0 = wide(a[0], b0) ^ wide(a[1], b3) ^ wide(a[2], b2) ^ wide(a[3], b1);
    const uint64_t z1 = wide(a[0], b1) ^ wide(a[1], b0) ^ wide(a[2], b3) ^ wide(a[3], b2);
    const uint64_t z2 = wide(a[0], b2) ^ wide(a[1], b1) ^ wide(a[2], b0) ^ wide(a[3], b3);
    const uint64_t z3 = wide(a[0], b3) ^ wide(a[1], b2) ^ wide(a[2], b1) ^ wide(a[3], b0);
    return (z0 & 0x1111111111111111ull) | (z1 & 0x2222222222222222ull) | (z2 & 0x4444444444444444ull) |
           (z3 & 0x8888888888888888ull);
  }
  PP_D uint64_t mul(uint64_t b) const {
    const uint32_t bl = (uint32_t)b, bh = (uint32_t)(b >> 32);
    const uint64_t lo = clmul(q[0], bl), hi = clmul(q[1], bh);
    const uint64_t mid = clmul(q[2], bl ^ bh) ^ lo ^ hi;
    return gf64_reduce(hi ^ (mid >> 32), lo ^ (mid << 32));
  }
};

constexpr int kTileBits = 9;   // at most 512 rows per tile
constexpr int kTileCols = 8;   // polynomials per tile (64-byte row segments)
constexpr int kTileThreads = 256;
constexpr int kMaxOps = 32;
static_assert((1 << (kTileBits - 1)) <= kTileThreads, "one butterfly pair index per thread");

constexpr int kClassThreads = 288;  // 9 warps: two rows per thread for the 515-row classes of n = 2^17
constexpr uint32_t kClassWords = 5376;  // 42 KiB of shared memory: 2^17 / 255 rows x 8 polynomials, 2^20 / 255 x 1
// words per class row of CC polynomials: the 16-byte chunks of any 8
// consecutive rows fall on distinct bank groups (row strides of 5, 3 and 1
// chunks are odd)
__host__ __device__ constexpr uint32_t class_stride(int CC) { return CC == 8 ? 10 : CC == 4 ? 6 : (uint32_t)CC; }
constexpr int kMaxClassOps = 16;

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

struct ClassOp {
  uint32_t polylen, dd, sl;
};
struct ClassPlan {
  uint32_t m;          // class modulus (every dd is a multiple)
  uint32_t cc_log;     // log2 of the polynomials per CTA
  uint32_t col_tiles;  // column chunks per class
  uint32_t n_ops;
  int32_t inverse;
  ClassOp op[kMaxClassOps];
};

// The class pass: CTA (rho, column chunk) holds rows rho, rho + m, rho + 2m,
// ... (J rows) x CC polynomials in shared memory and applies the phases in
// order, each from the old values (the two-link closed form).  Row j of the
// class starts at word j * class_stride(CC); its partner r + dd is row
// j + dd / m.  Global copies: consecutive threads take consecutive
// polynomials of a row; phases: one row per thread, its condition evaluated
// once for the row.  n <= 2^20, so row indices fit 32 bits.
template <int CC>
__global__ void __launch_bounds__(kClassThreads, 3) k_fft_cvt_class(uint64_t* __restrict__ d, size_t n, size_t batch,
                                                                 size_t ld, const __grid_constant__ ClassPlan P) {
  constexpr uint32_t S = class_stride(CC);
  constexpr int kChunk = CC >= 2 ? 2 : 1;  // words per shared-memory access
  constexpr int kChunks = CC / kChunk;
  constexpr int kRowsPer = (kClassWords / S + kClassThreads - 1) / kClassThreads;
  constexpr uint32_t kStep = kClassThreads / CC;  // rows per copy step
  __shared__ __align__(16) uint64_t s[kClassWords];
  const uint32_t rho = blockIdx.x / P.col_tiles;
  const size_t col0 = (size_t)(blockIdx.x - rho * P.col_tiles) * CC;
  const uint32_t J = min((uint32_t)((n - rho + P.m - 1) / P.m), kClassWords / S);  // the host sizes CC to fit
  const uint32_t c = threadIdx.x % CC, j0 = threadIdx.x / CC;
  const bool col_ok = col0 + c < batch;
  const size_t g0 = (rho + (size_t)P.m * j0) * ld + col0 + c, gstep = (size_t)P.m * kStep * ld;
  {
    size_t gi = g0;
    // unrolled: several loads in flight per thread
#pragma unroll 8
    for (uint32_t j = j0, si = j0 * S + c; j < J; j += kStep, si += kStep * S, gi += gstep) s[si] = col_ok ? d[gi] : 0;
  }
  __syncthreads();
  for (uint32_t oi = 0; oi < P.n_ops; oi++) {
    const ClassOp op = P.op[oi];
    const uint32_t qr = op.dd / P.m;  // partner distance in rows
    uint64_t nv[kRowsPer][CC];
    bool chg[kRowsPer];
#pragma unroll
    for (int k = 0; k < kRowsPer; k++) {
      const uint32_t j = threadIdx.x + k * kClassThreads;
      const uint32_t r = (rho + P.m * j) & (op.polylen - 1);
      chg[k] = j < J && r >= op.sl && r + op.dd < op.polylen && j + qr < J;
      if (!chg[k]) continue;
      const bool two = !P.inverse && r + 2 * op.dd < op.polylen && j + 2 * qr < J;
      const uint64_t* a0 = s + j * S;
      const uint64_t* a1 = a0 + qr * S;
      const uint64_t* a2 = a1 + qr * S;
#pragma unroll
      for (int x = 0; x < kChunks; x++) {
        if constexpr (kChunk == 2) {
          ulonglong2 v = *reinterpret_cast<const ulonglong2*>(a0 + 2 * x);
          const ulonglong2 p = *reinterpret_cast<const ulonglong2*>(a1 + 2 * x);
          v.x ^= p.x;
          v.y ^= p.y;
          if (two) {
            const ulonglong2 q = *reinterpret_cast<const ulonglong2*>(a2 + 2 * x);
            v.x ^= q.x;
            v.y ^= q.y;
          }
          nv[k][kChunk * x] = v.x;
          nv[k][(kChunk * x + 1) % CC] = v.y;
        } else {
          uint64_t v = a0[x] ^ a1[x];
          if (two) v ^= a2[x];
          nv[k][x] = v;
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kRowsPer; k++) {
      if (!chg[k]) continue;
      uint64_t* a0 = s + (threadIdx.x + k * kClassThreads) * S;
#pragma unroll
      for (int x = 0; x < kChunks; x++) {
        if constexpr (kChunk == 2)
          *reinterpret_cast<ulonglong2*>(a0 + 2 * x) = make_ulonglong2(nv[k][2 * x], nv[k][(2 * x + 1) % CC]);
        else
          a0[x] = nv[k][x];
      }
    }
    __syncthreads();
  }
  if (!col_ok) return;
  size_t gi = g0;
  for (uint32_t j = j0, si = j0 * S + c; j < J; j += kStep, si += kStep * S, gi += gstep) d[gi] = s[si];
}

// A tile pass: 2^p rows varying in bits [lo, lo+p) (the other bits fixed
// by the tile index) x kTileCols polynomials (the column chunk), in shared
// memory, column-major with a padded column stride.  Conversion phases and
// butterflies in the order of the plan.
__global__ void __launch_bounds__(kTileThreads, 3) k_fft_tile(uint64_t* __restrict__ d, size_t n, size_t batch,
                                                           size_t ld, const __grid_constant__ TilePlan P) {
  constexpr uint32_t kStride = (1u << kTileBits) + 1;
  constexpr int kRowsPerThread = (1 << kTileBits) / kTileThreads;  // 2
  __shared__ uint64_t s[kStride * kTileCols];
  const uint32_t p = P.p, T = 1u << p;
  // column chunk fastest: the CTAs resident together cover whole rows
  const uint64_t t = blockIdx.x / P.col_tiles;
  const size_t col0 = (size_t)(blockIdx.x - t * P.col_tiles) * kTileCols;
  const uint64_t low = t & ((1ull << P.lo) - 1), high = t >> P.lo;
  auto row_of = [&](uint32_t u) -> size_t { return low + ((size_t)u << P.lo) + (high << (P.lo + p)); };
  // load: consecutive threads read consecutive polynomials of a row
#pragma unroll 8
  for (uint32_t e = threadIdx.x; e < T * kTileCols; e += kTileThreads) {
    const uint32_t u = e >> 3, c = e & 7;
    s[c * kStride + u] = col0 + c < batch ? d[row_of(u) * ld + col0 + c] : 0;
  }
  __syncthreads();
  // butterflies: one pair index per thread (p <= kTileBits, so T / 2 <= the
  // thread count), its twiddle shared by the columns the thread takes
  const uint32_t pr = threadIdx.x & ((T >> 1) - 1);
  const uint32_t c_first = threadIdx.x >> (p - 1), c_step = kTileThreads >> (p - 1);
  for (uint32_t oi = 0; oi < P.n_ops; oi++) {
    const TileOp op = P.op[oi];
    if (op.kind == 0) {
      // conversion phase from the old values (at most two links): one row
      // per thread, all kTileCols polynomials; only changed rows are stored
      const uint32_t PL = op.a, DD = op.b, SL = op.c, HI = PL - DD;
      uint64_t nv[kRowsPerThread][kTileCols];
      bool chg[kRowsPerThread];
#pragma unroll
      for (int k = 0; k < kRowsPerThread; k++) {
        const uint32_t u = threadIdx.x + k * kTileThreads;
        const uint32_t r = u & (PL - 1);
        chg[k] = u < T && r >= SL && r < HI;
        if (!chg[k]) continue;
        const bool two = !P.inverse && r + 2 * DD < PL;
#pragma unroll
        for (int c = 0; c < kTileCols; c++) {
          const uint64_t* col = s + c * kStride;
          uint64_t v = col[u] ^ col[u + DD];
          if (two) v ^= col[u + 2 * DD];
          nv[k][c] = v;
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kRowsPerThread; k++) {
        if (!chg[k]) continue;
        const uint32_t u = threadIdx.x + k * kTileThreads;
#pragma unroll
        for (int c = 0; c < kTileCols; c++) s[c * kStride + u] = nv[k][c];
      }
    } else if (c_first < kTileCols) {
      const uint32_t kl = op.a, kg = op.b, depth = op.c, h = 1u << kl;
      const uint32_t u = ((pr >> kl) << (kl + 1)) | (pr & (h - 1));  // bit kl of u is 0
      const uint64_t tb = row_of(u) >> (kg + 1);                        // block index of the global row
      const MulByW W(cantor_v((1u << depth) ^ (uint32_t)(2 * tb)));
      for (uint32_t c = c_first; c < kTileCols; c += c_step) {
        uint64_t* col = s + c * kStride;
        const uint64_t a = col[u], b = col[u + h];
        if (!P.inverse) {
          const uint64_t lo = a ^ W.mul(b);
          col[u] = lo;
          col[u + h] = b ^ lo;
        } else {
          const uint64_t fh = a ^ b;
          col[u] = a ^ W.mul(fh);
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
struct CvtTile {  // a conversion subtree of at most kTileBits bits
  uint32_t lb, pl;
  std::vector<Phase> ph;
};
struct Pass {
  bool tile;
  ClassPlan cls;  // class pass
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

// The conversion as the top phases of the wide nodes (in their order) and
// the narrow subtrees.
static void collect_cvt(int lb, int pl, bool inverse, std::vector<Phase>& wide, std::vector<CvtTile>& tiles) {
  if (pl <= 1) return;
  if (pl <= kTileBits) {
    CvtTile t{(uint32_t)lb, (uint32_t)pl, {}};
    if (!inverse) sched_fwd(lb, pl, t.ph);
    else sched_inv(lb, pl, t.ph);
    tiles.push_back(std::move(t));
    return;
  }
  const int si = choose_si(pl);
  std::vector<Phase> top;
  if (!inverse)
    for (int i = pl - 1; i >= si; i--) top.push_back({1u << (i + lb + 1), 1u << (i + lb), 1u << (i + lb - si)});
  else
    for (int i = si; i < pl; i++) top.push_back({1u << (i + lb + 1), 1u << (i + lb), 1u << (i + lb - si)});
  if (!inverse) wide.insert(wide.end(), top.begin(), top.end());
  collect_cvt(lb, si, inverse, wide, tiles);
  collect_cvt(lb + si, pl - si, inverse, wide, tiles);
  if (inverse) wide.insert(wide.end(), top.begin(), top.end());
}

static bool add_op(TilePlan& tp, int32_t kind, uint32_t a, uint32_t b, uint32_t c) {
  if (tp.n_ops >= (uint32_t)kMaxOps) return false;
  tp.op[tp.n_ops++] = TileOp{kind, a, b, c};
  return true;
}
// a subtree's phases in the tile's local row units (every value of the
// subtree is a multiple of 2^lo)
static bool add_cvt_ops(TilePlan& tp, const CvtTile& t, uint32_t lo) {
  for (const Phase& f : t.ph)
    if (!add_op(tp, 0, f.polylen >> lo, (f.sh - f.sl) >> lo, f.sl >> lo)) return false;
  return true;
}
// butterflies of bits [lo, top): forward from the top bit down (depth
// d = L-1-k ascending), inverse from the bottom bit up
static bool add_bfly_ops(TilePlan& tp, uint32_t lo, uint32_t top, uint32_t L, bool inverse) {
  for (uint32_t i = 0; i < top - lo; i++) {
    const uint32_t k = inverse ? lo + i : top - 1 - i;
    if (!add_op(tp, 1, k - lo, k, L - 1 - k)) return false;
  }
  return true;
}

static bool make_plan(uint32_t L, size_t n, bool inverse, std::vector<Pass>& out) {
  std::vector<Phase> wide;
  std::vector<CvtTile> tiles;
  collect_cvt(0, (int)L, inverse, wide, tiles);
  // fused tiles, top group first
  std::vector<Pass> fused;
  for (uint32_t top = L; top > 0;) {
    uint32_t lo = top > (uint32_t)kTileBits ? top - kTileBits : 0;
    for (const CvtTile& t : tiles)
      if (t.lb < lo && lo < t.lb + t.pl) lo = t.lb + t.pl;  // keep each subtree in one group
    if (lo >= top) return false;
    Pass ps{};
    ps.tile = true;
    ps.plan.lo = lo;
    ps.plan.p = top - lo;
    ps.plan.L = L;
    ps.plan.inverse = inverse ? 1 : 0;
    if (inverse && !add_bfly_ops(ps.plan, lo, top, L, true)) return false;
    for (const CvtTile& t : tiles)
      if (t.lb >= lo && t.lb + t.pl <= top && !add_cvt_ops(ps.plan, t, lo)) return false;
    if (!inverse && !add_bfly_ops(ps.plan, lo, top, L, false)) return false;
    fused.push_back(ps);
    top = lo;
  }
  // the class pass of the wide nodes' phases
  Pass cls{};
  if (!wide.empty()) {
    if (wide.size() > (size_t)kMaxClassOps) return false;
    uint32_t m = 0;
    for (const Phase& f : wide) m = std::gcd(m, f.sh - f.sl);
    const size_t J = (n + m - 1) / m;
    if (m < 2 || J > kClassWords) return false;
    uint32_t cc_log = 3;
    while (cc_log > 0 && J * class_stride(1 << cc_log) > kClassWords) cc_log--;
    cls.tile = false;
    cls.cls.m = m;
    cls.cls.cc_log = cc_log;
    cls.cls.n_ops = (uint32_t)wide.size();
    cls.cls.inverse = inverse ? 1 : 0;
    for (size_t i = 0; i < wide.size(); i++) cls.cls.op[i] = ClassOp{wide[i].polylen, wide[i].sh - wide[i].sl, wide[i].sl};
  }
  if (!inverse) {
    if (!wide.empty()) out.push_back(cls);
    out.insert(out.end(), fused.begin(), fused.end());
  } else {
    out.insert(out.end(), fused.rbegin(), fused.rend());
    if (!wide.empty()) out.push_back(cls);
  }
  return true;
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
  if (!make_plan(L, n, inverse, passes)) return cudaErrorInvalidValue;
  const unsigned col_tiles = (unsigned)ceil_div(batch, (size_t)kTileCols);
  for (Pass& ps : passes) {
    if (ps.tile) {
      const size_t blocks = (n >> ps.plan.p) * col_tiles;
      if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
      ps.plan.col_tiles = col_tiles;
      k_fft_tile<<<(unsigned)blocks, kTileThreads, 0, s>>>(d_data, n, batch, ld, ps.plan);
    } else {
      ps.cls.col_tiles = (uint32_t)ceil_div(batch, (size_t)1 << ps.cls.cc_log);
      const size_t blocks = (size_t)ps.cls.m * ps.cls.col_tiles;
      if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
      switch (ps.cls.cc_log) {
        case 3: k_fft_cvt_class<8><<<(unsigned)blocks, kClassThreads, 0, s>>>(d_data, n, batch, ld, ps.cls); break;
        case 2: k_fft_cvt_class<4><<<(unsigned)blocks, kClassThreads, 0, s>>>(d_data, n, batch, ld, ps.cls); break;
        case 1: k_fft_cvt_class<2><<<(unsigned)blocks, kClassThreads, 0, s>>>(d_data, n, batch, ld, ps.cls); break;
        default: k_fft_cvt_class<1><<<(unsigned)blocks, kClassThreads, 0, s>>>(d_data, n, batch, ld, ps.cls); break;
      }
    }
    note_launch();
  }
  return cudaGetLastError();
}

}  // namespace pp
