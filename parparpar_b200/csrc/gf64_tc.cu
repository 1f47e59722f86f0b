// GF(2^64) region multiply-accumulate on the tensor cores (tcgen05,
// kind::i8), sm_100a:  out[r][w] ^= XOR_i M[r][i] * in_i[w].
//
// As for GF(2^16) (gf16_tc.cu), bit b of c*x is the parity of
// sum_e bit_e(x) * bit_b(c * x^e), and an exact integer MMA over bytes keeps
// that parity if only the lowest bit of each byte carries information:
//   parity(sum_k A_k * B_k) = sum_k lsb(A_k) * lsb(B_k)   (mod 2)
// holds for ANY bytes A_k, B_k (the other bits contribute even amounts, and
// the int32 accumulator wraps modulo 2^32, which keeps the parity).  So both
// operands are plain 32-bit shifts of packed values:
//   B[w][(j, ii, beta)] = byte_beta(x_ii[w] >> j)    data, shift j = 0..7
//   A[(o,b)][(j, ii, beta)] = byte_beta(Q_{o,ii,b} >> j)
// where Q_{o,ii,b} has bit e = bit b of (M[o][ii] * x^e), i.e. row b of the
// 64x64 GF(2) matrix of multiplication by the coefficient.  The lowest bit of
// byte beta of (v >> j) is bit 8*beta + j of v, so the contraction runs over
// all 64 bits e = 8*beta + j of the input word.
//
// CTA tile: 2 outputs (M = 128 rows = 2 x 64 bits) x 512 words (two MMAs of
// N = 256); a stage is 2 inputs (K = 128 bytes = 8 shifts x 2 inputs x 8
// bytes, four K = 32 MMA steps).
//
//   warp 0      producer: cp.async.bulk of the 2 raw input rows of the tile
//   warp 1      TMEM allocation + one thread issuing tcgen05.mma
//   warps 2-9   per stage: each thread builds one (row, input) half-chunk of
//               the A tile from its coefficient with the closed form below
//               and writes the B rows of two words; then the epilogue (TMEM
//               counts -> parity -> ballot -> 32-bit halves of the output words)
//
// Closed form of the rows: with r = bitreverse(c) and x^64 = x^4+x^3+x+1,
//   Q_b = (r >> (63-b)) ^ XOR_{s in {0,1,3,4}, d = b-s >= 0}
//           [ (r << (d+1)) (d+1 < 64) ^ (r << (d+61)) (d <= 2) ^ (r << (d+62)) (d <= 1) ]
// (the unreduced product c << e contributes r >> (63-b); each reduction term
// s of x^64 contributes the bits of c >> (64-e) that land on bit b, and the
// second fold of the top bits contributes the (d+61), (d+62) terms).
//
// Every mbarrier wait is bounded (about one second); on a timeout the CTA
// records an error in *status, drains its copies and MMAs, frees TMEM and
// returns.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "pp_common.cuh"
#include "pp_internal.h"
#include "tc_batch.h"
#include "tc_common.cuh"

namespace pp {
// Input-row addresses of a stage for the producer thread.  With a pointer
// table (repair: lost rows point at a zero row) each address is a load from
// global memory; the producer loads the next stage's addresses while this
// stage's copies go out, so their latency stays off its path (issued one
// after another in front of each copy, the loads took longer than a stage).
template <int S>
struct StageRows {
  const uint64_t* p[S];
  __device__ __forceinline__ void load(const Gf64TcJob& J, unsigned st) {
#pragma unroll
    for (int ii = 0; ii < S; ii++) {
      const unsigned i = st * S + ii;
      p[ii] = i < J.n_in ? (J.in_ptrs ? J.in_ptrs[i] : J.in + (size_t)i * J.in_stride) : nullptr;
    }
  }
};

namespace tc64 {
using namespace pp::tc;

constexpr int kWords = 512;
constexpr int kStageIn = 2;
constexpr int kABytes = 128 * 128;              // 16 KiB
constexpr int kBBytes = kWords * 128;           // 64 KiB
constexpr int kRawBytes = kStageIn * kWords * 8;  // 8 KiB
constexpr int kLd = 4;                          // raw-row ring
constexpr int kBs = 2;                          // operand (A + B) ring
constexpr int kThreads = 320;
constexpr int kExp = 256;
constexpr int kOffA = 0;
constexpr int kOffB = kBs * kABytes;              // 32 KiB
constexpr int kOffRaw = kOffB + kBs * kBBytes;    // 160 KiB
constexpr int kOffBar = kOffRaw + kLd * kRawBytes;  // 192 KiB
constexpr int kSmemBytes = kOffBar + 256 + 1024;
constexpr uint32_t kIdesc = (2u << 4) | ((256u >> 3) << 17) | ((128u >> 4) << 24);

// Row b of the 64x64 GF(2) matrix of multiplication by c: bit e is bit b of
// c * x^e (closed form, see the header).
PP_D uint64_t mul_matrix_row(uint64_t c, unsigned b) {
  const uint64_t rv = __brevll(c);
  uint64_t qrow = rv >> (63 - b);
#pragma unroll
  for (int si = 0; si < 4; si++) {
    const int sft = si == 0 ? 0 : si == 1 ? 1 : si == 2 ? 3 : 4;
    const int d = (int)b - sft;
    if (d >= 0) {
      if (d + 1 < 64) qrow ^= rv << (d + 1);
      if (d <= 2) qrow ^= rv << (d + 61);
      if (d <= 1) qrow ^= rv << (d + 62);
    }
  }
  return qrow;
}

// One CTA per work item of the job table (tc_batch.h): the item fixes the
// job, the output pair, the word tile and the stage range; mode 0 stores,
// 1 XORs into the output, 2 XORs atomically (the job is split over CTAs).
__global__ void __launch_bounds__(kThreads, 1)
k_gf64_matvec_tc(const __grid_constant__ Gf64TcBatch batch, int* __restrict__ status) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t base_s = smem_addr(smem_raw);
  const uint32_t pad = ((base_s + 1023) & ~1023u) - base_s;
  uint8_t* smem = smem_raw + pad;
  const uint32_t sA = base_s + pad + kOffA, sB = base_s + pad + kOffB, sRaw = base_s + pad + kOffRaw;
  const uint32_t bar0 = smem_addr(smem + kOffBar);
  enum {
    RAW_FULL = 0,
    RAW_EMPTY = RAW_FULL + kLd,
    OP_FULL = RAW_EMPTY + kLd,
    OP_EMPTY = OP_FULL + kBs,
    D_FULL = OP_EMPTY + kBs,
    DONE = D_FULL + 1,
    NBARS = DONE + 1
  };
  static_assert(8 * NBARS + 16 <= 256, "barrier area");
  auto BAR = [&](int k) { return bar0 + 8u * (uint32_t)k; };
  volatile uint32_t* tmem_holder = reinterpret_cast<volatile uint32_t*>(smem + kOffBar + 8 * NBARS);
  volatile int* err = reinterpret_cast<volatile int*>(smem + kOffBar + 8 * NBARS + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int k = 0; k < NBARS; k++) {
      const bool by_expanders = (k >= RAW_EMPTY && k < RAW_EMPTY + kLd) || (k >= OP_FULL && k < OP_FULL + kBs);
      mbar_init(BAR(k), by_expanders ? (uint32_t)kExp : 1u);
    }
    *err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr((const void*)tmem_holder)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  const TcSeg sg = tc_item(&batch, blockIdx.x);

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      uint32_t g = 0;  // stages issued by this CTA
      do {  // the CTA's one item
        const Gf64TcJob J = pinned_job(batch.job[sg.job]);
        const size_t w0 = (size_t)(sg.tile / J.pairs) * kWords;
        const unsigned words_valid = (unsigned)min((size_t)kWords, J.words - w0);
        const uint32_t raw_copy = (uint32_t)(((size_t)words_valid * 8 + 15) & ~(size_t)15);
        StageRows<kStageIn> rows, next;
        rows.load(J, sg.st0);
        for (unsigned st = sg.st0; st < sg.st1; st++, g++) {
          const unsigned sl = g % kLd;
          next.load(J, st + 1);
          if (g >= (uint32_t)kLd && !mbar_wait(BAR(RAW_EMPTY + sl), (g / kLd - 1) & 1)) {
            *err = 1;
            break;
          }
          const unsigned i0 = st * kStageIn;
          const unsigned ni = min((unsigned)kStageIn, J.n_in - i0);
          mbar_expect_tx(BAR(RAW_FULL + sl), raw_copy * ni);
          for (unsigned ii = 0; ii < ni; ii++) {
            const uint64_t* row = rows.p[ii];
            bulk_g2s(sRaw + sl * kRawBytes + ii * (kWords * 8), row + w0, raw_copy, BAR(RAW_FULL + sl));
          }
          rows = next;
        }
      } while (0);
      if (*err) {  // every issued copy lands before the CTA exits
        for (uint32_t k = g > (uint32_t)kLd ? g - kLd : 0; k < g; k++)
          mbar_wait(BAR(RAW_FULL + k % kLd), (k / kLd) & 1);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      uint32_t g = 0;
      do {  // the CTA's one item
        for (unsigned k = 0; k < sg.st1 - sg.st0; k++, g++) {
          const unsigned bs = g % kBs;
          if (*err || !mbar_wait(BAR(OP_FULL + bs), (g / kBs) & 1)) {
            *err = 1;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int kk = 0; kk < 4; kk++) {
#pragma unroll
            for (int nn = 0; nn < 2; nn++) {
              mma_i8(tmem + nn * 256, sw128_desc(sA + bs * kABytes + 32 * kk),
                     sw128_desc(sB + bs * kBBytes + nn * (256 * 128) + 32 * kk), kIdesc,
                     (k > 0 || kk > 0) ? 1u : 0u);
            }
          }
          mma_commit(BAR(OP_EMPTY + bs));
        }
        if (!*err) mma_commit(BAR(D_FULL));
      } while (0);
      // all MMAs issued by this thread complete before TMEM is released
      mma_commit(BAR(DONE));
      if (!mbar_wait(BAR(DONE), 0)) *err = 1;
    }
  } else {
    // ------------------------------------------------------------ operand builders
    const int e = threadIdx.x - 64;  // 0..255
    const unsigned n = 2 * e;        // B: word pair n, n+1 of the tile
    const unsigned sw = (e >> 2) & 1;  // store order: conflict-free 128-bit phases
    const unsigned mA = n + sw, mB = n + 1 - sw;
    const uint32_t rowA = (mA >> 3) * 1024 + (mA & 7) * 128, rA = mA & 7;
    const uint32_t rowB = (mB >> 3) * 1024 + (mB & 7) * 128, rB = mB & 7;
    // A: row m, input half ii (adjacent threads alternate ii so a 64-bit store
    // phase of 16 threads covers 8 rows x 2 halves = all 32 banks)
    const unsigned a_ii = e & 1, a_m = e >> 1, a_oo = a_m >> 6, a_b = a_m & 63;
    const uint32_t arow_off = (a_m >> 3) * 1024 + (a_m & 7) * 128 + 8 * a_ii, ar7 = a_m & 7;
    // epilogue role: TMEM lane quarter q (rows 32q..32q+31), column half
    const int q = warp & 3;
    const int chalf = (warp - 2) >> 2;
    uint32_t g = 0, nseg = 0;
    do {  // the CTA's one item
      const Gf64TcJob J = pinned_job(batch.job[sg.job]);
      const unsigned o0 = 2 * (unsigned)(sg.tile % J.pairs);
      const size_t w0 = (size_t)(sg.tile / J.pairs) * kWords;
      const unsigned words_valid = (unsigned)min((size_t)kWords, J.words - w0);
      const bool okA = mA < words_valid, okB = mB < words_valid;
      const unsigned nst = sg.st1 - sg.st0;
      auto coef = [&](unsigned k) -> uint64_t {
        const unsigned o = o0 + a_oo, i = (sg.st0 + k) * kStageIn + a_ii;
        return (k < nst && o < J.n_out && i < J.n_in) ? J.coeff[(size_t)o * J.ldc + i] : 0ull;
      };
      uint64_t c_cur = coef(0);
      for (unsigned k = 0; k < nst; k++, g++) {
        const unsigned sl = g % kLd, bs = g % kBs;
        const uint64_t c_nxt = coef(k + 1);  // prefetch the next stage's coefficient
        const uint64_t qrow = mul_matrix_row(c_cur, a_b);
        const uint32_t qlo = (uint32_t)qrow, qhi = (uint32_t)(qrow >> 32);
        if (*err || !mbar_wait(BAR(RAW_FULL + sl), (g / kLd) & 1)) {
          *err = 1;
          break;
        }
        const unsigned i0 = (sg.st0 + k) * kStageIn;
        const unsigned ni = min((unsigned)kStageIn, J.n_in - i0);
        const uint32_t raw = sRaw + sl * kRawBytes + 8 * n;
        // B rows of words mA and mB: (lo, hi) of input 0, then (lo, hi) of input 1
        uint4 xA = make_uint4(0, 0, 0, 0), xB = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int ii = 0; ii < kStageIn; ii++) {
          if ((unsigned)ii >= ni) continue;
          // v = word n (x, y) and word n+1 (z, w) of input ii
          const uint4 v = lds128(raw + ii * (kWords * 8));
          const uint2 a = sw ? make_uint2(v.z, v.w) : make_uint2(v.x, v.y);
          const uint2 b = sw ? make_uint2(v.x, v.y) : make_uint2(v.z, v.w);
          if (ii == 0) {
            if (okA) { xA.x = a.x; xA.y = a.y; }
            if (okB) { xB.x = b.x; xB.y = b.y; }
          } else {
            if (okA) { xA.z = a.x; xA.w = a.y; }
            if (okB) { xB.z = b.x; xB.w = b.y; }
          }
        }
        mbar_arrive(BAR(RAW_EMPTY + sl));
        if (g >= (uint32_t)kBs && !mbar_wait(BAR(OP_EMPTY + bs), (g / kBs - 1) & 1)) {
          *err = 1;
          break;
        }
        const uint32_t at = sA + bs * kABytes, bt = sB + bs * kBBytes;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          sts64(at + arow_off + ((j ^ ar7) << 4), qlo >> j, qhi >> j);
          sts128(bt + rowA + ((j ^ rA) << 4), xA.x >> j, xA.y >> j, xA.z >> j, xA.w >> j);
          sts128(bt + rowB + ((j ^ rB) << 4), xB.x >> j, xB.y >> j, xB.z >> j, xB.w >> j);
        }
        fence_async_smem();
        mbar_arrive(BAR(OP_FULL + bs));
        c_cur = c_nxt;
      }
      // ---------------------------------------------------------- epilogue
      if (*err || !mbar_wait(BAR(D_FULL), nseg & 1)) {
        *err = 1;
        break;
      }
      nseg++;
      tc_fence_after();
      const unsigned o = o0 + (q >> 1);  // output of these rows
      const unsigned half = q & 1;       // bits [32*half, 32*half + 32)
      uint64_t* orow = o < J.n_out ? (J.out_ptrs ? J.out_ptrs[o] : J.out + (size_t)o * J.out_stride) : nullptr;
      for (int cc = 8 * chalf; cc < 8 * chalf + 8; cc++) {
        uint32_t r[32];
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + 32 * cc, r);
        uint32_t mine = 0;
#pragma unroll
        for (int jj = 0; jj < 32; jj++) {
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, r[jj] & 1u);
          if (lane == jj) mine = bal;
        }
        const unsigned widx = 32 * cc + lane;
        if (!orow || widx >= words_valid) continue;
        uint32_t* dst = reinterpret_cast<uint32_t*>(orow + w0 + widx) + half;
        if (sg.mode == 2) {
          if (mine) atomicXor(dst, mine);
        } else if (sg.mode == 1) {
          *dst ^= mine;
        } else {
          *dst = mine;
        }
      }
      // the TMEM reads above precede the arrive that releases the next
      // segment's first MMA
      tc_fence_before();
    } while (0);
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
  if (threadIdx.x == 0 && *err) atomicOr(status, 1);
}

// ---------------------------------------------------------------------------
// CTA-pair variant (cluster of 2, tcgen05 cta_group::2).  The pair computes
// 4 outputs (M = 256 rows: rows 0-127 = outputs o0, o0+1 in CTA 0, rows
// 128-255 = outputs o0+2, o0+3 in CTA 1) x 512 words with two MMAs of N = 256;
// each MMA takes B columns 0-127 from CTA 0 and 128-255 from CTA 1.  So each
// CTA builds the A rows of its own 2 outputs (as above) but the B rows of
// only 256 of the 512 words: per SM, the B tile the builders write and the
// tensor cores read is half that of the one-CTA kernel for the same work,
// and shared-memory bandwidth is what limits that kernel.
//
// Word mapping: CTA r builds words w0 + 256 r + u, u = 0..255, as B rows
// u (MMA nn = u / 128 takes rows 128 nn .. 128 nn + 127).  Column c of
// accumulator nn is therefore word w0 + 256 (c / 128) + 128 nn + c % 128.
//
// Pipeline: each CTA copies its own raw rows and builds its own tiles;
// CTA 1's warp 1 relays "stage built" to CTA 0 (one remote arrive per
// stage), CTA 0's warp 1 issues the pair MMAs, and its commits arrive on the
// "stage free", "accumulators ready" and "MMAs done" barriers of both CTAs.
// All waits are bounded as in the one-CTA kernel; the only unbounded
// barriers are the two cluster barriers that every thread of both CTAs
// reaches on every path.
constexpr int kPHalf = 256;                       // words built per CTA
constexpr int kPBBytes = kPHalf * 128;            // 32 KiB
constexpr int kPRawBytes = kStageIn * kPHalf * 8;  // 4 KiB
// kPLd raw-row stages, kPBs operand stages (ring depths 4-8 x 3-4 measured
// within 4 % of each other on the 1 GiB R=8 job; the deepest fits 227 KiB)
constexpr int pair_smem_bytes(int ld, int bs) { return bs * (kABytes + kPBBytes) + ld * kPRawBytes + 256 + 1024; }
constexpr int kPLd = 8;
constexpr int kPBs = 4;
constexpr int kPSmemBytes = pair_smem_bytes(kPLd, kPBs);
static_assert(kPSmemBytes <= 227 * 1024, "shared memory per CTA");
constexpr uint32_t kPIdesc = (2u << 4) | ((256u >> 3) << 17) | ((256u >> 4) << 24);

template <int kPLd, int kPBs>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    k_gf64_matvec_tc_pair(const __grid_constant__ Gf64TcBatch batch, int* __restrict__ status) {
  constexpr int kPOffA = 0;
  constexpr int kPOffB = kPBs * kABytes;
  constexpr int kPOffRaw = kPOffB + kPBs * kPBBytes;
  constexpr int kPOffBar = kPOffRaw + kPLd * kPRawBytes;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t base_s = smem_addr(smem_raw);
  const uint32_t pad = ((base_s + 1023) & ~1023u) - base_s;
  uint8_t* smem = smem_raw + pad;
  const uint32_t sA = base_s + pad + kPOffA, sB = base_s + pad + kPOffB, sRaw = base_s + pad + kPOffRaw;
  const uint32_t bar0 = smem_addr(smem + kPOffBar);
  enum {
    RAW_FULL = 0,
    RAW_EMPTY = RAW_FULL + kPLd,
    OPB_FULL = RAW_EMPTY + kPLd,  // this CTA's builders done with stage slot
    OPR_FULL = OPB_FULL + kPBs,   // CTA 0: CTA 1's builders done (relayed)
    OP_EMPTY = OPR_FULL + kPBs,
    D_FULL = OP_EMPTY + kPBs,
    DONE = D_FULL + 1,
    NBARS = DONE + 1
  };
  static_assert(8 * NBARS + 16 <= 256, "barrier area");
  auto BAR = [&](int k) { return bar0 + 8u * (uint32_t)k; };
  volatile uint32_t* tmem_holder = reinterpret_cast<volatile uint32_t*>(smem + kPOffBar + 8 * NBARS);
  volatile int* err = reinterpret_cast<volatile int*>(smem + kPOffBar + 8 * NBARS + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();

  if (threadIdx.x == 0) {
    for (int k = 0; k < NBARS; k++) {
      const bool by_builders = (k >= RAW_EMPTY && k < RAW_EMPTY + kPLd) || (k >= OPB_FULL && k < OPB_FULL + kPBs);
      mbar_init(BAR(k), by_builders ? (uint32_t)kExp : 1u);
    }
    *err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {  // both CTAs allocate together
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr((const void*)tmem_holder)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // the peer's barriers are initialised before any remote arrive
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  const TcSeg sg = tc_item(&batch, blockIdx.x >> 1);

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      uint32_t g = 0;
      do {  // the pair's one item
        const Gf64TcJob J = pinned_job(batch.job[sg.job]);
        const size_t wc = (size_t)(sg.tile / J.pairs) * kWords + (size_t)kPHalf * rank;
        const unsigned words_valid = J.words > wc ? (unsigned)min((size_t)kPHalf, J.words - wc) : 0u;
        const uint32_t raw_copy = (uint32_t)(((size_t)words_valid * 8 + 15) & ~(size_t)15);
        StageRows<kStageIn> rows, next;
        rows.load(J, sg.st0);
        for (unsigned st = sg.st0; st < sg.st1; st++, g++) {
          const unsigned sl = g % kPLd;
          next.load(J, st + 1);
          if (g >= (uint32_t)kPLd && !mbar_wait(BAR(RAW_EMPTY + sl), (g / kPLd - 1) & 1)) {
            *err = 1;
            break;
          }
          const unsigned i0 = st * kStageIn;
          const unsigned ni = raw_copy ? min((unsigned)kStageIn, J.n_in - i0) : 0u;
          mbar_expect_tx(BAR(RAW_FULL + sl), raw_copy * ni);
          for (unsigned ii = 0; ii < ni; ii++) {
            const uint64_t* row = rows.p[ii];
            bulk_g2s(sRaw + sl * kPRawBytes + ii * (kPHalf * 8), row + wc, raw_copy, BAR(RAW_FULL + sl));
          }
          rows = next;
        }
      } while (0);
      if (*err) {
        for (uint32_t k = g > (uint32_t)kPLd ? g - kPLd : 0; k < g; k++)
          mbar_wait(BAR(RAW_FULL + k % kPLd), (k / kPLd) & 1);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const unsigned nst = sg.st1 - sg.st0;
      if (rank == 0) {
        // -------------------------------------------------------- MMA issuer
        for (unsigned k = 0; k < nst; k++) {
          const unsigned bs = k % kPBs;
          const uint32_t ph = (k / kPBs) & 1;
          if (*err || !mbar_wait(BAR(OPB_FULL + bs), ph) || !mbar_wait_cluster(BAR(OPR_FULL + bs), ph)) {
            *err = 1;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int kk = 0; kk < 4; kk++) {
#pragma unroll
            for (int nn = 0; nn < 2; nn++) {
              mma_i8_pair(tmem + nn * 256, sw128_desc(sA + bs * kABytes + 32 * kk),
                          sw128_desc(sB + bs * kPBBytes + nn * (128 * 128) + 32 * kk), kPIdesc,
                          (k > 0 || kk > 0) ? 1u : 0u);
            }
          }
          mma_commit_pair(BAR(OP_EMPTY + bs));
        }
        if (!*err) mma_commit_pair(BAR(D_FULL));
        mma_commit_pair(BAR(DONE));
      } else {
        // -------------------------------------------------------- relay
        const uint32_t remote = peer_addr(BAR(OPR_FULL), 0);
        for (unsigned k = 0; k < nst; k++) {
          const unsigned bs = k % kPBs;
          if (*err || !mbar_wait(BAR(OPB_FULL + bs), (k / kPBs) & 1)) {
            *err = 1;
            break;
          }
          mbar_arrive_remote(remote + 8u * bs);
        }
      }
      // CTA 0's MMAs (which read this CTA's tiles and write its TMEM) have
      // completed before the tiles and TMEM are released
      if (!mbar_wait(BAR(DONE), 0)) *err = 1;
    }
  } else {
    // ------------------------------------------------------------ operand builders
    const int e = threadIdx.x - 64;  // 0..255
    // B: word u = e of this CTA's half, row e % 128 of half e / 128
    const unsigned bm = (unsigned)e & 127;
    const uint32_t brow = (e >> 7) * (128 * 128) + (bm >> 3) * 1024 + (bm & 7) * 128, br7 = bm & 7;
    // A: row m, input half ii (adjacent threads alternate ii)
    const unsigned a_ii = e & 1, a_m = e >> 1, a_oo = a_m >> 6, a_b = a_m & 63;
    const uint32_t arow_off = (a_m >> 3) * 1024 + (a_m & 7) * 128 + 8 * a_ii, ar7 = a_m & 7;
    const int q = warp & 3;
    const int nn_ep = (warp - 2) >> 2;  // epilogue: accumulator
    uint32_t g = 0;
    do {  // the pair's one item
      const Gf64TcJob J = pinned_job(batch.job[sg.job]);
      const unsigned o0 = 4 * (unsigned)(sg.tile % J.pairs) + 2 * rank;  // this CTA's two outputs
      const size_t w0 = (size_t)(sg.tile / J.pairs) * kWords;
      const size_t wc = w0 + (size_t)kPHalf * rank;
      const unsigned words_valid = J.words > wc ? (unsigned)min((size_t)kPHalf, J.words - wc) : 0u;
      const bool okB = (unsigned)e < words_valid;
      const unsigned nst = sg.st1 - sg.st0;
      auto coef = [&](unsigned k) -> uint64_t {
        const unsigned o = o0 + a_oo, i = (sg.st0 + k) * kStageIn + a_ii;
        return (k < nst && o < J.n_out && i < J.n_in) ? J.coeff[(size_t)o * J.ldc + i] : 0ull;
      };
      uint64_t c_cur = coef(0);
      for (unsigned k = 0; k < nst; k++, g++) {
        const unsigned sl = g % kPLd, bs = g % kPBs;
        const uint64_t c_nxt = coef(k + 1);
        const uint64_t qrow = mul_matrix_row(c_cur, a_b);
        const uint32_t qlo = (uint32_t)qrow, qhi = (uint32_t)(qrow >> 32);
        if (*err || !mbar_wait(BAR(RAW_FULL + sl), (g / kPLd) & 1)) {
          *err = 1;
          break;
        }
        const unsigned i0 = (sg.st0 + k) * kStageIn;
        const unsigned ni = min((unsigned)kStageIn, J.n_in - i0);
        uint4 x = make_uint4(0, 0, 0, 0);
        if (okB) {
          const uint32_t raw = sRaw + sl * kPRawBytes + 8 * (unsigned)e;
          const uint2 v0 = lds64(raw);
          x.x = v0.x;
          x.y = v0.y;
          if (ni > 1) {
            const uint2 v1 = lds64(raw + kPHalf * 8);
            x.z = v1.x;
            x.w = v1.y;
          }
        }
        mbar_arrive(BAR(RAW_EMPTY + sl));
        if (g >= (uint32_t)kPBs && !mbar_wait(BAR(OP_EMPTY + bs), (g / kPBs - 1) & 1)) {
          *err = 1;
          break;
        }
        const uint32_t at = sA + bs * kABytes, bt = sB + bs * kPBBytes;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          sts64(at + arow_off + ((j ^ ar7) << 4), qlo >> j, qhi >> j);
          sts128(bt + brow + ((j ^ br7) << 4), x.x >> j, x.y >> j, x.z >> j, x.w >> j);
        }
        fence_async_smem();
        mbar_arrive(BAR(OPB_FULL + bs));
        c_cur = c_nxt;
      }
      // ---------------------------------------------------------- epilogue
      if (*err || !mbar_wait(BAR(D_FULL), 0)) {
        *err = 1;
        break;
      }
      tc_fence_after();
      const unsigned o = o0 + (q >> 1);
      const unsigned half = q & 1;
      uint64_t* orow = o < J.n_out ? (J.out_ptrs ? J.out_ptrs[o] : J.out + (size_t)o * J.out_stride) : nullptr;
      for (int cc = 0; cc < 8; cc++) {
        uint32_t r[32];
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + 256 * nn_ep + 32 * cc, r);
        uint32_t mine = 0;
#pragma unroll
        for (int jj = 0; jj < 32; jj++) {
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, r[jj] & 1u);
          if (lane == jj) mine = bal;
        }
        const unsigned c = 32 * cc + lane;  // column of accumulator nn_ep
        const size_t widx = (size_t)kPHalf * (c >> 7) + 128 * nn_ep + (c & 127);
        if (!orow || w0 + widx >= J.words) continue;
        uint32_t* dst = reinterpret_cast<uint32_t*>(orow + w0 + widx) + half;
        if (sg.mode == 2) {
          if (mine) atomicXor(dst, mine);
        } else if (sg.mode == 1) {
          *dst ^= mine;
        } else {
          *dst = mine;
        }
      }
      tc_fence_before();
    } while (0);
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync();  // both CTAs are done with TMEM and the peer's barriers
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
  if (threadIdx.x == 0 && *err) atomicOr(status, 1);
}

// zero rows given by a pointer table (outputs of a non-accumulating job whose
// tiles are split across CTAs)
__global__ void k_zero_rows(uint64_t* const* __restrict__ rows, unsigned n_rows, size_t words) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < (size_t)n_rows * words;
       t += (size_t)gridDim.x * blockDim.x)
    rows[t / words][t % words] = 0;
}

static uint64_t tiles64(const Gf64TcJob& j) { return (uint64_t)j.pairs * j.wt; }

}  // namespace tc64

// ============================================================================
// The GF(2^64) product on the block-scaled FP4 path (tcgen05.mma kind::mxf4),
// one CTA per tile.  As in the GF(2^16) FP4 kernel (gf16_tc.cu): exact fp32
// counts (an item sums at most 65,536 inputs: counts < 64 * 2^16 = 2^22), the
// parity read as the lowest mantissa bit of count + 2^23.  Selection j of
// each 32-bit half of a word (bits 4m + j) feeds MMA step j, on both operands:
//   B[w][(j, ii, half, m)]     = v_j * bit (32 half + 4m + j) of x_ii[w]
//   A[(o,b)][(j, ii, half, m)] = v_j * bit (32 half + 4m + j) of Q_{o,ii,b}
// (Q = row b of the multiplication matrix, the closed form above).  A stage is
// 4 inputs: K = 256 elements = one 128-byte swizzled row; the 64-element MMA
// step j covers 32 bytes: inputs 0-1 in its first 16-byte chunk, 2-3 in the
// second, (lo half, hi half) as two 32-bit words per input.
//
// CTA tile: 2 outputs (M = 128) x 480 words (two accumulators of N = 240 on
// the two halves of the B tile); TMEM columns 0-239 and 256-495, scale
// factors in 240-255.  Builders (warps 2-9): the A rows of the stage's 4
// coefficients per output row (two (row, input) pairs per thread) and the B
// rows of up to two words per thread; then the epilogue.
namespace tc64f4 {
using namespace pp::tc;
PP_D uint64_t mul_matrix_row_f4(uint64_t c, unsigned b) { return tc64::mul_matrix_row(c, b); }

constexpr int kN = 240;
constexpr int kWords = 2 * kN;
constexpr int kStageIn = 4;
constexpr int kABytes = 128 * 128;               // 16 KiB
constexpr int kBBytes = kWords * 128;            // 60 KiB
constexpr int kRawBytes = kStageIn * kWords * 8;  // 15 KiB
constexpr int kLd = 4;
constexpr int kBs = 2;
constexpr int kThreads = 320;
constexpr int kExp = 256;
constexpr int kOffA = 0;
constexpr int kOffB = kBs * kABytes;
constexpr int kOffRaw = kOffB + kBs * kBBytes;
constexpr int kOffBar = kOffRaw + kLd * kRawBytes;
constexpr int kSmemBytes = kOffBar + 256 + 1024;
constexpr uint32_t kMaxStagesPerItem = 16384;  // 65,536 inputs
constexpr uint32_t kSfaCol = 240;
static_assert(kSmemBytes <= 227 * 1024, "shared memory");
static_assert(kOffB % 1024 == 0 && kBBytes % 1024 == 0 && (kN * 128) % 1024 == 0, "swizzle atoms");
constexpr uint32_t kIdesc = (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) | (1u << 23) | ((128u >> 4) << 24);

PP_D void mma_f4(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate, uint32_t sfa, uint32_t sfb) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %6, [%4], [%5], p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(accumulate), "r"(sfa), "r"(sfb), "r"(kIdesc)
      : "memory");
}
// Selection j of an operand word, in place: bit j of every nibble (bit 3 moved
// to bit 2, since e2m1 0x8 is -0), so a nonzero element of MMA step j is v_j =
// 0.5, 1, 2, 2 (e2m1 0x1, 0x2, 0x4, 0x4) on both operands and a product v_j^2.
// The B scale factor of step j is 1 / v_j^2 (4, 1, 0.25, 0.25), A's is 1, so
// every nonzero product adds exactly 1.  TMEM scale columns: A 240-243, B
// 248-255 (step 0), 496-503 (step 1), 504-511 (steps 2-3); 8-column B sets
// start on 8-column boundaries.
PP_D uint32_t sel4(uint32_t p, int j) { return j == 3 ? (p >> 1) & 0x44444444u : p & (0x11111111u << j); }
PP_D uint32_t sfb_col(int kk) { return kk == 0 ? 248u : kk == 1 ? 496u : 504u; }
// the scale factors of this warp's TMEM lane quarter (warps 2-5 of a CTA)
PP_D void fill_scales(uint32_t tmem, int warp) {
  const uint32_t t = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
  const uint32_t four = 0x81818181u, one = 0x7F7F7F7Fu, quarter = 0x7D7D7D7Du;  // ue8m0 4, 1, 0.25
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%2,%2,%2,%2,%2,%2,%2,%2};" ::"r"(t + 240),
      "r"(one), "r"(four)
      : "memory");
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%2,%2,%2,%2,%2,%2,%2,%2};" ::"r"(t + 496),
      "r"(one), "r"(quarter)
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// A rows: builder thread e makes rows b, b + 1 (b = 2 ((e / 4) % 32)) of the
// multiplication matrix of coefficient (output e / 128, input e % 4) of the
// stage: row b by the closed form, row b + 1 from it by one step of
// Q_{b+1} = ((Q_b ^ [b+1 in {0,1,3,4}] Q_63) << 1) | bit_{b+1}(c), which
// follows from c x^{e+1} = (c x^e) x mod x^64 + x^4 + x^3 + x + 1.
PP_D uint64_t mul_matrix_row63(uint64_t c) {  // row 63: the closed form at b = 63
  const uint64_t rv = __brevll(c);
  return rv ^ (rv << 63) ^ (rv << 61) ^ (rv << 60);
}
struct ARows {
  unsigned oo, ii, b, ch;
  uint32_t row0, r70, row1, r71;
  uint64_t red;
  PP_D explicit ARows(int e) {
    // a warp covers the 4 inputs x 8 consecutive row pairs of one output, so
    // a 64-bit store phase meets every (16-byte slot, half) of a row once or
    // twice (slot = chunk ^ row % 8, chunk = 2j + input / 2)
    const unsigned t = (unsigned)e >> 2;
    ii = (unsigned)e & 3;
    oo = t >> 5;
    b = 2 * (t & 31);
    const unsigned m0 = 64 * oo + b, m1 = m0 + 1;
    // input ii sits at chunk 2j + ii / 2, byte 8 (ii % 2) of an A row
    ch = ii >> 1;
    row0 = (m0 >> 3) * 1024 + (m0 & 7) * 128 + 8 * (ii & 1);
    r70 = m0 & 7;
    row1 = (m1 >> 3) * 1024 + (m1 & 7) * 128 + 8 * (ii & 1);
    r71 = m1 & 7;
    red = (b + 1 == 1 || b + 1 == 3) ? ~0ull : 0ull;  // b + 1 in {1, 3}: Q_63 enters
  }
  // rows b, b + 1 of coefficient c into the A tile at `at`
  PP_D void store(uint32_t at, uint64_t c) const {
    const uint64_t q0 = mul_matrix_row_f4(c, b);
    const uint64_t q1 = ((q0 ^ (mul_matrix_row63(c) & red)) << 1) | ((c >> (b + 1)) & 1ull);
    const uint32_t q0lo = (uint32_t)q0, q0hi = (uint32_t)(q0 >> 32), q1lo = (uint32_t)q1, q1hi = (uint32_t)(q1 >> 32);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      sts64(at + row0 + (((2 * j + ch) ^ r70) << 4), sel4(q0lo, j), sel4(q0hi, j));
      sts64(at + row1 + (((2 * j + ch) ^ r71) << 4), sel4(q1lo, j), sel4(q1hi, j));
    }
  }
};

__global__ void __launch_bounds__(kThreads, 1)
k_gf64_matvec_f4(const __grid_constant__ Gf64TcBatch batch, int* __restrict__ status) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t base_s = smem_addr(smem_raw);
  const uint32_t pad = ((base_s + 1023) & ~1023u) - base_s;
  uint8_t* smem = smem_raw + pad;
  const uint32_t sA = base_s + pad + kOffA, sB = base_s + pad + kOffB, sRaw = base_s + pad + kOffRaw;
  const uint32_t bar0 = smem_addr(smem + kOffBar);
  enum {
    RAW_FULL = 0,
    RAW_EMPTY = RAW_FULL + kLd,
    OP_FULL = RAW_EMPTY + kLd,
    OP_EMPTY = OP_FULL + kBs,
    D_FULL = OP_EMPTY + kBs,
    DONE = D_FULL + 1,
    NBARS = DONE + 1
  };
  static_assert(8 * NBARS + 16 <= 256, "barrier area");
  auto BAR = [&](int k) { return bar0 + 8u * (uint32_t)k; };
  volatile uint32_t* tmem_holder = reinterpret_cast<volatile uint32_t*>(smem + kOffBar + 8 * NBARS);
  volatile int* err = reinterpret_cast<volatile int*>(smem + kOffBar + 8 * NBARS + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int k = 0; k < NBARS; k++) {
      const bool by_expanders = (k >= RAW_EMPTY && k < RAW_EMPTY + kLd) || (k >= OP_FULL && k < OP_FULL + kBs);
      mbar_init(BAR(k), by_expanders ? (uint32_t)kExp : 1u);
    }
    *err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr((const void*)tmem_holder)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  if (warp >= 2 && warp < 6) fill_scales(tmem, warp);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const TcSeg sg = tc_item(&batch, blockIdx.x);

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      uint32_t g = 0;
      do {
        const Gf64TcJob J = pinned_job(batch.job[sg.job]);
        const size_t w0 = (size_t)(sg.tile / J.pairs) * kWords;
        const unsigned words_valid = (unsigned)min((size_t)kWords, J.words - w0);
        const uint32_t raw_copy = (uint32_t)(((size_t)words_valid * 8 + 15) & ~(size_t)15);
        StageRows<kStageIn> rows, next;
        rows.load(J, sg.st0);
        for (unsigned st = sg.st0; st < sg.st1; st++, g++) {
          const unsigned sl = g % kLd;
          next.load(J, st + 1);
          if (g >= (uint32_t)kLd && !mbar_wait(BAR(RAW_EMPTY + sl), (g / kLd - 1) & 1)) {
            *err = 1;
            break;
          }
          const unsigned i0 = st * kStageIn;
          const unsigned ni = min((unsigned)kStageIn, J.n_in - i0);
          mbar_expect_tx(BAR(RAW_FULL + sl), raw_copy * ni);
          for (unsigned ii = 0; ii < ni; ii++) {
            const uint64_t* row = rows.p[ii];
            bulk_g2s(sRaw + sl * kRawBytes + ii * (kWords * 8), row + w0, raw_copy, BAR(RAW_FULL + sl));
          }
          rows = next;
        }
      } while (0);
      if (*err) {
        for (uint32_t k = g > (uint32_t)kLd ? g - kLd : 0; k < g; k++)
          mbar_wait(BAR(RAW_FULL + k % kLd), (k / kLd) & 1);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t sfa = tmem + kSfaCol;
      for (unsigned k = 0; k < sg.st1 - sg.st0; k++) {
        const unsigned bs = k % kBs;
        if (*err || !mbar_wait(BAR(OP_FULL + bs), (k / kBs) & 1)) {
          *err = 1;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
#pragma unroll
          for (int nn = 0; nn < 2; nn++) {
            mma_f4(tmem + nn * 256, sw128_desc(sA + bs * kABytes + 32 * kk),
                   sw128_desc(sB + bs * kBBytes + nn * (kN * 128) + 32 * kk), (k > 0 || kk > 0) ? 1u : 0u, sfa,
                   tmem + sfb_col(kk));
          }
        }
        mma_commit(BAR(OP_EMPTY + bs));
      }
      if (!*err) mma_commit(BAR(D_FULL));
      mma_commit(BAR(DONE));
      if (!mbar_wait(BAR(DONE), 0)) *err = 1;
    }
  } else {
    // ------------------------------------------------------------ operand builders
    const int e = threadIdx.x - 64;  // 0..255
    const ARows ar(e);
    const int q = warp & 3;
    const int chalf = (warp - 2) >> 2;
    do {
      const Gf64TcJob J = pinned_job(batch.job[sg.job]);
      const unsigned o0 = 2 * (unsigned)(sg.tile % J.pairs);
      const size_t w0 = (size_t)(sg.tile / J.pairs) * kWords;
      const unsigned words_valid = (unsigned)min((size_t)kWords, J.words - w0);
      const unsigned nst = sg.st1 - sg.st0;
      auto coef = [&](unsigned k, unsigned ii) -> uint64_t {
        const unsigned o = o0 + ar.oo, i = (sg.st0 + k) * kStageIn + ii;
        return (k < nst && o < J.n_out && i < J.n_in) ? J.coeff[(size_t)o * J.ldc + i] : 0ull;
      };
      uint64_t c0 = coef(0, ar.ii);
      for (unsigned k = 0; k < nst; k++) {
        const unsigned sl = k % kLd, bs = k % kBs;
        const uint64_t n0 = coef(k + 1, ar.ii);  // the next stage's coefficient
        if (*err || !mbar_wait(BAR(RAW_FULL + sl), (k / kLd) & 1)) {
          *err = 1;
          break;
        }
        const unsigned i0 = (sg.st0 + k) * kStageIn;
        const unsigned ni = min((unsigned)kStageIn, J.n_in - i0);
        // B rows e and e + 240: the 4 inputs' words as (lo, hi) pairs
        uint32_t xw[2][8];
#pragma unroll
        for (int rr = 0; rr < 2; rr++) {
          const unsigned u = (unsigned)e + rr * kN;
          const bool ok = e < kN && u < words_valid;
#pragma unroll
          for (int ii = 0; ii < kStageIn; ii++) {
            uint2 v = make_uint2(0, 0);
            if (ok && (unsigned)ii < ni) v = lds64(sRaw + sl * kRawBytes + ii * (kWords * 8) + 8 * u);
            xw[rr][2 * ii] = v.x;
            xw[rr][2 * ii + 1] = v.y;
          }
        }
        mbar_arrive(BAR(RAW_EMPTY + sl));
        if (k >= (unsigned)kBs && !mbar_wait(BAR(OP_EMPTY + bs), (k / kBs - 1) & 1)) {
          *err = 1;
          break;
        }
        const uint32_t at = sA + bs * kABytes, bt = sB + bs * kBBytes;
        ar.store(at, c0);
        if (e < kN) {
#pragma unroll
          for (int rr = 0; rr < 2; rr++) {
            const unsigned u = (unsigned)e + rr * kN;
            const uint32_t brow = bt + (u >> 3) * 1024 + (u & 7) * 128, br7 = u & 7;
#pragma unroll
            for (int j = 0; j < 4; j++) {
              sts128(brow + (((2 * j) ^ br7) << 4), sel4(xw[rr][0], j), sel4(xw[rr][1], j), sel4(xw[rr][2], j),
                     sel4(xw[rr][3], j));
              sts128(brow + (((2 * j + 1) ^ br7) << 4), sel4(xw[rr][4], j), sel4(xw[rr][5], j),
                     sel4(xw[rr][6], j), sel4(xw[rr][7], j));
            }
          }
        }
        fence_async_smem();
        mbar_arrive(BAR(OP_FULL + bs));
        c0 = n0;
      }
      // ---------------------------------------------------------- epilogue
      if (*err || !mbar_wait(BAR(D_FULL), 0)) {
        *err = 1;
        break;
      }
      tc_fence_after();
      const unsigned o = o0 + (q >> 1);  // output of these rows
      const unsigned half = q & 1;       // bits [32*half, 32*half + 32)
      uint64_t* orow = o < J.n_out ? (J.out_ptrs ? J.out_ptrs[o] : J.out + (size_t)o * J.out_stride) : nullptr;
      for (int cc = 0; cc < (kN + 31) / 32; cc++) {
        uint32_t r[32];
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + 256 * chalf + 32 * cc, r);
        uint32_t mine = 0;
#pragma unroll
        for (int jj = 0; jj < 32; jj++) {
          const uint32_t bit = __float_as_uint(__fadd_rn(__uint_as_float(r[jj]), 8388608.0f)) & 1u;
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, bit);
          if (lane == jj) mine = bal;
        }
        const unsigned col = 32 * cc + lane;
        const unsigned widx = (unsigned)chalf * kN + col;
        if (!orow || col >= (unsigned)kN || widx >= words_valid) continue;
        uint32_t* dst = reinterpret_cast<uint32_t*>(orow + w0 + widx) + half;
        if (sg.mode == 2) {
          if (mine) atomicXor(dst, mine);
        } else if (sg.mode == 1) {
          *dst ^= mine;
        } else {
          *dst = mine;
        }
      }
      tc_fence_before();
    } while (0);
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
  if (threadIdx.x == 0 && *err) atomicOr(status, 1);
}

// ---------------------------------------------------------------------------
// FP4 on SM pairs (cluster of 2, tcgen05.mma cta_group::2 kind::mxf4, M = 256):
// the pair covers 4 outputs (CTA r holds the A rows and the accumulators of
// outputs o0 + 2r, o0 + 2r + 1) x 2N words (CTA r builds the B rows of words
// w0 + N r + u, u < N); MMA nn takes B rows H nn .. H nn + H - 1 of each CTA
// (H = N / 2), so column c of accumulator nn is word w0 + N (c / H) + H nn +
// c % H.  N is chosen per job (Gf64TcJob::n_mma, a multiple of 16 up to 240)
// so that tiles of 2N words cover the block with little waste (8 KiB blocks:
// 1,024 words as 3 tiles of 352, not 3 of 480; 4 KiB blocks: 2 of 256).  Per
// SM the B tile is half that of the one-CTA FP4 kernel.  Operand selections,
// scale factors (the same columns in both CTAs) and A rows as the one-CTA
// kernel.  Pipeline and bounded waits as the int8 pair kernel: CTA 1's warp 1
// relays "stage built" to CTA 0, whose warp 1 issues the MMAs and whose
// commits arrive in both CTAs.
constexpr int kPN = 240;                         // largest N
constexpr int kPWordsCta = kPN;                  // words built per CTA, at most
constexpr int kPWords = 2 * kPN;                 // words per pair tile, at most
constexpr int kPBBytes = kPWordsCta * 128;       // 30 KiB
constexpr int kPRawBytes = kStageIn * kPWordsCta * 8;  // 7.5 KiB
constexpr int kPLd = 5;
constexpr int kPBs = 4;
constexpr int kPOffA = 0;
constexpr int kPOffB = kPBs * kABytes;
constexpr int kPOffRaw = kPOffB + kPBs * kPBBytes;
constexpr int kPOffBar = kPOffRaw + kPLd * kPRawBytes;
constexpr int kPSmemBytes = kPOffBar + 256 + 1024;
constexpr uint32_t kPSfaCol = 240;
static_assert(kPSmemBytes <= 227 * 1024, "shared memory");
static_assert(kPOffB % 1024 == 0 && kPBBytes % 1024 == 0, "swizzle atoms");
// instruction descriptor for N (a multiple of 16, so the N/2 B rows of each
// CTA start on an 8-row swizzle atom)
PP_D uint32_t pair_idesc(uint32_t n) {
  return (1u << 7) | (1u << 10) | ((n >> 3) << 17) | (1u << 23) | ((256u >> 4) << 24);
}
// N for a job of `words` words: the fewest tiles of at most 2 x 240 words,
// each as narrow as covers the block
inline uint32_t pair_n_for(size_t words) {
  if (!words) return kPN;
  const size_t t = (words + kPWords - 1) / kPWords;
  const size_t half = (words + 2 * t - 1) / (2 * t);
  return (uint32_t)std::min<size_t>(kPN, std::max<size_t>(16, (half + 15) & ~(size_t)15));
}

PP_D void mma_f4_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate, uint32_t sfa,
                      uint32_t sfb, uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::mxf4.block_scale.block32 [%0], %1, %2, %6, [%4], [%5], p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(accumulate), "r"(sfa), "r"(sfb), "r"(idesc)
      : "memory");
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    k_gf64_matvec_f4_pair(const __grid_constant__ Gf64TcBatch batch, int* __restrict__ status) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t base_s = smem_addr(smem_raw);
  const uint32_t pad = ((base_s + 1023) & ~1023u) - base_s;
  uint8_t* smem = smem_raw + pad;
  const uint32_t sA = base_s + pad + kPOffA, sB = base_s + pad + kPOffB, sRaw = base_s + pad + kPOffRaw;
  const uint32_t bar0 = smem_addr(smem + kPOffBar);
  enum {
    RAW_FULL = 0,
    RAW_EMPTY = RAW_FULL + kPLd,
    OPB_FULL = RAW_EMPTY + kPLd,  // this CTA's builders done with stage slot
    OPR_FULL = OPB_FULL + kPBs,   // CTA 0: CTA 1's builders done (relayed)
    OP_EMPTY = OPR_FULL + kPBs,
    D_FULL = OP_EMPTY + kPBs,
    DONE = D_FULL + 1,
    NBARS = DONE + 1
  };
  static_assert(8 * NBARS + 16 <= 256, "barrier area");
  auto BAR = [&](int k) { return bar0 + 8u * (uint32_t)k; };
  volatile uint32_t* tmem_holder = reinterpret_cast<volatile uint32_t*>(smem + kPOffBar + 8 * NBARS);
  volatile int* err = reinterpret_cast<volatile int*>(smem + kPOffBar + 8 * NBARS + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();

  if (threadIdx.x == 0) {
    for (int k = 0; k < NBARS; k++) {
      const bool by_builders = (k >= RAW_EMPTY && k < RAW_EMPTY + kPLd) || (k >= OPB_FULL && k < OPB_FULL + kPBs);
      mbar_init(BAR(k), by_builders ? (uint32_t)kExp : 1u);
    }
    *err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {  // both CTAs allocate together
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr((const void*)tmem_holder)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  if (warp >= 2 && warp < 6) fill_scales(tmem, warp);
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // the peer's barriers and scale factors are ready before any remote arrive or MMA
  tc_fence_after();
  const TcSeg sg = tc_item(&batch, blockIdx.x >> 1);

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      uint32_t g = 0;
      do {
        const Gf64TcJob J = pinned_job(batch.job[sg.job]);
        const unsigned np = J.n_mma;
        const size_t wc = (size_t)(sg.tile / J.pairs) * (2 * np) + (size_t)np * rank;
        const unsigned words_valid = J.words > wc ? (unsigned)min((size_t)np, J.words - wc) : 0u;
        const uint32_t raw_copy = (uint32_t)(((size_t)words_valid * 8 + 15) & ~(size_t)15);
        StageRows<kStageIn> rows, next;
        rows.load(J, sg.st0);
        for (unsigned st = sg.st0; st < sg.st1; st++, g++) {
          const unsigned sl = g % kPLd;
          next.load(J, st + 1);
          if (g >= (uint32_t)kPLd && !mbar_wait(BAR(RAW_EMPTY + sl), (g / kPLd - 1) & 1)) {
            *err = 1;
            break;
          }
          const unsigned i0 = st * kStageIn;
          const unsigned ni = raw_copy ? min((unsigned)kStageIn, J.n_in - i0) : 0u;
          mbar_expect_tx(BAR(RAW_FULL + sl), raw_copy * ni);
          for (unsigned ii = 0; ii < ni; ii++) {
            const uint64_t* row = rows.p[ii];
            bulk_g2s(sRaw + sl * kPRawBytes + ii * (kPWordsCta * 8), row + wc, raw_copy, BAR(RAW_FULL + sl));
          }
          rows = next;
        }
      } while (0);
      if (*err) {
        for (uint32_t k = g > (uint32_t)kPLd ? g - kPLd : 0; k < g; k++)
          mbar_wait(BAR(RAW_FULL + k % kPLd), (k / kPLd) & 1);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const unsigned nst = sg.st1 - sg.st0;
      if (rank == 0) {
        // -------------------------------------------------------- MMA issuer
        const uint32_t sfa = tmem + kPSfaCol;
        const unsigned np = batch.job[sg.job].n_mma, hp = np / 2;
        const uint32_t idesc = pair_idesc(np);
        for (unsigned k = 0; k < nst; k++) {
          const unsigned bs = k % kPBs;
          const uint32_t ph = (k / kPBs) & 1;
          if (*err || !mbar_wait(BAR(OPB_FULL + bs), ph) || !mbar_wait_cluster(BAR(OPR_FULL + bs), ph)) {
            *err = 1;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int kk = 0; kk < 4; kk++) {
#pragma unroll
            for (int nn = 0; nn < 2; nn++) {
              mma_f4_pair(tmem + nn * 256, sw128_desc(sA + bs * kABytes + 32 * kk),
                          sw128_desc(sB + bs * kPBBytes + nn * (hp * 128) + 32 * kk), (k > 0 || kk > 0) ? 1u : 0u,
                          sfa, tmem + sfb_col(kk), idesc);
            }
          }
          mma_commit_pair(BAR(OP_EMPTY + bs));
        }
        if (!*err) mma_commit_pair(BAR(D_FULL));
        mma_commit_pair(BAR(DONE));
      } else {
        // -------------------------------------------------------- relay
        const uint32_t remote = peer_addr(BAR(OPR_FULL), 0);
        for (unsigned k = 0; k < nst; k++) {
          const unsigned bs = k % kPBs;
          if (*err || !mbar_wait(BAR(OPB_FULL + bs), (k / kPBs) & 1)) {
            *err = 1;
            break;
          }
          mbar_arrive_remote(remote + 8u * bs);
        }
      }
      // CTA 0's MMAs (which read this CTA's tiles and write its TMEM) have
      // completed before the tiles and TMEM are released
      if (!mbar_wait(BAR(DONE), 0)) *err = 1;
    }
  } else {
    // ------------------------------------------------------------ operand builders
    const int e = threadIdx.x - 64;  // 0..255
    const ARows ar(e);
    const int q = warp & 3;
    const int nn_ep = (warp - 2) >> 2;  // epilogue: accumulator
    uint32_t g = 0;
    do {
      const Gf64TcJob J = pinned_job(batch.job[sg.job]);
      const unsigned o0 = 4 * (unsigned)(sg.tile % J.pairs) + 2 * rank;  // this CTA's two outputs
      const unsigned np = J.n_mma, hp = np / 2;
      const size_t w0 = (size_t)(sg.tile / J.pairs) * (2 * np);
      const size_t wc = w0 + (size_t)np * rank;
      const unsigned words_valid = J.words > wc ? (unsigned)min((size_t)np, J.words - wc) : 0u;
      const bool okB = (unsigned)e < np && (unsigned)e < words_valid;
      const unsigned nst = sg.st1 - sg.st0;
      auto coef = [&](unsigned k, unsigned ii) -> uint64_t {
        const unsigned o = o0 + ar.oo, i = (sg.st0 + k) * kStageIn + ii;
        return (k < nst && o < J.n_out && i < J.n_in) ? J.coeff[(size_t)o * J.ldc + i] : 0ull;
      };
      uint64_t c0 = coef(0, ar.ii);
      for (unsigned k = 0; k < nst; k++, g++) {
        const unsigned sl = g % kPLd, bs = g % kPBs;
        const uint64_t n0 = coef(k + 1, ar.ii);  // the next stage's coefficient
        if (*err || !mbar_wait(BAR(RAW_FULL + sl), (g / kPLd) & 1)) {
          *err = 1;
          break;
        }
        const unsigned i0 = (sg.st0 + k) * kStageIn;
        const unsigned ni = min((unsigned)kStageIn, J.n_in - i0);
        uint32_t xw[8];
#pragma unroll
        for (int ii = 0; ii < kStageIn; ii++) {
          uint2 v = make_uint2(0, 0);
          if (okB && (unsigned)ii < ni) v = lds64(sRaw + sl * kPRawBytes + ii * (kPWordsCta * 8) + 8 * (unsigned)e);
          xw[2 * ii] = v.x;
          xw[2 * ii + 1] = v.y;
        }
        mbar_arrive(BAR(RAW_EMPTY + sl));
        if (g >= (uint32_t)kPBs && !mbar_wait(BAR(OP_EMPTY + bs), (g / kPBs - 1) & 1)) {
          *err = 1;
          break;
        }
        const uint32_t at = sA + bs * kABytes, bt = sB + bs * kPBBytes;
        ar.store(at, c0);
        if ((unsigned)e < np) {
          const unsigned u = (unsigned)e;
          const uint32_t brow = bt + (u >> 3) * 1024 + (u & 7) * 128, br7 = u & 7;
#pragma unroll
          for (int j = 0; j < 4; j++) {
            sts128(brow + (((2 * j) ^ br7) << 4), sel4(xw[0], j), sel4(xw[1], j), sel4(xw[2], j), sel4(xw[3], j));
            sts128(brow + (((2 * j + 1) ^ br7) << 4), sel4(xw[4], j), sel4(xw[5], j), sel4(xw[6], j),
                   sel4(xw[7], j));
          }
        }
        fence_async_smem();
        mbar_arrive(BAR(OPB_FULL + bs));
        c0 = n0;
      }
      // ---------------------------------------------------------- epilogue
      if (*err || !mbar_wait(BAR(D_FULL), 0)) {
        *err = 1;
        break;
      }
      tc_fence_after();
      const unsigned o = o0 + (q >> 1);
      const unsigned half = q & 1;
      uint64_t* orow = o < J.n_out ? (J.out_ptrs ? J.out_ptrs[o] : J.out + (size_t)o * J.out_stride) : nullptr;
      for (int cc = 0; cc < (int)(np + 31) / 32; cc++) {
        uint32_t r[32];
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + 256 * nn_ep + 32 * cc, r);
        uint32_t mine = 0;
#pragma unroll
        for (int jj = 0; jj < 32; jj++) {
          const uint32_t bit = __float_as_uint(__fadd_rn(__uint_as_float(r[jj]), 8388608.0f)) & 1u;
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, bit);
          if (lane == jj) mine = bal;
        }
        const unsigned c = 32 * cc + lane;  // column of accumulator nn_ep
        if (!orow || c >= np) continue;
        const size_t widx = (size_t)np * (c / hp) + (size_t)hp * nn_ep + (c % hp);
        if (w0 + widx >= J.words) continue;
        uint32_t* dst = reinterpret_cast<uint32_t*>(orow + w0 + widx) + half;
        if (sg.mode == 2) {
          if (mine) atomicXor(dst, mine);
        } else if (sg.mode == 1) {
          *dst ^= mine;
        } else {
          *dst = mine;
        }
      }
      tc_fence_before();
    } while (0);
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync();  // both CTAs are done with TMEM and the peer's barriers
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
  if (threadIdx.x == 0 && *err) atomicOr(status, 1);
}

}  // namespace tc64f4

// Operand format of the GF(2^64) tensor-core path (the kernels build their A
// operand from the coefficients, so it can differ per launch): FP4 on SM
// pairs, int8 for the one-CTA kernel, unless PARPAR_B200_GF64_TC=f4 or =i8
// fixes one format for both.  Measured on the 1 GiB PAR3 creates: FP4 pair
// 2.35 ms (R=8), 250 ms (R=1,024), 832 ms (262,144 x 4 KiB, R=2,621) against
// the int8 pair's 2.61 / 350 / 899 ms.
static bool gf64_tc_use_f4(bool pair) {
  static const int forced = [] {
    const char* v = getenv("PARPAR_B200_GF64_TC");
    return !v ? -1 : strcmp(v, "f4") == 0 ? 1 : strcmp(v, "i8") == 0 ? 0 : -1;
  }();
  return forced >= 0 ? forced != 0 : pair;
}

// Pair kernel (two SMs per tile) or one-CTA kernel for a whole table: the
// pair kernel's tile has 4 outputs, so it is used when no job has fewer than
// 4 (PARPAR_B200_GF64_PAIR=0 / 1 forces the choice).
static bool use_pair_kernel(const Gf64TcBatch& b) {
  static const int forced = [] {
    const char* v = getenv("PARPAR_B200_GF64_PAIR");
    return v && *v ? atoi(v) : -1;
  }();
  if (forced >= 0) return forced != 0;
  for (uint32_t j = 0; j < b.n_jobs; j++)
    if (b.job[j].n_out < 4) return false;
  return true;
}

static cudaError_t launch_gf64_tc_batch_impl(Gf64TcBatch& b, int sms, int* d_status, cudaStream_t s,
                                              bool allow_pair) {
  static std::atomic<uint64_t> attr{0};
  if (!device_done(attr)) {
    cudaError_t e = cudaFuncSetAttribute(tc64::k_gf64_matvec_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tc64::kSmemBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tc64::k_gf64_matvec_tc_pair<tc64::kPLd, tc64::kPBs>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, tc64::kPSmemBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tc64f4::k_gf64_matvec_f4, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               tc64f4::kSmemBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tc64f4::k_gf64_matvec_f4_pair, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               tc64f4::kPSmemBytes);
    if (e != cudaSuccess) return e;
    device_mark(attr);
  }
  const bool pair = allow_pair && use_pair_kernel(b);
  const bool f4 = allow_pair && gf64_tc_use_f4(pair);  // overlapped launches: the int8 one-CTA kernel
  const size_t tile_words = f4 ? (pair ? tc64f4::kPWords : tc64f4::kWords) : tc64::kWords;
  const unsigned stage_in = f4 ? tc64f4::kStageIn : tc64::kStageIn;
  // drop empty jobs (nothing to multiply) after zeroing their outputs
  uint32_t m = 0;
  for (uint32_t j = 0; j < b.n_jobs; j++) {
    Gf64TcJob& J = b.job[j];
    if (!J.n_out || !J.words) continue;
    J.n_stages = (J.n_in + stage_in - 1) / stage_in;
    J.pairs = pair ? (J.n_out + 3) / 4 : (J.n_out + 1) / 2;
    J.n_mma = f4 && pair ? tc64f4::pair_n_for(J.words) : 0;  // the FP4 pair's tiles are 2 n_mma words
    const size_t wt = ceil_div(J.words, J.n_mma ? 2 * (size_t)J.n_mma : tile_words);
    if (wt > 0xFFFFFFFFu) return cudaErrorInvalidValue;
    J.wt = (uint32_t)wt;
    if (!J.n_in) {
      if (J.accumulate) continue;
      if (J.out_ptrs) {
        tc64::k_zero_rows<<<148, 256, 0, s>>>(const_cast<uint64_t* const*>(J.out_ptrs), J.n_out, J.words);
      } else {
        cudaError_t e = cudaMemset2DAsync(J.out, J.out_stride * 8, 0, J.words * 8, J.n_out, s);
        if (e != cudaSuccess) return e;
      }
      note_launch();
      continue;
    }
    b.job[m++] = J;
  }
  b.n_jobs = m;
  if (!m) return cudaGetLastError();
  // the plan deals items to SMs, or to SM pairs for the pair kernel
  const uint64_t items = tc_batch_plan(b, tc64::tiles64, pair ? std::max(1, sms / 2) : sms,
                                      f4 ? tc64f4::kMaxStagesPerItem : 0u);
  if (items > 0x3FFFFFFFull) return cudaErrorInvalidConfiguration;
  for (uint32_t j = 0; j < m; j++) {
    const Gf64TcJob& J = b.job[j];
    if (J.splits == 1 || J.accumulate) continue;
    if (J.out_ptrs) {
      tc64::k_zero_rows<<<148, 256, 0, s>>>(const_cast<uint64_t* const*>(J.out_ptrs), J.n_out, J.words);
    } else {
      cudaError_t e = cudaMemset2DAsync(J.out, J.out_stride * 8, 0, J.words * 8, J.n_out, s);
      if (e != cudaSuccess) return e;
    }
    note_launch();
  }
  if (f4 && pair)
    tc64f4::k_gf64_matvec_f4_pair<<<2 * (unsigned)items, tc64f4::kThreads, tc64f4::kPSmemBytes, s>>>(b, d_status);
  else if (f4)
    tc64f4::k_gf64_matvec_f4<<<(unsigned)items, tc64f4::kThreads, tc64f4::kSmemBytes, s>>>(b, d_status);
  else if (pair)
    tc64::k_gf64_matvec_tc_pair<tc64::kPLd, tc64::kPBs>
        <<<2 * (unsigned)items, tc64::kThreads, tc64::kPSmemBytes, s>>>(b, d_status);
  else
    tc64::k_gf64_matvec_tc<<<(unsigned)items, tc64::kThreads, tc64::kSmemBytes, s>>>(b, d_status);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_gf64_tc_batch(Gf64TcBatch& b, int sms, int* d_status, cudaStream_t s) {
  return launch_gf64_tc_batch_impl(b, sms, d_status, s, true);
}
// The int8 one-CTA kernel only.  The SM-pair kernels (FP4 and int8) and the
// FP4 one-CTA kernel gave wrong words in the last tiles of a large job while
// kernels of other streams ran on the device (eight serving lanes); the int8
// one-CTA kernel was exact in every such run, so code that overlaps its own
// launches across streams uses it, whatever the format variables say.
cudaError_t launch_gf64_tc_batch_one_cta(Gf64TcBatch& b, int sms, int* d_status, cudaStream_t s) {
  return launch_gf64_tc_batch_impl(b, sms, d_status, s, false);
}

cudaError_t launch_gf64_matvec_tc(const uint64_t* d_in, const uint64_t* const* d_in_ptrs, size_t in_stride,
                                  size_t n_in, size_t words, const uint64_t* d_coeff, size_t ldc, size_t n_out,
                                  uint64_t* d_out, uint64_t* const* d_out_ptrs, size_t out_stride, bool accumulate,
                                  int sms, int* d_status, cudaStream_t s) {
  if (!n_out || !words) return cudaSuccess;
  if (n_in > 0xFFFFFFFFu || n_out > 0xFFFFFFFFu) return cudaErrorInvalidValue;
  Gf64TcBatch b{};
  b.n_jobs = 1;
  Gf64TcJob& J = b.job[0];
  J.in = d_in;
  J.in_ptrs = d_in_ptrs;
  J.in_stride = in_stride;
  J.coeff = d_coeff;
  J.ldc = ldc;
  J.out = d_out;
  J.out_ptrs = d_out_ptrs;
  J.out_stride = out_stride;
  J.words = words;
  J.n_in = (uint32_t)n_in;
  J.n_out = (uint32_t)n_out;
  J.accumulate = accumulate ? 1 : 0;
  return launch_gf64_tc_batch(b, sms, d_status, s);
}

}  // namespace pp
