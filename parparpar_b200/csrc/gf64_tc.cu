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

#include "pp_common.cuh"
#include "pp_internal.h"
#include "tc_common.cuh"

namespace pp {
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

// mode: 0 overwrite, 1 xor into existing, 2 atomic xor (inputs split across CTAs)
// Rows: input i at in_ptrs ? in_ptrs[i] : in + i*in_stride (words); output r
// at out_ptrs ? out_ptrs[r] : out + r*out_stride.
__global__ void __launch_bounds__(kThreads, 1)
k_gf64_matvec_tc(const uint64_t* __restrict__ in, const uint64_t* const* __restrict__ in_ptrs, size_t in_stride,
                 unsigned n_in, size_t words, const uint64_t* __restrict__ coeff, size_t ldc, unsigned n_out,
                 uint64_t* __restrict__ out, uint64_t* const* __restrict__ out_ptrs, size_t out_stride,
                 unsigned stages_per_split, int mode, int* __restrict__ status) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t base_s = smem_addr(smem_raw);
  const uint32_t pad = ((base_s + 1023) & ~1023u) - base_s;
  uint8_t* smem = smem_raw + pad;
  const uint32_t sA = base_s + pad + kOffA, sB = base_s + pad + kOffB, sRaw = base_s + pad + kOffRaw;
  uint8_t* a_p = smem + kOffA;
  uint8_t* b_p = smem + kOffB;
  const uint8_t* raw_p = smem + kOffRaw;
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
  auto BAR = [&](int k) { return bar0 + 8u * (uint32_t)k; };
  volatile uint32_t* tmem_holder = reinterpret_cast<volatile uint32_t*>(smem + kOffBar + 8 * NBARS);
  volatile int* err = reinterpret_cast<volatile int*>(smem + kOffBar + 8 * NBARS + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned o0 = 2 * blockIdx.x;  // output pair
  const size_t w0 = (size_t)blockIdx.y * kWords;
  const unsigned n_stages_total = (n_in + kStageIn - 1) / kStageIn;
  const unsigned st_begin = blockIdx.z * stages_per_split;
  const unsigned st_end = min(n_stages_total, st_begin + stages_per_split);
  const unsigned nst = st_end > st_begin ? st_end - st_begin : 0;
  const unsigned words_valid = (unsigned)min((size_t)kWords, words - w0);
  const uint32_t raw_copy = (uint32_t)(((size_t)words_valid * 8 + 15) & ~(size_t)15);

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

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      unsigned issued = 0;
      for (unsigned k = 0; k < nst && !*err; k++) {
        const unsigned sl = k % kLd, use = k / kLd;
        if (k >= (unsigned)kLd && !mbar_wait(BAR(RAW_EMPTY + sl), (use - 1) & 1)) {
          *err = 1;
          break;
        }
        const unsigned i0 = (st_begin + k) * kStageIn;
        const unsigned ni = min((unsigned)kStageIn, n_in - i0);
        mbar_expect_tx(BAR(RAW_FULL + sl), raw_copy * ni);
        for (unsigned ii = 0; ii < ni; ii++) {
          const uint64_t* row = in_ptrs ? in_ptrs[i0 + ii] : in + (size_t)(i0 + ii) * in_stride;
          bulk_g2s(sRaw + sl * kRawBytes + ii * (kWords * 8), row + w0, raw_copy, BAR(RAW_FULL + sl));
        }
        issued = k + 1;
      }
      if (*err) {
        for (unsigned k = issued > (unsigned)kLd ? issued - kLd : 0; k < issued; k++)
          mbar_wait(BAR(RAW_FULL + k % kLd), (k / kLd) & 1);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      for (unsigned k = 0; k < nst; k++) {
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
            mma_i8(tmem + nn * 256, sw128_desc(sA + bs * kABytes + 32 * kk),
                   sw128_desc(sB + bs * kBBytes + nn * (256 * 128) + 32 * kk), kIdesc, (k > 0 || kk > 0) ? 1u : 0u);
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
    const unsigned n = 2 * e;        // B: word pair n, n+1 of the tile
    const unsigned sw = (e >> 2) & 1;  // store order: conflict-free 128-bit phases
    const unsigned mA = n + sw, mB = n + 1 - sw;
    const uint32_t rowA = (mA >> 3) * 1024 + (mA & 7) * 128, rA = mA & 7;
    const uint32_t rowB = (mB >> 3) * 1024 + (mB & 7) * 128, rB = mB & 7;
    const bool okA = mA < words_valid, okB = mB < words_valid;
    // A: row m, input half ii (adjacent threads alternate ii so a 64-bit store
    // phase of 16 threads covers 8 rows x 2 halves = all 32 banks)
    const unsigned a_ii = e & 1, a_m = e >> 1, a_oo = a_m >> 6, a_b = a_m & 63;
    const uint32_t arow_off = (a_m >> 3) * 1024 + (a_m & 7) * 128 + 8 * a_ii, ar7 = a_m & 7;
    auto coef = [&](unsigned k) -> uint64_t {
      const unsigned o = o0 + a_oo, i = (st_begin + k) * kStageIn + a_ii;
      return (k < nst && o < n_out && i < n_in) ? coeff[(size_t)o * ldc + i] : 0ull;
    };
    uint64_t c_cur = coef(0);
    for (unsigned k = 0; k < nst; k++) {
      const unsigned sl = k % kLd, bs = k % kBs;
      const uint64_t c_nxt = coef(k + 1);  // prefetch the next stage's coefficient
      // row b of the multiplication matrix of c_cur (closed form, see header)
      const uint64_t rv = __brevll(c_cur);
      uint64_t qrow = rv >> (63 - a_b);
#pragma unroll
      for (int si = 0; si < 4; si++) {
        const int sft = si == 0 ? 0 : si == 1 ? 1 : si == 2 ? 3 : 4;
        const int d = (int)a_b - sft;
        if (d >= 0) {
          if (d + 1 < 64) qrow ^= rv << (d + 1);
          if (d <= 2) qrow ^= rv << (d + 61);
          if (d <= 1) qrow ^= rv << (d + 62);
        }
      }
      const uint32_t qlo = (uint32_t)qrow, qhi = (uint32_t)(qrow >> 32);
      if (*err || !mbar_wait(BAR(RAW_FULL + sl), (k / kLd) & 1)) {
        *err = 1;
        break;
      }
      const unsigned i0 = (st_begin + k) * kStageIn;
      const unsigned ni = min((unsigned)kStageIn, n_in - i0);
      const uint8_t* raw = raw_p + sl * kRawBytes;
      // B rows of words mA and mB: (lo, hi) of input 0, then (lo, hi) of input 1
      uint4 xA = make_uint4(0, 0, 0, 0), xB = make_uint4(0, 0, 0, 0);
#pragma unroll
      for (int ii = 0; ii < kStageIn; ii++) {
        if ((unsigned)ii >= ni) continue;
        // v = word n (x, y) and word n+1 (z, w) of input ii
        const uint4 v = *reinterpret_cast<const uint4*>(raw + ii * (kWords * 8) + 8 * n);
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
      if (k >= (unsigned)kBs && !mbar_wait(BAR(OP_EMPTY + bs), (k / kBs - 1) & 1)) {
        *err = 1;
        break;
      }
      uint8_t* at = a_p + bs * kABytes;
      uint8_t* bt = b_p + bs * kBBytes;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        *reinterpret_cast<uint2*>(at + arow_off + ((j ^ ar7) << 4)) = make_uint2(qlo >> j, qhi >> j);
        *reinterpret_cast<uint4*>(bt + rowA + ((j ^ rA) << 4)) = make_uint4(xA.x >> j, xA.y >> j, xA.z >> j, xA.w >> j);
        *reinterpret_cast<uint4*>(bt + rowB + ((j ^ rB) << 4)) = make_uint4(xB.x >> j, xB.y >> j, xB.z >> j, xB.w >> j);
      }
      fence_async_smem();
      mbar_arrive(BAR(OP_FULL + bs));
      c_cur = c_nxt;
    }
    // ------------------------------------------------------------ epilogue
    const bool have = nst > 0 && !*err && mbar_wait(BAR(D_FULL), 0);
    if (nst > 0 && !have) *err = 1;
    tc_fence_after();
    const int q = warp & 3;             // TMEM lane quarter: rows 32q..32q+31
    const int chalf = (warp - 2) >> 2;  // columns [256*chalf, 256*chalf + 256)
    const unsigned o = o0 + (q >> 1);   // output of these rows
    const unsigned half = q & 1;        // bits [32*half, 32*half + 32)
    for (int cc = 8 * chalf; cc < 8 * chalf + 8; cc++) {
      uint32_t r[32];
      if (have) {
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + 32 * cc, r);
      } else {
#pragma unroll
        for (int jj = 0; jj < 32; jj++) r[jj] = 0;
      }
      uint32_t mine = 0;
#pragma unroll
      for (int jj = 0; jj < 32; jj++) {
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, r[jj] & 1u);
        if (lane == jj) mine = bal;
      }
      const unsigned widx = 32 * cc + lane;
      if (!have || o >= n_out || widx >= words_valid) continue;
      uint64_t* orow = out_ptrs ? out_ptrs[o] : out + (size_t)o * out_stride;
      uint32_t* dst = reinterpret_cast<uint32_t*>(orow + w0 + widx) + half;
      if (mode == 2) {
        if (mine) atomicXor(dst, mine);
      } else if (mode == 1) {
        *dst ^= mine;
      } else {
        *dst = mine;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
  if (threadIdx.x == 0 && *err) atomicOr(status, 1);
}

}  // namespace tc64

cudaError_t launch_gf64_matvec_tc(const uint64_t* d_in, const uint64_t* const* d_in_ptrs, size_t in_stride,
                                  size_t n_in, size_t words, const uint64_t* d_coeff, size_t ldc, size_t n_out,
                                  uint64_t* d_out, uint64_t* const* d_out_ptrs, size_t out_stride, bool accumulate,
                                  int sms, int* d_status, cudaStream_t s) {
  if (!n_out || !words) return cudaSuccess;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(tc64::k_gf64_matvec_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tc64::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const size_t pairs = ceil_div(n_out, 2);
  const size_t wt = ceil_div(words, tc64::kWords);
  const size_t n_stages = ceil_div(n_in, tc64::kStageIn);
  const size_t base = pairs * wt;
  const size_t target = (size_t)(sms > 0 ? sms : 148);
  // fill the SMs in one wave: floor, never more CTAs than SMs from splitting
  size_t splits = base >= target ? 1 : std::max<size_t>(1, target / base);
  size_t max_splits = std::max<size_t>(1, n_stages / 16);
  if (splits > max_splits) splits = max_splits;
  size_t per = ceil_div(n_stages, splits);
  splits = ceil_div(n_stages, per);
  int mode;
  if (splits == 1) {
    mode = accumulate ? 1 : 0;
  } else {
    mode = 2;
    if (!accumulate) {
      if (d_out_ptrs) return cudaErrorInvalidValue;
      cudaError_t e = cudaMemset2DAsync(d_out, out_stride * 8, 0, words * 8, n_out, s);
      note_launch();
      if (e != cudaSuccess) return e;
    }
  }
  if (pairs > 0x7FFFFFFF || wt > 65535 || splits > 65535) return cudaErrorInvalidConfiguration;
  dim3 grid((unsigned)pairs, (unsigned)wt, (unsigned)splits);
  tc64::k_gf64_matvec_tc<<<grid, tc64::kThreads, tc64::kSmemBytes, s>>>(
      d_in, d_in_ptrs, in_stride, (unsigned)n_in, words, d_coeff, ldc, (unsigned)n_out, d_out, d_out_ptrs,
      out_stride, (unsigned)per, mode, d_status);
  note_launch();
  return cudaGetLastError();
}

}  // namespace pp
