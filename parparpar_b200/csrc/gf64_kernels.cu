// GF(2^64) kernels for the PAR3 hot path (sm_100a).
//
//  * k_gf64_cauchy       Cauchy coefficients inv((fI+c) ^ (fR+r)), 0 -> 1
//                        (reference src/par3_engine.cc:358-425), inverted in
//                        runs of 16 with one Itoh-Tsujii inverse per run
//                        (Montgomery's simultaneous-inversion trick).
//  * k_gf64_matvec_lut   out[r][w] ^= XOR_c M[r][c] * in[c][w]
//                        (the work of GF64Controller::WorkerThread,
//                        reference src/par3_engine.cc:784-917, semantics of
//                        gf64/gf64_region_scalar.c:63-91).
//  * region element ops  gf64_region_mul_arr / muladd_arr semantics
//                        (reference gf64/gf64_region_scalar.c:8-28).
//  * solve steps         GF64Controller::SolveAndReconstruct
//                        (reference src/par3_engine.cc:980-1053).
//
// Constant multiplication uses sixteen 4-bit split tables per coefficient,
// T_q[n] = c * n * x^(4q).  Each table is 16 x 8 B = 128 B = one full row of
// shared-memory banks, so a warp's 32 lookups into it are conflict-free.
#include "pp_common.cuh"
#include "pp_internal.h"

#include <algorithm>

namespace pp {

// ---------------------------------------------------------------- Cauchy
constexpr int kInvRun = 8;

__global__ void __launch_bounds__(128)
k_gf64_cauchy(uint64_t* __restrict__ m, size_t n_in, size_t n_rec, uint64_t fI, uint64_t fR, size_t ld) {
  const size_t runs_per_row = (n_in + kInvRun - 1) / kInvRun;
  const size_t total = runs_per_row * n_rec;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const size_t r = t / runs_per_row;
    const size_t c0 = (t % runs_per_row) * kInvRun;
    const uint64_t y = fR + r;
    uint64_t d[kInvRun], p[kInvRun];
#pragma unroll
    for (int j = 0; j < kInvRun; j++) {
      uint64_t v = (c0 + j < n_in) ? ((fI + c0 + j) ^ y) : 1;
      d[j] = v ? v : 1;
      p[j] = j ? gf64_mul(p[j - 1], d[j]) : d[j];
    }
    uint64_t inv = gf64_inv(p[kInvRun - 1]);
    uint64_t* row = m + r * ld;
#pragma unroll
    for (int j = kInvRun - 1; j >= 1; j--) {
      uint64_t v = gf64_mul(inv, p[j - 1]);
      inv = gf64_mul(inv, d[j]);
      if (c0 + j < n_in) row[c0 + j] = v;
    }
    row[c0] = inv;
  }
}

cudaError_t launch_gf64_cauchy(uint64_t* d_m, size_t n_in, size_t n_rec, uint64_t first_in, uint64_t first_rec,
                               size_t ld, cudaStream_t s) {
  size_t total = ceil_div(n_in, kInvRun) * n_rec;
  if (!total) return cudaSuccess;
  size_t blocks = ceil_div(total, 128);
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_gf64_cauchy<<<(unsigned)blocks, 128, 0, s>>>(d_m, n_in, n_rec, first_in, first_rec, ld);
  note_launch();
  return cudaGetLastError();
}

// A[r][c] = inv((fI + cols[c]) ^ (fR + r)), zero denominators mapped to 1:
// the repair system of lib/par3gen.js:3864-3880 (rows = the first n recovery
// equations, columns = the lost input blocks).
__global__ void k_gf64_cauchy_cols(uint64_t* __restrict__ A, size_t n_rows, const uint64_t* __restrict__ cols,
                                   size_t n_cols, uint64_t fI, uint64_t fR) {
  const size_t total = n_rows * n_cols;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const size_t r = t / n_cols, c = t % n_cols;
    uint64_t d = (fI + cols[c]) ^ (fR + r);
    A[t] = gf64_inv(d ? d : 1);
  }
}

cudaError_t launch_gf64_cauchy_cols(uint64_t* d_A, size_t n_rows, const uint64_t* d_cols, size_t n_cols, uint64_t fI,
                                    uint64_t fR, cudaStream_t s) {
  const size_t total = n_rows * n_cols;
  if (!total) return cudaSuccess;
  size_t blocks = std::min<size_t>(ceil_div(total, 128), 148 * 64);
  k_gf64_cauchy_cols<<<(unsigned)blocks, 128, 0, s>>>(d_A, n_rows, d_cols, n_cols, fI, fR);
  note_launch();
  return cudaGetLastError();
}

// Closed-form inverse of the repair system when it is a true Cauchy matrix
// (rows x_j = fR + j, columns y_i = fI + cols[i], all x_j != y_i so that no
// denominator was mapped to 1).  Over GF(2^m) (signs vanish):
//   (A^-1)[i][j] = b_i * a_j / (x_j + y_i)
//   a_j = prod_k (x_j + y_k) / prod_{k != j} (x_j + x_k)
//   b_i = prod_k (x_k + y_i) / prod_{k != i} (y_i + y_k)
// The solution of a nonsingular system is unique, so A^-1 * rhs equals the
// Gauss-Jordan result of the reference's SolveAndReconstruct
// (src/par3_engine.cc:980-1053) word for word.
//
// One warp per weight: lanes take every 32nd factor, then a shuffle tree
// multiplies the 32 partial products.
__device__ __forceinline__ uint64_t warp_gf64_prod(uint64_t v) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = gf64_mul(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void __launch_bounds__(256) k_gf64_cauchy_inv_weights(const uint64_t* __restrict__ cols, size_t n,
                                                                 uint64_t fI, uint64_t fR, uint64_t* __restrict__ wa,
                                                                 uint64_t* __restrict__ wb) {
  const unsigned lane = threadIdx.x & 31;
  const size_t w = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= 2 * n) return;
  uint64_t num = 1, den = 1;
  if (w < n) {  // a_j, j = w
    const uint64_t xj = fR + w;
    for (size_t k = lane; k < n; k += 32) {
      num = gf64_mul(num, xj ^ (fI + cols[k]));
      if (k != w) den = gf64_mul(den, xj ^ (fR + k));
    }
  } else {  // b_i, i = w - n
    const size_t i = w - n;
    const uint64_t yi = fI + cols[i];
    for (size_t k = lane; k < n; k += 32) {
      num = gf64_mul(num, (fR + k) ^ yi);
      if (k != i) den = gf64_mul(den, yi ^ (fI + cols[k]));
    }
  }
  num = warp_gf64_prod(num);
  den = warp_gf64_prod(den);
  if (lane == 0) {
    const uint64_t v = gf64_mul(num, gf64_inv(den));
    if (w < n) wa[w] = v;
    else wb[w - n] = v;
  }
}

// Ainv[i][j] = wb[i] * wa[j] * A[j][i]  (A[j][i] = 1 / (x_j + y_i))
__global__ void k_gf64_cauchy_inv_assemble(const uint64_t* __restrict__ A, const uint64_t* __restrict__ wa,
                                           const uint64_t* __restrict__ wb, size_t n, uint64_t* __restrict__ Ainv) {
  const size_t total = n * n;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const size_t i = t / n, j = t % n;
    Ainv[t] = gf64_mul(gf64_mul(wb[i], wa[j]), A[j * n + i]);
  }
}

cudaError_t launch_gf64_cauchy_inverse(const uint64_t* d_A, const uint64_t* d_cols, size_t n, uint64_t fI,
                                       uint64_t fR, uint64_t* d_w, uint64_t* d_Ainv, cudaStream_t s) {
  if (!n) return cudaSuccess;
  const size_t warps = 2 * n;
  k_gf64_cauchy_inv_weights<<<(unsigned)ceil_div(warps * 32, 256), 256, 0, s>>>(d_cols, n, fI, fR, d_w, d_w + n);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t blocks = std::min<size_t>(ceil_div(n * n, 256), 148 * 32);
  k_gf64_cauchy_inv_assemble<<<(unsigned)blocks, 256, 0, s>>>(d_A, d_w, d_w + n, n, d_Ainv);
  note_launch();
  return cudaGetLastError();
}

// inverse of every element, inverse(0) = 0 (reference gf64/gf64_invert.c:29-75)
__global__ void __launch_bounds__(128)
k_gf64_inverse_batch(uint64_t* __restrict__ out, const uint64_t* __restrict__ in, size_t n) {
  const size_t runs = (n + kInvRun - 1) / kInvRun;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < runs; t += (size_t)gridDim.x * blockDim.x) {
    const size_t c0 = t * kInvRun;
    uint64_t d[kInvRun], p[kInvRun];
    uint32_t zero = 0;
#pragma unroll
    for (int j = 0; j < kInvRun; j++) {
      uint64_t v = (c0 + j < n) ? in[c0 + j] : 1;
      if (!v) zero |= 1u << j;
      d[j] = v ? v : 1;
      p[j] = j ? gf64_mul(p[j - 1], d[j]) : d[j];
    }
    uint64_t inv = gf64_inv(p[kInvRun - 1]);
    uint64_t res[kInvRun];
#pragma unroll
    for (int j = kInvRun - 1; j >= 1; j--) {
      res[j] = gf64_mul(inv, p[j - 1]);
      inv = gf64_mul(inv, d[j]);
    }
    res[0] = inv;
#pragma unroll
    for (int j = 0; j < kInvRun; j++)
      if (c0 + j < n) out[c0 + j] = ((zero >> j) & 1) ? 0 : res[j];
  }
}

cudaError_t launch_gf64_inverse_batch(uint64_t* d_out, const uint64_t* d_in, size_t n, cudaStream_t s) {
  size_t runs = ceil_div(n, kInvRun);
  if (!runs) return cudaSuccess;
  size_t blocks = ceil_div(runs, 128);
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_gf64_inverse_batch<<<(unsigned)blocks, 128, 0, s>>>(d_out, d_in, n);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- matvec
constexpr int kMvT = 256;         // threads
constexpr int kMvW = 4;           // words per thread
constexpr int kMvTile = kMvT * kMvW;
constexpr int kMvR = 8;           // outputs per block
constexpr int kMvStage = 2;       // inputs per table stage (double buffered)
constexpr size_t kMvTabWords = (size_t)kMvStage * kMvR * 256;  // u64 per buffer
constexpr size_t kMvSmem = 2 * kMvTabWords * sizeof(uint64_t);  // 64 KiB

// Fill the 16 tables of coefficient c: T[q][n] = c * n * x^(4q).
PP_D void gf64_build_tables(uint64_t* T, uint64_t c, int q) {
  uint64_t b0 = (q == 0) ? c : gf64_reduce(c >> (64 - 4 * q), c << (4 * q));
  uint64_t b1 = gf64_dbl(b0), b2 = gf64_dbl(b1), b3 = gf64_dbl(b2);
  uint64_t* t = T + q * 16;
  t[0] = 0;
  t[1] = b0;
  t[2] = b1;
  t[3] = b1 ^ b0;
  t[4] = b2;
  t[5] = b2 ^ b0;
  t[6] = b2 ^ b1;
  t[7] = b2 ^ b1 ^ b0;
  t[8] = b3;
  t[9] = b3 ^ b0;
  t[10] = b3 ^ b1;
  t[11] = b3 ^ b1 ^ b0;
  t[12] = b3 ^ b2;
  t[13] = b3 ^ b2 ^ b0;
  t[14] = b3 ^ b2 ^ b1;
  t[15] = b3 ^ b2 ^ b1 ^ b0;
}

// mode: 0 overwrite, 1 xor into existing, 2 atomic xor (split inputs)
// Row addressing: input c is in_ptrs ? in_ptrs[c] : in + c*in_stride; output
// r likewise.
__global__ void __launch_bounds__(kMvT, 2)
k_gf64_matvec_lut(const uint64_t* __restrict__ in, const uint64_t* const* __restrict__ in_ptrs, size_t in_stride,
                  size_t n_in, size_t words, const uint64_t* __restrict__ coeff, size_t ldc, size_t n_out,
                  uint64_t* __restrict__ out, uint64_t* const* __restrict__ out_ptrs, size_t out_stride,
                  size_t inputs_per_split, int mode) {
  extern __shared__ __align__(16) uint64_t smem[];
  const size_t r0 = (size_t)blockIdx.x * kMvR;
  const size_t w0 = (size_t)blockIdx.y * kMvTile;
  const size_t i_begin = (size_t)blockIdx.z * inputs_per_split;
  const size_t i_end = min(n_in, i_begin + inputs_per_split);
  if (i_begin >= i_end) return;

  uint64_t acc[kMvW][kMvR];
#pragma unroll
  for (int j = 0; j < kMvW; j++)
#pragma unroll
    for (int o = 0; o < kMvR; o++) acc[j][o] = 0;

  // table layout per buffer: [stage input][output][q][n]
  auto build = [&](size_t ib, uint64_t* buf) {
    for (int t = threadIdx.x; t < kMvStage * kMvR * 16; t += kMvT) {
      int q = t & 15, o = (t >> 4) % kMvR, j = (t >> 4) / kMvR;
      size_t c = ib + j;
      uint64_t k = (c < i_end && r0 + o < n_out) ? coeff[(r0 + o) * ldc + c] : 0;
      gf64_build_tables(buf + ((size_t)j * kMvR + o) * 256, k, q);
    }
  };

  const size_t nstages = (i_end - i_begin + kMvStage - 1) / kMvStage;
  build(i_begin, smem);
  __syncthreads();
  for (size_t s = 0; s < nstages; s++) {
    const size_t ib = i_begin + s * kMvStage;
    uint64_t* cur = smem + (s & 1) * kMvTabWords;
    if (s + 1 < nstages) build(ib + kMvStage, smem + ((s + 1) & 1) * kMvTabWords);
    const int ns = (int)min((size_t)kMvStage, i_end - ib);
    for (int j = 0; j < ns; j++) {
      const uint64_t* row = in_ptrs ? in_ptrs[ib + j] : in + (ib + j) * in_stride;
      uint64_t x[kMvW];
#pragma unroll
      for (int u = 0; u < kMvW; u++) {
        size_t w = w0 + threadIdx.x + u * kMvT;
        x[u] = w < words ? __ldg(row + w) : 0;
      }
      const uint64_t* T = cur + (size_t)j * kMvR * 256;
#pragma unroll
      for (int u = 0; u < kMvW; u++) {
        uint32_t lo = (uint32_t)x[u], hi = (uint32_t)(x[u] >> 32);
        uint32_t nib[16];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          nib[q] = (lo >> (4 * q)) & 15;
          nib[q + 8] = (hi >> (4 * q)) & 15;
        }
#pragma unroll
        for (int o = 0; o < kMvR; o++) {
          const uint64_t* To = T + o * 256;
          uint64_t a = 0;
#pragma unroll
          for (int q = 0; q < 16; q++) a ^= To[q * 16 + nib[q]];
          acc[u][o] ^= a;
        }
      }
    }
    __syncthreads();
  }

#pragma unroll
  for (int o = 0; o < kMvR; o++) {
    if (r0 + o >= n_out) continue;
    uint64_t* orow = out_ptrs ? out_ptrs[r0 + o] : out + (r0 + o) * out_stride;
#pragma unroll
    for (int u = 0; u < kMvW; u++) {
      size_t w = w0 + threadIdx.x + u * kMvT;
      if (w >= words) continue;
      if (mode == 2) {
        if (acc[u][o]) atomicXor(reinterpret_cast<unsigned long long*>(orow + w), (unsigned long long)acc[u][o]);
      } else if (mode == 1) {
        orow[w] ^= acc[u][o];
      } else {
        orow[w] = acc[u][o];
      }
    }
  }
}

static cudaError_t matvec_common(const uint64_t* d_in, const uint64_t* const* d_in_ptrs, size_t in_stride,
                                 size_t n_in, size_t words, const uint64_t* d_coeff, size_t ldc, size_t n_out,
                                 uint64_t* d_out, uint64_t* const* d_out_ptrs, size_t out_stride, bool accumulate,
                                 int sms, cudaStream_t s) {
  if (!n_out || !words) return cudaSuccess;
  static std::atomic<uint64_t> attr{0};
  if (!device_done(attr)) {
    cudaError_t e = cudaFuncSetAttribute(k_gf64_matvec_lut, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMvSmem);
    if (e != cudaSuccess) return e;
    device_mark(attr);
  }
  const size_t rt = ceil_div(n_out, kMvR);
  const size_t wt = ceil_div(words, kMvTile);
  const size_t base = rt * wt;
  const size_t target = (size_t)(sms > 0 ? sms : 148) * 3;
  size_t splits = base >= target ? 1 : ceil_div(target, base);
  size_t max_splits = ceil_div(n_in, kMvStage * 4);
  if (splits > max_splits) splits = max_splits;
  if (splits < 1) splits = 1;
  size_t per = ceil_div(ceil_div(n_in, splits), kMvStage) * kMvStage;
  splits = ceil_div(n_in, per);
  if (splits > 65535) {
    splits = 65535;
    per = ceil_div(n_in, splits);
    splits = ceil_div(n_in, per);
  }
  int mode;
  if (splits <= 1) {
    mode = accumulate ? 1 : 0;
    splits = 1;
    per = n_in;
  } else {
    mode = 2;
    if (!accumulate) {
      if (d_out_ptrs) return cudaErrorInvalidValue;  // caller zeroes pointer-table outputs
      cudaError_t e = cudaMemset2DAsync(d_out, out_stride * 8, 0, words * 8, n_out, s);
      note_launch();
      if (e != cudaSuccess) return e;
    }
  }
  if (rt > 65535 || wt > 65535) return cudaErrorInvalidConfiguration;
  dim3 grid((unsigned)rt, (unsigned)wt, (unsigned)splits);
  k_gf64_matvec_lut<<<grid, kMvT, kMvSmem, s>>>(d_in, d_in_ptrs, in_stride, n_in, words, d_coeff, ldc, n_out, d_out,
                                               d_out_ptrs, out_stride, per, mode);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_gf64_matvec(const uint64_t* d_in, size_t in_stride, size_t n_in, size_t words,
                               const uint64_t* d_coeff, size_t ldc, size_t n_out, uint64_t* d_out,
                               size_t out_stride, bool accumulate, int sms, cudaStream_t s) {
  if (!n_in) {
    if (accumulate || !n_out || !words) return cudaSuccess;
    note_launch();
    return cudaMemset2DAsync(d_out, out_stride * 8, 0, words * 8, n_out, s);
  }
  return matvec_common(d_in, nullptr, in_stride, n_in, words, d_coeff, ldc, n_out, d_out, nullptr, out_stride,
                       accumulate, sms, s);
}

cudaError_t launch_gf64_2d_gather(uint64_t* const* d_outs, size_t K, const uint64_t* const* d_ins, size_t G,
                                  const uint64_t* d_coeff, size_t kstride, size_t len, int sms, cudaStream_t s) {
  if (!G) return cudaSuccess;
  return matvec_common(nullptr, d_ins, 0, G, len, d_coeff, kstride, K, nullptr, d_outs, 0, true, sms, s);
}

// ---------------------------------------------------------------- region
__global__ void k_gf64_region_mul_arr(uint64_t* __restrict__ out, const uint64_t* __restrict__ in,
                                      const uint64_t* __restrict__ coeff, size_t len, size_t n_coeff) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x)
    out[i] = gf64_mul(in[i], coeff[n_coeff == 1 ? 0 : i % n_coeff]);
}

// XOR over coefficients of in*coeff_c == in * (XOR of the coefficients):
// multiplication distributes over field addition, so the fold is exact.
__global__ void k_gf64_region_muladd_arr(uint64_t* __restrict__ out, const uint64_t* __restrict__ in,
                                         const uint64_t* __restrict__ coeff, size_t len, size_t n_coeff) {
  __shared__ uint64_t csum;
  if (threadIdx.x == 0) {
    uint64_t s = 0;
    for (size_t c = 0; c < n_coeff; c++) s ^= coeff[c];
    csum = s;
  }
  __syncthreads();
  const uint64_t k = csum;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x)
    out[i] ^= gf64_mul(in[i], k);
}

cudaError_t launch_gf64_region_mul_arr(uint64_t* d_out, const uint64_t* d_in, const uint64_t* d_coeff, size_t len,
                                       size_t n_coeff, cudaStream_t s) {
  if (!len) return cudaSuccess;
  size_t blocks = ceil_div(len, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_gf64_region_mul_arr<<<(unsigned)blocks, 256, 0, s>>>(d_out, d_in, d_coeff, len, n_coeff);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_gf64_region_muladd_arr(uint64_t* d_out, const uint64_t* d_in, const uint64_t* d_coeff,
                                          size_t len, size_t n_coeff, cudaStream_t s) {
  if (!len) return cudaSuccess;
  size_t blocks = ceil_div(len, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_gf64_region_muladd_arr<<<(unsigned)blocks, 256, 0, s>>>(d_out, d_in, d_coeff, len, n_coeff);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- solve
// Step `col`: pivot search (first nonzero at or below the diagonal), row swap
// of A, pivot-row scaling of A, and the multiplier column fcol[r] = A[r][col].
// piv[0] = pivot row, piv[1] = inverse of the pivot.
__global__ void k_gf64_solve_pivot(uint64_t* __restrict__ A, size_t n, size_t col, uint64_t* __restrict__ fcol,
                                   uint64_t* __restrict__ piv, int* __restrict__ status) {
  __shared__ unsigned long long best;
  if (*(volatile int*)status != 0) return;
  if (threadIdx.x == 0) best = ~0ull;
  __syncthreads();
  for (size_t r = col + threadIdx.x; r < n; r += blockDim.x)
    if (A[r * n + col] != 0) {
      atomicMin(&best, (unsigned long long)r);
      break;
    }
  __syncthreads();
  const size_t p = (size_t)best;
  if (p == ~0ull || p >= n) {
    if (threadIdx.x == 0) *status = -1;
    return;
  }
  if (p != col) {
    for (size_t j = threadIdx.x; j < n; j += blockDim.x) {
      uint64_t t = A[col * n + j];
      A[col * n + j] = A[p * n + j];
      A[p * n + j] = t;
    }
    __syncthreads();
  }
  const uint64_t pv = A[col * n + col];
  const uint64_t pinv = gf64_inv(pv);
  __syncthreads();
  if (pv != 1)
    for (size_t j = threadIdx.x; j < n; j += blockDim.x) A[col * n + j] = gf64_mul(A[col * n + j], pinv);
  for (size_t r = threadIdx.x; r < n; r += blockDim.x) fcol[r] = (r == col) ? 0 : A[r * n + col];
  if (threadIdx.x == 0) {
    piv[0] = p;
    piv[1] = pinv;
  }
}

// Swap RHS rows col <-> pivot and scale the pivot row (SET, not accumulate).
__global__ void k_gf64_solve_rhs_pivot(uint64_t* __restrict__ rhs, size_t B, size_t col,
                                       const uint64_t* __restrict__ piv, const int* __restrict__ status) {
  if (*(volatile const int*)status != 0) return;
  const size_t p = (size_t)piv[0];
  const uint64_t pinv = piv[1];
  for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < B; w += (size_t)gridDim.x * blockDim.x) {
    uint64_t a = rhs[col * B + w];
    uint64_t b = rhs[p * B + w];
    if (p != col) rhs[p * B + w] = a;
    rhs[col * B + w] = pinv == 1 ? b : gf64_mul(b, pinv);
  }
}

// Eliminate column `col` from every row r != col of [A | rhs]:
//   A[r][j] ^= f_r * A[col][j] (j >= col), rhs[r][w] ^= f_r * rhs[col][w].
// grid.y = row; grid.x = chunks over (n - col) + B elements.
__global__ void __launch_bounds__(256)
k_gf64_solve_eliminate(uint64_t* __restrict__ A, uint64_t* __restrict__ rhs, size_t n, size_t B, size_t col,
                       const uint64_t* __restrict__ fcol, const int* __restrict__ status) {
  __shared__ uint64_t T[256];
  const size_t r = blockIdx.y;
  if (*(volatile const int*)status != 0) return;
  const uint64_t f = fcol[r];
  if (r == col || f == 0) return;
  if (threadIdx.x < 16) gf64_build_tables(T, f, threadIdx.x);
  __syncthreads();
  const size_t na = n - col;
  const size_t total = na + B;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    uint64_t src, *dst;
    if (e < na) {
      src = A[col * n + col + e];
      dst = A + r * n + col + e;
    } else {
      src = rhs[col * B + (e - na)];
      dst = rhs + r * B + (e - na);
    }
    uint32_t lo = (uint32_t)src, hi = (uint32_t)(src >> 32);
    uint64_t a = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      a ^= T[q * 16 + ((lo >> (4 * q)) & 15)];
      a ^= T[(q + 8) * 16 + ((hi >> (4 * q)) & 15)];
    }
    *dst ^= a;
  }
}

cudaError_t launch_gf64_solve(uint64_t* d_A, uint64_t* d_rhs, size_t n, size_t B, uint64_t* d_fcol, int* d_status,
                              cudaStream_t s) {
  // d_fcol holds n multipliers followed by 2 words of pivot info
  uint64_t* piv = d_fcol + n;
  for (size_t col = 0; col < n; col++) {
    k_gf64_solve_pivot<<<1, 1024, 0, s>>>(d_A, n, col, d_fcol, piv, d_status);
    unsigned rb = (unsigned)std::min<size_t>(ceil_div(B, 256), 148 * 4);
    if (rb < 1) rb = 1;
    if (B) k_gf64_solve_rhs_pivot<<<rb, 256, 0, s>>>(d_rhs, B, col, piv, d_status);
    size_t per_row = (n - col) + B;
    unsigned cx = (unsigned)std::min<size_t>(ceil_div(per_row, 256 * 4), 64);
    if (cx < 1) cx = 1;
    dim3 grid(cx, (unsigned)n);
    k_gf64_solve_eliminate<<<grid, 256, 0, s>>>(d_A, d_rhs, n, B, col, d_fcol, d_status);
    note_launch(B ? 3 : 2);
  }
  return cudaGetLastError();
}

// dst ^= src over `bytes` bytes (16-byte vectors where both are aligned,
// bytes otherwise)
__global__ void k_xor_bytes(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, size_t bytes, bool vec) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t done = 0;
  if (vec) {
    const size_t nv = bytes / 16;
    uint4* d = reinterpret_cast<uint4*>(dst);
    const uint4* q = reinterpret_cast<const uint4*>(src);
    for (size_t i = t; i < nv; i += stride) {
      uint4 a = d[i];
      const uint4 b = q[i];
      a.x ^= b.x;
      a.y ^= b.y;
      a.z ^= b.z;
      a.w ^= b.w;
      d[i] = a;
    }
    done = nv * 16;
  }
  for (size_t i = done + t; i < bytes; i += stride) dst[i] ^= src[i];
}

cudaError_t launch_xor_bytes(uint8_t* d_dst, const uint8_t* d_src, size_t bytes, cudaStream_t s) {
  if (!bytes) return cudaSuccess;
  const bool vec = ((uintptr_t)d_dst % 16) == 0 && ((uintptr_t)d_src % 16) == 0;
  const size_t units = vec ? bytes / 16 + 16 : bytes;
  const unsigned blocks = (unsigned)std::min<size_t>(ceil_div(units, 256), 148 * 8);
  k_xor_bytes<<<std::max(1u, blocks), 256, 0, s>>>(d_dst, d_src, bytes, vec);
  note_launch();
  return cudaGetLastError();
}

}  // namespace pp
