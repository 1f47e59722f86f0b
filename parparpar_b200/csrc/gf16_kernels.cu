// GF(2^16) kernels for the PAR2 hot path (sm_100a).
//
//  * k_gf16_coeff_matrix   PAR2 coefficients 2^(L_i * e_o mod 65535)
//                          (reference gf16/gfmat_coeff.c:84-101).
//  * k_gf16_muladd_lut     the region multiply-accumulate
//                          out[o] ^= XOR_i c[o][i] * in[i]
//                          (the work of Galois16Mul::mul_add_multi_packpf as
//                          driven by PAR2ProcCPU::compute_worker,
//                          reference gf16/controller_cpu.cpp:463-537).
//  * k_gf16_pivot / k_gf16_eliminate
//                          one Gauss-Jordan step of Galois16RecMatrix::Compute
//                          (reference gf16/gfmat_inv.cpp:137-278,560-690).
//
// Multiplication by a per-(output,input) constant c is done with 4-bit split
// tables T_q[n] = c * (n << 4q), q = 0..3, kept in shared memory.  A 16-entry
// table of 64-bit entries occupies exactly the 32 banks, so a warp's 32
// lookups into one table never conflict (distinct entries sit in distinct
// banks, equal entries broadcast).  Each 64-bit entry packs the partial
// products of FOUR outputs, so the nibble indices of one input word are
// extracted once and serve four outputs per lookup.
#include "pp_common.cuh"
#include "pp_internal.h"

namespace pp {

// ---------------------------------------------------------------- coeffs
PP_D uint16_t gf16_pow2(uint32_t e) {
  uint32_t r = 1, b = 2;
  while (e) {
    if (e & 1) r = gf16_mul(r, b);
    b = gf16_mul(b, b);
    e >>= 1;
  }
  return (uint16_t)r;
}

// 2^k for k = 0..65535 (2^65535 = 2^0): a PAR2 coefficient
// 2^(L * e mod 65535) is one lookup.  128 KiB per device, filled once per
// device (pp_ctx_create waits for it; a launch that finds it unfilled fills it
// first on its own stream).
// g_gf16_inv[x] = 1/x (0 for x = 0), for the inversion kernels.
__device__ uint16_t g_gf16_exp[65536];
__device__ __align__(16) uint16_t g_gf16_inv[65536];
static std::atomic<uint64_t> g_gf16_exp_ready{0};

__global__ void k_gf16_exp_init() {
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < 65536; k += gridDim.x * blockDim.x) {
    g_gf16_exp[k] = gf16_pow2(k % 65535u);
    g_gf16_inv[k] = gf16_inv_euclid((uint16_t)k);
  }
}

static cudaError_t exp_table_on(cudaStream_t s) {
  if (device_done(g_gf16_exp_ready)) return cudaSuccess;
  k_gf16_exp_init<<<64, 256, 0, s>>>();
  note_launch();
  return cudaGetLastError();
}

cudaError_t gf16_exp_table_init(cudaStream_t s) {
  if (device_done(g_gf16_exp_ready)) return cudaSuccess;
  cudaError_t e = exp_table_on(s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) device_mark(g_gf16_exp_ready);
  return e;
}

__global__ void k_gf16_coeff_matrix(const uint16_t* __restrict__ logs, unsigned n_in,
                                    const uint16_t* __restrict__ exps, unsigned n_out,
                                    uint16_t* __restrict__ coeffs) {
  size_t total = (size_t)n_in * n_out;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    unsigned o = (unsigned)(idx / n_in), i = (unsigned)(idx % n_in);
    uint32_t e = (uint32_t)(((uint64_t)logs[i] * exps[o]) % 65535u);
    coeffs[idx] = g_gf16_exp[e];
  }
}

cudaError_t launch_gf16_coeff_matrix(const uint16_t* d_logs, unsigned n_in, const uint16_t* d_exps,
                                     unsigned n_out, uint16_t* d_coeffs, cudaStream_t s) {
  size_t total = (size_t)n_in * n_out;
  if (!total) return cudaSuccess;
  if (cudaError_t e = exp_table_on(s)) return e;
  unsigned blocks = (unsigned)((total + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  k_gf16_coeff_matrix<<<blocks, 256, 0, s>>>(d_logs, n_in, d_exps, n_out, d_coeffs);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- muladd
constexpr int kT = 256;                   // threads per block
constexpr int kChunks = 2;                // 16-byte chunks per thread per input
constexpr int kTileBytes = kT * kChunks * 16;  // 8 KiB of each slice per block
constexpr int kStage = 8;                 // inputs whose tables are built together

// mode: 0 = overwrite, 1 = xor into existing (single writer), 2 = atomic xor
template <int QUADS>
__global__ void __launch_bounds__(kT, 2)
k_gf16_muladd_lut(const uint8_t* __restrict__ in, size_t in_stride, unsigned n_in, size_t slice_bytes,
                  const uint16_t* __restrict__ coeffs, size_t ldc, unsigned n_out, uint8_t* __restrict__ out,
                  size_t out_stride, unsigned inputs_per_split, int mode) {
  __shared__ uint64_t tab[kStage][QUADS][4][16];
  __shared__ uint16_t pw[kStage][QUADS * 4][16];

  const unsigned o0 = blockIdx.x * QUADS * 4;
  const unsigned i_begin = blockIdx.z * inputs_per_split;
  const unsigned i_end = min(n_in, i_begin + inputs_per_split);

  size_t coff[kChunks];
  int cvalid[kChunks];
#pragma unroll
  for (int j = 0; j < kChunks; j++) {
    coff[j] = (size_t)blockIdx.y * kTileBytes + (size_t)(j * kT + threadIdx.x) * 16;
    long long v = (long long)slice_bytes - (long long)coff[j];
    cvalid[j] = v <= 0 ? 0 : (v >= 16 ? 16 : (int)v);
  }
  // byte masks for a partial final chunk
  uint32_t cmask[kChunks][4];
#pragma unroll
  for (int j = 0; j < kChunks; j++)
#pragma unroll
    for (int u = 0; u < 4; u++) {
      int keep = cvalid[j] - 4 * u;
      cmask[j][u] = keep >= 4 ? 0xFFFFFFFFu : (keep <= 0 ? 0u : ((1u << (8 * keep)) - 1u));
    }

  uint64_t acc[kChunks * 8][QUADS];
#pragma unroll
  for (int k = 0; k < kChunks * 8; k++)
#pragma unroll
    for (int q = 0; q < QUADS; q++) acc[k][q] = 0;

  auto load = [&](unsigned i, uint4 (&d)[kChunks]) {
    const uint8_t* row = in + (size_t)i * in_stride;
#pragma unroll
    for (int j = 0; j < kChunks; j++) {
      if (cvalid[j] > 0) {
        uint4 v = __ldg(reinterpret_cast<const uint4*>(row + coff[j]));
        if (cvalid[j] < 16) {
          v.x &= cmask[j][0];
          v.y &= cmask[j][1];
          v.z &= cmask[j][2];
          v.w &= cmask[j][3];
        }
        d[j] = v;
      } else {
        d[j] = make_uint4(0, 0, 0, 0);
      }
    }
  };

  for (unsigned ib = i_begin; ib < i_end; ib += kStage) {
    const unsigned ns = min((unsigned)kStage, i_end - ib);
    __syncthreads();  // previous stage's tables fully consumed
    // c * x^k for k < 16, per (input, output) of the stage
    for (int t = threadIdx.x; t < kStage * QUADS * 4; t += kT) {
      int j = t / (QUADS * 4), o = t % (QUADS * 4);
      uint32_t c = 0;
      if ((unsigned)j < ns && o0 + o < n_out) c = coeffs[(size_t)(o0 + o) * ldc + ib + j];
#pragma unroll
      for (int k = 0; k < 16; k++) {
        pw[j][o][k] = (uint16_t)c;
        c = gf16_dbl(c);
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < kStage * QUADS * 64; t += kT) {
      int n = t & 15, q = (t >> 4) & 3, qd = (t >> 6) % QUADS, j = (t >> 6) / QUADS;
      uint64_t e = 0;
#pragma unroll
      for (int oo = 0; oo < 4; oo++) {
        uint32_t v = 0;
#pragma unroll
        for (int b = 0; b < 4; b++)
          if ((n >> b) & 1) v ^= pw[j][qd * 4 + oo][4 * q + b];
        e |= (uint64_t)v << (16 * oo);
      }
      tab[j][qd][q][n] = e;
    }
    __syncthreads();

    uint4 cur[kChunks], nxt[kChunks];
    load(ib, cur);
    for (unsigned j = 0; j < ns; j++) {
      if (j + 1 < ns) load(ib + j + 1, nxt);
#pragma unroll
      for (int k = 0; k < kChunks * 8; k++) {
        const uint4& c4 = cur[k >> 3];
        uint32_t w32 = ((k & 7) >> 1) == 0 ? c4.x : ((k & 7) >> 1) == 1 ? c4.y : ((k & 7) >> 1) == 2 ? c4.z : c4.w;
        uint32_t x = (k & 1) ? (w32 >> 16) : (w32 & 0xFFFFu);
        uint32_t n0 = x & 15, n1 = (x >> 4) & 15, n2 = (x >> 8) & 15, n3 = x >> 12;
#pragma unroll
        for (int qd = 0; qd < QUADS; qd++) {
          const uint64_t* T = &tab[j][qd][0][0];
          acc[k][qd] ^= T[n0] ^ T[16 + n1] ^ T[32 + n2] ^ T[48 + n3];
        }
      }
      if (j + 1 < ns) {
#pragma unroll
        for (int c = 0; c < kChunks; c++) cur[c] = nxt[c];
      }
    }
  }

  // epilogue
#pragma unroll
  for (int qd = 0; qd < QUADS; qd++) {
#pragma unroll
    for (int oo = 0; oo < 4; oo++) {
      unsigned o = o0 + qd * 4 + oo;
      if (o >= n_out) continue;
      uint8_t* row = out + (size_t)o * out_stride;
#pragma unroll
      for (int j = 0; j < kChunks; j++) {
        if (cvalid[j] <= 0) continue;
        uint32_t w[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          uint32_t lo = (uint32_t)(acc[j * 8 + 2 * u][qd] >> (16 * oo)) & 0xFFFFu;
          uint32_t hi = (uint32_t)(acc[j * 8 + 2 * u + 1][qd] >> (16 * oo)) & 0xFFFFu;
          w[u] = (lo | (hi << 16)) & cmask[j][u];
        }
        uint8_t* dst = row + coff[j];
        if (mode == 2) {
          uint32_t* d32 = reinterpret_cast<uint32_t*>(dst);
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (w[u]) atomicXor(d32 + u, w[u]);
        } else if (cvalid[j] == 16) {
          uint4 v = make_uint4(w[0], w[1], w[2], w[3]);
          if (mode == 1) {
            uint4 old = *reinterpret_cast<const uint4*>(dst);
            v.x ^= old.x;
            v.y ^= old.y;
            v.z ^= old.z;
            v.w ^= old.w;
          }
          *reinterpret_cast<uint4*>(dst) = v;
        } else {
          for (int b = 0; b < cvalid[j]; b++) {
            uint8_t nb = (uint8_t)(w[b >> 2] >> (8 * (b & 3)));
            dst[b] = mode == 1 ? (uint8_t)(dst[b] ^ nb) : nb;
          }
        }
      }
    }
  }
}

cudaError_t launch_gf16_muladd(const uint8_t* d_in, size_t in_stride, unsigned n_in, size_t slice_bytes,
                               const uint16_t* d_coeffs, size_t ldc, unsigned n_out, uint8_t* d_out,
                               size_t out_stride, bool accumulate, int sms, cudaStream_t s) {
  if (!n_out || !slice_bytes) return cudaSuccess;
  if (!n_in) {
    if (accumulate) return cudaSuccess;
    note_launch();
    return cudaMemset2DAsync(d_out, out_stride, 0, slice_bytes, n_out, s);
  }
  const int quads = n_out <= 4 ? 1 : 2;
  const unsigned rt = (unsigned)ceil_div(n_out, quads * 4);
  const unsigned wt = (unsigned)ceil_div(slice_bytes, kTileBytes);
  const unsigned base = rt * wt;
  const unsigned target = (unsigned)(sms > 0 ? sms : 148) * 4;
  unsigned splits = base >= target ? 1 : (unsigned)ceil_div(target, base);
  unsigned max_splits = (unsigned)ceil_div(n_in, kStage);
  if (splits > max_splits) splits = max_splits;
  if (splits < 1) splits = 1;
  unsigned per = (unsigned)ceil_div(ceil_div(n_in, splits), kStage) * kStage;
  splits = (unsigned)ceil_div(n_in, per);
  int mode;
  if (splits == 1) {
    mode = accumulate ? 1 : 0;
  } else {
    mode = 2;
    if (!accumulate) {
      cudaError_t e = cudaMemset2DAsync(d_out, out_stride, 0, slice_bytes, n_out, s);
      note_launch();
      if (e != cudaSuccess) return e;
    }
  }
  dim3 grid(rt, wt, splits);
  if (quads == 1)
    k_gf16_muladd_lut<1><<<grid, kT, 0, s>>>(d_in, in_stride, n_in, slice_bytes, d_coeffs, ldc, n_out, d_out,
                                             out_stride, per, mode);
  else
    k_gf16_muladd_lut<2><<<grid, kT, 0, s>>>(d_in, in_stride, n_in, slice_bytes, d_coeffs, ldc, n_out, d_out,
                                             out_stride, per, mode);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- invert
__global__ void k_gf16_build_rec_matrix(const uint16_t* __restrict__ logs, const uint32_t* __restrict__ col_of,
                                        unsigned n_in, const uint16_t* __restrict__ rec, unsigned m,
                                        uint16_t* __restrict__ mat, size_t ld) {
  size_t total = (size_t)n_in * m;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    unsigned r = (unsigned)(idx / n_in), i = (unsigned)(idx % n_in);
    uint32_t e = (uint32_t)(((uint64_t)logs[i] * rec[r]) % 65535u);
    mat[(size_t)r * ld + col_of[i]] = g_gf16_exp[e];
  }
}

cudaError_t launch_gf16_build_rec_matrix(const uint16_t* d_logs, const uint32_t* d_col_of, unsigned n_in,
                                         const uint16_t* d_rec, unsigned m, uint16_t* d_mat, size_t ld,
                                         cudaStream_t s) {
  size_t total = (size_t)n_in * m;
  if (!total) return cudaSuccess;
  if (cudaError_t e = exp_table_on(s)) return e;
  unsigned blocks = (unsigned)ceil_div(total, 256);
  if (blocks > 8192) blocks = 8192;
  k_gf16_build_rec_matrix<<<blocks, 256, 0, s>>>(d_logs, d_col_of, n_in, d_rec, m, d_mat, ld);
  note_launch();
  return cudaGetLastError();
}

// Pivot k: check, gather the pivot column, scale row k in place with the
// identity column substituted (reference gfmat_inv.cpp:146-153, SCALE_ROW).
__global__ void k_gf16_pivot(uint16_t* __restrict__ mat, unsigned m, unsigned ncols, size_t ld, unsigned pc0,
                             unsigned k, uint16_t* __restrict__ fcol, int* __restrict__ status) {
  if (*(volatile int*)status >= 0) return;
  uint16_t* rowk = mat + (size_t)k * ld;
  const uint16_t p = rowk[pc0 + k];
  if (p == 0) {
    if (threadIdx.x == 0) *status = (int)k;
    return;
  }
  for (unsigned r = threadIdx.x; r < m; r += blockDim.x) fcol[r] = mat[(size_t)r * ld + pc0 + k];
  __syncthreads();
  const uint16_t ip = gf16_inv_euclid(p);
  for (unsigned c = threadIdx.x; c < ncols; c += blockDim.x) {
    uint16_t v = (c == pc0 + k) ? (uint16_t)1 : rowk[c];
    rowk[c] = gf16_mul(v, ip);
  }
}

// Eliminate column pc0+k from every row r != k:
//   row_r ^= f_r * row_k, with the column itself replaced by f_r * row_k[col]
// (reference gfmat_inv.cpp:154-166, MULADD_ROW with REPLACE_WORD(...,0)).
__global__ void __launch_bounds__(256)
k_gf16_eliminate(uint16_t* __restrict__ mat, unsigned m, unsigned ncols, size_t ld, unsigned pc0, unsigned k,
                 const uint16_t* __restrict__ fcol, const int* __restrict__ status) {
  __shared__ uint16_t T[4][16];
  const unsigned r = blockIdx.y;
  if (r == k || *(volatile const int*)status >= 0) return;
  const uint16_t f = fcol[r];
  if (f == 0) return;  // the pivot column entry is already zero
  if (threadIdx.x < 64) {
    int q = threadIdx.x >> 4, n = threadIdx.x & 15;
    T[q][n] = gf16_mul(f, (uint32_t)n << (4 * q));
  }
  __syncthreads();
  const size_t c0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 8;
  if (c0 >= ncols) return;
  const uint16_t* rowk = mat + (size_t)k * ld;
  uint16_t* rowr = mat + (size_t)r * ld;
  uint4 a = *reinterpret_cast<const uint4*>(rowk + c0);
  uint4 b = *reinterpret_cast<const uint4*>(rowr + c0);
  uint32_t av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
  for (int u = 0; u < 4; u++) {
    uint32_t res = 0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      uint32_t x = (av[u] >> (16 * h)) & 0xFFFFu;
      uint32_t y = T[0][x & 15] ^ T[1][(x >> 4) & 15] ^ T[2][(x >> 8) & 15] ^ T[3][x >> 12];
      uint32_t col = (uint32_t)c0 + 2 * u + h;
      uint32_t old = (bv[u] >> (16 * h)) & 0xFFFFu;
      res |= ((col == pc0 + k) ? y : (y ^ old)) << (16 * h);
    }
    bv[u] = res;
  }
  *reinterpret_cast<uint4*>(rowr + c0) = make_uint4(bv[0], bv[1], bv[2], bv[3]);
}

// The whole elimination of an m x m matrix (m <= kInvSmall; row stride ld,
// 16-byte aligned rows) by one CTA in shared memory: the same steps as
// k_gf16_pivot + k_gf16_eliminate with pc0 = 0, all m pivots in one launch.
// The m pivot steps are serial, so each is kept short: the pivot inverse is
// one load from a shared-memory copy of the inverse table, and row r's update
// row_r ^= f_r * row_k uses 4-bit split tables of f_r (64 entries from three
// doublings and XORs) instead of a multiplication per element.
constexpr unsigned kInvSmall = 128;
constexpr unsigned kInvThreads = 1024;
constexpr unsigned kInvPer = kInvSmall * kInvSmall / kInvThreads;  // elements per thread, at most
constexpr int kInvTableBytes = 65536 * 2;                          // inverse table
constexpr int kInvDynBytes = kInvTableBytes + kInvSmall * 64 * 2;  // + split tables of every row
__global__ void __launch_bounds__(kInvThreads) k_gf16_invert_small(uint16_t* __restrict__ mat, unsigned m, size_t ld,
                                                                   int* __restrict__ status) {
  extern __shared__ __align__(16) uint16_t dyn[];
  uint16_t* sinv = dyn;                        // 1/x for every x
  uint16_t* T = dyn + kInvTableBytes / 2;      // T[(r * 4 + q) * 16 + n] = f_r * (n << 4q)
  __shared__ uint16_t a[kInvSmall * kInvSmall];
  // pivot columns: col[k & 1][r] = a[r][k] as step k begins (written by the
  // elimination of step k - 1, so a step needs two barriers, not three)
  __shared__ uint16_t col[2][kInvSmall];
  const unsigned mm = m * m, t = threadIdx.x;
  for (unsigned x = t; x < 65536 / 8; x += kInvThreads)
    reinterpret_cast<uint4*>(sinv)[x] = reinterpret_cast<const uint4*>(g_gf16_inv)[x];
  unsigned rr[kInvPer], cc[kInvPer];  // this thread's elements (row kInvSmall: none)
#pragma unroll
  for (unsigned u = 0; u < kInvPer; u++) {
    const unsigned e = t + kInvThreads * u;
    rr[u] = e < mm ? e / m : kInvSmall;
    cc[u] = e < mm ? e % m : 0;
  }
  for (unsigned e = t; e < mm; e += kInvThreads) {
    const uint16_t v = mat[(size_t)(e / m) * ld + e % m];
    a[e] = v;
    if (e % m == 0) col[0][e / m] = v;
  }
  __syncthreads();
  for (unsigned k = 0; k < m; k++) {
    const uint16_t* fcol = col[k & 1];
    uint16_t* fnext = col[(k + 1) & 1];
    const uint16_t p = fcol[k];
    if (p == 0) {  // uniform across the CTA
      if (t == 0) *status = (int)k;
      return;
    }
    if (t < 4 * m) {  // split tables of row r = t / 4, nibble q = t % 4
      const unsigned r = t >> 2, q = t & 3;
      uint32_t b0 = fcol[r];
      for (unsigned d = 0; d < 4 * q; d++) b0 = gf16_dbl(b0);
      const uint32_t b1 = gf16_dbl(b0), b2 = gf16_dbl(b1), b3 = gf16_dbl(b2);
      uint16_t* tq = T + (r * 4 + q) * 16;
#pragma unroll
      for (unsigned n = 0; n < 16; n++)
        tq[n] = (uint16_t)(((n & 1) ? b0 : 0u) ^ ((n & 2) ? b1 : 0u) ^ ((n & 4) ? b2 : 0u) ^ ((n & 8) ? b3 : 0u));
    } else if (t < 5 * m) {  // scale row k, the identity column substituted
      const unsigned c = t - 4 * m;
      const uint16_t v = gf16_mul(c == k ? (uint16_t)1 : a[k * m + c], sinv[p]);
      a[k * m + c] = v;
      if (c == k + 1) fnext[k] = v;  // row k's entry of the next pivot column
    }
    __syncthreads();
#pragma unroll
    for (unsigned u = 0; u < kInvPer; u++) {
      const unsigned r = rr[u], c = cc[u];
      if (r < m && r != k) {
        uint16_t v = a[r * m + c];
        if (fcol[r]) {
          const uint32_t x = a[k * m + c];
          const uint16_t* tr = T + r * 64;
          const uint16_t y =
              (uint16_t)(tr[x & 15] ^ tr[16 + ((x >> 4) & 15)] ^ tr[32 + ((x >> 8) & 15)] ^ tr[48 + (x >> 12)]);
          v = c == k ? y : (uint16_t)(v ^ y);
          a[r * m + c] = v;
        }
        if (c == k + 1) fnext[r] = v;
      }
    }
    __syncthreads();
  }
  for (unsigned e = t; e < mm; e += kInvThreads) mat[(size_t)(e / m) * ld + e % m] = a[e];
}

cudaError_t launch_gf16_invert(uint16_t* d_mat, unsigned m, unsigned ncols, size_t ld, unsigned pc0,
                               uint16_t* d_fcol, int* d_status, cudaStream_t s) {
  if (pc0 == 0 && ncols == m && m <= kInvSmall) {
    static std::atomic<uint64_t> attr{0};
    if (!device_done(attr)) {
      cudaError_t e = cudaFuncSetAttribute(k_gf16_invert_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kInvDynBytes);
      if (e != cudaSuccess) return e;
      device_mark(attr);
    }
    if (cudaError_t e = exp_table_on(s)) return e;
    k_gf16_invert_small<<<1, kInvThreads, kInvDynBytes, s>>>(d_mat, m, ld, d_status);
    note_launch();
    return cudaGetLastError();
  }
  dim3 grid((unsigned)ceil_div(ncols, 256 * 8), m);
  for (unsigned k = 0; k < m; k++) {
    k_gf16_pivot<<<1, 1024, 0, s>>>(d_mat, m, ncols, ld, pc0, k, d_fcol, d_status);
    k_gf16_eliminate<<<grid, 256, 0, s>>>(d_mat, m, ncols, ld, pc0, k, d_fcol, d_status);
    note_launch(2);
  }
  return cudaGetLastError();
}

}  // namespace pp
