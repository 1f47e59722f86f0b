// Internal host-side declarations shared by the C-ABI layer and the kernel
// translation units.  Not part of the public interface (include/parpar_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <string>

#include "tc_batch.h"

#include <mutex>

struct pp_ctx;

namespace pp {

// One-time setup per device (kernel attributes are set per device): whether
// the current device's bit is set in `mask`, and setting it.
inline bool device_done(const std::atomic<uint64_t>& mask) {
  int d = 0;
  cudaGetDevice(&d);
  return d >= 0 && d < 64 && ((mask.load(std::memory_order_acquire) >> d) & 1u);
}
inline void device_mark(std::atomic<uint64_t>& mask) {
  int d = 0;
  cudaGetDevice(&d);
  if (d >= 0 && d < 64) mask.fetch_or(1ull << d, std::memory_order_acq_rel);
}

// Launch counter: every kernel launch issued by this library increments it
// (reported by pp_ctx_launch_count so callers can account for native work).
void note_launch(int n = 1);
uint64_t launches();

// context internals for the host translation units other than capi.cpp
int ctx_device(const pp_ctx* c);
int ctx_sms(const pp_ctx* c);
cudaStream_t ctx_stream(const pp_ctx* c);
int* ctx_status_word(const pp_ctx* c);
std::mutex& ctx_mutex(pp_ctx* c);
int ctx_fail(pp_ctx* c, int code, const char* msg);  // records the message, returns code

// ------------------------------------------------------------ GF(2^16)
// The device table of 2^k in GF(2^16) behind the coefficient kernels:
// filled on stream s and waited for, once per device (at context creation).
cudaError_t gf16_exp_table_init(cudaStream_t s);
// the same for the table behind launch_gf16_tc_expand (gf16_tc.cu)
cudaError_t gf16_tc_tables_init(cudaStream_t s);
// coeffs[o*N + i] = 2^(logs[i] * exps[o] mod 65535)   (device buffers)
cudaError_t launch_gf16_coeff_matrix(const uint16_t* d_logs, unsigned n_in, const uint16_t* d_exps,
                                     unsigned n_out, uint16_t* d_coeffs, cudaStream_t s);

// Region multiply-accumulate over 16-byte-aligned rows:
//   out[o] (^)= XOR_i coeffs[o*N + i] * in[i]   for the first slice_bytes bytes
// in/out rows are in_stride/out_stride bytes apart (multiples of 16).
// Bytes past slice_bytes are neither read as data nor written.
// If !accumulate the outputs are overwritten.
// coeffs rows are ldc elements apart.
cudaError_t launch_gf16_muladd(const uint8_t* d_in, size_t in_stride, unsigned n_in, size_t slice_bytes,
                               const uint16_t* d_coeffs, size_t ldc, unsigned n_out, uint8_t* d_out,
                               size_t out_stride, bool accumulate, int sms, cudaStream_t s);

// Tensor-core (tcgen05, kind::mxf4 or kind::i8) variant.  launch_gf16_tc_expand builds
// the coefficient bit-matrix tiles (gf16_tc_coeff_bytes(n_in, n_out) bytes)
// that launch_gf16_muladd_tc consumes; *d_status is set nonzero if a bounded
// device wait timed out.
size_t gf16_tc_coeff_bytes(unsigned n_in, unsigned n_out);
// inputs per stage of the tiles (8: int8 operands; 16: block-scaled FP4,
// the default; fixed for the process)
unsigned gf16_tc_stage_inputs();
cudaError_t launch_gf16_tc_expand(const uint16_t* d_coeffs, size_t ldc, unsigned n_in, unsigned n_out,
                                  uint8_t* d_aexp, cudaStream_t s);
cudaError_t launch_gf16_muladd_tc(const uint8_t* d_in, size_t in_stride, unsigned n_in, size_t slice_bytes,
                                  const uint8_t* d_aexp, unsigned n_out, uint8_t* d_out, size_t out_stride,
                                  bool accumulate, int sms, int* d_status, cudaStream_t s,
                                  unsigned a_stride = 0);  // 0: the tiles of exactly these n_in inputs

// PAR2 inversion (Gauss-Jordan without pivoting, identity columns in place).
// d_mat: m rows x ncols (row stride ld elements, rows 16-byte aligned).  Runs
// all m pivot steps; d_status[0] (set to -1 by the caller) receives the first
// row whose pivot was zero.  A square matrix (pc0 = 0, ncols = m) of at most
// 128 rows is eliminated by one CTA in one launch.
cudaError_t launch_gf16_invert(uint16_t* d_mat, unsigned m, unsigned ncols, size_t ld, unsigned pivot_col0,
                               uint16_t* d_fcol, int* d_status, cudaStream_t s);

// Build the PAR2 repair matrix: mat[r][col_of[i]] = coeff(logs[i], rec[r]).
cudaError_t launch_gf16_build_rec_matrix(const uint16_t* d_logs, const uint32_t* d_col_of, unsigned n_in,
                                         const uint16_t* d_rec, unsigned m, uint16_t* d_mat, size_t ld,
                                         cudaStream_t s);

// ------------------------------------------------------------ GF(2^64)
cudaError_t launch_gf64_cauchy(uint64_t* d_m, size_t n_in, size_t n_rec, uint64_t first_in, uint64_t first_rec,
                               size_t ld, cudaStream_t s);
cudaError_t launch_gf64_cauchy_cols(uint64_t* d_A, size_t n_rows, const uint64_t* d_cols, size_t n_cols, uint64_t fI,
                                    uint64_t fR, cudaStream_t s);
cudaError_t launch_gf64_inverse_batch(uint64_t* d_out, const uint64_t* d_in, size_t n, cudaStream_t s);
// inverse of the n x n Cauchy system built by launch_gf64_cauchy_cols (rows
// fR + j, columns fI + cols[i], no zero denominator): d_w holds 2n words of
// weights, d_Ainv receives A^-1 (n x n, row-major)
cudaError_t launch_gf64_cauchy_inverse(const uint64_t* d_A, const uint64_t* d_cols, size_t n, uint64_t fI,
                                       uint64_t fR, uint64_t* d_w, uint64_t* d_Ainv, cudaStream_t s);

// out[r][w] (^)= XOR_c coeff[r*ldc + c] * in[c][w]
// in rows in_stride words apart, out rows out_stride words apart.
cudaError_t launch_gf64_matvec(const uint64_t* d_in, size_t in_stride, size_t n_in, size_t words,
                               const uint64_t* d_coeff, size_t ldc, size_t n_out, uint64_t* d_out,
                               size_t out_stride, bool accumulate, int sms, cudaStream_t s);

// Tensor-core (tcgen05) variant of the matvec; optional device pointer tables
// for the rows (NULL: strided).  Requires 16-byte aligned rows and an even
// word count.  *d_status is set nonzero if a bounded device wait gave up.
// Tensor-core launches over a job table (tc_batch.h): one launch for all
// jobs; the job fields the kernels derive (n_stages, groups / pairs,
// wt) are filled in here and empty jobs are dropped, so the table is modified.
cudaError_t launch_gf16_tc_batch(Gf16TcBatch& b, int sms, int* d_status, cudaStream_t s);
cudaError_t launch_gf64_tc_batch(Gf64TcBatch& b, int sms, int* d_status, cudaStream_t s);
cudaError_t launch_gf64_tc_batch_one_cta(Gf64TcBatch& b, int sms, int* d_status, cudaStream_t s);

cudaError_t launch_gf64_matvec_tc(const uint64_t* d_in, const uint64_t* const* d_in_ptrs, size_t in_stride,
                                  size_t n_in, size_t words, const uint64_t* d_coeff, size_t ldc, size_t n_out,
                                  uint64_t* d_out, uint64_t* const* d_out_ptrs, size_t out_stride, bool accumulate,
                                  int sms, int* d_status, cudaStream_t s);

// Gather form used by the region entry points: pointer tables on the device.
//   outs[k][w] ^= XOR_g in_blocks[g][w] * coeff[k*kstride + g]
cudaError_t launch_gf64_2d_gather(uint64_t* const* d_outs, size_t K, const uint64_t* const* d_ins, size_t G,
                                  const uint64_t* d_coeff, size_t kstride, size_t len, int sms,
                                  cudaStream_t s);

// Element-wise region ops (n_coeff cycling / summing semantics of the
// reference's gf64_region_mul_arr / gf64_region_muladd_arr).
cudaError_t launch_gf64_region_mul_arr(uint64_t* d_out, const uint64_t* d_in, const uint64_t* d_coeff, size_t len,
                                       size_t n_coeff, cudaStream_t s);
cudaError_t launch_gf64_region_muladd_arr(uint64_t* d_out, const uint64_t* d_in, const uint64_t* d_coeff,
                                          size_t len, size_t n_coeff, cudaStream_t s);

// SolveAndReconstruct: Gauss-Jordan on A (n x n) with the RHS (n x B words).
// d_status[0] = 0 on success, -1 if singular.
cudaError_t launch_gf64_solve(uint64_t* d_A, uint64_t* d_rhs, size_t n, size_t B, uint64_t* d_fcol,
                              int* d_status, cudaStream_t s);

// dst ^= src over `bytes` bytes (any alignment)
cudaError_t launch_xor_bytes(uint8_t* d_dst, const uint8_t* d_src, size_t bytes, cudaStream_t s);

// Batched additive FFT, in place (column-major: coefficient c of polynomial
// b at data[c*ld + b]).
cudaError_t launch_gf64_fft(uint64_t* d_data, size_t n, size_t batch, size_t ld, bool inverse, cudaStream_t s);

// ------------------------------------------------------------ block hashes
// PAR2 input-slice checksums: out[20*i..] = MD5 || CRC32le of the first
// min(lengths[i], slice) bytes of row i followed by zeros up to slice bytes
// (lengths NULL: every row is slice bytes).  Rows 16-byte aligned.  d_idx
// (optional): row i's entry goes to d_out + 20 * d_idx[i], none for 0xFFFF.
cudaError_t launch_par2_block_hash(const uint8_t* d_data, size_t stride, size_t n, uint64_t slice,
                                   const uint64_t* d_lengths, uint8_t* d_out, cudaStream_t s,
                                   const uint16_t* d_idx = nullptr);

// The same hashes over column bands of slices that are all `slice` bytes:
// 64-byte blocks [k0, k1) of every row; d_state (5 words per row) carries the
// MD5 and CRC32 state from band to band; `first` starts it, `last` (k1 =
// slice / 64) finishes the message and writes the entries to d_out.
cudaError_t launch_par2_block_hash_band(const uint8_t* d_data, size_t stride, size_t n, uint64_t slice,
                                        uint64_t k0, uint64_t k1, uint32_t* d_state, uint8_t* d_out, bool first,
                                        bool last, cudaStream_t s);

// BLAKE3 over n messages "prefix || data_i": the prefix is P bytes (32 or 40)
// made of pre[0..6) (24 bytes), u64le(first_index + i) and, when P == 40,
// u64le(extra).  The 16-byte truncated digest of message i goes to
// hash_out + i * hash_stride; with copy_to set, the data bytes are also
// written to copy_to + i * copy_stride.  C is derived by the launcher.
struct B3Job {
  const uint8_t* data = nullptr;
  size_t stride = 0;
  uint64_t D = 0;
  uint32_t P = 32;
  uint32_t pre[6] = {};
  uint64_t first_index = 0;
  uint64_t extra = 0;
  uint64_t n = 0;
  uint64_t C = 0;
  uint8_t* copy_to = nullptr;
  size_t copy_stride = 0;
  uint8_t* hash_out = nullptr;
  size_t hash_stride = 16;
  uint32_t one = 1;  // set by the launcher
};
size_t blake3_scratch_words(size_t n, uint64_t message_bytes);  // chunk chaining values (2 levels)
cudaError_t launch_blake3_blocks(const B3Job& job, uint32_t* d_scratch, cudaStream_t s);
// headers of n PAR3 recovery packets (64 + block_size bytes each), all but
// the checksum field
cudaError_t launch_par3_packet_headers(uint8_t* d_pkts, size_t n, size_t block_size, uint64_t set_id_le,
                                       uint64_t first, cudaStream_t s);

// PAR2 memory checksum of each row's first len bytes (16-byte blocks, see
// hash_kernels.cu).  d_valid NULL: write the 16-byte checksum of row i to
// d_out + i * out_stride; else set d_valid[i] to whether it equals the 16
// bytes stored there.  Rows 16-byte aligned; d_out 4-byte aligned.
cudaError_t launch_par2_cksum(const uint8_t* d_rows, size_t stride, size_t n, uint64_t len, uint8_t* d_out,
                              size_t out_stride, int* d_valid, cudaStream_t s);

// PAR2 recovery packet headers (68 bytes each, MD5 included) of n slices of
// `slice` bytes (a multiple of 4; rows 4-byte aligned); pre = set id and
// type words; d_out 4-byte aligned.
cudaError_t launch_par2_packet_headers(const uint8_t* d_data, size_t stride, size_t n, uint64_t slice,
                                       const uint32_t pre[8], const uint16_t* d_exps, uint8_t* d_out,
                                       cudaStream_t s);

}  // namespace pp
