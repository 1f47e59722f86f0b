/*
 * parpar_b200 — C ABI of the B200 (sm_100a) parity engine.
 *
 * This is the drop-in boundary for the two GF hot paths of ParParPar:
 *   PAR2: the GF(2^16) region multiply-accumulate behind the gf16 controller
 *         (gf16/controller.h:77-217, IPAR2ProcBackend) and the repair-matrix
 *         inversion (gf16/gfmat_inv.h:16-50, Galois16RecMatrix);
 *   PAR3: the GF(2^64) Cauchy-matrix engine behind the gf64_addon N-API entry
 *         points (src/par3_engine.h:11-244, GF64Controller) and the gf64 region
 *         dispatch table (gf64/gf64_global.h:23-37).
 * All reference citations are path:line inside the ParParPar source tree.
 *
 * Conventions
 *   - Every function returns an int status: PP_OK (0) or a negative PP_ERR_*
 *     code; pp_ctx_last_error() gives the message of the last failure on that
 *     context.  No C++ exception crosses this boundary.
 *   - Buffer arguments may be HOST memory (pageable or pinned) or DEVICE
 *     memory of the context's GPU; the library detects which.  Calls that take
 *     host buffers are synchronous, like the reference: outputs are complete on
 *     return.  Calls whose buffers are all device memory are enqueued on the
 *     context's stream and return without waiting (pp_ctx_synchronize waits).
 *   - Words are little-endian: u16 for GF(2^16), u64 for GF(2^64).
 *   - No CPU fallback: without a usable CUDA device every compute entry point
 *     fails with PP_ERR_NO_DEVICE.
 */
#ifndef PARPAR_B200_H
#define PARPAR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define PP_API __declspec(dllexport)
#else
#define PP_API __attribute__((visibility("default")))
#endif

/* ------------------------------------------------------------------ status */
#define PP_OK 0
#define PP_ERR_INVALID_ARG (-1)
#define PP_ERR_CUDA (-2)
#define PP_ERR_NO_MEMORY (-3)
#define PP_ERR_SINGULAR (-4)      /* PAR3 solve: matrix singular (reference returns -1) */
#define PP_ERR_NOT_INVERTIBLE (-5) /* PAR2 invert: not enough usable recovery (reference returns false) */
#define PP_ERR_BUSY (-6)          /* PAR2 processor staging area full (reference PROC_ADD_FULL) */
#define PP_ERR_NO_DEVICE (-7)
#define PP_ERR_UNSUPPORTED (-8)
#define PP_ERR_TIMEOUT (-9)       /* a bounded device-side wait gave up (kernel returned early) */
#define PP_ERR_TOO_LARGE (-10)    /* size above a fixed maximum of an allocation-free entry point */
#define PP_ERR_IO (-11)           /* a file could not be opened or read (streaming create) */

/* reference PAR2ProcBackendAddResult (gf16/controller.h:38-43) */
#define PP_PROC_ADD_OK 0
#define PP_PROC_ADD_OK_BUSY 1
#define PP_PROC_ADD_FULL 2

/* kernel selection for pp_gf64_compute_recovery (the reference's entry points
 * ComputeRecoveryBlocks / …Barycentric / …Fenger / …Full, src/par3_engine.h:23-243,
 * all compute the same Cauchy product bit-for-bit) */
#define PP_GF64_KERNEL_AUTO 0
#define PP_GF64_KERNEL_MATVEC 1
#define PP_GF64_KERNEL_BARYCENTRIC 2
#define PP_GF64_KERNEL_FENGER 3

/* Region kernel selection (pp_ctx_set_gf16_kernel / pp_ctx_set_gf64_kernel) */
#define PP_GF16_KERNEL_AUTO 0
#define PP_GF16_KERNEL_LUT 1      /* shared-memory 4-bit split tables */
#define PP_GF16_KERNEL_TENSOR 2   /* tcgen05 u8 MMA over the GF(2) bit matrices */

typedef struct pp_ctx pp_ctx;
typedef struct pp_par2_proc pp_par2_proc;

/* ----------------------------------------------------------------- context */
PP_API const char* pp_version(void);
PP_API const char* pp_status_string(int status);
/* Create a context on CUDA device `device` with its own stream. */
PP_API int pp_ctx_create(int device, pp_ctx** out);
PP_API void pp_ctx_destroy(pp_ctx* ctx);
/* Use an external cudaStream_t (NULL restores the context's own stream). */
PP_API int pp_ctx_set_stream(pp_ctx* ctx, void* cuda_stream);
PP_API void* pp_ctx_get_stream(pp_ctx* ctx);
PP_API int pp_ctx_synchronize(pp_ctx* ctx);
PP_API const char* pp_ctx_last_error(pp_ctx* ctx);
/* Number of kernels (and device memsets) this library has launched so far. */
PP_API uint64_t pp_launch_count(void);
/* Drop cached device buffers (scratch, coefficient matrices). */
PP_API int pp_ctx_free_cache(pp_ctx* ctx);
/* Kernel timing, for measurement tools (off by default).  With `on` != 0 the
 * context brackets each region product it issues on its stream for a
 * device-resident single job (pp_par2_create / pp_gf16_muladd: the region
 * kernel and its output zeroing; pp_gf64_compute_recovery: the region
 * kernel) with a pair of CUDA events.  pp_ctx_kernel_time waits for the
 * bracketed launches, returns their summed device time in ms and their count
 * since the previous call, and clears them.  No counterpart in the reference. */
PP_API int pp_ctx_set_kernel_timing(pp_ctx* ctx, int on);
PP_API int pp_ctx_kernel_time(pp_ctx* ctx, double* ms, uint64_t* launches);
/* Choose the GF(2^16) region kernel used by this context (PP_GF16_KERNEL_*). */
PP_API int pp_ctx_set_gf16_kernel(pp_ctx* ctx, int kernel);
/* Choose the GF(2^64) region kernel used by this context (same constants). */
PP_API int pp_ctx_set_gf64_kernel(pp_ctx* ctx, int kernel);

/* ============================================================ PAR2 / GF16 */

/* Coefficient of input slice `input_block` for recovery exponent `exp`,
 * 2^(L_i * exp mod 65535) with L_i the i-th log coprime to 65535
 * (replaces gfmat_coeff, gf16/gfmat_coeff.c:99-101; host scalar helper). */
PP_API uint16_t pp_par2_coeff(uint16_t input_block, uint16_t exp);
PP_API uint16_t pp_par2_input_log(uint16_t input_block);

/* coeffs[o * num_inputs + i] = coeff(input_idx[i], exps[o]), computed on the
 * device (replaces the per-input set_coeffs loop, gf16/controller_cpu.cpp:372-378). */
PP_API int pp_par2_coeff_matrix(pp_ctx* ctx, const uint16_t* input_idx, unsigned num_inputs,
                                const uint16_t* exps, unsigned num_outputs, uint16_t* coeffs);

/* Region multiply-accumulate (the work of Galois16Mul::mul_add_multi_packpf
 * driven by PAR2ProcCPU::run_kernel/compute_worker, gf16/controller_cpu.cpp:463-624,
 * gf16/gf16mul.h:360-412):
 *   outputs[o] (^)= XOR_i coeffs[o * coeff_stride + i] * inputs[i]
 * over the first slice_bytes bytes of each row; rows are input_stride /
 * output_stride bytes apart.  An odd final byte is a word with a zero high
 * byte.  accumulate=0 overwrites the outputs. */
PP_API int pp_gf16_muladd(pp_ctx* ctx, const void* inputs, size_t input_stride, unsigned num_inputs,
                          size_t slice_bytes, const uint16_t* coeffs, size_t coeff_stride,
                          unsigned num_outputs, void* outputs, size_t output_stride, int accumulate);

/* PAR2 create in one call: recovery[o] = XOR_i coeff(input_idx[i], exps[o]) * inputs[i]. */
PP_API int pp_par2_create(pp_ctx* ctx, const void* inputs, size_t input_stride, unsigned num_inputs,
                          size_t slice_bytes, const uint16_t* input_idx, const uint16_t* exps,
                          unsigned num_outputs, void* outputs, size_t output_stride);

/* PAR2 repair-matrix inversion (replaces Galois16RecMatrix::Compute +
 * GetFactor, gf16/gfmat_inv.cpp:560-690, gf16/gfmat_inv.h:40-45).
 *   valid[num_inputs]      nonzero = input slice present
 *   recovery[*num_recovery] recovery exponents available; sorted on return and
 *                          truncated to the rows used (a row whose pivot is
 *                          zero is dropped and the inversion retried, as the
 *                          reference does for the PAR2 flaw)
 *   factors                num_missing x num_inputs, row k = missing slice k:
 *                          columns [0, valid_count) weight the valid slices in
 *                          index order, columns [valid_count, num_inputs) the
 *                          recovery slices in the order of recovery[].
 * Returns PP_ERR_NOT_INVERTIBLE where the reference returns false. */
PP_API int pp_par2_invert(pp_ctx* ctx, const uint8_t* valid, unsigned num_inputs, uint16_t* recovery,
                          unsigned* num_recovery, uint16_t* factors);

/* ---- PAR2 processor: IPAR2ProcBackend for a CUDA device -----------------
 * Mirrors gf16/controller.h:77-217 (and PAR2ProcCPU's behaviour,
 * gf16/controller_cpu.cpp): staging areas of `input_batch` slices, inputs
 * added one at a time (canAdd back-pressure), the kernel runs per full
 * staging area, outputs read back per recovery slice. */
PP_API int pp_par2_proc_create(pp_ctx* ctx, size_t slice_size, unsigned staging_areas, unsigned input_batch,
                               pp_par2_proc** out);
PP_API void pp_par2_proc_destroy(pp_par2_proc* proc);
/* setCurrentSliceSize (may shrink; growing reallocates) */
PP_API int pp_par2_proc_set_current_slice_size(pp_par2_proc* proc, size_t size);
/* setRecoverySlices(n, exps); exps NULL -> every exponent 1 (custom-coefficient use) */
PP_API int pp_par2_proc_set_recovery_slices(pp_par2_proc* proc, unsigned num, const uint16_t* exps);
/* canAdd -> PP_PROC_ADD_OK / _OK_BUSY / _FULL */
PP_API int pp_par2_proc_can_add(pp_par2_proc* proc);
/* Block until an add is possible (waitForAdd). */
PP_API int pp_par2_proc_wait_for_add(pp_par2_proc* proc);
/* addInput(buffer, size, inputNum, flush): the buffer may be reused on return. */
PP_API int pp_par2_proc_add_input(pp_par2_proc* proc, const void* buffer, size_t size, uint16_t input_num,
                                  int flush);
/* addInput(buffer, size, coeffs[num_recovery], flush) — decode overload. */
PP_API int pp_par2_proc_add_input_coeffs(pp_par2_proc* proc, const void* buffer, size_t size,
                                         const uint16_t* coeffs, int flush);
PP_API int pp_par2_proc_flush(pp_par2_proc* proc);
/* endInput: flush and wait for all processing. */
PP_API int pp_par2_proc_end_input(pp_par2_proc* proc);
/* getOutput(index, output) -> *valid (1 = output passed the integrity check). */
PP_API int pp_par2_proc_get_output(pp_par2_proc* proc, unsigned index, void* output, int* valid);
PP_API int pp_par2_proc_discard_output(pp_par2_proc* proc);
/* Device address of recovery slice `index` in the processor's output area
 * (rows of the slice size rounded up to 16 bytes; the recovery data once
 * end_input has returned).  No counterpart in the reference, whose output
 * area is host memory that getOutput unpacks (gf16/controller_cpu.cpp:423-443):
 * a caller that consumes recovery slices on the device (packet MD5, a copy to
 * another device) reads them here in place.  Valid until the next
 * set_recovery_slices, free_processing_mem or destroy.  Writing through it
 * before the first get_output of a job makes get_output report the slices so
 * changed invalid (their memory checksum no longer matches). */
PP_API int pp_par2_proc_output_ptr(pp_par2_proc* proc, unsigned index, void** dev_ptr);
/* Input hashing in the processor's own pass (replaces feeding the same
 * buffers to HasherInput::update / getBlock(md5crc, zeroPad),
 * hasher/hasher_input_base.h:104-117, beside the backend's addInput): with
 * max_inputs > 0, every slice added by input number afterwards gets its IFSC
 * entry (MD5 || CRC32le of the slice zero-padded to the current slice size)
 * computed on the device from its staged row, at index input_num (which must
 * be < max_inputs); decode inputs (add_input_coeffs) are not hashed.
 * max_inputs = 0 turns it off.  get_input_hashes waits for the submitted
 * batches and copies entries [0, count) (20 bytes each, host or device
 * buffer); entries of inputs not added since enabling read as zero. */
PP_API int pp_par2_proc_set_input_hashes(pp_par2_proc* proc, unsigned max_inputs);
PP_API int pp_par2_proc_get_input_hashes(pp_par2_proc* proc, uint8_t* out, unsigned count);
PP_API int pp_par2_proc_free_processing_mem(pp_par2_proc* proc);
PP_API unsigned pp_par2_proc_input_batch_size(pp_par2_proc* proc);
PP_API unsigned pp_par2_proc_batches_started(pp_par2_proc* proc);
/* Staging areas whose device work has finished, counted in submission order
 * (the PAR2ProcCPU counterpart is the compute thread's _queueProc notify,
 * gf16/controller_cpu.cpp:520-530, that drives progressCb).  wait_batches
 * blocks until at least `count` batches have finished (PP_ERR_TIMEOUT after
 * a minute); it waits on host-side state only, so a watcher thread may call
 * it while the owning thread keeps adding inputs -- the libuv backend shim
 * reports finished batches to PAR2Proc::onBackendProcess this way. */
PP_API unsigned pp_par2_proc_batches_done(pp_par2_proc* proc);
PP_API int pp_par2_proc_wait_batches(pp_par2_proc* proc, unsigned count);

/* ============================================================ PAR3 / GF64 */

/* Cauchy matrix M[r][c] = inv((first_input + c) XOR (first_recovery + r)),
 * zero denominators mapped to 1, row-major num_recovery x num_inputs
 * (replaces GF64Controller::BuildCauchyMatrix, src/par3_engine.cc:358-425). */
PP_API int pp_gf64_build_cauchy(pp_ctx* ctx, uint64_t* coeff, size_t num_inputs, size_t num_recovery,
                                uint64_t first_input, uint64_t first_recovery);

/* Recovery blocks from the Cauchy product (replaces
 * GF64Controller::ComputeRecoveryBlocks / …Full / …Barycentric / …Fenger,
 * src/par3_engine.h:23-243; N-API compute_recovery*, src/gf64_addon.cc:1266-1434).
 *   recovery[r][w] (^)= XOR_c inputs[c][w] * M[r][c]
 * inputs: num_inputs blocks of block_size64 words; recovery: num_recovery
 * blocks.  accumulate=0 overwrites.  Empty problems return PP_OK untouched. */
PP_API int pp_gf64_compute_recovery(pp_ctx* ctx, const uint64_t* inputs, size_t num_inputs, uint64_t* recovery,
                                    size_t num_recovery, size_t block_size64, uint64_t first_input,
                                    uint64_t first_recovery, int accumulate, int kernel);

/* Same with a caller-supplied coefficient matrix (num_recovery x num_inputs)
 * (replaces ComputeRecoveryBlocksWithCoeff, src/par3_engine.h:61-68). */
PP_API int pp_gf64_compute_recovery_with_coeff(pp_ctx* ctx, const uint64_t* inputs, size_t num_inputs,
                                               uint64_t* recovery, size_t num_recovery, size_t block_size64,
                                               const uint64_t* coeff, int accumulate);

/* Gauss-Jordan solve of A (n x n, modified) with the same row operations on
 * rhs (n blocks of block_size64 words, becomes the solution)
 * (replaces GF64Controller::SolveAndReconstruct, src/par3_engine.cc:980-1053).
 * Returns PP_ERR_SINGULAR where the reference returns -1; on that error the
 * contents of A and rhs are unspecified. */
PP_API int pp_gf64_solve_and_reconstruct(pp_ctx* ctx, uint64_t* A, uint64_t* rhs, size_t n, size_t block_size64);

/* PAR3 repair in one call (the decode of lib/par3gen.js:3840-4010 on the
 * device): with y_eq = first_recovery + eq for eq < n and x_k = first_input + k,
 *   A[eq][col] = inv(x_{missing[col]} ^ y_eq)                 (0 -> 1)
 *   rhs[eq]    = recovery[eq] (zero where recovery_present[eq] == 0)
 *                ^ XOR_{k not missing} inv(x_k ^ y_eq) * inputs[k]
 *   restored   = solution of A * restored = rhs  (Gauss-Jordan, as SolveAndReconstruct)
 * inputs: num_inputs blocks of block_size64 words (rows of lost blocks are not
 * read); missing: n distinct block indices; recovery: n blocks (block eq holds
 * recovery block first_recovery + eq); recovery_present: n flags or NULL (all
 * present); restored: n blocks, restored[col] = input block missing[col].
 * Returns PP_ERR_SINGULAR where the reference's solve returns -1. */
PP_API int pp_gf64_repair(pp_ctx* ctx, const uint64_t* inputs, size_t num_inputs, const uint64_t* missing, size_t n,
                          const uint64_t* recovery, const uint8_t* recovery_present, size_t block_size64,
                          uint64_t first_input, uint64_t first_recovery, uint64_t* restored);

/* Region primitives (replace the gf64_region_* dispatch pointers,
 * gf64/gf64_global.h:23-37; semantics gf64/gf64_region_scalar.c:8-91). */
PP_API int pp_gf64_region_mul(pp_ctx* ctx, uint64_t* out, const uint64_t* in, size_t len, uint64_t constant);
/* out[i] = in[i] * coeff[i % n_coeff] */
PP_API int pp_gf64_region_mul_arr(pp_ctx* ctx, uint64_t* out, const uint64_t* in, const uint64_t* coeff, size_t len,
                                  size_t n_coeff);
/* out[i] ^= XOR_c in[i] * coeff[c] */
PP_API int pp_gf64_region_muladd_arr(pp_ctx* ctx, uint64_t* out, const uint64_t* in, const uint64_t* coeff,
                                     size_t len, size_t n_coeff);
/* out[w] ^= XOR_g in_blocks[g][w] * coeff_blocks[g] */
PP_API int pp_gf64_region_coupled_muladd_arr(pp_ctx* ctx, uint64_t* out, const uint64_t* const* in_blocks,
                                             const uint64_t* coeff_blocks, size_t len, size_t G);
/* outs[k][w] ^= in[w] * coeff_block_starts[k][0] */
PP_API int pp_gf64_region_fused_output_muladd_arr(pp_ctx* ctx, uint64_t* const* outs, const uint64_t* in,
                                                  const uint64_t* const* coeff_block_starts, size_t len, size_t K);
/* outs[k][w] ^= XOR_g in_blocks[g][w] * coeff_block_2d[k * K_stride + g] */
PP_API int pp_gf64_region_2d_muladd_arr(pp_ctx* ctx, uint64_t* const* outs, size_t K, const uint64_t* const* in_blocks,
                                        size_t G, const uint64_t* coeff_block_2d, size_t K_stride, size_t len);
/* out[i] = inverse(in[i]), inverse(0) = 0 (replaces gf64_inverse_batch,
 * gf64/gf64_invert.c:71-75). */
PP_API int pp_gf64_inverse_batch(pp_ctx* ctx, uint64_t* out, const uint64_t* in, size_t n);

/* dst ^= src over `bytes` bytes (replaces the xor_buffers export,
 * src/gf64_addon.cc:3216-3265, used to reduce chunked recovery partials).
 * The caller checks equal lengths (the reference's RangeError). */
PP_API int pp_xor_buffers(pp_ctx* ctx, void* dst, const void* src, size_t bytes);

/* ---- One job over several GPUs ------------------------------------------
 * Each context (one per GPU) computes a contiguous byte range
 * [range_begin[i], range_end[i]) of every slice / block and writes the same
 * range of the outputs, with no data exchanged between devices: the split
 * PAR2Proc makes over its backends (gf16/controller.cpp:42-84, ranges checked
 * by the rule of checkBackendAllocation: no gaps or overlaps, starts on 16-bit
 * words, an odd size only for the range that ends the slice) and the Fenger
 * path's word ranges (src/par3_engine_fenger.cc:266-290; PAR3 ranges on 8-byte
 * words, 16 bytes keeps the tensor-core path's aligned rows).  Buffers are
 * host memory or device memory of every context's own GPU (a device buffer of
 * another GPU -> PP_ERR_INVALID_ARG).  Each range runs on its own host
 * thread; the call returns when every range is done.  Arguments otherwise as
 * pp_par2_create / pp_gf64_compute_recovery (create: fI, fR; no accumulate). */
PP_API int pp_par2_create_split(pp_ctx* const* ctxs, const size_t* range_begin, const size_t* range_end,
                                unsigned n_ranges, const void* inputs, size_t input_stride, unsigned num_inputs,
                                size_t slice_bytes, const uint16_t* input_idx, const uint16_t* exps,
                                unsigned num_outputs, void* outputs, size_t output_stride);
PP_API int pp_gf64_compute_recovery_split(pp_ctx* const* ctxs, const size_t* range_begin, const size_t* range_end,
                                          unsigned n_ranges, const uint64_t* inputs, size_t num_inputs,
                                          uint64_t* recovery, size_t num_recovery, size_t block_size64,
                                          uint64_t first_input, uint64_t first_recovery);

/* Allocation-free solve.  No counterpart in the reference: an addition for
 * callers that cannot allocate device memory where they need the repair solve
 * (a device pool owned by another allocator with no headroom, latency-bound
 * loops that cannot take cudaMalloc's device-wide synchronisation, services
 * that must not fail for lack of memory after start-up).
 * Same result and return codes as pp_gf64_solve_and_reconstruct, but: A and
 * rhs must be device memory of the current device (or managed memory; other
 * pointers -> PP_ERR_INVALID_ARG before any work is enqueued); work is enqueued on `cuda_stream` (NULL = the
 * legacy default stream) and the call waits for it; nothing is allocated.
 * Working storage is a fixed array inside the library (about 32 KiB, held on
 * every GPU that loads the library until exit), so n is limited to
 * PP_NOALLOC_SOLVE_MAX_N (larger n -> PP_ERR_TOO_LARGE), and calls that overlap
 * on the GPU share that array and race.  The first call on a device looks up
 * the array's device address (with that device current); make that first
 * call before any stream capture. */
#define PP_NOALLOC_SOLVE_MAX_N 4096
PP_API int pp_gf64_solve_and_reconstruct_noalloc(uint64_t* A, uint64_t* rhs, size_t n, size_t block_size64,
                                                 void* cuda_stream);

/* Additive FFT over GF(2^64), novel-polynomial basis on the Cantor basis
 * (replaces gf64_addfft64_fwd_recursive_scratch / _inv_recursive_scratch,
 * gf64/gf64_additive_fft_hqc2026.c:1656-1705).  Batched: `batch` polynomials
 * of n coefficients, coefficient c of polynomial b at data[c * ld + b]
 * (batch = ld = 1 is the reference's single-array call).  n must be a power
 * of two <= 2^20; n <= 1 is a no-op.  The inverse is not normalised, as in the
 * reference. */
PP_API int pp_gf64_fft_fwd(pp_ctx* ctx, uint64_t* data, size_t n, size_t batch, size_t ld);
PP_API int pp_gf64_fft_inv(pp_ctx* ctx, uint64_t* data, size_t n, size_t batch, size_t ld);

/* ------------------------------------------------------------ block hashes
 * Buffers may be host or device memory; device inputs are hashed where they
 * lie (slices already resident for a region pass are not re-read from the
 * host).  Host outputs are written before the call returns. */

/* PAR2 input-slice checksums, the 20-byte IFSC entries: for each block i,
 * MD5 (16 bytes) then CRC32 (4 bytes, little-endian) of the block's first
 * lengths[i] bytes followed by slice_size - lengths[i] zero bytes.  Replaces
 * HasherInput::getBlock(md5crc, zeroPad) (hasher/hasher_input_base.h:104-117)
 * as the PAR2 hasher binding drives it per slice (src/gf.cc:928-957 with
 * zeroPad 0, :1034-1036 for the zero-padded last slice of a file).  Block i
 * starts at blocks + i * block_stride; lengths NULL means every block is
 * slice_size bytes; lengths[i] > slice_size is an error.  block_stride must
 * cover the longest block.  The whole-file MD5 that HasherInput::end also
 * returns is a serial hash of the file stream and stays with the caller. */
PP_API int pp_par2_block_hashes(pp_ctx* ctx, const void* blocks, size_t block_stride, size_t num_blocks,
                                size_t slice_size, const uint64_t* lengths, uint8_t* md5crc);

/* pp_par2_create that also returns the inputs' IFSC entries (as
 * pp_par2_block_hashes with every input a full slice_bytes row, the caller
 * having zero-padded a file's last slice as pp_par2_create requires) computed
 * in the same pass over the inputs: each staged chunk of input rows is hashed
 * on the device beside the region kernels, so host inputs cross PCIe once for
 * both.  md5crc: num_inputs x 20 bytes, host or device. */
PP_API int pp_par2_create_hashed(pp_ctx* ctx, const void* inputs, size_t input_stride, unsigned num_inputs,
                                 size_t slice_bytes, const uint16_t* input_idx, const uint16_t* exps,
                                 unsigned num_outputs, void* outputs, size_t output_stride, uint8_t* md5crc);

/* PAR2 memory checksums: the checksum block the reference's PAR2 staging
 * appends to every slice (gf16/gf16_cksum_base.h:40-55 with the block step of
 * gf16/gf16_checksum_generic.h gf16_multi_mul2: C = 2*C ^ block), here with
 * 16-byte blocks of 8 little-endian GF(2^16) lanes: row i's first
 * slice_bytes bytes, zero-extended to a multiple of 16, as blocks B_0..B_nb-1
 * give out16[16*i..] = sum_j 2^(nb-1-j) * B_j lane-wise.  The function is
 * linear, so the PAR2 processor stages each input row with its checksum
 * block, multiplies it along with the data and reports, per output, whether
 * the carried block still equals the checksum of the output data
 * (pp_par2_proc_get_output's valid, as finish_packed_cksum,
 * gf16/controller_cpu.cpp:423-443). */
PP_API int pp_par2_memory_checksums(pp_ctx* ctx, const void* rows, size_t row_stride, size_t num_rows,
                                    size_t slice_bytes, uint8_t* out16);

/* PAR2 recovery-slice packet headers (getRecoveryHeader with the packet MD5
 * of _pullRecData / _getRecoveryPacketMD5, lib/par2.js:240-330,517-530):
 * headers receives num_slices x 68 bytes -- "PAR2\0PKT", u64le(68 +
 * slice_bytes), the MD5 of packet bytes [32, 68 + slice_bytes) (set id,
 * "PAR 2.0\0RecvSlic", u32le(exps[i]), slice i), the 16-byte set id, the type
 * and u32le(exps[i]); the packet is this header followed by the slice.
 * slice_bytes a multiple of 4 (PAR2). set_id is host or device memory. */
PP_API int pp_par2_recovery_packet_headers(pp_ctx* ctx, const void* slices, size_t slice_stride, size_t num_slices,
                                           size_t slice_bytes, const uint8_t* set_id, const uint16_t* exps,
                                           uint8_t* headers);

/* PAR3 data-block checksums (lib/par3gen.js:1001-1017, _inlineHashBlock):
 * hashes[16*i..] = BLAKE3(after_checksum[0..24) || u64le(first_index + i) ||
 * block_i)[0..16), block_i = block_size bytes at blocks + i * block_stride.
 * after_checksum is the data packet's 24 header bytes after its checksum
 * field (total length, input-set id, type; lib/par3gen.js:1237), host memory. */
PP_API int pp_par3_block_hashes(pp_ctx* ctx, const void* blocks, size_t block_stride, size_t num_blocks,
                                size_t block_size, uint64_t first_index, const uint8_t* after_checksum,
                                uint8_t* hashes);

/* PAR3 recovery packets (replaces assemble_recovery_packets,
 * src/gf64_addon.cc:2784-2936): packets receives num_recovery packets of
 * 64 + block_size bytes -- magic "PAR3\0PKT", the 16-byte BLAKE3 checksum of
 * packet bytes [24, 64 + block_size), u64le total length, the 8-byte
 * input-set id (host memory), type "PAR REC\0", u64le(first_recovery_index +
 * i), u64le(1), then recovery block i (recovery + i * block_size).
 * num_recovery or block_size 0, or num_recovery * block_size above 1 TiB,
 * is PP_ERR_INVALID_ARG (the reference's RangeErrors). */
PP_API int pp_par3_assemble_recovery_packets(pp_ctx* ctx, const void* recovery, size_t num_recovery,
                                             size_t block_size, const uint8_t* input_set_id,
                                             uint64_t first_recovery_index, uint8_t* packets);

/* One PAR3 create pass over the input blocks: the num_recovery recovery
 * blocks first_recovery.. (as pp_gf64_compute_recovery) come back as
 * assembled RECOVERY packets (as pp_par3_assemble_recovery_packets,
 * num_recovery x (64 + 8 * block_size64) bytes), and, when data_hashes is not
 * NULL, every input block's data-packet checksum (as pp_par3_block_hashes
 * with first_index = first_input; num_inputs x 16 bytes) is computed from the
 * same staged input rows.  This is the reference's create flow of
 * _processRecoveryBatch + _finalizeRecoveryBlocks + assemble_recovery_packets
 * (lib/par3gen.js:1686-1712,1750-1898) plus the data-packet hashing of its
 * read loop (lib/par3gen.js:2790-2830), with the input crossing PCIe once. */
PP_API int pp_par3_create_packets(pp_ctx* ctx, const uint64_t* inputs, size_t num_inputs, size_t block_size64,
                                  uint64_t first_input, size_t num_recovery, uint64_t first_recovery,
                                  const uint8_t* data_after_checksum, uint8_t* data_hashes,
                                  const uint8_t* input_set_id, uint8_t* packets);

/* Streaming PAR3 create from a file (replaces par3_create_streaming,
 * src/gf64_create_streaming.cc:93-245): the file at source_path is cut into
 * ceil(size / block_size) input blocks, the last zero-padded; recovery
 * receives the num_recovery recovery blocks first_recovery.. of inputs
 * first_input.. (num_recovery x block_size bytes, host or device), as
 * ComputeRecoveryBlocksFull.  The file is read in chunks by parallel preads
 * into pinned buffers; each chunk is copied to the device and multiplied into
 * the recovery while the next chunk is read, so reading, copying and the
 * products overlap and the input is never held whole in memory.  With
 * data_hashes not NULL, every input block's data-packet checksum (as
 * pp_par3_block_hashes with first_index = first_input and
 * data_after_checksum) is computed from the same staged chunks
 * (ceil(size / block_size) x 16 bytes).  block_size must be a positive
 * multiple of 8 and num_recovery positive (PP_ERR_INVALID_ARG, the
 * reference's RangeErrors); a file that cannot be opened or read, or is
 * empty, gives PP_ERR_IO with the reference's message. */
typedef struct pp_stream_stats {
  uint64_t bytes_read;  /* file bytes read */
  uint64_t num_inputs;  /* input blocks */
  double seconds;       /* wall time of the call */
  double read_seconds;  /* time spent waiting for file reads */
} pp_stream_stats;
PP_API int pp_par3_create_streaming(pp_ctx* ctx, const char* source_path, size_t block_size, size_t num_recovery,
                                    uint64_t first_input, uint64_t first_recovery, uint8_t* recovery,
                                    const uint8_t* data_after_checksum, uint8_t* data_hashes,
                                    pp_stream_stats* stats);

/* ------------------------------------------------------------ batches
 * No counterpart in the reference (it runs one job at a time on its CPU
 * threads).  A batch is a plan over device-resident jobs of mixed kinds and
 * sizes: pp_batch_create builds every coefficient table the jobs need
 * (PAR2 expanded coefficient bit matrices, PAR3 Cauchy matrices, the inverse
 * of each repair system) and keeps them on the device, fuses the region
 * products of all jobs into one tensor-core launch per field and phase, and
 * captures the whole batch in a CUDA graph; pp_batch_run replays it on the
 * context's stream (asynchronous; pp_ctx_synchronize reports the status).
 * Results are bit-identical to running the jobs one by one through the
 * single-job entry points.
 *
 * All job buffers are device memory and stay bound to the plan: inputs rows
 * 16-byte aligned (base and stride), PAR3 outputs 8-byte aligned, PAR2
 * outputs 4-byte aligned.  Creation runs the batch once (the outputs are
 * written).  With PP_BATCH_TUNE it also times candidate work splits of each
 * fused launch on the jobs' own buffers and keeps the fastest; the choice is
 * remembered per shape for the process. */
#define PP_JOB_PAR2_CREATE 1 /* outputs[e] = XOR_i c(input_ids[i], exponents[e]) * inputs[i] */
#define PP_JOB_PAR3_CREATE 2 /* outputs[r] = XOR_c inv((fI+c)^(fR+r)) * inputs[c] */
#define PP_JOB_PAR3_REPAIR 3 /* restored[k] = input block missing[k], from the first n recovery blocks */
#define PP_JOB_GF16_MULADD 4 /* outputs[o] = XOR_i coeffs[o][i] * inputs[i] (e.g. the PAR2 repair decode
                              * with the factors of pp_par2_invert) */

typedef struct pp_job {
  int kind;
  const void* inputs;        /* num_inputs rows (PAR3 repair: lost rows are not read) */
  size_t input_stride;       /* bytes between input rows */
  size_t num_inputs;
  size_t slice_bytes;        /* PAR2: bytes per slice; PAR3: block bytes, a multiple of 8 */
  const uint16_t* input_ids; /* PAR2: input slice numbers (host), NULL = 0..num_inputs-1 */
  const uint16_t* exponents; /* PAR2: recovery exponents (host) */
  size_t num_recovery;       /* PAR2 / PAR3 create: output rows; repair: ignored */
  void* outputs;             /* PAR2 / PAR3 create: recovery rows; repair: restored rows */
  size_t output_stride;      /* bytes between output rows */
  uint64_t first_input;      /* PAR3 */
  uint64_t first_recovery;   /* PAR3 */
  const uint64_t* missing;   /* PAR3 repair: lost input indices (host), n of them */
  size_t num_missing;
  const void* recovery;      /* PAR3 repair: the first n recovery blocks (device) */
  size_t recovery_stride;    /* bytes between recovery rows */
  const uint8_t* recovery_present; /* PAR3 repair: NULL, or n flags (host); absent rows count as zero */
  const uint16_t* coeffs;    /* GF16 muladd: num_recovery x num_inputs coefficients, row-major (host) */
} pp_job;

typedef struct pp_batch pp_batch;
#define PP_BATCH_TUNE 1
/* PP_BATCH_NO_GRAPH: for jobs seen once -- creation builds the tables only
 * (no eager run, no capture, no tuning) and pp_batch_run issues the fused
 * launches directly, so creation plus one run is the work of running the
 * jobs once. */
#define PP_BATCH_NO_GRAPH 2
PP_API int pp_batch_create(pp_ctx* ctx, const pp_job* jobs, size_t n_jobs, int flags, pp_batch** out);
PP_API int pp_batch_run(pp_batch* batch);
/* launches the batch's graph issues per run (kernels and memset/copy nodes) */
PP_API int pp_batch_launches(const pp_batch* batch);
PP_API void pp_batch_destroy(pp_batch* batch);

/* ------------------------------------------------------------ serving loop
 * No counterpart in the reference.  A server owns a context and a scheduler
 * thread.  Submitted jobs (pp_job, host or device buffers; the small host
 * arrays of the job are copied at submit, the data buffers must stay valid
 * until the job completes) are admitted in arrival order while the device
 * memory they need fits in hbm_budget_bytes (staging of host buffers, repair
 * temporaries and the resident coefficient tables all count); admitted jobs
 * are grouped into waves of at most max_jobs_per_wave and each wave runs as
 * fused tensor-core launches on one of `lanes` streams, so a wave admitted
 * while others are on the GPU overlaps with them (continuous batching).
 * PAR3 Cauchy matrices and PAR2 coefficient tiles stay resident (LRU within
 * the budget).  Every job's result is identical to running it alone.  Host
 * buffers should be pinned for copies to overlap. */
typedef struct pp_server pp_server;
typedef struct pp_server_stats {
  uint64_t submitted, completed, failed;
  uint64_t waves;              /* fused waves launched */
  uint64_t input_bytes;        /* input bytes of the completed jobs */
  double elapsed_s;            /* first submit -> last completion */
  double gbps;                 /* input_bytes / elapsed_s / 1e9 */
  double p50_ms, p99_ms, max_ms; /* submit -> completion latency of completed jobs */
  uint64_t hbm_peak_bytes;     /* most device memory held at once (jobs + tables) */
  uint64_t tables_resident, table_bytes;
} pp_server_stats;
PP_API int pp_server_create(int device, size_t hbm_budget_bytes, int max_jobs_per_wave, int lanes, pp_server** out);
PP_API int pp_server_submit(pp_server* srv, const pp_job* job, uint64_t* ticket);
/* the job's status (PP_OK or its error), or PP_ERR_TIMEOUT if still running after timeout_ms (< 0: no limit) */
PP_API int pp_server_wait(pp_server* srv, uint64_t ticket, int timeout_ms);
PP_API int pp_server_get_stats(pp_server* srv, pp_server_stats* out);
PP_API void pp_server_reset_stats(pp_server* srv);
PP_API const char* pp_server_last_error(pp_server* srv);
PP_API void pp_server_destroy(pp_server* srv); /* waits for every submitted job */

#ifdef __cplusplus
}
#endif
#endif /* PARPAR_B200_H */
