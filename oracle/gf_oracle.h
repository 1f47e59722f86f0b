/* Test infrastructure only: the oracle.
 *
 * A plain-C restatement of the reference's GF arithmetic on the PAR2/PAR3
 * hot path.  It exists to check the CUDA product on the same inputs; it is
 * never linked into, called by or shipped with the product.  Each function
 * names the reference file:line whose behaviour it restates.  Parity of this
 * restatement is pinned by the tests against the reference's own build
 * (oracle/_ref, compiled from the reference sources) and against the golden
 * fixtures under tests/golden/.
 */
#ifndef PP_GF_ORACLE_H
#define PP_GF_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- GF(2^16), poly x^16+x^12+x^3+x+1 (0x1100B) ---------- */
uint16_t or_gf16_mul(uint16_t a, uint16_t b);
uint16_t or_gf16_exp(uint32_t e);
uint16_t or_gf16_inv(uint16_t a);
uint16_t or_par2_input_log(uint16_t inputBlock);
uint16_t or_par2_coeff(uint16_t inputBlock, uint16_t recoveryExp);

/* dst[o] (sliceSize bytes each) = XOR_i coeffs[o*numInputs+i] * src_i,
 * src_i of sizes[i] <= sliceSize bytes (bytes beyond sizes[i] read as 0). */
void or_par2_muladd(const uint8_t* const* src, const size_t* sizes, unsigned numInputs,
                    size_t sliceSize, const uint16_t* coeffs, unsigned numOutputs,
                    uint8_t* dst);

/* PAR2 repair inversion; returns 1 on success (factors: numMissing x numInputs,
 * recovery/numRec updated to the rows used), 0 if not invertible. */
int or_par2_invert(const uint8_t* valid, unsigned numInputs, uint16_t* recovery,
                   unsigned* numRec, uint16_t* factors);

/* ---------------- GF(2^64), poly x^64+x^4+x^3+x+1 ---------------------- */
uint64_t or_gf64_mul(uint64_t a, uint64_t b);
uint64_t or_gf64_inv(uint64_t a);
void or_gf64_build_cauchy(uint64_t* m, size_t numInputs, size_t numRecovery,
                          uint64_t firstInput, uint64_t firstRecovery);
void or_gf64_matvec(const uint64_t* in, size_t numInputs, uint64_t* out, size_t numRecovery,
                    size_t blockSize64, const uint64_t* coeff, int accumulate);
void or_gf64_compute_recovery(const uint64_t* in, size_t numInputs, uint64_t* out,
                              size_t numRecovery, size_t blockSize64, uint64_t firstInput,
                              uint64_t firstRecovery, int accumulate);
int or_gf64_solve_and_reconstruct(uint64_t* A, uint64_t* rhs, size_t n, size_t blockSize64);

void or_gf64_region_mul(uint64_t* out, const uint64_t* in, size_t len, uint64_t c);
void or_gf64_region_mul_arr(uint64_t* out, const uint64_t* in, const uint64_t* coeff,
                            size_t len, size_t nCoeff);
void or_gf64_region_muladd_arr(uint64_t* out, const uint64_t* in, const uint64_t* coeff,
                               size_t len, size_t nCoeff);

/* additive FFT, novel-polynomial basis on the Cantor basis; n a power of 2 */
uint64_t or_gf64_cantor(int i);
void or_gf64_fft_fwd(uint64_t* a, size_t n);
void or_gf64_fft_inv(uint64_t* a, size_t n);

/* ---------------- PAR2 memory checksum --------------------------------- */
/* gf16/gf16_cksum_base.h:40-55 with gf16_multi_mul2 (gf16_checksum_generic.h):
 * C = 2*C ^ B_j over 16-byte blocks (8 LE GF(2^16) lanes) of the first len
 * bytes zero-extended to a multiple of 16; out: 16 bytes */
void or_par2_mem_cksum(const uint8_t* data, size_t len, uint8_t* out);

/* ---------------- block hashes ---------------------------------------- */
/* BLAKE3, default hash mode; out_len <= 32 */
void or_blake3(const uint8_t* in, size_t len, uint8_t* out, size_t out_len);
/* PAR3 data-block hashes (lib/par3gen.js:1001-1017):
 * out[16*i..] = BLAKE3(after_checksum[24] || u64le(first_index+i) || block_i)[0:16] */
void or_par3_block_hashes(const uint8_t* blocks, size_t stride, size_t n, size_t block_size,
                          uint64_t first_index, const uint8_t* after_checksum, uint8_t* out16);
/* PAR3 recovery packets (src/gf64_addon.cc:2884-2934): n packets of 64 + block_size bytes */
void or_par3_recovery_packets(const uint8_t* recovery, size_t n, size_t block_size,
                              const uint8_t* input_set_id, uint64_t first_index, uint8_t* packets);

#ifdef __cplusplus
}
#endif
#endif
