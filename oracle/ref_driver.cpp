// Test infrastructure only: a thin extern "C" driver over the reference's own
// C/C++ implementation of the GF hot paths (trafgals/ParParPar).  It is
// compiled from the reference sources where they lie (see oracle/Makefile)
// into oracle/_ref/libppref.so and is used by the tests to pin the oracle
// restatement, and by bench.py's reference arm as the timed CPU baseline.
// Nothing in the product links or calls it.
//
// Reference entry points driven here:
//   PAR2 create  : PAR2Proc + PAR2ProcCPU (gf16/controller.h:248-326,
//                  gf16/controller_cpu.cpp:291-331,423-443), non-libuv build
//                  exactly as test/gf16/test-ctrl.cpp drives it.
//   PAR2 invert  : Galois16RecMatrix::Compute / GetFactor (gf16/gfmat_inv.h:16-50)
//   PAR3 create  : GF64Controller::ComputeRecoveryBlocks{,Barycentric,Fenger}
//                  (src/par3_engine.h:23-243)
//   PAR3 repair  : GF64Controller::BuildCauchyMatrix + SolveAndReconstruct
//   region ops   : gf64_region_* dispatch table (gf64/gf64_global.h:23-37)
//   FFT          : gf64_addfft64_{fwd,inv}_recursive_scratch
//                  (gf64/gf64_additive_fft_hqc2026.c:1656,1680)
//   block hashes : setup_hasher + HasherInput_Create (hasher/hasher.cpp: the
//                  fastest variant the CPU supports) update / getBlock / end
//                  (hasher/hasher_input_base.h:44-128), driven like the PAR2
//                  hasher binding (src/gf.cc:928-1037); blake3_hash
//                  (hasher/hasher_blake3.h:50)

#include "controller.h"
#include "controller_cpu.h"
#include "gfmat_coeff.h"
#include "gfmat_inv.h"
#include "par3_engine.h"
extern "C" {
#include "gf64_additive_fft.h"
#include "hasher_blake3.h"
}
#include "hasher.h"
#include <cstdint>
#include <cstring>
#include <future>
#include <vector>

extern "C" {
extern gf64_t gf64_mul_reference(gf64_t a, gf64_t b);
extern gf64_t gf64_inverse(gf64_t a);
}

// The N-API addon binds the gf64 dispatch table at module load; a plain C++
// caller has to do the same before the first engine call.
static void ensure_gf64_dispatch() {
	static const bool bound = (gf64_init_dispatch(), true);
	(void)bound;
}

static const char* g_par2_method = "";

extern "C" {

// ---------------------------------------------------------------- PAR2 ----
// inputs: numInputs slices back to back, each sliceSize bytes (the last one
// may be shorter: lastSize bytes).  out: numOutputs * sliceSize bytes.
// Returns 1 if every output passed the controller's memory checksum.
int ref_par2_create(const uint8_t* inputs, unsigned numInputs, size_t sliceSize,
                    size_t lastSize, const uint16_t* inputIdx,
                    const uint16_t* exps, unsigned numOutputs, uint8_t* out,
                    int threads) {
	PAR2Proc par2;
	PAR2ProcCPU cpu(2);
	std::vector<PAR2ProcBackendAlloc> be{{&cpu, 0, sliceSize}};
	par2.init(sliceSize, be);
	cpu.init(GF16_AUTO);
	if (threads > 0) cpu.setNumThreads(threads);
	g_par2_method = cpu.getMethodName();
	if (!par2.setRecoverySlices(numOutputs, exps)) return -1;
	for (unsigned i = 0; i < numInputs; i++) {
		par2.waitForAdd();
		size_t sz = (i == numInputs - 1) ? lastSize : sliceSize;
		par2.addInput(inputs + (size_t)i * sliceSize, sz, inputIdx[i], false);
	}
	par2.endInput().get();
	int ok = 1;
	for (unsigned o = 0; o < numOutputs; o++) {
		if (!par2.getOutput(o, out + (size_t)o * sliceSize).get()) ok = 0;
	}
	par2.deinit();
	return ok;
}

// Same, with explicit per-input coefficient columns: coeffs[i*numOutputs+o]
// (the decode overload addInput(buf, size, const uint16_t* coeffs, …),
// gf16/controller.h:170).
int ref_par2_create_coeffs(const uint8_t* inputs, unsigned numInputs, size_t sliceSize,
                           const uint16_t* coeffs, unsigned numOutputs, uint8_t* out,
                           int threads) {
	PAR2Proc par2;
	PAR2ProcCPU cpu(2);
	std::vector<PAR2ProcBackendAlloc> be{{&cpu, 0, sliceSize}};
	par2.init(sliceSize, be);
	cpu.init(GF16_AUTO);
	if (threads > 0) cpu.setNumThreads(threads);
	if (!par2.setRecoverySlices(numOutputs, nullptr)) return -1;
	for (unsigned i = 0; i < numInputs; i++) {
		par2.waitForAdd();
		par2.addInput(inputs + (size_t)i * sliceSize, sliceSize, coeffs + (size_t)i * numOutputs, false);
	}
	par2.endInput().get();
	int ok = 1;
	for (unsigned o = 0; o < numOutputs; o++) {
		if (!par2.getOutput(o, out + (size_t)o * sliceSize).get()) ok = 0;
	}
	par2.deinit();
	return ok;
}

const char* ref_par2_method(void) { return g_par2_method; }

uint16_t ref_gfmat_coeff(uint16_t inputBlock, uint16_t recoveryBlock) {
	gfmat_init();
	return gfmat_coeff(inputBlock, recoveryBlock);
}
uint16_t ref_gfmat_input_log(uint16_t inputBlock) {
	gfmat_init();
	return gfmat_input_log(inputBlock);
}

// Galois16RecMatrix::Compute.  valid[numInputs] (0/1); recovery[*numRec] is
// sorted and may shrink (rows dropped by the PAR2 flaw).  factors receives
// numMissing rows x numInputs columns of GetFactor(col,row).
// Returns 1 on success, 0 if not invertible.
int ref_par2_invert(const uint8_t* valid, unsigned numInputs, uint16_t* recovery,
                    unsigned* numRec, uint16_t* factors, int threads) {
	gfmat_init();
	std::vector<bool> iv(numInputs);
	unsigned validCount = 0;
	for (unsigned i = 0; i < numInputs; i++) { iv[i] = valid[i] != 0; validCount += iv[i]; }
	std::vector<uint16_t> rec(recovery, recovery + *numRec);
	Galois16RecMatrix mat;
	if (threads > 0) mat.setNumThreads(threads);
	bool ok = mat.Compute(iv, validCount, rec);
	if (!ok) return 0;
	unsigned missing = numInputs - validCount;
	for (unsigned r = 0; r < missing; r++)
		for (unsigned c = 0; c < numInputs; c++)
			factors[(size_t)r * numInputs + c] = mat.GetFactor(c, r);
	*numRec = (unsigned)rec.size();
	memcpy(recovery, rec.data(), rec.size() * sizeof(uint16_t));
	return 1;
}

// ---------------------------------------------------------------- PAR3 ----
uint64_t ref_gf64_mul(uint64_t a, uint64_t b) { return gf64_mul_reference(a, b); }
uint64_t ref_gf64_inverse(uint64_t a) { return gf64_inverse(a); }

// kind: 0 = ComputeRecoveryBlocks (matvec), 1 = Barycentric, 2 = Fenger,
//       3 = ComputeRecoveryBlocksFull
void ref_gf64_compute_recovery(int kind, const uint64_t* inputs, size_t numInputs,
                               uint64_t* recovery, size_t numRecovery, size_t blockSize64,
                               uint64_t firstInput, uint64_t firstRecovery, int threads,
                               int accumulate) {
	ensure_gf64_dispatch();
	switch (kind) {
	case 0:
		GF64Controller::ComputeRecoveryBlocks(inputs, numInputs, recovery, numRecovery, blockSize64,
		                                      firstInput, firstRecovery, threads, accumulate != 0);
		break;
	case 1:
		GF64Controller::ComputeRecoveryBlocksBarycentric(inputs, numInputs, recovery, numRecovery,
		                                                 blockSize64, firstInput, firstRecovery,
		                                                 threads, accumulate != 0);
		break;
	case 2:
		GF64Controller::ComputeRecoveryBlocksFenger(inputs, numInputs, recovery, numRecovery,
		                                            blockSize64, firstInput, firstRecovery, threads);
		break;
	default:
		GF64Controller::ComputeRecoveryBlocksFull(inputs, numInputs, recovery, numRecovery,
		                                          blockSize64, firstInput, firstRecovery, threads,
		                                          accumulate != 0);
		break;
	}
}

void ref_gf64_compute_recovery_with_coeff(const uint64_t* inputs, size_t numInputs,
                                          uint64_t* recovery, size_t numRecovery,
                                          size_t blockSize64, const uint64_t* coeff,
                                          int threads, int accumulate) {
	ensure_gf64_dispatch();
	GF64Controller::ComputeRecoveryBlocksWithCoeff(inputs, numInputs, recovery, numRecovery,
	                                               blockSize64, coeff, threads, accumulate != 0);
}

void ref_gf64_build_cauchy(uint64_t* m, size_t numInputs, size_t numRecovery,
                           uint64_t firstInput, uint64_t firstRecovery) {
	ensure_gf64_dispatch();
	GF64Controller::BuildCauchyMatrix(m, numInputs, numRecovery, firstInput, firstRecovery);
}

int ref_gf64_solve_and_reconstruct(uint64_t* A, uint64_t* rhs, size_t n, size_t blockSize64) {
	ensure_gf64_dispatch();
	return GF64Controller::SolveAndReconstruct(A, rhs, n, blockSize64, 1);
}

void ref_gf64_fft_fwd(uint64_t* arr, size_t n) {
	ensure_gf64_dispatch();
	std::vector<gf64_t> scratch(gf64_addfft64_fwd_recursive_scratch_words(n) + 1);
	gf64_addfft64_fwd_recursive_scratch(arr, n, scratch.data(), scratch.size());
}
void ref_gf64_fft_inv(uint64_t* arr, size_t n) {
	ensure_gf64_dispatch();
	std::vector<gf64_t> scratch(gf64_addfft64_inv_recursive_scratch_words(n) + 1);
	gf64_addfft64_inv_recursive_scratch(arr, n, scratch.data(), scratch.size());
}
void ref_gf64_poly_mul(uint64_t* out, const uint64_t* a, size_t la, const uint64_t* b,
                       size_t lb, size_t outLen) {
	ensure_gf64_dispatch();
	size_t n = 1;
	while (n < la + lb - 1) n <<= 1;
	std::vector<gf64_t> scratch(gf64_addfft64_poly_mul_recursive_scratch_words(n) + 1);
	gf64_addfft64_poly_mul_recursive_scratch(out, a, la, b, lb, outLen, scratch.data(), scratch.size());
}

// One PAR2 input file through the reference hasher, as the binding feeds it:
// every full slice gets getBlock(md5crc, 0); a trailing partial slice gets
// getBlock(md5crc, slice - tail) (zero padding); then end() gives the file MD5.
// ifsc receives ceil(len / slice) 20-byte entries.
static void ensure_hasher() {
	static bool done = false;
	if (!done) {
		setup_hasher();
		done = true;
	}
}

const char* ref_par2_hasher_method() {
	ensure_hasher();
	return hasherInput_methodName();
}

void ref_par2_hash_file(const uint8_t* data, size_t len, size_t slice, uint8_t* ifsc, uint8_t* file_md5) {
	ensure_hasher();
	IHasherInput* h = HasherInput_Create();
	size_t pos = 0;
	while (len - pos >= slice) {
		h->update(data + pos, slice);
		h->getBlock(ifsc, 0);
		ifsc += 20;
		pos += slice;
	}
	if (pos < len) {
		h->update(data + pos, len - pos);
		h->getBlock(ifsc, slice - (len - pos));
	}
	h->end(file_md5);
	h->destroy();
}

void ref_blake3(const uint8_t* in, size_t len, uint8_t* out, size_t out_len) { blake3_hash(in, len, out, out_len); }

// PAR3 data-block checksums as lib/par3gen.js:1001-1017 computes them
// (createHash().update(afterChecksum).update(u64le index).update(block)),
// here with the reference's own BLAKE3.
void ref_par3_block_hashes(const uint8_t* blocks, size_t n, size_t bs, uint64_t first, const uint8_t* after,
                           uint8_t* out16) {
	for (size_t i = 0; i < n; i++) {
		uint8_t idx[8];
		for (int b = 0; b < 8; b++) idx[b] = (uint8_t)((first + i) >> (8 * b));
		blake3_hasher h;
		blake3_hasher_init(&h);
		blake3_hasher_update(&h, after, 24);
		blake3_hasher_update(&h, idx, 8);
		blake3_hasher_update(&h, blocks + i * bs, bs);
		blake3_hasher_finalize(&h, out16 + 16 * i, 16);
	}
}

// The body of AssembleRecoveryPackets_NAPI (src/gf64_addon.cc:2884-2934; the
// N-API wrapper needs node headers, so its loop is driven directly): header
// fields, block copy, BLAKE3 of packet[24 .. 64 + bs) with the reference's
// hasher, truncated to 16 bytes at packet[8].
void ref_par3_assemble_recovery_packets(const uint8_t* rec, size_t n, size_t bs, const uint8_t* sid,
                                        uint64_t first, uint8_t* out) {
	static const uint8_t magic[8] = {'P', 'A', 'R', '3', 0, 'P', 'K', 'T'};
	static const uint8_t type[8] = {'P', 'A', 'R', ' ', 'R', 'E', 'C', 0};
	const size_t pkt_size = 64 + bs;
	for (size_t i = 0; i < n; i++) {
		uint8_t* pkt = out + i * pkt_size;
		memcpy(pkt, magic, 8);
		memset(pkt + 8, 0, 16);
		for (int b = 0; b < 8; b++) pkt[24 + b] = (uint8_t)((uint64_t)pkt_size >> (8 * b));
		memcpy(pkt + 32, sid, 8);
		memcpy(pkt + 40, type, 8);
		for (int b = 0; b < 8; b++) pkt[48 + b] = (uint8_t)((first + i) >> (8 * b));
		for (int b = 0; b < 8; b++) pkt[56 + b] = (uint8_t)(b == 0);
		memcpy(pkt + 64, rec + i * bs, bs);
		blake3_hasher h;
		blake3_hasher_init(&h);
		blake3_hasher_update(&h, pkt + 24, 24);
		blake3_hasher_update(&h, pkt + 48, 16 + bs);
		uint8_t full[32];
		blake3_hasher_finalize(&h, full, 32);
		memcpy(pkt + 8, full, 16);
	}
}

}  // extern "C"
