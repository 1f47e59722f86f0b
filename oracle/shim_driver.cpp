// Test infrastructure only: drives the reference's own PAR2 front controller
// (PAR2Proc, gf16/controller.cpp, non-libuv build, as test/gf16/test-ctrl.cpp
// drives it) over the CUDA backend shim PAR2ProcCUDA
// (parparpar_b200/shim/controller_cuda.cpp) -- alone, or beside the
// reference's PAR2ProcCPU with each slice split by byte range
// (controller.cpp:42-84).  Built by `make -C oracle shim` into
// oracle/_ref/libppshim.so against the reference's sources and
// parparpar_b200/libparpar_b200.so.

#include "controller.h"
#include "controller_cpu.h"
#include "controller_cuda.h"

#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

namespace {

// backends for [0, split) on the CPU and [split, slice) on the GPU; split 0 =
// the GPU alone, split = slice = the CPU alone
struct Procs {
	std::unique_ptr<PAR2ProcCPU> cpu;
	std::unique_ptr<PAR2ProcCUDA> cuda;
	std::vector<PAR2ProcBackendAlloc> be;
	bool ok = true;
	Procs(size_t slice, size_t split, int device, int threads) {
		if (split > 0) {
			cpu.reset(new PAR2ProcCPU(2));
			be.push_back({cpu.get(), 0, split});
		}
		if (split < slice) {
			cuda.reset(new PAR2ProcCUDA(device));
			ok = cuda->init();
			be.push_back({cuda.get(), split, slice - split});
		}
	}
	// after PAR2Proc::init has set the slice sizes (the order of test-ctrl.cpp)
	void initCpu(int threads) {
		if (!cpu) return;
		cpu->init(GF16_AUTO);
		if (threads > 0) cpu->setNumThreads(threads);
	}
};

template <class AddFn>
int run(size_t slice, size_t split, int device, int threads, unsigned numInputs, unsigned numOutputs,
        const uint16_t* exps, uint8_t* out, AddFn add) {
	// the controller splits on 16-bit word boundaries (an odd split only at the slice's end)
	if (split > slice || ((split & 1) && split != slice)) return -2;
	Procs P(slice, split, device, threads);
	if (!P.ok) return -3;
	PAR2Proc par2;
	if (!par2.init(slice, P.be)) return -4;
	P.initCpu(threads);
	if (!par2.setRecoverySlices(numOutputs, exps)) return -5;
	for (unsigned i = 0; i < numInputs; i++) {
		par2.waitForAdd();
		add(par2, i);
	}
	par2.endInput().get();
	int ok = 1;
	for (unsigned o = 0; o < numOutputs; o++)
		if (!par2.getOutput(o, out + (size_t)o * slice).get()) ok = 0;
	par2.deinit();
	return ok;
}

}  // namespace

extern "C" {

// PAR2 create through PAR2Proc: inputs back to back (the last `lastSize`
// bytes long), input numbers, recovery exponents.  Returns 1 if every output
// passed its memory checksum, 0 if one did not, < 0 on a set-up error.
int shim_par2_create(const uint8_t* inputs, unsigned numInputs, size_t sliceSize, size_t lastSize,
                     const uint16_t* inputIdx, const uint16_t* exps, unsigned numOutputs, uint8_t* out,
                     size_t split, int device, int threads) {
	return run(sliceSize, split, device, threads, numInputs, numOutputs, exps, out, [&](PAR2Proc& p, unsigned i) {
		const size_t sz = (i == numInputs - 1) ? lastSize : sliceSize;
		p.addInput(inputs + (size_t)i * sliceSize, sz, inputIdx[i], false);
	});
}

// The decode overload: coeffs[i * numOutputs + o] per input.
int shim_par2_create_coeffs(const uint8_t* inputs, unsigned numInputs, size_t sliceSize, const uint16_t* coeffs,
                            unsigned numOutputs, uint8_t* out, size_t split, int device, int threads) {
	return run(sliceSize, split, device, threads, numInputs, numOutputs, nullptr, out, [&](PAR2Proc& p, unsigned i) {
		p.addInput(inputs + (size_t)i * sliceSize, sliceSize, coeffs + (size_t)i * numOutputs, false);
	});
}

// A second setSliceSize with a different size on the same backend (the
// shim reallocates), then a create: returns what shim_par2_create returns.
int shim_par2_resize_then_create(const uint8_t* inputs, unsigned numInputs, size_t firstSize, size_t sliceSize,
                                 const uint16_t* inputIdx, const uint16_t* exps, unsigned numOutputs, uint8_t* out,
                                 int device) {
	PAR2ProcCUDA cuda(device);
	if (!cuda.init()) return -3;
	cuda.setSliceSize(firstSize);
	std::vector<PAR2ProcBackendAlloc> be{{&cuda, 0, sliceSize}};
	PAR2Proc par2;
	if (!par2.init(sliceSize, be)) return -4;
	if (!par2.setRecoverySlices(numOutputs, exps)) return -5;
	for (unsigned i = 0; i < numInputs; i++) {
		par2.waitForAdd();
		par2.addInput(inputs + (size_t)i * sliceSize, sliceSize, inputIdx[i], false);
	}
	par2.endInput().get();
	int ok = 1;
	for (unsigned o = 0; o < numOutputs; o++)
		if (!par2.getOutput(o, out + (size_t)o * sliceSize).get()) ok = 0;
	par2.deinit();
	return ok;
}

}  // extern "C"
