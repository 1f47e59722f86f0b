// PAR2ProcCUDA (see controller_cuda.h): IPAR2ProcBackend over the
// parparpar_b200 processor.  Error handling follows PAR2ProcCPU / PAR2ProcOCL:
// bool returns for set-up calls, PROC_ADD_FULL for back-pressure; a failed
// device call leaves the backend unusable and getOutput reports invalid.
#include "controller_cuda.h"

#include <cstdio>
#include <cstring>
#include <vector>

namespace {
#ifndef USE_LIBUV
std::future<void> ready() {
	std::promise<void> p;
	p.set_value();
	return p.get_future();
}
std::future<bool> ready(bool v) {
	std::promise<bool> p;
	p.set_value(v);
	return p.get_future();
}
#endif
}  // namespace

#ifdef USE_LIBUV
PAR2ProcCUDA::PAR2ProcCUDA(uv_loop_t* loop, int dev, unsigned areas, unsigned batch)
: IPAR2ProcBackend(loop), ctx(nullptr), proc(nullptr), device(dev), sliceSize(0), stagingAreas(areas ? areas : 2),
  batchHint(batch), addedSinceEnd(false), watchStop(false), watchSubmitted(0), watchReported(0) {
#else
PAR2ProcCUDA::PAR2ProcCUDA(int dev, unsigned areas, unsigned batch)
: IPAR2ProcBackend(), ctx(nullptr), proc(nullptr), device(dev), sliceSize(0), stagingAreas(areas ? areas : 2),
  batchHint(batch), addedSinceEnd(false) {
#endif
	processingAdd = false;
	currentStagingArea = currentStagingInputs = 0;
	inputBatchSize = minInBatchSize = batch;
	statBatchesStarted = 0;
}

PAR2ProcCUDA::~PAR2ProcCUDA() {
	_deinit();
}

bool PAR2ProcCUDA::init() {
	if (ctx) return true;
	if (pp_ctx_create(device, &ctx) != PP_OK) {
		ctx = nullptr;
		return false;
	}
	return true;
}

const char* PAR2ProcCUDA::getLastError() const {
	return ctx ? pp_ctx_last_error(ctx) : "no CUDA context";
}

void PAR2ProcCUDA::_deinit() {
#ifdef USE_LIBUV
	if (watcher.joinable()) {
		{
			std::lock_guard<std::mutex> g(watchMu);
			watchStop = true;
		}
		watchCv.notify_all();
		watcher.join();
	}
#endif
	if (proc) pp_par2_proc_destroy(proc);
	proc = nullptr;
	if (ctx) pp_ctx_destroy(ctx);
	ctx = nullptr;
}

// (Re)create the processor for slices of `size` bytes: a different size from
// a second setSliceSize call gets a new allocation, as PAR2ProcCPU reallocates
// its staging (gf16/controller_cpu.cpp:93-117).
bool PAR2ProcCUDA::reopen(size_t size) {
	if (!init()) return false;
	if (proc && size == sliceSize) return true;
	if (proc) pp_par2_proc_destroy(proc);
	proc = nullptr;
	if (pp_par2_proc_create(ctx, size, stagingAreas, batchHint, &proc) != PP_OK) {
		proc = nullptr;
		return false;
	}
	sliceSize = size;
	inputBatchSize = pp_par2_proc_input_batch_size(proc);
	if (!minInBatchSize) minInBatchSize = inputBatchSize;
	if (!outputExponents.empty())
		return pp_par2_proc_set_recovery_slices(proc, (unsigned)outputExponents.size(), outputExponents.data()) ==
		       PP_OK;
	return true;
}

void PAR2ProcCUDA::syncStats() {
	if (!proc) return;
	const unsigned started = pp_par2_proc_batches_started(proc);
#ifdef USE_LIBUV
	if (started > statBatchesStarted) {
		// each newly submitted batch holds a staging area until the device is done with it
		for (unsigned k = statBatchesStarted; k < started; k++) stagingActiveCount_inc();
		{
			std::lock_guard<std::mutex> g(watchMu);
			watchSubmitted = started;
		}
		watchCv.notify_one();
		if (!watcher.joinable()) watcher = std::thread(&PAR2ProcCUDA::watchLoop, this);
	}
#endif
	statBatchesStarted = started;
}

void PAR2ProcCUDA::setSliceSize(size_t size) {
	reopen(size);
}

bool PAR2ProcCUDA::setCurrentSliceSize(size_t size) {
	if (!proc) return reopen(size);
	// shrinking keeps the allocation; growing reallocates inside the processor
	return pp_par2_proc_set_current_slice_size(proc, size) == PP_OK;
}

bool PAR2ProcCUDA::setRecoverySlices(unsigned numSlices, const uint16_t* exponents) {
	outputExponents.resize(numSlices);
	for (unsigned i = 0; i < numSlices; i++) outputExponents[i] = exponents ? exponents[i] : 1;
	if (!proc) return true;  // applied when the processor is created
	return pp_par2_proc_set_recovery_slices(proc, numSlices, exponents) == PP_OK;
}

PAR2ProcBackendAddResult PAR2ProcCUDA::canAdd() const {
	if (!proc) return PROC_ADD_FULL;
	switch (pp_par2_proc_can_add(proc)) {
		case PP_PROC_ADD_OK: return PROC_ADD_OK;
		case PP_PROC_ADD_OK_BUSY: return PROC_ADD_OK_BUSY;
		default: return PROC_ADD_FULL;
	}
}

#ifndef USE_LIBUV
void PAR2ProcCUDA::waitForAdd() {
	if (proc) pp_par2_proc_wait_for_add(proc);
}

std::future<void> PAR2ProcCUDA::addInput(const void* buffer, size_t size, uint16_t inputNum, bool flush) {
	// the processor copies the slice before returning: the caller's buffer is free at once
	if (proc && pp_par2_proc_add_input(proc, buffer, size, inputNum, flush ? 1 : 0) == PP_OK) {
		processingAdd = true;
		addedSinceEnd = true;
	}
	syncStats();
	return ready();
}

std::future<void> PAR2ProcCUDA::addInput(const void* buffer, size_t size, const uint16_t* coeffs, bool flush) {
	if (proc && pp_par2_proc_add_input_coeffs(proc, buffer, size, coeffs, flush ? 1 : 0) == PP_OK) {
		processingAdd = true;
		addedSinceEnd = true;
	}
	syncStats();
	return ready();
}

std::future<void> PAR2ProcCUDA::endInput() {
	if (proc) pp_par2_proc_end_input(proc);
	syncStats();
	addedSinceEnd = false;
	processing_finished();
	return ready();
}

std::future<bool> PAR2ProcCUDA::getOutput(unsigned index, void* output) {
	int valid = 0;
	if (!proc || pp_par2_proc_get_output(proc, index, output, &valid) != PP_OK) return ready(false);
	return ready(valid != 0);
}
#endif

// Benchmark-only calls of the interface (PAR2Proc::dummyInput / fillInput):
// a dummy input adds a zero slice under that input number; fillInput has no
// staging of its own to fill.
void PAR2ProcCUDA::dummyInput(uint16_t inputNum, bool flush) {
	if (!proc) return;
	std::vector<uint8_t> zero(sliceSize, 0);
	if (pp_par2_proc_add_input(proc, zero.data(), zero.size(), inputNum, flush ? 1 : 0) == PP_OK) processingAdd = true;
	syncStats();
}

bool PAR2ProcCUDA::fillInput(const void*) {
	return true;
}

void PAR2ProcCUDA::flush() {
	if (proc) pp_par2_proc_flush(proc);
	syncStats();
}

void PAR2ProcCUDA::freeProcessingMem() {
	if (proc) pp_par2_proc_free_processing_mem(proc);
}

#ifdef USE_LIBUV
// -------- libuv build: callbacks on the loop thread --------------------------
// The processor finishes an add before pp_par2_proc_add_input returns, so the
// add's callback is queued at once; finished batches are reported by the
// watcher thread, which waits for them with pp_par2_proc_wait_batches (a wait
// on host-side counters only, safe beside the loop thread's calls).
void PAR2ProcCUDA::watchLoop() {
	for (;;) {
		unsigned target;
		{
			std::unique_lock<std::mutex> g(watchMu);
			watchCv.wait(g, [this] { return watchStop || watchSubmitted > watchReported; });
			if (watchStop) return;
			target = watchReported + 1;
		}
		pp_par2_proc_wait_batches(proc, target);
		{
			std::lock_guard<std::mutex> g(watchMu);
			watchReported = target;
		}
		auto* req = new Req{2, nullptr, nullptr, true, target};
		_queueProc.notify(req);
	}
}

void PAR2ProcCUDA::addInput(const void* buffer, size_t size, uint16_t inputNum, bool flush, const PAR2ProcPlainCb& cb) {
	if (proc && pp_par2_proc_add_input(proc, buffer, size, inputNum, flush ? 1 : 0) == PP_OK) processingAdd = true;
	pendingInCallbacks++;
	syncStats();
	_queueSent.notify(new Req{0, cb, nullptr, true, 0});
}

void PAR2ProcCUDA::addInput(const void* buffer, size_t size, const uint16_t* coeffs, bool flush, const PAR2ProcPlainCb& cb) {
	if (proc && pp_par2_proc_add_input_coeffs(proc, buffer, size, coeffs, flush ? 1 : 0) == PP_OK)
		processingAdd = true;
	pendingInCallbacks++;
	syncStats();
	_queueSent.notify(new Req{0, cb, nullptr, true, 0});
}

void PAR2ProcCUDA::endInput() {
	// PAR2Proc calls the base class's endInput (endSignalled = true) after
	// flush(); completion reaches it through progressCb -> onBackendProcess
	endSignalled = true;
}

void PAR2ProcCUDA::getOutput(unsigned index, void* output, const PAR2ProcOutputCb& cb) {
	int valid = 0;
	const bool ok = proc && pp_par2_proc_get_output(proc, index, output, &valid) == PP_OK;
	pendingOutCallbacks++;
	_queueRecv.notify(new Req{1, nullptr, cb, ok && valid != 0, 0});
}

void PAR2ProcCUDA::_notifySent(void* r) {
	auto* req = static_cast<Req*>(r);
	pendingInCallbacks--;
	if (req->plain) req->plain();
	delete req;
	// the last add's callback may come after the last batch finished
	if (endSignalled && isEmpty() && progressCb) progressCb(0);
}

void PAR2ProcCUDA::_notifyRecv(void* r) {
	auto* req = static_cast<Req*>(r);
	pendingOutCallbacks--;
	if (req->output) req->output(req->valid);
	delete req;
	if (pendingOutCallbacks < 1 && deinitCallback) deinit(deinitCallback);
}

void PAR2ProcCUDA::_notifyProc(void* r) {
	auto* req = static_cast<Req*>(r);
	stagingActiveCount_dec();
	delete req;
	if (endSignalled && isEmpty()) {
		endSignalled = false;
		processing_finished();
	}
	// one finished staging area: PAR2Proc::onBackendProcess resumes adds
	if (progressCb) progressCb(inputBatchSize);
}
#endif
