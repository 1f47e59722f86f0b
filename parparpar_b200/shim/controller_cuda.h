// PAR2ProcCUDA: the CUDA backend of the reference's PAR2 front controller.
//
// This file belongs in the reference's tree beside gf16/controller_cpu.h and
// gf16/controller_ocl.h: it implements IPAR2ProcBackend (gf16/controller.h:
// 77-217) over the parparpar_b200 C ABI (include/parpar_b200.h, the
// pp_par2_proc_* processor), so PAR2Proc (gf16/controller.cpp) can drive a
// B200 alone or split each slice by byte range between it and PAR2ProcCPU
// (controller.cpp:42-84), and GfProc (src/gf.cc:700-724) can construct it
// from a `proc_cuda` option the way it constructs PAR2ProcOCL.
//
// Both controller builds are covered:
//  * without USE_LIBUV (the futures build, test/gf16/test-ctrl.cpp): addInput,
//    endInput and getOutput return ready futures -- the processor copies a
//    caller's slice before pp_par2_proc_add_input returns, and end_input /
//    get_output wait for the device;
//  * with USE_LIBUV (the Node addon): every callback is delivered on the loop
//    thread through the base class's ThreadNotifyQueues, and a watcher thread
//    reports finished batches to progressCb, which PAR2Proc::onBackendProcess
//    needs to resume adds after canAdd() said PROC_ADD_FULL.
#ifndef __GF16_CONTROLLER_CUDA
#define __GF16_CONTROLLER_CUDA

#include "controller.h"
#include "parpar_b200.h"

#ifdef USE_LIBUV
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#endif

class PAR2ProcCUDA : public IPAR2ProcBackend {
	pp_ctx* ctx;
	pp_par2_proc* proc;
	int device;
	size_t sliceSize;
	unsigned stagingAreas, batchHint;
	bool addedSinceEnd;

	void run_kernel(unsigned, unsigned) override {}  // the processor launches its own kernels
	void _deinit() override;
	bool reopen(size_t size);
	void syncStats();

#ifdef USE_LIBUV
	struct Req {
		int kind;  // 0: add done, 1: output ready, 2: end of input
		PAR2ProcPlainCb plain;
		PAR2ProcOutputCb output;
		bool valid;
		unsigned batches;
	};
	void _notifySent(void* req) override;
	void _notifyRecv(void* req) override;
	void _notifyProc(void* req) override;
	// batches-started watcher: reports finished staging areas to progressCb
	std::thread watcher;
	std::mutex watchMu;
	std::condition_variable watchCv;
	std::atomic<bool> watchStop;
	unsigned watchSubmitted, watchReported;
	void watchLoop();
#endif

public:
#ifdef USE_LIBUV
	explicit PAR2ProcCUDA(uv_loop_t* loop, int device = 0, unsigned stagingAreas = 2, unsigned inputBatch = 0);
#else
	explicit PAR2ProcCUDA(int device = 0, unsigned stagingAreas = 2, unsigned inputBatch = 0);
#endif
	~PAR2ProcCUDA() override;
	bool init();  // false when no device / library error (GfProc then skips the backend)
	const char* getLastError() const;

	void setSliceSize(size_t size) override;
	bool setCurrentSliceSize(size_t size) override;
	bool setRecoverySlices(unsigned numSlices, const uint16_t* exponents = nullptr) override;
	PAR2ProcBackendAddResult canAdd() const override;
	FUTURE_RETURN_T addInput(const void* buffer, size_t size, uint16_t inputNum, bool flush IF_LIBUV(, const PAR2ProcPlainCb& cb)) override;
	FUTURE_RETURN_T addInput(const void* buffer, size_t size, const uint16_t* coeffs, bool flush IF_LIBUV(, const PAR2ProcPlainCb& cb)) override;
	void dummyInput(uint16_t inputNum, bool flush = false) override;
	bool fillInput(const void* buffer) override;
	void flush() override;
#ifndef USE_LIBUV
	FUTURE_RETURN_T endInput() override;
	void waitForAdd() override;
#else
	void endInput();
#endif
	FUTURE_RETURN_BOOL_T getOutput(unsigned index, void* output IF_LIBUV(, const PAR2ProcOutputCb& cb)) override;
	void freeProcessingMem() override;
};

#endif
