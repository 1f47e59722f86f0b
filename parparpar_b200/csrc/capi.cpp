// C ABI implementation (include/parpar_b200.h): contexts, host/device buffer
// staging, the PAR2 processor and the PAR3 engine entry points.  All GF
// arithmetic on data runs in the CUDA kernels (gf16_kernels.cu,
// gf64_kernels.cu); the host side does argument checking, layout, and the
// scalar bookkeeping the reference also does on its host threads
// (coefficient columns, permutations, retry of a dropped recovery row).
#include "../../include/parpar_b200.h"

#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <list>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pp_internal.h"

namespace pp {
static std::atomic<uint64_t> g_launches{0};
void note_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }
uint64_t launches() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace pp

using namespace pp;

// ------------------------------------------------------------- host GF(2^16)
// Log/antilog tables of the PAR2 field with generator 2, and the table of
// input-constant logs (the i-th positive integer coprime to 65535).  These
// serve the scalar host bookkeeping only (coefficient columns of the
// processor, the permutation of the repair matrix); region data never goes
// through them.
namespace {
struct Gf16Host {
  uint16_t exp[65535 * 2];
  uint16_t log[65536];
  uint16_t ilog[32768];
  Gf16Host() {
    uint32_t n = 1;
    for (uint32_t e = 0; e < 65535; e++) {
      exp[e] = exp[e + 65535] = (uint16_t)n;
      log[n] = (uint16_t)e;
      n <<= 1;
      if (n & 0x10000) n ^= 0x1100B;
    }
    log[0] = 0;
    uint32_t e = 0;
    for (uint32_t i = 0; i < 32768; i++) {
      do {
        e++;
      } while (!(e % 3) || !(e % 5) || !(e % 17) || !(e % 257));
      ilog[i] = (uint16_t)e;
    }
  }
  uint16_t coeff(uint16_t idx, uint16_t ex) const {
    uint32_t l = ilog[idx & 32767];
    return exp[(uint32_t)(((uint64_t)l * ex) % 65535)];
  }
};
const Gf16Host& gf16h() {
  static Gf16Host* t = new Gf16Host();
  return *t;
}
}  // namespace

// -------------------------------------------------------------------- ctx
enum Slot { S_IN = 0, S_OUT, S_COEF, S_A, S_B, S_C, S_D, S_E, S_AEXP, S_HASH, S_HCV, S_PKT, S_STREAM, S_HSTATE, S_NSLOTS };

struct CauchyEntry {
  size_t n_in, n_rec;
  uint64_t fI, fR;
  uint64_t* d;  // from the context's memory pool, in the context stream's order
  size_t bytes;
};
// Resident Cauchy matrices per context: the reference keeps an LRU of 8
// (src/par3_engine.cc:451-482); on the device the bound is 32 matrices and
// 16 GiB, so a rotating set of repair shapes (a batch of different jobs run
// one after another) stays resident instead of being rebuilt every pass.
constexpr size_t kCauchyEntries = 32;
constexpr size_t kCauchyBytes = (size_t)16 << 30;
// Idle memory the context's pool keeps between calls (scratch growth and
// evicted matrices are recarved from it without driver calls).
constexpr uint64_t kPoolKeepBytes = (uint64_t)16 << 30;

// Resident PAR2 coefficient table: the coefficient matrix of (input slice
// numbers, exponents) and, for the tensor-core kernel, its expanded bit-matrix
// tiles; keyed by the two index lists.
struct Par2Entry {
  std::string key;
  uint16_t* d_coef = nullptr;
  uint8_t* d_aexp = nullptr;
  size_t bytes = 0;
};
constexpr size_t kPar2CacheEntries = 4;
constexpr size_t kPar2CacheBytes = (size_t)4 << 30;

struct pp_ctx {
  int device = 0;
  int sms = 148;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  void* slot_p[S_NSLOTS] = {};
  size_t slot_n[S_NSLOTS] = {};
  std::list<CauchyEntry> cauchy;  // LRU, front = most recent
  cudaMemPool_t pool = nullptr;   // stream-ordered pool of the scratch slots and Cauchy matrices (first use)
  cudaEvent_t alloc_ev = nullptr; // orders the side streams against pool allocations and frees
  std::list<Par2Entry> par2;      // LRU, front = most recent
  std::deque<size_t> par2_seen;   // hashes of recent PAR2 keys without a table
  int gf16_kernel = PP_GF16_KERNEL_AUTO;
  int gf64_kernel = PP_GF16_KERNEL_AUTO;
  int* d_status = nullptr;  // set nonzero by a kernel whose bounded wait gave up
  cudaStream_t copy = nullptr;     // host-to-device copies overlapped with the region kernels
  cudaEvent_t copy_ev = nullptr, start_ev = nullptr;
  cudaStream_t hash = nullptr;     // block hashes of staged inputs, beside the region kernels
  cudaEvent_t hash_ev = nullptr, staged_ev = nullptr;
  uint8_t* pinned = nullptr;       // streaming reads: two pinned chunk buffers
  size_t pinned_n = 0;
  // kernel timing (pp_ctx_set_kernel_timing): event pairs around region products
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> t_pending, t_free;
  std::mutex mu;
};

// Bracket one region product on the context's stream with CUDA events when
// kernel timing is on (measurement only; off by default).
static std::pair<cudaEvent_t, cudaEvent_t>* timing_begin(pp_ctx* ctx) {
  if (!ctx->timing) return nullptr;
  std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
  if (!ctx->t_free.empty()) {
    ev = ctx->t_free.back();
    ctx->t_free.pop_back();
  } else if (cudaEventCreate(&ev.first) != cudaSuccess || cudaEventCreate(&ev.second) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  ctx->t_pending.push_back(ev);
  cudaEventRecord(ev.first, ctx->stream);
  return &ctx->t_pending.back();
}
static void timing_end(pp_ctx* ctx, std::pair<cudaEvent_t, cudaEvent_t>* ev) {
  if (ev) cudaEventRecord(ev->second, ctx->stream);
}

static int set_err(pp_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

#define CUDA_TRY(ctx, expr)                                                                          \
  do {                                                                                               \
    cudaError_t _e = (expr);                                                                         \
    if (_e != cudaSuccess) {                                                                         \
      return set_err(ctx, PP_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, \
                     __LINE__);                                                                      \
    }                                                                                                \
  } while (0)

// ---- tracing: with PARPAR_B200_TRACE set (and not "0"), host-side spans of
// the single-job entry points and of the allocation / synchronisation calls
// their caches make are written to stderr, one line per span of at least
// 0.5 ms: "pp-trace <what> <bytes> <ms>".  Off by default (one getenv).
static bool trace_on() {
  static const bool on = [] {
    const char* e = getenv("PARPAR_B200_TRACE");
    return e && *e && strcmp(e, "0") != 0;
  }();
  return on;
}
struct TraceSpan {
  const char* what;
  size_t bytes;
  std::chrono::steady_clock::time_point t0;
  TraceSpan(const char* w, size_t b) : what(w), bytes(b), t0(std::chrono::steady_clock::now()) {}
  ~TraceSpan() {
    if (!trace_on()) return;
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (ms >= 0.5) fprintf(stderr, "pp-trace %s %zu %.3f\n", what, bytes, ms);
  }
};
#define PP_TRACE_CAT2(a, b) a##b
#define PP_TRACE_CAT(a, b) PP_TRACE_CAT2(a, b)
#define PP_TRACE(what, bytes) TraceSpan PP_TRACE_CAT(pp_span_, __LINE__)(what, bytes)

static int bind(pp_ctx* ctx) {
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return set_err(ctx, PP_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return PP_OK;
}

// accessors for the other host translation units (batch.cpp, server.cpp)
namespace pp {
int ctx_device(const pp_ctx* c) { return c->device; }
int ctx_sms(const pp_ctx* c) { return c->sms; }
cudaStream_t ctx_stream(const pp_ctx* c) { return c->stream; }
int* ctx_status_word(const pp_ctx* c) { return c->d_status; }
std::mutex& ctx_mutex(pp_ctx* c) { return c->mu; }
int ctx_fail(pp_ctx* c, int code, const char* msg) { return set_err(c, code, "%s", msg); }
}  // namespace pp

// Read and clear the device status word (after a synchronize).
static int device_status(pp_ctx* ctx) {
  int h = 0;
  if (cudaMemcpy(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, PP_ERR_CUDA, "status read failed");
  }
  if (h) {
    cudaMemset(ctx->d_status, 0, sizeof(int));
    return set_err(ctx, PP_ERR_TIMEOUT, "a device-side wait timed out; the kernel returned early");
  }
  return PP_OK;
}

// The context's stream-ordered memory pool, created on first use.  It keeps
// up to kPoolKeepBytes of freed memory, so buffers that are freed and
// allocated again (scratch growth, evicted Cauchy matrices) cost no driver
// call and no synchronisation: a cudaFree of a large buffer waits for the
// whole device and unmaps its pages, a cudaMalloc maps new ones, tens to
// hundreds of milliseconds each under load.
static cudaMemPool_t ctx_pool(pp_ctx* ctx) {
  if (ctx->pool) return ctx->pool;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = ctx->device;
  if (cudaMemPoolCreate(&ctx->pool, &props) != cudaSuccess) {
    cudaGetLastError();
    ctx->pool = nullptr;
    return nullptr;
  }
  if (cudaEventCreateWithFlags(&ctx->alloc_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    cudaMemPoolDestroy(ctx->pool);
    ctx->pool = nullptr;
    return nullptr;
  }
  uint64_t keep = kPoolKeepBytes;
  cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  return ctx->pool;
}

// Pool allocations and frees are ordered on the context stream.  The copy and
// hash streams also touch scratch buffers, so before a free the context
// stream waits for their work so far (join), and after an allocation they
// wait for the context stream (follow).
static void side_streams_join(pp_ctx* ctx) {
  for (cudaStream_t side : {ctx->copy, ctx->hash}) {
    if (!side) continue;
    cudaEventRecord(ctx->alloc_ev, side);
    cudaStreamWaitEvent(ctx->stream, ctx->alloc_ev, 0);
  }
}
static void side_streams_follow(pp_ctx* ctx) {
  if (!ctx->alloc_ev) return;
  cudaEventRecord(ctx->alloc_ev, ctx->stream);
  for (cudaStream_t side : {ctx->copy, ctx->hash})
    if (side) cudaStreamWaitEvent(side, ctx->alloc_ev, 0);
}

static void* pool_alloc(pp_ctx* ctx, size_t n) {
  cudaMemPool_t pool = ctx_pool(ctx);
  if (!pool) return nullptr;
  void* p = nullptr;
  if (cudaMallocFromPoolAsync(&p, n, pool, ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    // return the pool's idle memory to the device and retry once
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolTrimTo(pool, 0);
    if (cudaMallocFromPoolAsync(&p, n, pool, ctx->stream) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
  }
  side_streams_follow(ctx);
  return p;
}
static void pool_free(pp_ctx* ctx, void* p) {
  if (!p) return;
  side_streams_join(ctx);
  cudaFreeAsync(p, ctx->stream);
}

static void* scratch(pp_ctx* ctx, Slot s, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (ctx->slot_n[s] >= bytes) return ctx->slot_p[s];
  PP_TRACE("scratch-grow", bytes);
  const size_t prev_n = ctx->slot_n[s];
  if (ctx->slot_p[s]) {
    pool_free(ctx, ctx->slot_p[s]);
    ctx->slot_p[s] = nullptr;
    ctx->slot_n[s] = 0;
  }
  // headroom against regrowth: at least twice the previous size, so a stream
  // of growing jobs reallocates O(log) times
  size_t n = std::max(bytes + bytes / 8, 2 * prev_n);
  n = (n + 255) & ~(size_t)255;
  void* p = pool_alloc(ctx, n);
  if (!p) {
    p = pool_alloc(ctx, bytes);
    if (!p) return nullptr;
    n = bytes;
  }
  ctx->slot_p[s] = p;
  ctx->slot_n[s] = n;
  return p;
}

static bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static inline size_t round16(size_t v) { return (v + 15) & ~(size_t)15; }
static inline bool aligned16(const void* p, size_t stride) {
  return ((uintptr_t)p % 16) == 0 && (stride % 16) == 0;
}

// Upload a small host array into a scratch slot (pageable source: safe to
// reuse on return).  Device arrays are returned as is.
template <class T>
static const T* to_device(pp_ctx* ctx, Slot s, const T* p, size_t n, int* status) {
  *status = PP_OK;
  if (n == 0) return p;
  if (is_device_ptr(p)) return p;
  T* d = (T*)scratch(ctx, s, n * sizeof(T));
  if (!d) {
    *status = set_err(ctx, PP_ERR_NO_MEMORY, "device allocation of %zu bytes failed", n * sizeof(T));
    return nullptr;
  }
  cudaError_t e = cudaMemcpyAsync(d, p, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) {
    *status = set_err(ctx, PP_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
    return nullptr;
  }
  return d;
}

extern "C" {

PP_API const char* pp_version(void) { return "parpar_b200 0.1 (sm_100a)"; }

PP_API const char* pp_status_string(int s) {
  switch (s) {
    case PP_OK: return "ok";
    case PP_ERR_INVALID_ARG: return "invalid argument";
    case PP_ERR_CUDA: return "CUDA error";
    case PP_ERR_NO_MEMORY: return "out of device memory";
    case PP_ERR_SINGULAR: return "singular matrix";
    case PP_ERR_NOT_INVERTIBLE: return "recovery matrix not invertible";
    case PP_ERR_BUSY: return "staging area busy";
    case PP_ERR_NO_DEVICE: return "no CUDA device";
    case PP_ERR_UNSUPPORTED: return "unsupported";
    case PP_ERR_TIMEOUT: return "device wait timed out";
    case PP_ERR_TOO_LARGE: return "size above the entry point's fixed maximum";
    case PP_ERR_IO: return "file open or read failed";
    default: return "unknown status";
  }
}

PP_API uint64_t pp_launch_count(void) { return launches(); }

PP_API int pp_ctx_create(int device, pp_ctx** out) {
  if (!out) return PP_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return PP_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return PP_ERR_INVALID_ARG;
  pp_ctx* ctx = new pp_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete ctx;
    return PP_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return PP_ERR_CUDA;
  }
  if (cudaMalloc(&ctx->d_status, sizeof(int)) != cudaSuccess || cudaMemset(ctx->d_status, 0, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(ctx->own);
    delete ctx;
    return PP_ERR_CUDA;
  }
  ctx->stream = ctx->own;
  if (gf16_exp_table_init(ctx->own) != cudaSuccess || gf16_tc_tables_init(ctx->own) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(ctx->d_status);
    cudaStreamDestroy(ctx->own);
    delete ctx;
    return PP_ERR_CUDA;
  }
  if (const char* k = getenv("PP_GF16_KERNEL")) {
    if (!strcmp(k, "lut")) ctx->gf16_kernel = PP_GF16_KERNEL_LUT;
    else if (!strcmp(k, "tensor")) ctx->gf16_kernel = PP_GF16_KERNEL_TENSOR;
  }
  if (const char* k = getenv("PP_GF64_KERNEL")) {
    if (!strcmp(k, "lut")) ctx->gf64_kernel = PP_GF16_KERNEL_LUT;
    else if (!strcmp(k, "tensor")) ctx->gf64_kernel = PP_GF16_KERNEL_TENSOR;
  }
  *out = ctx;
  return PP_OK;
}

PP_API int pp_ctx_free_cache(pp_ctx* ctx) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  bind(ctx);
  cudaStreamSynchronize(ctx->stream);
  for (int s = 0; s < S_NSLOTS; s++) {
    pool_free(ctx, ctx->slot_p[s]);
    ctx->slot_p[s] = nullptr;
    ctx->slot_n[s] = 0;
  }
  for (auto& e : ctx->cauchy) pool_free(ctx, e.d);
  ctx->cauchy.clear();
  for (auto& e : ctx->par2) {
    pool_free(ctx, e.d_coef);
    pool_free(ctx, e.d_aexp);
  }
  ctx->par2.clear();
  if (ctx->pool) {
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolTrimTo(ctx->pool, 0);
  }
  return PP_OK;
}

PP_API int pp_ctx_set_kernel_timing(pp_ctx* ctx, int on) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->timing = on != 0;
  return PP_OK;
}

PP_API int pp_ctx_kernel_time(pp_ctx* ctx, double* ms, uint64_t* launches) {
  if (!ctx || !ms) return PP_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  double total = 0;
  for (auto& ev : ctx->t_pending) {
    CUDA_TRY(ctx, cudaEventSynchronize(ev.second));
    float t = 0;
    CUDA_TRY(ctx, cudaEventElapsedTime(&t, ev.first, ev.second));
    total += t;
  }
  *ms = total;
  if (launches) *launches = ctx->t_pending.size();
  ctx->t_free.insert(ctx->t_free.end(), ctx->t_pending.begin(), ctx->t_pending.end());
  ctx->t_pending.clear();
  return PP_OK;
}

PP_API void pp_ctx_destroy(pp_ctx* ctx) {
  if (!ctx) return;
  pp_ctx_free_cache(ctx);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& ev : ctx->t_pending) ctx->t_free.push_back(ev);
  for (auto& ev : ctx->t_free) {
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->copy) cudaStreamDestroy(ctx->copy);
  if (ctx->copy_ev) cudaEventDestroy(ctx->copy_ev);
  if (ctx->start_ev) cudaEventDestroy(ctx->start_ev);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->hash) cudaStreamDestroy(ctx->hash);
  if (ctx->hash_ev) cudaEventDestroy(ctx->hash_ev);
  if (ctx->staged_ev) cudaEventDestroy(ctx->staged_ev);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  if (ctx->alloc_ev) cudaEventDestroy(ctx->alloc_ev);
  delete ctx;
}

PP_API int pp_ctx_set_stream(pp_ctx* ctx, void* s) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  cudaStream_t n = s ? (cudaStream_t)s : ctx->own;
  if (n != ctx->stream && ctx->stream) {
    // resident buffers are freed and reused in the stream's order: finish
    // the old stream's work before another stream takes over
    std::lock_guard<std::mutex> g(ctx->mu);
    bind(ctx);
    cudaStreamSynchronize(ctx->stream);
  }
  ctx->stream = n;
  return PP_OK;
}
PP_API void* pp_ctx_get_stream(pp_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
PP_API int pp_ctx_synchronize(pp_ctx* ctx) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  bind(ctx);
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return device_status(ctx);
}

PP_API int pp_ctx_set_gf16_kernel(pp_ctx* ctx, int kernel) {
  if (!ctx || kernel < PP_GF16_KERNEL_AUTO || kernel > PP_GF16_KERNEL_TENSOR) return PP_ERR_INVALID_ARG;
  ctx->gf16_kernel = kernel;
  return PP_OK;
}

PP_API int pp_ctx_set_gf64_kernel(pp_ctx* ctx, int kernel) {
  if (!ctx || kernel < PP_GF16_KERNEL_AUTO || kernel > PP_GF16_KERNEL_TENSOR) return PP_ERR_INVALID_ARG;
  ctx->gf64_kernel = kernel;
  return PP_OK;
}
PP_API const char* pp_ctx_last_error(pp_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

// ============================================================ PAR2 / GF16
PP_API uint16_t pp_par2_coeff(uint16_t input_block, uint16_t exp) { return gf16h().coeff(input_block, exp); }
PP_API uint16_t pp_par2_input_log(uint16_t input_block) { return gf16h().ilog[input_block & 32767]; }

static int par2_coeff_matrix_dev(pp_ctx* ctx, const uint16_t* input_idx, unsigned n_in, const uint16_t* exps,
                                 unsigned n_out, uint16_t* d_coeffs) {
  // per-input logs (host bookkeeping: a table lookup per input) -> device
  std::vector<uint16_t> logs(n_in);
  std::vector<uint16_t> hidx(n_in);
  if (is_device_ptr(input_idx)) {
    CUDA_TRY(ctx, cudaMemcpyAsync(hidx.data(), input_idx, n_in * 2, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  } else {
    memcpy(hidx.data(), input_idx, n_in * 2);
  }
  for (unsigned i = 0; i < n_in; i++) {
    if (hidx[i] >= 32768) return set_err(ctx, PP_ERR_INVALID_ARG, "input index %u >= 32768", hidx[i]);
    logs[i] = gf16h().ilog[hidx[i]];
  }
  int st;
  const uint16_t* d_logs = to_device(ctx, S_A, logs.data(), n_in, &st);
  if (st) return st;
  const uint16_t* d_exps = to_device(ctx, S_B, exps, n_out, &st);
  if (st) return st;
  CUDA_TRY(ctx, launch_gf16_coeff_matrix(d_logs, n_in, d_exps, n_out, d_coeffs, ctx->stream));
  return PP_OK;
}

static bool use_tensor(int sel, unsigned n_in, unsigned n_out);

// The resident coefficient table of (input_idx, exps): built the second time
// a key is used (coefficient matrix, plus the expanded tiles when the
// tensor-core kernel is selected), then found by key; least recently used
// tables are dropped beyond kPar2CacheEntries / kPar2CacheBytes.
static int par2_table(pp_ctx* ctx, const uint16_t* input_idx, unsigned n_in, const uint16_t* exps, unsigned n_out,
                      const Par2Entry** out) {
  std::string key(2 * (size_t)(n_in + n_out) + 1, '\0');
  if (is_device_ptr(input_idx)) {
    CUDA_TRY(ctx, cudaMemcpy(&key[0], input_idx, n_in * 2, cudaMemcpyDeviceToHost));
  } else {
    memcpy(&key[0], input_idx, n_in * 2);
  }
  memcpy(&key[2 * (size_t)n_in], exps, n_out * 2);
  const bool tc = use_tensor(ctx->gf16_kernel, n_in, n_out);
  key.back() = tc ? 1 : 0;
  for (auto it = ctx->par2.begin(); it != ctx->par2.end(); ++it) {
    if (it->key == key) {
      ctx->par2.splice(ctx->par2.begin(), ctx->par2, it);
      *out = &ctx->par2.front();
      return PP_OK;
    }
  }
  // a key seen for the first time gets no table (*out = nullptr: the caller
  // uses the context's reusable scratch buffers); a table is built when the
  // key comes back, so a stream of one-off jobs allocates nothing per call
  const size_t h = std::hash<std::string>()(key);
  if (std::find(ctx->par2_seen.begin(), ctx->par2_seen.end(), h) == ctx->par2_seen.end()) {
    ctx->par2_seen.push_back(h);
    if (ctx->par2_seen.size() > 64) ctx->par2_seen.pop_front();
    *out = nullptr;
    return PP_OK;
  }
  Par2Entry e;
  e.key = std::move(key);
  const size_t cbytes = (size_t)n_in * n_out * 2, tbytes = tc ? gf16_tc_coeff_bytes(n_in, n_out) : 0;
  e.bytes = cbytes + tbytes;
  size_t total = e.bytes;
  for (auto& x : ctx->par2) total += x.bytes;
  // tables come from the context's pool; an evicted table is freed in the
  // stream's order, after every kernel that read it
  while (!ctx->par2.empty() && (ctx->par2.size() >= kPar2CacheEntries || total > kPar2CacheBytes)) {
    total -= ctx->par2.back().bytes;
    pool_free(ctx, ctx->par2.back().d_coef);
    pool_free(ctx, ctx->par2.back().d_aexp);
    ctx->par2.pop_back();
  }
  PP_TRACE("par2-table-alloc", e.bytes);
  e.d_coef = (uint16_t*)pool_alloc(ctx, cbytes);
  e.d_aexp = tbytes ? (uint8_t*)pool_alloc(ctx, tbytes) : nullptr;
  if (!e.d_coef || (tbytes && !e.d_aexp)) {
    pool_free(ctx, e.d_coef);
    pool_free(ctx, e.d_aexp);
    return set_err(ctx, PP_ERR_NO_MEMORY, "PAR2 coefficient table (%zu bytes)", e.bytes);
  }
  int r = par2_coeff_matrix_dev(ctx, input_idx, n_in, exps, n_out, e.d_coef);
  if (!r && tc) {
    cudaError_t ce = launch_gf16_tc_expand(e.d_coef, n_in, n_in, n_out, e.d_aexp, ctx->stream);
    if (ce != cudaSuccess) r = set_err(ctx, PP_ERR_CUDA, "tile expansion: %s", cudaGetErrorString(ce));
  }
  if (r) {
    pool_free(ctx, e.d_coef);
    pool_free(ctx, e.d_aexp);
    return r;
  }
  ctx->par2.push_front(std::move(e));
  *out = &ctx->par2.front();
  return PP_OK;
}

PP_API int pp_par2_coeff_matrix(pp_ctx* ctx, const uint16_t* input_idx, unsigned num_inputs, const uint16_t* exps,
                                unsigned num_outputs, uint16_t* coeffs) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if ((num_inputs && !input_idx) || (num_outputs && !exps) || !coeffs) return PP_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  size_t n = (size_t)num_inputs * num_outputs;
  if (!n) return PP_OK;
  bool dev = is_device_ptr(coeffs);
  uint16_t* d = dev ? coeffs : (uint16_t*)scratch(ctx, S_COEF, n * 2);
  if (!d) return set_err(ctx, PP_ERR_NO_MEMORY, "coefficient buffer");
  if (int r = par2_coeff_matrix_dev(ctx, input_idx, num_inputs, exps, num_outputs, d)) return r;
  if (!dev) {
    CUDA_TRY(ctx, cudaMemcpyAsync(coeffs, d, n * 2, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return PP_OK;
}

// GF(2^16) region kernel dispatch.  The tensor-core kernel needs its
// coefficient bit-matrix tiles, expanded into `aexp` (device scratch of
// gf16_tc_coeff_bytes bytes).
// AUTO: the tensor-core kernel whenever a full 8-input stage exists (it is
// 1.9x (R=8) to 2.2x (R=64) faster than the lookup kernel on 1 GiB jobs);
// the lookup kernel for fewer than 8 inputs.
static bool use_tensor(int sel, unsigned n_in, unsigned n_out) {
  if (sel == PP_GF16_KERNEL_LUT) return false;
  if (sel == PP_GF16_KERNEL_TENSOR) return true;
  return n_in >= 8 && n_out >= 1;
}
// aexp_ready: aexp already holds the expanded tiles of d_coeffs (a resident
// table), so the expansion is skipped
static cudaError_t gf16_region(int sel, const uint8_t* din, size_t dstride, unsigned n_in, size_t slice,
                               const uint16_t* d_coeffs, size_t ldc, unsigned n_out, uint8_t* dout, size_t ostride,
                               bool accumulate, int sms, uint8_t* aexp, int* d_status, cudaStream_t s,
                               bool aexp_ready = false) {
  if (use_tensor(sel, n_in, n_out) && aexp) {
    if (!aexp_ready) {
      cudaError_t e = launch_gf16_tc_expand(d_coeffs, ldc, n_in, n_out, aexp, s);
      if (e != cudaSuccess) return e;
    }
    return launch_gf16_muladd_tc(din, dstride, n_in, slice, aexp, n_out, dout, ostride, accumulate, sms, d_status, s);
  }
  return launch_gf16_muladd(din, dstride, n_in, slice, d_coeffs, ldc, n_out, dout, ostride, accumulate, sms, s);
}

// Region muladd with staging of host / unaligned buffers.
// Host inputs of a large tensor-core job are copied in chunks of
// kCopyChunk slices on the context's copy stream; the region kernel of chunk
// c (accumulating from the second chunk on) waits only for that chunk, so the
// copies overlap the products and the job takes about as long as its copies.
constexpr unsigned kCopyChunk = 4096;
constexpr unsigned kCopyTail = 256;
constexpr size_t kBandMinBytes = (size_t)128 << 20;  // column bands for staged inputs of at least this size
constexpr size_t kBandMinWidth = 4096;               // bytes of every slice per band, at least (multiple of 64)
constexpr size_t kGf16TileBytes = 128 * 128;  // one expanded tile (8 outputs x one stage of inputs)

static int ensure_copy_stream(pp_ctx* ctx) {
  if (ctx->copy) return PP_OK;
  if (cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->copy_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->start_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, PP_ERR_CUDA, "copy stream");
  }
  side_streams_follow(ctx);  // after the pool allocations made so far
  return PP_OK;
}

static int ensure_hash_stream(pp_ctx* ctx) {
  if (ctx->hash) return PP_OK;
  if (cudaStreamCreateWithFlags(&ctx->hash, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->hash_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->staged_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, PP_ERR_CUDA, "hash stream");
  }
  side_streams_follow(ctx);  // after the pool allocations made so far
  return PP_OK;
}

// Where the IFSC entries of a hashed region pass go on the device.
static uint8_t* hash_buffer(pp_ctx* ctx, uint8_t* hashes, unsigned n_in) {
  if (!hashes) return nullptr;
  if (is_device_ptr(hashes) && ((uintptr_t)hashes % 4) == 0) return hashes;
  return (uint8_t*)scratch(ctx, S_HASH, (size_t)20 * n_in);
}

// hashes: optional IFSC entries (MD5 || CRC32 of each input row's slice
// bytes), computed on the hash stream from the device rows as they are staged,
// concurrently with the region kernels; host or device memory, n_in x 20.
static int gf16_muladd_impl(pp_ctx* ctx, const void* inputs, size_t in_stride, unsigned n_in, size_t slice,
                            const uint16_t* d_coeffs, size_t ldc, unsigned n_out, void* outputs, size_t out_stride,
                            bool accumulate, uint8_t* aexp_ready = nullptr, uint8_t* hashes = nullptr) {
  const bool in_dev = is_device_ptr(inputs);
  const bool out_dev = is_device_ptr(outputs);
  const size_t row = round16(slice);
  if (hashes && n_in == 0) hashes = nullptr;
  uint8_t* dh = hash_buffer(ctx, hashes, n_in);
  if (hashes) {
    if (!dh) return set_err(ctx, PP_ERR_NO_MEMORY, "hash output");
    if (int r = ensure_hash_stream(ctx)) return r;
  }
  // after the region work: the hash stream's work joins the context's stream,
  // and host hash outputs are copied back
  auto join_hashes = [&]() -> int {
    if (!hashes) return PP_OK;
    CUDA_TRY(ctx, cudaEventRecord(ctx->hash_ev, ctx->hash));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->hash_ev, 0));
    if (dh != hashes)
      CUDA_TRY(ctx, cudaMemcpyAsync(hashes, dh, (size_t)20 * n_in, cudaMemcpyDefault, ctx->stream));
    return PP_OK;
  };
  if (!in_dev && n_in >= 2 * kCopyChunk && use_tensor(ctx->gf16_kernel, n_in, n_out)) {
    // ---- chunked: copies of chunk c+1 overlap the products of chunk c
    if (int r = ensure_copy_stream(ctx)) return r;
    uint8_t* din = (uint8_t*)scratch(ctx, S_IN, row * n_in);
    if (!din) return set_err(ctx, PP_ERR_NO_MEMORY, "input staging (%zu bytes)", row * n_in);
    uint8_t* dout = (uint8_t*)outputs;
    size_t ostride = out_stride;
    const bool stage_out = !out_dev || !aligned16(outputs, out_stride);
    if (stage_out) {
      dout = (uint8_t*)scratch(ctx, S_OUT, row * n_out);
      if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "output staging (%zu bytes)", row * n_out);
      ostride = row;
      if (accumulate)
        CUDA_TRY(ctx, cudaMemcpy2DAsync(dout, row, outputs, out_stride, slice, n_out,
                                        out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    }
    uint8_t* aexp = aexp_ready;
    if (!aexp) {
      aexp = (uint8_t*)scratch(ctx, S_AEXP, gf16_tc_coeff_bytes(n_in, n_out));
      if (!aexp) return set_err(ctx, PP_ERR_NO_MEMORY, "coefficient tiles");
      CUDA_TRY(ctx, launch_gf16_tc_expand(d_coeffs, ldc, n_in, n_out, aexp, ctx->stream));
    }
    const unsigned si = gf16_tc_stage_inputs();  // inputs per tile stage (8 int8, 16 FP4)
    const unsigned stages = (n_in + si - 1) / si;
    // the staging rows are free once earlier work on the context's stream is done
    CUDA_TRY(ctx, cudaEventRecord(ctx->start_ev, ctx->stream));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy, ctx->start_ev, 0));
    if (hashes) CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->hash, ctx->start_ev, 0));
    unsigned hashed = 0;  // slices whose hashes are launched
    for (unsigned c0 = 0, nc = 0; c0 < n_in; c0 += nc) {
      // the last kCopyChunk slices go in halving pieces (down to kCopyTail),
      // so little product work is left once the final copy has landed
      const unsigned rest = n_in - c0;
      // (pieces are multiples of 16 slices: whole tile stages of either operand format)
      nc = rest > kCopyChunk ? kCopyChunk : rest > kCopyTail ? std::max(kCopyTail, (rest / 2 + 15) & ~15u) : rest;
      CUDA_TRY(ctx, cudaMemcpy2DAsync(din + (size_t)c0 * row, row, (const uint8_t*)inputs + (size_t)c0 * in_stride,
                                      in_stride, slice, nc, cudaMemcpyHostToDevice, ctx->copy));
      CUDA_TRY(ctx, cudaEventRecord(ctx->copy_ev, ctx->copy));
      CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->copy_ev, 0));
      // hashes: one launch per full chunk, one for all the tail pieces (an
      // MD5 takes as long for 256 slices as for 4,096, its chain being serial
      // within each slice, so per-piece launches would queue up after the
      // last copy)
      if (hashes && (nc == kCopyChunk || c0 + nc == n_in)) {
        CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->hash, ctx->copy_ev, 0));
        CUDA_TRY(ctx, launch_par2_block_hash(din + (size_t)hashed * row, row, c0 + nc - hashed, slice, nullptr,
                                             dh + (size_t)20 * hashed, ctx->hash));
        hashed = c0 + nc;
      }
      CUDA_TRY(ctx, launch_gf16_muladd_tc(din + (size_t)c0 * row, row, nc, slice, aexp + (size_t)(c0 / si) * kGf16TileBytes,
                                          n_out, dout, ostride, accumulate || c0 > 0, ctx->sms, ctx->d_status,
                                          ctx->stream, stages));
    }
    if (stage_out)
      CUDA_TRY(ctx, cudaMemcpy2DAsync(outputs, out_stride, dout, row, slice, n_out,
                                      out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    if (int r = join_hashes()) return r;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return device_status(ctx);
  }
  // ---- column bands: host inputs of few large slices with their hashes.
  // An MD5 chain runs through a whole slice, so hashing after the last copy
  // would add a full slice's chain (about 17 ms for 1 MiB) to the call.  The
  // copies go instead as column bands of every slice (bytes [c0, c1) of all
  // rows, about 64 MiB per band); each band's product (the region product is
  // column-separable) and the band's MD5 / CRC32 blocks (state carried from
  // band to band) run as it lands.
  const size_t band_w = std::max<size_t>(kBandMinWidth, (((size_t)64 << 20) / std::max(1u, n_in)) & ~(size_t)63);
  if (hashes && !in_dev && n_in < 2 * kCopyChunk && use_tensor(ctx->gf16_kernel, n_in, n_out) &&
      (size_t)row * n_in >= kBandMinBytes && slice > band_w) {
    if (int r = ensure_copy_stream(ctx)) return r;
    uint8_t* din = (uint8_t*)scratch(ctx, S_IN, row * n_in);
    uint32_t* hst = (uint32_t*)scratch(ctx, S_HSTATE, (size_t)20 * n_in);
    if (!din || !hst) return set_err(ctx, PP_ERR_NO_MEMORY, "input staging (%zu bytes)", row * n_in);
    uint8_t* dout = (uint8_t*)outputs;
    size_t ostride = out_stride;
    const bool stage_out = !out_dev || !aligned16(outputs, out_stride);
    if (stage_out) {
      dout = (uint8_t*)scratch(ctx, S_OUT, row * n_out);
      if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "output staging (%zu bytes)", row * n_out);
      ostride = row;
      if (accumulate)
        CUDA_TRY(ctx, cudaMemcpy2DAsync(dout, row, outputs, out_stride, slice, n_out,
                                        out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    }
    uint8_t* aexp = aexp_ready;
    if (!aexp) {
      aexp = (uint8_t*)scratch(ctx, S_AEXP, gf16_tc_coeff_bytes(n_in, n_out));
      if (!aexp) return set_err(ctx, PP_ERR_NO_MEMORY, "coefficient tiles");
      CUDA_TRY(ctx, launch_gf16_tc_expand(d_coeffs, ldc, n_in, n_out, aexp, ctx->stream));
    }
    CUDA_TRY(ctx, cudaEventRecord(ctx->start_ev, ctx->stream));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy, ctx->start_ev, 0));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->hash, ctx->start_ev, 0));
    for (size_t c0 = 0; c0 < slice; c0 += band_w) {
      const size_t c1 = std::min(slice, c0 + band_w);
      CUDA_TRY(ctx, cudaMemcpy2DAsync(din + c0, row, (const uint8_t*)inputs + c0, in_stride, c1 - c0, n_in,
                                      cudaMemcpyHostToDevice, ctx->copy));
      CUDA_TRY(ctx, cudaEventRecord(ctx->copy_ev, ctx->copy));
      CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->copy_ev, 0));
      CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->hash, ctx->copy_ev, 0));
      const bool last = c1 == slice;
      CUDA_TRY(ctx, launch_par2_block_hash_band(din, row, n_in, slice, c0 / 64, last ? slice / 64 : c1 / 64, hst, dh,
                                                c0 == 0, last, ctx->hash));
      CUDA_TRY(ctx, launch_gf16_muladd_tc(din + c0, row, n_in, c1 - c0, aexp, n_out, dout + c0, ostride, accumulate,
                                          ctx->sms, ctx->d_status, ctx->stream));
    }
    if (stage_out)
      CUDA_TRY(ctx, cudaMemcpy2DAsync(outputs, out_stride, dout, row, slice, n_out,
                                      out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    if (int r = join_hashes()) return r;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return device_status(ctx);
  }
  const uint8_t* din = (const uint8_t*)inputs;
  size_t dstride = in_stride;
  if (n_in && (!in_dev || !aligned16(inputs, in_stride))) {
    uint8_t* s = (uint8_t*)scratch(ctx, S_IN, row * n_in);
    if (!s) return set_err(ctx, PP_ERR_NO_MEMORY, "input staging (%zu bytes)", row * n_in);
    CUDA_TRY(ctx, cudaMemcpy2DAsync(s, row, inputs, in_stride, slice, n_in,
                                    in_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    din = s;
    dstride = row;
  }
  if (hashes) {  // hash the staged rows beside the region kernel
    CUDA_TRY(ctx, cudaEventRecord(ctx->staged_ev, ctx->stream));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->hash, ctx->staged_ev, 0));
    CUDA_TRY(ctx, launch_par2_block_hash(din, dstride, n_in, slice, nullptr, dh, ctx->hash));
  }
  uint8_t* dout = (uint8_t*)outputs;
  size_t ostride = out_stride;
  const bool stage_out = !out_dev || !aligned16(outputs, out_stride);
  if (stage_out) {
    dout = (uint8_t*)scratch(ctx, S_OUT, row * n_out);
    if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "output staging (%zu bytes)", row * n_out);
    ostride = row;
    if (accumulate)
      CUDA_TRY(ctx, cudaMemcpy2DAsync(dout, row, outputs, out_stride, slice, n_out,
                                      out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
  }
  uint8_t* aexp = aexp_ready;
  if (!aexp && use_tensor(ctx->gf16_kernel, n_in, n_out)) {
    aexp = (uint8_t*)scratch(ctx, S_AEXP, gf16_tc_coeff_bytes(n_in, n_out));
    if (!aexp) return set_err(ctx, PP_ERR_NO_MEMORY, "coefficient tiles");
  }
  auto* tev = timing_begin(ctx);
  CUDA_TRY(ctx, gf16_region(ctx->gf16_kernel, din, dstride, n_in, slice, d_coeffs, ldc, n_out, dout, ostride,
                            accumulate, ctx->sms, aexp, ctx->d_status, ctx->stream, aexp_ready != nullptr));
  timing_end(ctx, tev);
  if (stage_out) {
    CUDA_TRY(ctx, cudaMemcpy2DAsync(outputs, out_stride, dout, row, slice, n_out,
                                    out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (int r = join_hashes()) return r;
  if (!in_dev || !out_dev || (hashes && dh != hashes)) {
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return device_status(ctx);
  }
  return PP_OK;
}

PP_API int pp_gf16_muladd(pp_ctx* ctx, const void* inputs, size_t input_stride, unsigned num_inputs,
                          size_t slice_bytes, const uint16_t* coeffs, size_t coeff_stride, unsigned num_outputs,
                          void* outputs, size_t output_stride, int accumulate) {
  PP_TRACE("call-gf16_muladd", 0);
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!outputs || (num_inputs && (!inputs || !coeffs))) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if (num_inputs && input_stride < slice_bytes) return set_err(ctx, PP_ERR_INVALID_ARG, "input_stride < slice_bytes");
  if (num_outputs > 1 && output_stride < slice_bytes)
    return set_err(ctx, PP_ERR_INVALID_ARG, "output_stride < slice_bytes");
  if (num_outputs && coeff_stride < num_inputs) return set_err(ctx, PP_ERR_INVALID_ARG, "coeff_stride < num_inputs");
  if (!num_outputs || !slice_bytes) return PP_OK;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  if (output_stride < slice_bytes) output_stride = round16(slice_bytes);
  int st = PP_OK;
  const uint16_t* dc = coeffs;
  if (num_inputs) {
    // pack coefficients densely on the device
    std::vector<uint16_t> hc;
    if (!is_device_ptr(coeffs)) {
      hc.resize((size_t)num_outputs * num_inputs);
      for (unsigned o = 0; o < num_outputs; o++)
        memcpy(&hc[(size_t)o * num_inputs], coeffs + (size_t)o * coeff_stride, num_inputs * 2);
      dc = to_device(ctx, S_COEF, hc.data(), hc.size(), &st);
      if (st) return st;
      coeff_stride = num_inputs;
    }
  }
  return gf16_muladd_impl(ctx, inputs, input_stride, num_inputs, slice_bytes, dc, coeff_stride, num_outputs, outputs,
                          output_stride, accumulate != 0);
}

static int par2_create_impl(pp_ctx* ctx, const void* inputs, size_t input_stride, unsigned num_inputs,
                            size_t slice_bytes, const uint16_t* input_idx, const uint16_t* exps, unsigned num_outputs,
                            void* outputs, size_t output_stride, uint8_t* hashes) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!outputs || (num_inputs && (!inputs || !input_idx)) || (num_outputs && !exps))
    return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if (num_inputs && input_stride < slice_bytes) return set_err(ctx, PP_ERR_INVALID_ARG, "input_stride < slice_bytes");
  if (num_inputs > 32768) return set_err(ctx, PP_ERR_INVALID_ARG, "PAR2 allows at most 32768 input slices");
  if (!num_outputs || !slice_bytes) return PP_OK;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  if (output_stride < slice_bytes) output_stride = round16(slice_bytes);
  if (!num_inputs)
    return gf16_muladd_impl(ctx, inputs, input_stride, 0, slice_bytes, nullptr, 0, num_outputs, outputs,
                            output_stride, false);
  const Par2Entry* t = nullptr;
  if (int r = par2_table(ctx, input_idx, num_inputs, exps, num_outputs, &t)) return r;
  if (t)
    return gf16_muladd_impl(ctx, inputs, input_stride, num_inputs, slice_bytes, t->d_coef, num_inputs, num_outputs,
                            outputs, output_stride, false, t->d_aexp, hashes);
  uint16_t* dc = (uint16_t*)scratch(ctx, S_COEF, (size_t)num_inputs * num_outputs * 2);
  if (!dc) return set_err(ctx, PP_ERR_NO_MEMORY, "coefficients");
  if (int r = par2_coeff_matrix_dev(ctx, input_idx, num_inputs, exps, num_outputs, dc)) return r;
  return gf16_muladd_impl(ctx, inputs, input_stride, num_inputs, slice_bytes, dc, num_inputs, num_outputs, outputs,
                          output_stride, false, nullptr, hashes);
}

PP_API int pp_par2_create(pp_ctx* ctx, const void* inputs, size_t input_stride, unsigned num_inputs,
                          size_t slice_bytes, const uint16_t* input_idx, const uint16_t* exps, unsigned num_outputs,
                          void* outputs, size_t output_stride) {
  PP_TRACE("call-par2_create", 0);
  return par2_create_impl(ctx, inputs, input_stride, num_inputs, slice_bytes, input_idx, exps, num_outputs, outputs,
                          output_stride, nullptr);
}

PP_API int pp_par2_create_hashed(pp_ctx* ctx, const void* inputs, size_t input_stride, unsigned num_inputs,
                                 size_t slice_bytes, const uint16_t* input_idx, const uint16_t* exps,
                                 unsigned num_outputs, void* outputs, size_t output_stride, uint8_t* md5crc) {
  if (ctx && num_inputs && !md5crc) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if (ctx && num_inputs && (!num_outputs || !slice_bytes))  // nothing to create: the hashes alone
    return pp_par2_block_hashes(ctx, inputs, input_stride, num_inputs, slice_bytes, nullptr, md5crc);
  return par2_create_impl(ctx, inputs, input_stride, num_inputs, slice_bytes, input_idx, exps, num_outputs, outputs,
                          output_stride, md5crc);
}

PP_API int pp_par2_invert(pp_ctx* ctx, const uint8_t* valid, unsigned num_inputs, uint16_t* recovery,
                          unsigned* num_recovery, uint16_t* factors) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!valid || !recovery || !num_recovery || !factors) return set_err(ctx, PP_ERR_INVALID_ARG, "null argument");
  if (num_inputs == 0 || num_inputs > 32768) return set_err(ctx, PP_ERR_INVALID_ARG, "num_inputs out of range");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  // host bookkeeping: column permutation, row list (Construct, gfmat_inv.cpp:462-558)
  std::vector<uint32_t> col_of(num_inputs);
  unsigned vc = 0;
  for (unsigned i = 0; i < num_inputs; i++) vc += valid[i] ? 1 : 0;
  const unsigned m = num_inputs - vc;
  if (m == 0) return set_err(ctx, PP_ERR_INVALID_ARG, "no missing input slices");
  {
    unsigned a = 0, b = vc;
    for (unsigned i = 0; i < num_inputs; i++) col_of[i] = valid[i] ? a++ : b++;
  }
  std::vector<uint16_t> rec(recovery, recovery + *num_recovery);
  std::sort(rec.begin(), rec.end());
  std::vector<uint16_t> logs(num_inputs);
  for (unsigned i = 0; i < num_inputs; i++) logs[i] = gf16h().ilog[i];
  // The matrix [valid columns | lost columns] is reduced by eliminating on
  // the lost columns; row operations never mix the two blocks, so the same
  // pivots (and zero pivots) arise from the m x m lost block B alone.  The
  // factors are then [B^-1 * valid block | B^-1]: an m x m elimination plus
  // one region product, instead of m pivot steps over all n columns.
  const size_t ld = (num_inputs + 7) & ~(size_t)7;
  const size_t ldb = (m + 7) & ~(size_t)7;
  uint16_t* d_mat = (uint16_t*)scratch(ctx, S_D, (size_t)m * ld * 2);
  uint16_t* d_fcol = (uint16_t*)scratch(ctx, S_E, (size_t)m * 2 + 64);
  uint16_t* d_blk = (uint16_t*)scratch(ctx, S_PKT, (size_t)m * ldb * 2);
  uint16_t* d_fac = (uint16_t*)scratch(ctx, S_OUT, (size_t)m * ld * 2);
  if (!d_mat || !d_fcol || !d_blk || !d_fac) return set_err(ctx, PP_ERR_NO_MEMORY, "inversion matrix");
  int* d_status = (int*)((char*)d_fcol + (((size_t)m * 2 + 15) & ~(size_t)15));
  int st;
  const uint16_t* d_logs = to_device(ctx, S_A, logs.data(), num_inputs, &st);
  if (st) return st;
  const uint32_t* d_col = to_device(ctx, S_B, col_of.data(), num_inputs, &st);
  if (st) return st;
  for (;;) {
    if (rec.size() < m) return set_err(ctx, PP_ERR_NOT_INVERTIBLE, "not enough recovery slices to invert");
    const uint16_t* d_rec = to_device(ctx, S_C, rec.data(), m, &st);
    if (st) return st;
    CUDA_TRY(ctx, cudaMemsetAsync(d_mat, 0, (size_t)m * ld * 2, ctx->stream));
    CUDA_TRY(ctx, launch_gf16_build_rec_matrix(d_logs, d_col, num_inputs, d_rec, m, d_mat, ld, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy2DAsync(d_blk, ldb * 2, d_mat + vc, ld * 2, (size_t)m * 2, m, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(d_status, 0xFF, sizeof(int), ctx->stream));
    CUDA_TRY(ctx, launch_gf16_invert(d_blk, m, m, ldb, 0, d_fcol, d_status, ctx->stream));
    int hs = -1;
    CUDA_TRY(ctx, cudaMemcpyAsync(&hs, d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (hs < 0) break;
    rec.erase(rec.begin() + hs);  // PAR2 flaw: drop the recovery row and retry
  }
  // factors = [B^-1 * valid block | B^-1]
  if (vc) {
    uint8_t* aexp = nullptr;
    if (use_tensor(ctx->gf16_kernel, m, m)) {
      aexp = (uint8_t*)scratch(ctx, S_AEXP, gf16_tc_coeff_bytes(m, m));
      if (!aexp) return set_err(ctx, PP_ERR_NO_MEMORY, "coefficient tiles");
    }
    CUDA_TRY(ctx, gf16_region(ctx->gf16_kernel, (const uint8_t*)d_mat, ld * 2, m, (size_t)vc * 2, d_blk, ldb, m,
                              (uint8_t*)d_fac, ld * 2, false, ctx->sms, aexp, ctx->d_status, ctx->stream));
  }
  CUDA_TRY(ctx, cudaMemcpy2DAsync(d_fac + vc, ld * 2, d_blk, ldb * 2, (size_t)m * 2, m, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
  CUDA_TRY(ctx, cudaMemcpy2DAsync(factors, (size_t)num_inputs * 2, d_fac, ld * 2, (size_t)num_inputs * 2, m,
                                  is_device_ptr(factors) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (int r = device_status(ctx)) return r;
  memcpy(recovery, rec.data(), m * 2);
  *num_recovery = m;
  return PP_OK;
}

// ------------------------------------------------------------ PAR2 processor
struct pp_par2_proc {
  pp_ctx* ctx = nullptr;
  size_t alloc_size = 0, cur_size = 0, row = 0;
  unsigned batch = 12, n_areas = 2;
  unsigned batch_alloc = 12;  // rows allocated per staging area
  bool batch_fixed = false;   // the caller chose the batch size
  struct Area {
    uint8_t* d_in = nullptr;
    uint8_t* d_ck = nullptr;        // memory checksum block of each staged row (16 B rows)
    uint8_t* h_in = nullptr;        // pinned host rows: host inputs are staged here
    std::vector<uint8_t> host_row;  // row i of this batch sits in h_in (else already in d_in)
    uint16_t* d_coeff = nullptr;  // [n_out][batch]
    uint8_t* d_aexp = nullptr;    // tensor-core coefficient tiles
    std::vector<uint16_t> h_coeff;
    std::vector<uint16_t> h_idx;  // input number of each staged row (0xFFFF: not hashed)
    uint16_t* d_idx = nullptr;
    unsigned d_idx_n = 0;
    unsigned count = 0;
    cudaEvent_t done = nullptr;
    bool active = false;
  };
  std::vector<Area> areas;
  unsigned cur = 0;
  std::vector<uint16_t> exps;
  uint8_t* d_out = nullptr;
  size_t d_out_n = 0;
  bool has_output = false;
  uint8_t* d_out_ck = nullptr;    // the outputs' carried checksum blocks (16 B rows)
  int* d_valid = nullptr;         // per-output memory-checksum result
  std::vector<int> valid;         // its host copy, once checked
  bool checked = false;
  unsigned batches_started = 0;
  cudaStream_t s_copy = nullptr, s_comp = nullptr;
  cudaEvent_t copied = nullptr;
  uint8_t* d_hash = nullptr;  // IFSC entries of the staged inputs, by input number
  unsigned hash_cap = 0;
  // batches whose device work has finished: counted by a host function queued
  // behind each batch's kernels, waited for without touching CUDA
  std::mutex done_mu;
  std::condition_variable done_cv;
  unsigned batches_done = 0;
};

// host function queued on the compute stream after each batch (no CUDA calls)
static void CUDART_CB proc_batch_finished(void* arg) {
  auto* p = static_cast<pp_par2_proc*>(arg);
  {
    std::lock_guard<std::mutex> g(p->done_mu);
    p->batches_done++;
  }
  p->done_cv.notify_all();
}

// host slices of at least this many bytes are copied straight from the
// caller's buffer (one DMA beats a host memcpy into the pinned rows)
constexpr size_t kProcDirectBytes = 256 << 10;

// Staged rows and output rows: the slice rounded up to 16 bytes.  The memory
// checksum block of each row (the reference's packed staging appends one per
// slice, gf16/gf16_global.h:214-218) lives in a separate array of 16-byte
// rows that the same coefficients multiply in a second, small launch.
static size_t proc_row(size_t slice) { return round16(slice); }

static int proc_alloc_inputs(pp_par2_proc* p) {
  for (auto& a : p->areas) {
    if (a.d_in) cudaFree(a.d_in);
    if (a.d_ck) cudaFree(a.d_ck);
    if (a.h_in) cudaFreeHost(a.h_in);
    a.d_in = nullptr;
    a.d_ck = nullptr;
    a.h_in = nullptr;
    // pinned rows only for slices small enough to be staged (larger ones are
    // copied straight from the caller's buffer)
    if (cudaMalloc(&a.d_in, p->row * p->batch_alloc) != cudaSuccess ||
        cudaMalloc(&a.d_ck, (size_t)16 * p->batch_alloc) != cudaSuccess ||
        (p->row < kProcDirectBytes && cudaMallocHost(&a.h_in, p->row * p->batch_alloc) != cudaSuccess)) {
      cudaGetLastError();
      return PP_ERR_NO_MEMORY;
    }
    a.host_row.assign(p->batch_alloc, 0);
  }
  return PP_OK;
}

// Default batch: about 128 MiB of input per staging area (64-8192 slices),
// so one tensor-core launch covers many stages; set_recovery_slices lowers it
// so that an area's coefficient tiles stay within 256 MiB.
static unsigned proc_batch_for(const pp_par2_proc* p, size_t n_out) {
  size_t b = std::max<size_t>(64, std::min<size_t>(8192, (128u << 20) / p->row));
  if (n_out) b = std::min(b, std::max<size_t>(64, ((size_t)256 << 20) / (n_out * 256)));
  return (unsigned)std::min<size_t>(b, p->batch_alloc);
}

PP_API int pp_par2_proc_create(pp_ctx* ctx, size_t slice_size, unsigned staging_areas, unsigned input_batch,
                               pp_par2_proc** out) {
  if (!ctx || !out || slice_size == 0) return PP_ERR_INVALID_ARG;
  *out = nullptr;
  if (int r = bind(ctx)) return r;
  auto* p = new pp_par2_proc();
  p->ctx = ctx;
  p->alloc_size = p->cur_size = slice_size;
  p->row = proc_row(slice_size);
  p->n_areas = staging_areas ? staging_areas : 2;
  // A GPU batch amortises launch latency and the tensor-core pipeline fill
  if (input_batch) {
    p->batch = p->batch_alloc = input_batch;
    p->batch_fixed = true;
  } else {
    p->batch_alloc = std::max<unsigned>(64, std::min<size_t>(8192, (128u << 20) / p->row));
    p->batch = proc_batch_for(p, 0);
  }
  p->areas.resize(p->n_areas);
  if (cudaStreamCreateWithFlags(&p->s_copy, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&p->s_comp, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->copied, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    pp_par2_proc_destroy(p);
    return PP_ERR_CUDA;
  }
  for (auto& a : p->areas) {
    if (cudaEventCreateWithFlags(&a.done, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      pp_par2_proc_destroy(p);
      return PP_ERR_CUDA;
    }
  }
  if (proc_alloc_inputs(p) != PP_OK) {
    pp_par2_proc_destroy(p);
    return PP_ERR_NO_MEMORY;
  }
  *out = p;
  return PP_OK;
}

PP_API void pp_par2_proc_destroy(pp_par2_proc* p) {
  if (!p) return;
  bind(p->ctx);
  if (p->s_comp) cudaStreamSynchronize(p->s_comp);
  if (p->s_copy) cudaStreamSynchronize(p->s_copy);
  for (auto& a : p->areas) {
    if (a.d_in) cudaFree(a.d_in);
    if (a.d_ck) cudaFree(a.d_ck);
    if (a.h_in) cudaFreeHost(a.h_in);
    if (a.d_coeff) cudaFree(a.d_coeff);
    if (a.d_aexp) cudaFree(a.d_aexp);
    if (a.d_idx) cudaFree(a.d_idx);
    if (a.done) cudaEventDestroy(a.done);
  }
  if (p->d_hash) cudaFree(p->d_hash);
  if (p->d_out) cudaFree(p->d_out);
  if (p->d_out_ck) cudaFree(p->d_out_ck);
  if (p->d_valid) cudaFree(p->d_valid);
  if (p->copied) cudaEventDestroy(p->copied);
  if (p->s_copy) cudaStreamDestroy(p->s_copy);
  if (p->s_comp) cudaStreamDestroy(p->s_comp);
  delete p;
}

static bool area_busy(pp_par2_proc::Area& a) {
  if (!a.active) return false;
  cudaError_t e = cudaEventQuery(a.done);
  if (e == cudaSuccess) {
    a.active = false;
    return false;
  }
  if (e != cudaErrorNotReady) cudaGetLastError();
  return true;
}

PP_API int pp_par2_proc_set_current_slice_size(pp_par2_proc* p, size_t size) {
  if (!p || size == 0) return PP_ERR_INVALID_ARG;
  bind(p->ctx);
  if (size > p->alloc_size) {
    cudaStreamSynchronize(p->s_comp);
    p->alloc_size = size;
    p->row = proc_row(size);
    if (!p->batch_fixed) {  // larger rows: fewer of them (never more than the coefficient buffers hold)
      p->batch_alloc = std::max<unsigned>(64, std::min<size_t>(8192, (128u << 20) / p->row));
      p->batch = std::min(p->batch, proc_batch_for(p, p->exps.size()));
    }
    if (proc_alloc_inputs(p) != PP_OK) return set_err(p->ctx, PP_ERR_NO_MEMORY, "staging realloc");
    if (p->d_out) {
      cudaFree(p->d_out);
      p->d_out = nullptr;
      p->d_out_n = 0;
    }
  }
  p->cur_size = size;
  return PP_OK;
}

static int proc_ensure_out(pp_par2_proc* p) {
  size_t need = p->row * std::max<size_t>(1, p->exps.size());
  if (p->d_valid) cudaFree(p->d_valid);
  if (p->d_out_ck) cudaFree(p->d_out_ck);
  p->d_valid = nullptr;
  p->d_out_ck = nullptr;
  if (cudaMalloc(&p->d_valid, sizeof(int) * std::max<size_t>(1, p->exps.size())) != cudaSuccess ||
      cudaMalloc(&p->d_out_ck, (size_t)16 * std::max<size_t>(1, p->exps.size())) != cudaSuccess) {
    cudaGetLastError();
    return set_err(p->ctx, PP_ERR_NO_MEMORY, "checksum flags");
  }
  if (p->d_out_n >= need) return PP_OK;
  if (p->d_out) cudaFree(p->d_out);
  p->d_out = nullptr;
  if (cudaMalloc(&p->d_out, need) != cudaSuccess) {
    cudaGetLastError();
    p->d_out_n = 0;
    return set_err(p->ctx, PP_ERR_NO_MEMORY, "processing buffer");
  }
  p->d_out_n = need;
  return PP_OK;
}

PP_API int pp_par2_proc_set_recovery_slices(pp_par2_proc* p, unsigned num, const uint16_t* exps) {
  if (!p) return PP_ERR_INVALID_ARG;
  bind(p->ctx);
  cudaStreamSynchronize(p->s_comp);
  p->exps.assign(num, 1);  // default 1 (custom-coefficient use), as gf16/controller_cpu.cpp:176
  if (exps) memcpy(p->exps.data(), exps, num * 2);
  if (!p->batch_fixed) p->batch = proc_batch_for(p, num);
  for (auto& a : p->areas) {
    a.h_coeff.assign((size_t)num * p->batch, 0);
    if (a.d_coeff) cudaFree(a.d_coeff);
    a.d_coeff = nullptr;
    if (a.d_aexp) cudaFree(a.d_aexp);
    a.d_aexp = nullptr;
    if (num && cudaMalloc(&a.d_coeff, (size_t)num * p->batch * 2) != cudaSuccess) {
      cudaGetLastError();
      return set_err(p->ctx, PP_ERR_NO_MEMORY, "coefficient buffer");
    }
    if (num && cudaMalloc(&a.d_aexp, gf16_tc_coeff_bytes(p->batch, num)) != cudaSuccess) {
      cudaGetLastError();
      return set_err(p->ctx, PP_ERR_NO_MEMORY, "coefficient tiles");
    }
  }
  p->has_output = false;
  return num ? proc_ensure_out(p) : PP_OK;
}

PP_API int pp_par2_proc_can_add(pp_par2_proc* p) {
  if (!p) return PP_ERR_INVALID_ARG;
  bind(p->ctx);
  if (area_busy(p->areas[p->cur])) return PP_PROC_ADD_FULL;
  unsigned prev = (p->cur == 0 ? p->n_areas : p->cur) - 1;
  return area_busy(p->areas[prev]) ? PP_PROC_ADD_OK_BUSY : PP_PROC_ADD_OK;
}

PP_API int pp_par2_proc_wait_for_add(pp_par2_proc* p) {
  if (!p) return PP_ERR_INVALID_ARG;
  bind(p->ctx);
  auto& a = p->areas[p->cur];
  if (a.active) {
    CUDA_TRY(p->ctx, cudaEventSynchronize(a.done));
    a.active = false;
  }
  return PP_OK;
}

static int proc_submit(pp_par2_proc* p) {
  auto& a = p->areas[p->cur];
  if (!a.count) return PP_OK;
  const unsigned n_out = (unsigned)p->exps.size();
  // host-staged rows: one copy per run of consecutive rows
  for (unsigned i = 0; i < a.count;) {
    if (!a.host_row[i]) {
      i++;
      continue;
    }
    unsigned j = i;
    while (j < a.count && a.host_row[j]) a.host_row[j++] = 0;
    CUDA_TRY(p->ctx, cudaMemcpyAsync(a.d_in + (size_t)i * p->row, a.h_in + (size_t)i * p->row,
                                     (size_t)(j - i) * p->row, cudaMemcpyHostToDevice, p->s_copy));
    i = j;
  }
  // coefficient block [n_out][batch] (only the first `count` columns are used)
  CUDA_TRY(p->ctx, cudaMemcpyAsync(a.d_coeff, a.h_coeff.data(), (size_t)n_out * p->batch * 2,
                                   cudaMemcpyHostToDevice, p->s_copy));
  if (p->d_hash) {  // the rows' input numbers, for the IFSC entries
    if (a.d_idx_n < a.count) {
      CUDA_TRY(p->ctx, cudaStreamSynchronize(p->s_copy));
      if (a.d_idx) cudaFree(a.d_idx);
      a.d_idx = nullptr;
      a.d_idx_n = 0;
      if (cudaMalloc(&a.d_idx, sizeof(uint16_t) * p->batch_alloc) != cudaSuccess) {
        cudaGetLastError();
        return set_err(p->ctx, PP_ERR_NO_MEMORY, "hash index table");
      }
      a.d_idx_n = p->batch_alloc;
    }
    CUDA_TRY(p->ctx, cudaMemcpyAsync(a.d_idx, a.h_idx.data(), sizeof(uint16_t) * a.count, cudaMemcpyHostToDevice,
                                     p->s_copy));
  }
  CUDA_TRY(p->ctx, cudaEventRecord(p->copied, p->s_copy));
  CUDA_TRY(p->ctx, cudaStreamWaitEvent(p->s_comp, p->copied, 0));
  if (p->d_hash)
    CUDA_TRY(p->ctx, launch_par2_block_hash(a.d_in, p->row, a.count, p->cur_size, nullptr, p->d_hash, p->s_comp,
                                            a.d_idx));
  // each row's memory checksum, then the products of the data rows and of
  // the checksum rows (the second launch reuses the expanded coefficient tiles)
  // An odd slice's last word is (byte, 0); the product of that word has a
  // high byte too, which the checksum identity needs, so the internal rows
  // are multiplied and checksummed over whole words (the staged rows are
  // zero past the slice; getOutput copies out only the slice's bytes).
  const size_t len_w = (p->cur_size + 1) & ~(size_t)1;
  CUDA_TRY(p->ctx, launch_par2_cksum(a.d_in, p->row, a.count, len_w, a.d_ck, 16, nullptr, p->s_comp));
  CUDA_TRY(p->ctx, gf16_region(p->ctx->gf16_kernel, a.d_in, p->row, a.count, len_w, a.d_coeff, p->batch,
                               n_out, p->d_out, p->row, p->has_output, p->ctx->sms, a.d_aexp, p->ctx->d_status,
                               p->s_comp));
  CUDA_TRY(p->ctx, gf16_region(p->ctx->gf16_kernel, a.d_ck, 16, a.count, 16, a.d_coeff, p->batch, n_out,
                               p->d_out_ck, 16, p->has_output, p->ctx->sms, a.d_aexp, p->ctx->d_status, p->s_comp,
                               true));
  p->checked = false;
  CUDA_TRY(p->ctx, cudaEventRecord(a.done, p->s_comp));
  CUDA_TRY(p->ctx, cudaLaunchHostFunc(p->s_comp, proc_batch_finished, p));
  a.active = true;
  a.count = 0;
  p->has_output = true;
  p->batches_started++;
  p->cur = (p->cur + 1) % p->n_areas;
  return PP_OK;
}

static int proc_add(pp_par2_proc* p, const void* buf, size_t size, const uint16_t* coeffs, uint16_t input_num,
                    bool flush) {
  if (!buf && size) return PP_ERR_INVALID_ARG;
  if (p->exps.empty()) return set_err(p->ctx, PP_ERR_INVALID_ARG, "setRecoverySlices not called");
  if (size > p->cur_size) return set_err(p->ctx, PP_ERR_INVALID_ARG, "input larger than the current slice size");
  bind(p->ctx);
  auto& a = p->areas[p->cur];
  if (area_busy(a)) return set_err(p->ctx, PP_ERR_BUSY, "staging area busy");
  const unsigned n_out = (unsigned)p->exps.size();
  const unsigned idx = a.count;
  if (p->d_hash) {
    if (!coeffs && input_num >= p->hash_cap)
      return set_err(p->ctx, PP_ERR_INVALID_ARG, "input number %u beyond the %u-entry input hash table",
                     (unsigned)input_num, p->hash_cap);
    if (a.h_idx.size() < p->batch_alloc) a.h_idx.resize(p->batch_alloc);
    a.h_idx[idx] = coeffs ? (uint16_t)0xFFFF : input_num;  // decode inputs are not hashed
  }
  for (unsigned o = 0; o < n_out; o++)
    a.h_coeff[(size_t)o * p->batch + idx] = coeffs ? coeffs[o] : gf16h().coeff(input_num, p->exps[o]);
  if (size && (size >= kProcDirectBytes || !a.h_in || is_device_ptr(buf))) {
    // device input, or a large host slice (one DMA beats a host memcpy into
    // the pinned rows): copied into the area now, so that the caller may
    // reuse the buffer on return
    uint8_t* dst = a.d_in + (size_t)idx * p->row;
    CUDA_TRY(p->ctx, cudaMemcpyAsync(dst, buf, size, cudaMemcpyDefault, p->s_copy));
    if (size < p->row) CUDA_TRY(p->ctx, cudaMemsetAsync(dst + size, 0, p->row - size, p->s_copy));
    CUDA_TRY(p->ctx, cudaStreamSynchronize(p->s_copy));
    a.host_row[idx] = 0;
  } else {
    // host input: into the area's pinned rows; the whole batch goes to the
    // device in one copy at submit
    uint8_t* dst = a.h_in + (size_t)idx * p->row;
    if (size) memcpy(dst, buf, size);
    if (size < p->row) memset(dst + size, 0, p->row - size);
    a.host_row[idx] = 1;
  }
  a.count++;
  if (flush || a.count == p->batch) return proc_submit(p);
  return PP_OK;
}

PP_API int pp_par2_proc_add_input(pp_par2_proc* p, const void* buffer, size_t size, uint16_t input_num, int flush) {
  if (!p) return PP_ERR_INVALID_ARG;
  if (input_num >= 32768) return set_err(p->ctx, PP_ERR_INVALID_ARG, "input index >= 32768");
  return proc_add(p, buffer, size, nullptr, input_num, flush != 0);
}

PP_API int pp_par2_proc_add_input_coeffs(pp_par2_proc* p, const void* buffer, size_t size, const uint16_t* coeffs,
                                         int flush) {
  if (!p || !coeffs) return PP_ERR_INVALID_ARG;
  return proc_add(p, buffer, size, coeffs, 0, flush != 0);
}

PP_API int pp_par2_proc_flush(pp_par2_proc* p) {
  if (!p) return PP_ERR_INVALID_ARG;
  bind(p->ctx);
  return proc_submit(p);
}

PP_API int pp_par2_proc_end_input(pp_par2_proc* p) {
  if (!p) return PP_ERR_INVALID_ARG;
  bind(p->ctx);
  if (int r = proc_submit(p)) return r;
  CUDA_TRY(p->ctx, cudaStreamSynchronize(p->s_comp));
  for (auto& a : p->areas) a.active = false;
  return device_status(p->ctx);
}

PP_API int pp_par2_proc_get_output(pp_par2_proc* p, unsigned index, void* output, int* valid) {
  if (!p || !output) return PP_ERR_INVALID_ARG;
  if (index >= p->exps.size()) return set_err(p->ctx, PP_ERR_INVALID_ARG, "output index out of range");
  bind(p->ctx);
  if (valid) *valid = 0;
  CUDA_TRY(p->ctx, cudaStreamSynchronize(p->s_comp));
  const unsigned n_out = (unsigned)p->exps.size();
  if (!p->has_output) {
    // no input was added: the recovery data is all zero
    CUDA_TRY(p->ctx, cudaMemsetAsync(p->d_out + (size_t)index * p->row, 0, p->cur_size, p->s_copy));
  } else if (!p->checked) {
    // verify every output's carried checksum against its data once
    // (finish_packed_cksum, gf16/controller_cpu.cpp:423-443)
    CUDA_TRY(p->ctx, launch_par2_cksum(p->d_out, p->row, n_out, (p->cur_size + 1) & ~(size_t)1, p->d_out_ck, 16,
                                       p->d_valid, p->s_copy));
    p->valid.assign(n_out, 0);
    CUDA_TRY(p->ctx, cudaMemcpyAsync(p->valid.data(), p->d_valid, sizeof(int) * n_out, cudaMemcpyDeviceToHost,
                                     p->s_copy));
    p->checked = true;
  }
  CUDA_TRY(p->ctx, cudaMemcpyAsync(output, p->d_out + (size_t)index * p->row, p->cur_size, cudaMemcpyDefault,
                                   p->s_copy));
  CUDA_TRY(p->ctx, cudaStreamSynchronize(p->s_copy));
  if (valid) *valid = p->has_output ? p->valid[index] : 1;
  return PP_OK;
}

PP_API unsigned pp_par2_proc_batches_done(pp_par2_proc* p) {
  if (!p) return 0;
  std::lock_guard<std::mutex> g(p->done_mu);
  return p->batches_done;
}

PP_API int pp_par2_proc_wait_batches(pp_par2_proc* p, unsigned count) {
  if (!p) return PP_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> g(p->done_mu);
  // bounded: a batch that has not finished within a minute is reported, not waited for
  if (!p->done_cv.wait_for(g, std::chrono::seconds(60), [&] { return p->batches_done >= count; }))
    return PP_ERR_TIMEOUT;
  return PP_OK;
}

PP_API int pp_par2_proc_output_ptr(pp_par2_proc* p, unsigned index, void** dev_ptr) {
  if (!p || !dev_ptr) return PP_ERR_INVALID_ARG;
  *dev_ptr = nullptr;
  if (index >= p->exps.size()) return set_err(p->ctx, PP_ERR_INVALID_ARG, "output index out of range");
  if (!p->d_out) return set_err(p->ctx, PP_ERR_INVALID_ARG, "no output area");
  *dev_ptr = p->d_out + (size_t)index * p->row;
  return PP_OK;
}

PP_API int pp_par2_proc_set_input_hashes(pp_par2_proc* p, unsigned max_inputs) {
  if (!p) return PP_ERR_INVALID_ARG;
  if (max_inputs > 32768) return set_err(p->ctx, PP_ERR_INVALID_ARG, "max_inputs > 32768");
  bind(p->ctx);
  CUDA_TRY(p->ctx, cudaStreamSynchronize(p->s_comp));
  if (p->d_hash) cudaFree(p->d_hash);
  p->d_hash = nullptr;
  p->hash_cap = 0;
  if (!max_inputs) return PP_OK;
  if (cudaMalloc(&p->d_hash, (size_t)20 * max_inputs) != cudaSuccess) {
    cudaGetLastError();
    return set_err(p->ctx, PP_ERR_NO_MEMORY, "input hash table");
  }
  CUDA_TRY(p->ctx, cudaMemset(p->d_hash, 0, (size_t)20 * max_inputs));
  p->hash_cap = max_inputs;
  // rows already staged in the open batch were added without an entry
  auto& a = p->areas[p->cur];
  if (a.h_idx.size() < p->batch_alloc) a.h_idx.resize(p->batch_alloc);
  for (unsigned i = 0; i < a.count; i++) a.h_idx[i] = 0xFFFF;
  return PP_OK;
}

PP_API int pp_par2_proc_get_input_hashes(pp_par2_proc* p, uint8_t* out, unsigned count) {
  if (!p || (count && !out)) return PP_ERR_INVALID_ARG;
  if (!p->d_hash) return set_err(p->ctx, PP_ERR_INVALID_ARG, "input hashing is not enabled");
  if (count > p->hash_cap) return set_err(p->ctx, PP_ERR_INVALID_ARG, "count beyond the input hash table");
  bind(p->ctx);
  CUDA_TRY(p->ctx, cudaStreamSynchronize(p->s_comp));
  CUDA_TRY(p->ctx, cudaMemcpy(out, p->d_hash, (size_t)20 * count, cudaMemcpyDefault));
  return device_status(p->ctx);
}

PP_API int pp_par2_proc_discard_output(pp_par2_proc* p) {
  if (!p) return PP_ERR_INVALID_ARG;
  p->has_output = false;
  return PP_OK;
}

PP_API int pp_par2_proc_free_processing_mem(pp_par2_proc* p) {
  if (!p) return PP_ERR_INVALID_ARG;
  bind(p->ctx);
  cudaStreamSynchronize(p->s_comp);
  if (p->d_out) cudaFree(p->d_out);
  p->d_out = nullptr;
  p->d_out_n = 0;
  p->has_output = false;
  return PP_OK;
}

PP_API unsigned pp_par2_proc_input_batch_size(pp_par2_proc* p) { return p ? p->batch : 0; }
PP_API unsigned pp_par2_proc_batches_started(pp_par2_proc* p) { return p ? p->batches_started : 0; }

// ============================================================ PAR3 / GF64
static uint64_t* cauchy_get(pp_ctx* ctx, size_t n_in, size_t n_rec, uint64_t fI, uint64_t fR, int* st) {
  *st = PP_OK;
  for (auto it = ctx->cauchy.begin(); it != ctx->cauchy.end(); ++it) {
    if (it->n_in == n_in && it->n_rec == n_rec && it->fI == fI && it->fR == fR) {
      ctx->cauchy.splice(ctx->cauchy.begin(), ctx->cauchy, it);
      return ctx->cauchy.front().d;
    }
  }
  // LRU within kCauchyEntries / kCauchyBytes; matrices come from the
  // context's pool, an evicted one is freed in the stream's order (after
  // every kernel that read it)
  const size_t need = n_in * n_rec * 8;
  size_t total = need;
  for (auto& e : ctx->cauchy) total += e.bytes;
  while (!ctx->cauchy.empty() && (ctx->cauchy.size() >= kCauchyEntries || total > kCauchyBytes)) {
    total -= ctx->cauchy.back().bytes;
    pool_free(ctx, ctx->cauchy.back().d);
    ctx->cauchy.pop_back();
  }
  PP_TRACE("cauchy-alloc", need);
  void* d = pool_alloc(ctx, need);
  if (!d) {
    // make room: drop every cached matrix and retry once
    for (auto& e : ctx->cauchy) pool_free(ctx, e.d);
    ctx->cauchy.clear();
    d = pool_alloc(ctx, need);
    if (!d) {
      *st = set_err(ctx, PP_ERR_NO_MEMORY, "Cauchy matrix %zu x %zu", n_rec, n_in);
      return nullptr;
    }
  }
  cudaError_t e = launch_gf64_cauchy((uint64_t*)d, n_in, n_rec, fI, fR, n_in, ctx->stream);
  if (e != cudaSuccess) {
    pool_free(ctx, d);
    *st = set_err(ctx, PP_ERR_CUDA, "Cauchy build: %s", cudaGetErrorString(e));
    return nullptr;
  }
  ctx->cauchy.push_front({n_in, n_rec, fI, fR, (uint64_t*)d, need});
  return (uint64_t*)d;
}

PP_API int pp_gf64_build_cauchy(pp_ctx* ctx, uint64_t* coeff, size_t num_inputs, size_t num_recovery,
                                uint64_t first_input, uint64_t first_recovery) {
  if (!ctx || !coeff) return PP_ERR_INVALID_ARG;
  if (!num_inputs || !num_recovery) return PP_OK;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  if (is_device_ptr(coeff)) {
    CUDA_TRY(ctx, launch_gf64_cauchy(coeff, num_inputs, num_recovery, first_input, first_recovery, num_inputs,
                                     ctx->stream));
    return PP_OK;
  }
  uint64_t* d = (uint64_t*)scratch(ctx, S_COEF, num_inputs * num_recovery * 8);
  if (!d) return set_err(ctx, PP_ERR_NO_MEMORY, "Cauchy matrix");
  CUDA_TRY(ctx, launch_gf64_cauchy(d, num_inputs, num_recovery, first_input, first_recovery, num_inputs,
                                   ctx->stream));
  CUDA_TRY(ctx, cudaMemcpyAsync(coeff, d, num_inputs * num_recovery * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

// GF(2^64) region dispatch.  The tensor-core kernel copies rows with 16-byte
// bulk copies, so it needs 16-byte aligned rows and an even word count;
// otherwise (or when the lookup kernel is selected) the lookup kernel runs.
static bool aligned_rows64(const uint64_t* base, size_t stride) {
  return ((uintptr_t)base % 16) == 0 && (stride % 2) == 0;
}
static cudaError_t gf64_region(pp_ctx* ctx, const uint64_t* din, const uint64_t* const* d_in_ptrs, size_t in_stride,
                               size_t n_in, size_t words, const uint64_t* d_coeff, size_t ldc, size_t n_out,
                               uint64_t* dout, uint64_t* const* d_out_ptrs, size_t out_stride, bool accumulate,
                               bool rows_aligned) {
  const bool tc_ok = rows_aligned && (words % 2) == 0 && n_in >= 2;
  const bool tc = ctx->gf64_kernel == PP_GF16_KERNEL_TENSOR ? tc_ok
                  : ctx->gf64_kernel == PP_GF16_KERNEL_LUT   ? false
                                                             : tc_ok;
  if (tc)
    return launch_gf64_matvec_tc(din, d_in_ptrs, in_stride, n_in, words, d_coeff, ldc, n_out, dout, d_out_ptrs,
                                 out_stride, accumulate, ctx->sms, ctx->d_status, ctx->stream);
  if (d_in_ptrs || d_out_ptrs)
    return launch_gf64_2d_gather(d_out_ptrs, n_out, d_in_ptrs, n_in, d_coeff, ldc, words, ctx->sms, ctx->stream);
  return launch_gf64_matvec(din, in_stride, n_in, words, d_coeff, ldc, n_out, dout, out_stride, accumulate, ctx->sms,
                            ctx->stream);
}

// hj: optional BLAKE3 block-hash job over the input blocks (prefix fields and
// hash_out for block 0 set; data, n and the offsets are filled per staged
// chunk), run on the hash stream beside the products; hcv = its chaining-value
// scratch, sized for the whole input.  The hash work is joined into the
// context's stream before return.
// in_ld / out_ld: row strides of the caller's blocks in words (0 = B, the
// reference's contiguous layout); a word range of every block is a view with
// the full block length as its stride.
static int gf64_matvec_impl(pp_ctx* ctx, const uint64_t* inputs, size_t n_in, uint64_t* recovery, size_t n_rec,
                            size_t B, const uint64_t* d_coeff, bool accumulate, const B3Job* hj = nullptr,
                            uint32_t* hcv = nullptr, size_t in_ld = 0, size_t out_ld = 0) {
  if (!in_ld) in_ld = B;
  if (!out_ld) out_ld = B;
  if (hj && in_ld != B) return set_err(ctx, PP_ERR_INVALID_ARG, "block hashes need whole blocks");
  const bool in_dev = is_device_ptr(inputs);
  const bool out_dev = is_device_ptr(recovery);
  const uint64_t* din = inputs;
  // host <-> staging copies of [rows, B words] views with the caller's strides
  auto h2d_rows = [&](uint64_t* dst, const uint64_t* src, size_t ld, size_t rows, cudaStream_t st) {
    return ld == B ? cudaMemcpyAsync(dst, src, rows * B * 8, cudaMemcpyHostToDevice, st)
                   : cudaMemcpy2DAsync(dst, B * 8, src, ld * 8, B * 8, rows, cudaMemcpyHostToDevice, st);
  };
  auto d2h_rows = [&](uint64_t* dst, size_t ld, const uint64_t* src, size_t rows, cudaStream_t st) {
    return ld == B ? cudaMemcpyAsync(dst, src, rows * B * 8, cudaMemcpyDeviceToHost, st)
                   : cudaMemcpy2DAsync(dst, ld * 8, src, B * 8, B * 8, rows, cudaMemcpyDeviceToHost, st);
  };
  if (hj)
    if (int r = ensure_hash_stream(ctx)) return r;
  auto hash_rows = [&](const uint64_t* rows, size_t first, size_t count) -> cudaError_t {
    B3Job J = *hj;
    J.data = (const uint8_t*)rows;
    J.stride = B * 8;
    J.D = B * 8;
    J.n = count;
    J.first_index = hj->first_index + first;
    J.hash_out = hj->hash_out + first * hj->hash_stride;
    return launch_blake3_blocks(J, hcv, ctx->hash);
  };
  auto join_hash = [&]() -> int {
    if (!hj) return PP_OK;
    CUDA_TRY(ctx, cudaEventRecord(ctx->hash_ev, ctx->hash));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->hash_ev, 0));
    return PP_OK;
  };
  const size_t chunk = std::max<size_t>(1024, (64u << 20) / (B * 8));  // input blocks per ~64 MiB copy
  if (!in_dev && n_in >= 2 * chunk) {
    // ---- chunked: the copy of chunk c+1 overlaps the product of chunk c
    // (each chunk's product accumulates into the outputs after the first)
    if (int r = ensure_copy_stream(ctx)) return r;
    uint64_t* s = (uint64_t*)scratch(ctx, S_IN, n_in * B * 8);
    if (!s) return set_err(ctx, PP_ERR_NO_MEMORY, "input staging (%zu bytes)", n_in * B * 8);
    uint64_t* dout = recovery;
    size_t dout_ld = out_ld;
    if (!out_dev) {
      dout = (uint64_t*)scratch(ctx, S_OUT, n_rec * B * 8);
      if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "output staging");
      dout_ld = B;
      if (accumulate) CUDA_TRY(ctx, h2d_rows(dout, recovery, out_ld, n_rec, ctx->stream));
    }
    CUDA_TRY(ctx, cudaEventRecord(ctx->start_ev, ctx->stream));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy, ctx->start_ev, 0));
    const size_t tail = std::max<size_t>(2, chunk / 16);
    for (size_t c0 = 0, nc = 0; c0 < n_in; c0 += nc) {
      // the last chunk goes in halving pieces (down to chunk / 16 blocks), so
      // little product work is left once the final copy has landed
      const size_t rest = n_in - c0;
      nc = rest > chunk ? chunk : rest > tail ? std::max(tail, (rest / 2 + 1) & ~(size_t)1) : rest;
      CUDA_TRY(ctx, h2d_rows(s + c0 * B, inputs + c0 * in_ld, in_ld, nc, ctx->copy));
      CUDA_TRY(ctx, cudaEventRecord(ctx->copy_ev, ctx->copy));
      CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->copy_ev, 0));
      if (hj) {
        CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->hash, ctx->copy_ev, 0));
        CUDA_TRY(ctx, hash_rows(s + c0 * B, c0, nc));
      }
      CUDA_TRY(ctx, gf64_region(ctx, s + c0 * B, nullptr, B, nc, B, d_coeff + c0, n_in, n_rec, dout, nullptr, dout_ld,
                                accumulate || c0 > 0, aligned_rows64(s, B) && aligned_rows64(dout, dout_ld)));
    }
    if (!out_dev) CUDA_TRY(ctx, d2h_rows(recovery, out_ld, dout, n_rec, ctx->stream));
    if (int r = join_hash()) return r;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return device_status(ctx);
  }
  size_t din_ld = in_ld;
  if (!in_dev) {
    uint64_t* s = (uint64_t*)scratch(ctx, S_IN, n_in * B * 8);
    if (!s) return set_err(ctx, PP_ERR_NO_MEMORY, "input staging (%zu bytes)", n_in * B * 8);
    CUDA_TRY(ctx, h2d_rows(s, inputs, in_ld, n_in, ctx->stream));
    din = s;
    din_ld = B;
  }
  if (hj) {  // hash the device rows beside the product
    CUDA_TRY(ctx, cudaEventRecord(ctx->staged_ev, ctx->stream));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->hash, ctx->staged_ev, 0));
    CUDA_TRY(ctx, hash_rows(din, 0, n_in));
  }
  uint64_t* dout = recovery;
  size_t dout_ld = out_ld;
  if (!out_dev) {
    dout = (uint64_t*)scratch(ctx, S_OUT, n_rec * B * 8);
    if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "output staging");
    dout_ld = B;
    if (accumulate) CUDA_TRY(ctx, h2d_rows(dout, recovery, out_ld, n_rec, ctx->stream));
  }
  auto* tev = timing_begin(ctx);
  CUDA_TRY(ctx, gf64_region(ctx, din, nullptr, din_ld, n_in, B, d_coeff, n_in, n_rec, dout, nullptr, dout_ld,
                            accumulate, aligned_rows64(din, din_ld) && aligned_rows64(dout, dout_ld)));
  timing_end(ctx, tev);
  if (!out_dev) CUDA_TRY(ctx, d2h_rows(recovery, out_ld, dout, n_rec, ctx->stream));
  if (int r = join_hash()) return r;
  if (!in_dev || !out_dev) {
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return device_status(ctx);
  }
  return PP_OK;
}

PP_API int pp_gf64_compute_recovery(pp_ctx* ctx, const uint64_t* inputs, size_t num_inputs, uint64_t* recovery,
                                    size_t num_recovery, size_t block_size64, uint64_t first_input,
                                    uint64_t first_recovery, int accumulate, int kernel) {
  PP_TRACE("call-gf64_compute_recovery", 0);
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (num_inputs == 0 || num_recovery == 0 || block_size64 == 0) return PP_OK;
  if (!inputs || !recovery) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if (kernel < PP_GF64_KERNEL_AUTO || kernel > PP_GF64_KERNEL_FENGER)
    return set_err(ctx, PP_ERR_INVALID_ARG, "unknown kernel %d", kernel);
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  int st;
  uint64_t* M = cauchy_get(ctx, num_inputs, num_recovery, first_input, first_recovery, &st);
  if (!M) return st;
  return gf64_matvec_impl(ctx, inputs, num_inputs, recovery, num_recovery, block_size64, M, accumulate != 0);
}

PP_API int pp_gf64_compute_recovery_with_coeff(pp_ctx* ctx, const uint64_t* inputs, size_t num_inputs,
                                               uint64_t* recovery, size_t num_recovery, size_t block_size64,
                                               const uint64_t* coeff, int accumulate) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (num_inputs == 0 || num_recovery == 0 || block_size64 == 0) return PP_OK;
  if (!inputs || !recovery || !coeff) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  int st;
  const uint64_t* dc = to_device(ctx, S_COEF, coeff, num_inputs * num_recovery, &st);
  if (st) return st;
  return gf64_matvec_impl(ctx, inputs, num_inputs, recovery, num_recovery, block_size64, dc, accumulate != 0);
}

PP_API int pp_gf64_solve_and_reconstruct(pp_ctx* ctx, uint64_t* A, uint64_t* rhs, size_t n, size_t B) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (n == 0) return PP_OK;
  if (!A || (!rhs && B)) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const bool a_dev = is_device_ptr(A), r_dev = rhs ? is_device_ptr(rhs) : true;
  uint64_t* dA = A;
  uint64_t* dR = rhs;
  if (!a_dev) {
    dA = (uint64_t*)scratch(ctx, S_D, n * n * 8);
    if (!dA) return set_err(ctx, PP_ERR_NO_MEMORY, "solve matrix");
    CUDA_TRY(ctx, cudaMemcpyAsync(dA, A, n * n * 8, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (!r_dev) {
    dR = (uint64_t*)scratch(ctx, S_IN, n * B * 8);
    if (!dR) return set_err(ctx, PP_ERR_NO_MEMORY, "solve rhs");
    CUDA_TRY(ctx, cudaMemcpyAsync(dR, rhs, n * B * 8, cudaMemcpyHostToDevice, ctx->stream));
  }
  uint64_t* dF = (uint64_t*)scratch(ctx, S_E, (n + 2) * 8 + 64);
  if (!dF) return set_err(ctx, PP_ERR_NO_MEMORY, "solve scratch");
  int* dS = (int*)(dF + n + 2);
  CUDA_TRY(ctx, cudaMemsetAsync(dS, 0, sizeof(int), ctx->stream));
  CUDA_TRY(ctx, launch_gf64_solve(dA, dR, n, B, dF, dS, ctx->stream));
  int hs = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&hs, dS, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  if (!a_dev) CUDA_TRY(ctx, cudaMemcpyAsync(A, dA, n * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (!r_dev) CUDA_TRY(ctx, cudaMemcpyAsync(rhs, dR, n * B * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (hs != 0) return set_err(ctx, PP_ERR_SINGULAR, "matrix is singular");
  return PP_OK;
}

// element-wise region ops ---------------------------------------------------
static int region_elem(pp_ctx* ctx, uint64_t* out, const uint64_t* in, const uint64_t* coeff, size_t len,
                       size_t n_coeff, bool add) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!len) return PP_OK;
  if (!out || !in || !coeff || !n_coeff) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const bool in_dev = is_device_ptr(in), out_dev = is_device_ptr(out);
  int st;
  const uint64_t* dc = to_device(ctx, S_COEF, coeff, n_coeff, &st);
  if (st) return st;
  const uint64_t* din = in;
  if (!in_dev) {
    uint64_t* s = (uint64_t*)scratch(ctx, S_IN, len * 8);
    if (!s) return set_err(ctx, PP_ERR_NO_MEMORY, "staging");
    CUDA_TRY(ctx, cudaMemcpyAsync(s, in, len * 8, cudaMemcpyHostToDevice, ctx->stream));
    din = s;
  }
  uint64_t* dout = out;
  if (!out_dev) {
    dout = (uint64_t*)scratch(ctx, S_OUT, len * 8);
    if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "staging");
    if (add) CUDA_TRY(ctx, cudaMemcpyAsync(dout, out, len * 8, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (add)
    CUDA_TRY(ctx, launch_gf64_region_muladd_arr(dout, din, dc, len, n_coeff, ctx->stream));
  else
    CUDA_TRY(ctx, launch_gf64_region_mul_arr(dout, din, dc, len, n_coeff, ctx->stream));
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(out, dout, len * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (!in_dev || !out_dev || !is_device_ptr(coeff)) CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

PP_API int pp_gf64_region_mul(pp_ctx* ctx, uint64_t* out, const uint64_t* in, size_t len, uint64_t constant) {
  return region_elem(ctx, out, in, &constant, len, 1, false);
}
PP_API int pp_gf64_region_mul_arr(pp_ctx* ctx, uint64_t* out, const uint64_t* in, const uint64_t* coeff, size_t len,
                                  size_t n_coeff) {
  return region_elem(ctx, out, in, coeff, len, n_coeff, false);
}
PP_API int pp_gf64_region_muladd_arr(pp_ctx* ctx, uint64_t* out, const uint64_t* in, const uint64_t* coeff,
                                     size_t len, size_t n_coeff) {
  return region_elem(ctx, out, in, coeff, len, n_coeff, true);
}

// 2-D gather form: all three pointer-table entry points reduce to
//   outs[k][w] ^= XOR_g ins[g][w] * C[k][g]
static int region_2d(pp_ctx* ctx, uint64_t* const* outs, size_t K, const uint64_t* const* ins, size_t G,
                     const std::vector<uint64_t>& C, size_t len) {
  if (!K || !G || !len) return PP_OK;
  bool all_dev = true;
  for (size_t k = 0; k < K && all_dev; k++) all_dev = is_device_ptr(outs[k]);
  for (size_t g = 0; g < G && all_dev; g++) all_dev = is_device_ptr(ins[g]);
  int st;
  const uint64_t* dC = to_device(ctx, S_COEF, C.data(), C.size(), &st);
  if (st) return st;
  std::vector<const uint64_t*> din(G);
  std::vector<uint64_t*> dout(K);
  uint64_t *sin = nullptr, *sout = nullptr;
  if (all_dev) {
    for (size_t g = 0; g < G; g++) din[g] = ins[g];
    for (size_t k = 0; k < K; k++) dout[k] = outs[k];
  } else {
    sin = (uint64_t*)scratch(ctx, S_IN, G * len * 8);
    sout = (uint64_t*)scratch(ctx, S_OUT, K * len * 8);
    if (!sin || !sout) return set_err(ctx, PP_ERR_NO_MEMORY, "staging");
    for (size_t g = 0; g < G; g++) {
      CUDA_TRY(ctx, cudaMemcpyAsync(sin + g * len, ins[g], len * 8, cudaMemcpyDefault, ctx->stream));
      din[g] = sin + g * len;
    }
    for (size_t k = 0; k < K; k++) {
      CUDA_TRY(ctx, cudaMemcpyAsync(sout + k * len, outs[k], len * 8, cudaMemcpyDefault, ctx->stream));
      dout[k] = sout + k * len;
    }
  }
  const uint64_t* const* dpin = to_device(ctx, S_A, din.data(), G, &st);
  if (st) return st;
  uint64_t* const* dpout = (uint64_t* const*)to_device(ctx, S_B, (const uint64_t* const*)dout.data(), K, &st);
  if (st) return st;
  bool al = (len % 2) == 0;
  for (size_t g2 = 0; g2 < G && al; g2++) al = ((uintptr_t)din[g2] % 16) == 0;
  for (size_t k = 0; k < K && al; k++) al = ((uintptr_t)dout[k] % 16) == 0;
  CUDA_TRY(ctx, gf64_region(ctx, nullptr, dpin, 0, G, len, dC, G, K, nullptr, dpout, 0, true, al));
  if (!all_dev) {
    for (size_t k = 0; k < K; k++)
      CUDA_TRY(ctx, cudaMemcpyAsync(outs[k], sout + k * len, len * 8, cudaMemcpyDefault, ctx->stream));
  }
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return device_status(ctx);
}

PP_API int pp_gf64_region_coupled_muladd_arr(pp_ctx* ctx, uint64_t* out, const uint64_t* const* in_blocks,
                                             const uint64_t* coeff_blocks, size_t len, size_t G) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!G || !len) return PP_OK;
  if (!out || !in_blocks || !coeff_blocks) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  std::vector<uint64_t> C(G);
  if (is_device_ptr(coeff_blocks))
    CUDA_TRY(ctx, cudaMemcpy(C.data(), coeff_blocks, G * 8, cudaMemcpyDeviceToHost));
  else
    memcpy(C.data(), coeff_blocks, G * 8);
  uint64_t* outs[1] = {out};
  return region_2d(ctx, outs, 1, in_blocks, G, C, len);
}

PP_API int pp_gf64_region_fused_output_muladd_arr(pp_ctx* ctx, uint64_t* const* outs, const uint64_t* in,
                                                  const uint64_t* const* coeff_block_starts, size_t len, size_t K) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!K || !len) return PP_OK;
  if (!outs || !in || !coeff_block_starts) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  std::vector<uint64_t> C(K);
  for (size_t k = 0; k < K; k++) {
    if (is_device_ptr(coeff_block_starts[k]))
      CUDA_TRY(ctx, cudaMemcpy(&C[k], coeff_block_starts[k], 8, cudaMemcpyDeviceToHost));
    else
      C[k] = coeff_block_starts[k][0];
  }
  const uint64_t* ins[1] = {in};
  return region_2d(ctx, outs, K, ins, 1, C, len);
}

PP_API int pp_gf64_region_2d_muladd_arr(pp_ctx* ctx, uint64_t* const* outs, size_t K, const uint64_t* const* in_blocks,
                                        size_t G, const uint64_t* coeff_block_2d, size_t K_stride, size_t len) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!K || !G || !len) return PP_OK;
  if (!outs || !in_blocks || !coeff_block_2d || K_stride < G)
    return set_err(ctx, PP_ERR_INVALID_ARG, "bad arguments");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  std::vector<uint64_t> C(K * G);
  std::vector<uint64_t> raw((K - 1) * K_stride + G);
  if (is_device_ptr(coeff_block_2d))
    CUDA_TRY(ctx, cudaMemcpy(raw.data(), coeff_block_2d, raw.size() * 8, cudaMemcpyDeviceToHost));
  else
    memcpy(raw.data(), coeff_block_2d, raw.size() * 8);
  for (size_t k = 0; k < K; k++)
    for (size_t gg = 0; gg < G; gg++) C[k * G + gg] = raw[k * K_stride + gg];
  return region_2d(ctx, outs, K, in_blocks, G, C, len);
}

PP_API int pp_gf64_inverse_batch(pp_ctx* ctx, uint64_t* out, const uint64_t* in, size_t n) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!n) return PP_OK;
  if (!out || !in) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const bool in_dev = is_device_ptr(in), out_dev = is_device_ptr(out);
  const uint64_t* din = in;
  if (!in_dev) {
    uint64_t* s = (uint64_t*)scratch(ctx, S_IN, n * 8);
    if (!s) return set_err(ctx, PP_ERR_NO_MEMORY, "staging");
    CUDA_TRY(ctx, cudaMemcpyAsync(s, in, n * 8, cudaMemcpyHostToDevice, ctx->stream));
    din = s;
  }
  uint64_t* dout = out_dev ? out : (uint64_t*)scratch(ctx, S_OUT, n * 8);
  if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "staging");
  CUDA_TRY(ctx, launch_gf64_inverse_batch(dout, din, n, ctx->stream));
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(out, dout, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (!in_dev || !out_dev) CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

static int gf64_fft_common(pp_ctx* ctx, uint64_t* data, size_t n, size_t batch, size_t ld, bool inverse) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (n <= 1 || batch == 0) return PP_OK;
  if (!data) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if ((n & (n - 1)) != 0 || n > ((size_t)1 << 20))
    return set_err(ctx, PP_ERR_INVALID_ARG, "n must be a power of two <= 2^20");
  if (ld < batch) return set_err(ctx, PP_ERR_INVALID_ARG, "ld < batch");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const bool dev = is_device_ptr(data);
  uint64_t* d = data;
  size_t dld = ld;
  if (!dev) {
    dld = batch;
    d = (uint64_t*)scratch(ctx, S_IN, n * batch * 8);
    if (!d) return set_err(ctx, PP_ERR_NO_MEMORY, "fft staging");
    CUDA_TRY(ctx, cudaMemcpy2DAsync(d, dld * 8, data, ld * 8, batch * 8, n, cudaMemcpyHostToDevice, ctx->stream));
  }
  CUDA_TRY(ctx, launch_gf64_fft(d, n, batch, dld, inverse, ctx->stream));
  if (!dev) {
    CUDA_TRY(ctx, cudaMemcpy2DAsync(data, ld * 8, d, dld * 8, batch * 8, n, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return PP_OK;
}

PP_API int pp_gf64_fft_fwd(pp_ctx* ctx, uint64_t* data, size_t n, size_t batch, size_t ld) {
  return gf64_fft_common(ctx, data, n, batch, ld, false);
}
PP_API int pp_gf64_fft_inv(pp_ctx* ctx, uint64_t* data, size_t n, size_t batch, size_t ld) {
  return gf64_fft_common(ctx, data, n, batch, ld, true);
}

PP_API int pp_gf64_repair(pp_ctx* ctx, const uint64_t* inputs, size_t num_inputs, const uint64_t* missing, size_t n,
                          const uint64_t* recovery, const uint8_t* recovery_present, size_t B, uint64_t first_input,
                          uint64_t first_recovery, uint64_t* restored) {
  PP_TRACE("call-gf64_repair", 0);
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (n == 0 || B == 0) return PP_OK;
  if (!inputs || !missing || !recovery || !restored) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if (n > num_inputs) return set_err(ctx, PP_ERR_INVALID_ARG, "more lost blocks than inputs");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  // host bookkeeping: lost-block set and the per-input row pointers
  std::vector<uint64_t> miss(n);
  if (is_device_ptr(missing))
    CUDA_TRY(ctx, cudaMemcpy(miss.data(), missing, n * 8, cudaMemcpyDeviceToHost));
  else
    memcpy(miss.data(), missing, n * 8);
  std::vector<uint8_t> lost(num_inputs, 0);
  // the system is a true Cauchy matrix (closed-form inverse) unless some lost
  // column id fI + c equals a row id fR + j, whose entry the reference maps to 1
  bool cauchy = true;
  for (size_t c = 0; c < n; c++) {
    if (miss[c] >= num_inputs || lost[miss[c]]) return set_err(ctx, PP_ERR_INVALID_ARG, "bad missing index list");
    lost[miss[c]] = 1;
    if (first_input + miss[c] - first_recovery < n) cauchy = false;
  }
  const bool in_dev = is_device_ptr(inputs), out_dev = is_device_ptr(restored), rec_dev = is_device_ptr(recovery);
  const uint64_t* din = inputs;
  if (!in_dev) {
    uint64_t* st = (uint64_t*)scratch(ctx, S_IN, num_inputs * B * 8);
    if (!st) return set_err(ctx, PP_ERR_NO_MEMORY, "input staging");
    CUDA_TRY(ctx, cudaMemcpyAsync(st, inputs, num_inputs * B * 8, cudaMemcpyHostToDevice, ctx->stream));
    din = st;
  }
  // rhs = recovery rows (absent rows zero), then the known-input sum.  With
  // the closed-form inverse the rhs is kept apart from the restored blocks.
  uint64_t* rhs = (out_dev && !cauchy) ? restored : (uint64_t*)scratch(ctx, S_OUT, n * B * 8);
  uint64_t* zero = (uint64_t*)scratch(ctx, S_C, B * 8);
  uint64_t* dA = (uint64_t*)scratch(ctx, S_D, (cauchy ? 2 * n * n + 3 * n : n * n + n) * 8);
  uint64_t* dF = (uint64_t*)scratch(ctx, S_E, (n + 2) * 8 + 64);
  if (!rhs || !zero || !dA || !dF) return set_err(ctx, PP_ERR_NO_MEMORY, "repair buffers");
  uint64_t* dcols = dA + n * n;
  CUDA_TRY(ctx, cudaMemsetAsync(zero, 0, B * 8, ctx->stream));
  CUDA_TRY(ctx, cudaMemcpyAsync(rhs, recovery, n * B * 8, rec_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                ctx->stream));
  if (recovery_present) {
    for (size_t eq = 0; eq < n; eq++)
      if (!recovery_present[eq]) CUDA_TRY(ctx, cudaMemsetAsync(rhs + eq * B, 0, B * 8, ctx->stream));
  }
  int st;
  uint64_t* M = cauchy_get(ctx, num_inputs, n, first_input, first_recovery, &st);
  if (!M) return st;
  std::vector<const uint64_t*> in_ptrs(num_inputs);
  for (size_t k = 0; k < num_inputs; k++) in_ptrs[k] = lost[k] ? zero : din + k * B;
  std::vector<uint64_t*> out_ptrs(n);
  for (size_t eq = 0; eq < n; eq++) out_ptrs[eq] = rhs + eq * B;
  const uint64_t* const* dpin = to_device(ctx, S_A, in_ptrs.data(), num_inputs, &st);
  if (st) return st;
  uint64_t* const* dpout = (uint64_t* const*)to_device(ctx, S_B, (const uint64_t* const*)out_ptrs.data(), n, &st);
  if (st) return st;
  bool al = (B % 2) == 0 && ((uintptr_t)din % 16) == 0 && ((uintptr_t)rhs % 16) == 0 && ((uintptr_t)zero % 16) == 0;
  CUDA_TRY(ctx, gf64_region(ctx, nullptr, dpin, 0, num_inputs, B, M, num_inputs, n, nullptr, dpout, 0, true, al));
  // the n x n system over the lost columns, then the solve
  CUDA_TRY(ctx, cudaMemcpyAsync(dcols, miss.data(), n * 8, cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(ctx, launch_gf64_cauchy_cols(dA, n, dcols, n, first_input, first_recovery, ctx->stream));
  if (cauchy) {
    // restored = A^-1 * rhs: O(n^2) weights + one n x n region product
    uint64_t* dW = dcols + n;
    uint64_t* dAinv = dW + 2 * n;
    uint64_t* dout = out_dev ? restored : (uint64_t*)scratch(ctx, S_COEF, n * B * 8);
    if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "repair output");
    CUDA_TRY(ctx, launch_gf64_cauchy_inverse(dA, dcols, n, first_input, first_recovery, dW, dAinv, ctx->stream));
    const bool al2 = (B % 2) == 0 && ((uintptr_t)rhs % 16) == 0 && ((uintptr_t)dout % 16) == 0;
    CUDA_TRY(ctx, gf64_region(ctx, rhs, nullptr, B, n, B, dAinv, n, n, dout, nullptr, B, false, al2));
    if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(restored, dout, n * B * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return device_status(ctx);
  }
  int* dS = (int*)(dF + n + 2);
  CUDA_TRY(ctx, cudaMemsetAsync(dS, 0, sizeof(int), ctx->stream));
  CUDA_TRY(ctx, launch_gf64_solve(dA, rhs, n, B, dF, dS, ctx->stream));
  int hs = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&hs, dS, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(restored, rhs, n * B * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (hs != 0) return set_err(ctx, PP_ERR_SINGULAR, "repair matrix is singular");
  return device_status(ctx);
}

// ------------------------------------------------------------ block hashes
// A strided list of n rows as device rows: device rows are used in place when
// they meet the alignment asked for; otherwise they are copied into scratch
// slot `s` with a 16-byte rounded stride.  `width` bytes are read from each of
// the first n - 1 rows and `last` from the last one.
static const uint8_t* rows_on_device(pp_ctx* ctx, Slot s, const void* rows, size_t stride, size_t n, size_t width,
                                     size_t last, bool need16, size_t* dstride, int* st) {
  *st = PP_OK;
  const bool dev = is_device_ptr(rows);
  if (dev && (!need16 || aligned16(rows, n > 1 ? stride : 0))) {
    *dstride = stride;
    return (const uint8_t*)rows;
  }
  const size_t ds = round16(std::max(width, last));
  uint8_t* d = (uint8_t*)scratch(ctx, s, ds * n);
  if (!d) {
    *st = set_err(ctx, PP_ERR_NO_MEMORY, "device allocation of %zu bytes failed", ds * n);
    return nullptr;
  }
  const cudaMemcpyKind k = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaError_t e = cudaSuccess;
  if (n > 1 && width) e = cudaMemcpy2DAsync(d, ds, rows, stride, width, n - 1, k, ctx->stream);
  if (e == cudaSuccess && last)
    e = cudaMemcpyAsync(d + ds * (n - 1), (const uint8_t*)rows + stride * (n - 1), last, k, ctx->stream);
  if (e != cudaSuccess) {
    *st = set_err(ctx, PP_ERR_CUDA, "row staging: %s", cudaGetErrorString(e));
    return nullptr;
  }
  *dstride = ds;
  return d;
}

// Read a small argument that may live on either side.
static int host_bytes(pp_ctx* ctx, const void* p, size_t n, void* out) {
  if (is_device_ptr(p)) {
    CUDA_TRY(ctx, cudaMemcpy(out, p, n, cudaMemcpyDeviceToHost));
  } else {
    memcpy(out, p, n);
  }
  return PP_OK;
}

static inline uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}

PP_API int pp_par2_block_hashes(pp_ctx* ctx, const void* blocks, size_t block_stride, size_t num_blocks,
                                size_t slice_size, const uint64_t* lengths, uint8_t* md5crc) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (num_blocks == 0) return PP_OK;
  if (!blocks || !md5crc) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const size_t n = num_blocks;
  size_t width = slice_size, last = slice_size;
  const uint64_t* dlen = nullptr;
  int st = PP_OK;
  if (lengths) {
    std::vector<uint64_t> hl(n);
    if (int r = host_bytes(ctx, lengths, n * 8, hl.data())) return r;
    uint64_t mx = 0;
    for (size_t i = 0; i < n; i++) {
      if (hl[i] > slice_size)
        return set_err(ctx, PP_ERR_INVALID_ARG, "block %zu: length %llu exceeds the slice size %zu", i,
                       (unsigned long long)hl[i], slice_size);
      mx = std::max<uint64_t>(mx, hl[i]);
    }
    width = (size_t)mx;
    last = (size_t)hl[n - 1];
    dlen = to_device(ctx, S_A, lengths, n, &st);
    if (st) return st;
  }
  if (n > 1 && block_stride < width) return set_err(ctx, PP_ERR_INVALID_ARG, "block_stride is shorter than a block");
  size_t dstride = 0;
  const uint8_t* drows = rows_on_device(ctx, S_IN, blocks, block_stride, n, width, last, true, &dstride, &st);
  if (!drows) return st;
  const bool out_dev = is_device_ptr(md5crc) && ((uintptr_t)md5crc % 4) == 0;
  uint8_t* dout = out_dev ? md5crc : (uint8_t*)scratch(ctx, S_OUT, 20 * n);
  if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "hash output");
  CUDA_TRY(ctx, launch_par2_block_hash(drows, dstride, n, slice_size, dlen, dout, ctx->stream));
  if (!out_dev)
    CUDA_TRY(ctx, cudaMemcpyAsync(md5crc, dout, 20 * n, cudaMemcpyDefault, ctx->stream));
  if (!out_dev || drows != blocks || lengths) CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

PP_API int pp_par3_block_hashes(pp_ctx* ctx, const void* blocks, size_t block_stride, size_t num_blocks,
                                size_t block_size, uint64_t first_index, const uint8_t* after_checksum,
                                uint8_t* hashes) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (num_blocks == 0) return PP_OK;
  if (!blocks || !after_checksum || !hashes) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if (num_blocks > 1 && block_stride < block_size)
    return set_err(ctx, PP_ERR_INVALID_ARG, "block_stride is shorter than a block");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const size_t n = num_blocks;
  uint8_t after[24];
  if (int r = host_bytes(ctx, after_checksum, 24, after)) return r;
  int st = PP_OK;
  size_t dstride = 0;
  const uint8_t* drows =
      rows_on_device(ctx, S_IN, blocks, block_stride, n, block_size, block_size, false, &dstride, &st);
  if (!drows) return st;
  const bool out_dev = is_device_ptr(hashes);
  uint8_t* dout = out_dev ? hashes : (uint8_t*)scratch(ctx, S_OUT, 16 * n);
  const size_t sw = blake3_scratch_words(n, 32 + (uint64_t)block_size);
  uint32_t* dcv = sw ? (uint32_t*)scratch(ctx, S_B, sw * 4) : nullptr;
  if (!dout || (sw && !dcv)) return set_err(ctx, PP_ERR_NO_MEMORY, "hash buffers");
  B3Job J;
  J.data = drows;
  J.stride = dstride;
  J.D = block_size;
  J.P = 32;
  for (int k = 0; k < 6; k++) J.pre[k] = le32(after + 4 * k);
  J.first_index = first_index;
  J.n = n;
  J.hash_out = dout;
  J.hash_stride = 16;
  CUDA_TRY(ctx, launch_blake3_blocks(J, dcv, ctx->stream));
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(hashes, dout, 16 * n, cudaMemcpyDeviceToHost, ctx->stream));
  if (!out_dev || drows != blocks) CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

// Headers + BLAKE3 of n recovery packets built from device recovery rows
// (dstride bytes apart) into device packets dpk; enqueued on the context's
// stream.
static int assemble_packets(pp_ctx* ctx, const uint8_t* drows, size_t dstride, size_t n, size_t block_size,
                            const uint8_t sid[8], uint64_t first, uint8_t* dpk) {
  const size_t pkt = 64 + block_size;
  const size_t sw = blake3_scratch_words(n, 40 + (uint64_t)block_size);
  uint32_t* dcv = sw ? (uint32_t*)scratch(ctx, S_B, sw * 4) : nullptr;
  if (sw && !dcv) return set_err(ctx, PP_ERR_NO_MEMORY, "packet hash scratch");
  uint64_t sid64 = 0;
  for (int b = 0; b < 8; b++) sid64 |= (uint64_t)sid[b] << (8 * b);
  CUDA_TRY(ctx, launch_par3_packet_headers(dpk, n, block_size, sid64, first, ctx->stream));
  // checksum input: header bytes [24, 48) = total length, set id, "PAR REC\0";
  // then the body u64le(index), u64le(1), block
  B3Job J;
  J.data = drows;
  J.stride = dstride;
  J.D = block_size;
  J.P = 40;
  J.pre[0] = (uint32_t)pkt;
  J.pre[1] = (uint32_t)((uint64_t)pkt >> 32);
  J.pre[2] = le32(sid);
  J.pre[3] = le32(sid + 4);
  J.pre[4] = 0x20524150u;  // "PAR "
  J.pre[5] = 0x00434552u;  // "REC\0"
  J.first_index = first;
  J.extra = 1;
  J.n = n;
  J.copy_to = dpk + 64;
  J.copy_stride = pkt;
  J.hash_out = dpk + 8;
  J.hash_stride = pkt;
  CUDA_TRY(ctx, launch_blake3_blocks(J, dcv, ctx->stream));
  return PP_OK;
}

static int check_packet_args(pp_ctx* ctx, size_t num_recovery, size_t block_size) {
  if (num_recovery == 0) return set_err(ctx, PP_ERR_INVALID_ARG, "numRecovery must be a positive integer");
  if (block_size == 0) return set_err(ctx, PP_ERR_INVALID_ARG, "blockSize must be a positive integer");
  if (num_recovery > ((size_t)1 << 40) / block_size)
    return set_err(ctx, PP_ERR_INVALID_ARG, "numRecovery * blockSize exceeds 1 TiB cap");
  return PP_OK;
}

PP_API int pp_par3_assemble_recovery_packets(pp_ctx* ctx, const void* recovery, size_t num_recovery,
                                             size_t block_size, const uint8_t* input_set_id,
                                             uint64_t first_recovery_index, uint8_t* packets) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (int r = check_packet_args(ctx, num_recovery, block_size)) return r;
  if (!recovery || !input_set_id || !packets) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const size_t n = num_recovery, pkt = 64 + block_size;
  uint8_t sid[8];
  if (int r = host_bytes(ctx, input_set_id, 8, sid)) return r;
  int st = PP_OK;
  size_t dstride = 0;
  const uint8_t* drows = rows_on_device(ctx, S_IN, recovery, block_size, n, block_size, block_size, false,
                                        &dstride, &st);
  if (!drows) return st;
  const bool out_dev = is_device_ptr(packets);
  uint8_t* dpk = out_dev ? packets : (uint8_t*)scratch(ctx, S_OUT, n * pkt);
  if (!dpk) return set_err(ctx, PP_ERR_NO_MEMORY, "packet buffer");
  if (int r = assemble_packets(ctx, drows, dstride, n, block_size, sid, first_recovery_index, dpk)) return r;
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(packets, dpk, n * pkt, cudaMemcpyDeviceToHost, ctx->stream));
  if (!out_dev || drows != recovery) CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

PP_API int pp_par3_create_packets(pp_ctx* ctx, const uint64_t* inputs, size_t num_inputs, size_t block_size64,
                                  uint64_t first_input, size_t num_recovery, uint64_t first_recovery,
                                  const uint8_t* data_after_checksum, uint8_t* data_hashes,
                                  const uint8_t* input_set_id, uint8_t* packets) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (num_inputs == 0 || block_size64 == 0) return set_err(ctx, PP_ERR_INVALID_ARG, "no input blocks");
  const size_t bs = block_size64 * 8;
  if (int r = check_packet_args(ctx, num_recovery, bs)) return r;
  if (!inputs || !input_set_id || !packets || (data_hashes && !data_after_checksum))
    return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  uint8_t sid[8];
  if (int r = host_bytes(ctx, input_set_id, 8, sid)) return r;
  int st;
  uint64_t* M = cauchy_get(ctx, num_inputs, num_recovery, first_input, first_recovery, &st);
  if (!M) return st;
  uint64_t* drec = (uint64_t*)scratch(ctx, S_PKT, num_recovery * bs);
  if (!drec) return set_err(ctx, PP_ERR_NO_MEMORY, "recovery blocks (%zu bytes)", num_recovery * bs);
  // data-block hashes of the inputs, in the same pass
  B3Job hj;
  uint32_t* hcv = nullptr;
  uint8_t* dh = nullptr;
  if (data_hashes) {
    uint8_t after[24];
    if (int r = host_bytes(ctx, data_after_checksum, 24, after)) return r;
    dh = is_device_ptr(data_hashes) ? data_hashes : (uint8_t*)scratch(ctx, S_HASH, 16 * num_inputs);
    const size_t sw = blake3_scratch_words(num_inputs, 32 + (uint64_t)bs);
    hcv = sw ? (uint32_t*)scratch(ctx, S_HCV, sw * 4) : nullptr;
    if (!dh || (sw && !hcv)) return set_err(ctx, PP_ERR_NO_MEMORY, "hash buffers");
    hj.P = 32;
    for (int k = 0; k < 6; k++) hj.pre[k] = le32(after + 4 * k);
    hj.first_index = first_input;
    hj.hash_out = dh;
    hj.hash_stride = 16;
  }
  if (int r = gf64_matvec_impl(ctx, inputs, num_inputs, drec, num_recovery, block_size64, M, false,
                               data_hashes ? &hj : nullptr, hcv))
    return r;
  const bool out_dev = is_device_ptr(packets);
  const size_t pkt = 64 + bs;
  uint8_t* dpk = out_dev ? packets : (uint8_t*)scratch(ctx, S_OUT, num_recovery * pkt);
  if (!dpk) return set_err(ctx, PP_ERR_NO_MEMORY, "packet buffer");
  if (int r = assemble_packets(ctx, (const uint8_t*)drec, bs, num_recovery, bs, sid, first_recovery, dpk)) return r;
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(packets, dpk, num_recovery * pkt, cudaMemcpyDeviceToHost, ctx->stream));
  if (data_hashes && dh != data_hashes)
    CUDA_TRY(ctx, cudaMemcpyAsync(data_hashes, dh, 16 * num_inputs, cudaMemcpyDeviceToHost, ctx->stream));
  if (!out_dev || (data_hashes && dh != data_hashes) || !is_device_ptr(inputs)) {
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return device_status(ctx);
  }
  return PP_OK;
}

PP_API int pp_par2_memory_checksums(pp_ctx* ctx, const void* rows, size_t row_stride, size_t num_rows,
                                    size_t slice_bytes, uint8_t* out16) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (num_rows == 0) return PP_OK;
  if (!rows || !out16) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if (num_rows > 1 && row_stride < slice_bytes) return set_err(ctx, PP_ERR_INVALID_ARG, "row_stride < slice_bytes");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  int st = PP_OK;
  size_t dstride = 0;
  const uint8_t* drows =
      rows_on_device(ctx, S_IN, rows, row_stride, num_rows, slice_bytes, slice_bytes, true, &dstride, &st);
  if (!drows) return st;
  const bool out_dev = is_device_ptr(out16) && ((uintptr_t)out16 % 4) == 0;
  uint8_t* dout = out_dev ? out16 : (uint8_t*)scratch(ctx, S_OUT, 16 * num_rows);
  if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "checksum output");
  CUDA_TRY(ctx, launch_par2_cksum(drows, dstride, num_rows, slice_bytes, dout, 16, nullptr, ctx->stream));
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(out16, dout, 16 * num_rows, cudaMemcpyDefault, ctx->stream));
  if (!out_dev || drows != rows) CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

// ------------------------------------------------------------ streaming create
namespace {
// pread `n` bytes at `off` with `threads` parallel readers; returns 0, an
// errno, or -1 for a file that ended early
int pread_all(int fd, uint8_t* dst, size_t n, uint64_t off, unsigned threads) {
  std::atomic<int> err{0};
  auto work = [&](size_t a, size_t b) {
    size_t pos = a;
    while (pos < b && !err.load(std::memory_order_relaxed)) {
      ssize_t r = ::pread(fd, dst + pos, b - pos, (off_t)(off + pos));
      if (r < 0) {
        if (errno == EINTR) continue;
        err = errno;
        return;
      }
      if (r == 0) {
        err = -1;
        return;
      }
      pos += (size_t)r;
    }
  };
  const size_t per = std::max<size_t>((size_t)4 << 20, (n + threads - 1) / threads);
  std::vector<std::thread> ts;
  for (size_t a = per; a < n; a += per) ts.emplace_back(work, a, std::min(n, a + per));
  work(0, std::min(n, per));
  for (auto& t : ts) t.join();
  return err.load();
}
}  // namespace

PP_API int pp_par3_create_streaming(pp_ctx* ctx, const char* source_path, size_t block_size, size_t num_recovery,
                                    uint64_t first_input, uint64_t first_recovery, uint8_t* recovery,
                                    const uint8_t* data_after_checksum, uint8_t* data_hashes,
                                    pp_stream_stats* stats) {
  using clk = std::chrono::steady_clock;
  const auto t_start = clk::now();
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (num_recovery == 0) return set_err(ctx, PP_ERR_INVALID_ARG, "recoverySlices must be a positive integer");
  if (block_size == 0 || block_size % 8)
    return set_err(ctx, PP_ERR_INVALID_ARG, "blockSize must be positive and a multiple of 8");
  if (!source_path || !recovery || (data_hashes && !data_after_checksum))
    return set_err(ctx, PP_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const int fd = ::open(source_path, O_RDONLY);
  if (fd < 0) {
    const int e = errno;
    return set_err(ctx, PP_ERR_IO, "open failed for sourcePath: errno=%d (%s)", e, strerror(e));
  }
  struct FdGuard {
    int fd;
    ~FdGuard() { ::close(fd); }
  } guard{fd};
  struct stat st;
  if (::fstat(fd, &st) != 0) {
    const int e = errno;
    return set_err(ctx, PP_ERR_IO, "fstat failed: errno=%d (%s)", e, strerror(e));
  }
  if (st.st_size <= 0) return set_err(ctx, PP_ERR_IO, "sourcePath is empty");
  const uint64_t total = (uint64_t)st.st_size;
  const size_t bs = block_size, B = bs / 8;
  const size_t N = (size_t)((total + bs - 1) / bs);
  const size_t R = num_recovery;
  int rc;
  uint64_t* M = cauchy_get(ctx, N, R, first_input, first_recovery, &rc);
  if (!M) return rc;
  // chunks of about 64 MiB of whole blocks; two pinned and two device buffers
  const size_t chunk = std::max<size_t>(1, ((size_t)64 << 20) / bs);
  const size_t cbytes = chunk * bs;
  if (ctx->pinned_n < 2 * cbytes) {
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_n = 0;
    if (cudaMallocHost(&ctx->pinned, 2 * cbytes) != cudaSuccess) {
      cudaGetLastError();
      return set_err(ctx, PP_ERR_NO_MEMORY, "pinned read buffers (%zu bytes)", 2 * cbytes);
    }
    ctx->pinned_n = 2 * cbytes;
  }
  uint8_t* dbuf = (uint8_t*)scratch(ctx, S_STREAM, 2 * cbytes);
  const bool out_dev = is_device_ptr(recovery);
  uint64_t* drec = out_dev ? (uint64_t*)recovery : (uint64_t*)scratch(ctx, S_OUT, R * bs);
  if (!dbuf || !drec) return set_err(ctx, PP_ERR_NO_MEMORY, "streaming device buffers");
  if (int r = ensure_copy_stream(ctx)) return r;
  B3Job hj;
  uint32_t* hcv = nullptr;
  uint8_t* dh = nullptr;
  if (data_hashes) {
    if (int r = ensure_hash_stream(ctx)) return r;
    uint8_t after[24];
    if (int r = host_bytes(ctx, data_after_checksum, 24, after)) return r;
    dh = is_device_ptr(data_hashes) ? data_hashes : (uint8_t*)scratch(ctx, S_HASH, 16 * N);
    const size_t sw = blake3_scratch_words(chunk, 32 + (uint64_t)bs);
    hcv = sw ? (uint32_t*)scratch(ctx, S_HCV, sw * 4) : nullptr;
    if (!dh || (sw && !hcv)) return set_err(ctx, PP_ERR_NO_MEMORY, "hash buffers");
    hj.P = 32;
    for (int k = 0; k < 6; k++) hj.pre[k] = le32(after + 4 * k);
    hj.stride = bs;
    hj.D = bs;
    hj.hash_stride = 16;
  }
  // per device buffer: the copy into it waits for the work that last read it
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 4; i++)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } eg{ev};
  for (int i = 0; i < 4; i++)
    if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return set_err(ctx, PP_ERR_CUDA, "streaming events");
    }
  cudaEvent_t* freed = ev;       // [2]: the product (and hash) of the buffer's last chunk is done
  cudaEvent_t* copied = ev + 2;  // [2]: the buffer's copy to the device is done
  const unsigned readers = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  double read_s = 0;
  auto read_chunk = [&](size_t c, uint8_t* dst) -> int {
    const uint64_t off = (uint64_t)c * cbytes;
    const size_t want = (size_t)std::min<uint64_t>(cbytes, total - off);
    const size_t nblk = std::min(chunk, N - c * chunk);
    const auto t0 = clk::now();
    const int e = pread_all(fd, dst, want, off, readers);
    read_s += std::chrono::duration<double>(clk::now() - t0).count();
    if (e == -1) return set_err(ctx, PP_ERR_IO, "unexpected EOF while reading sourcePath");
    if (e) return set_err(ctx, PP_ERR_IO, "read failed: errno=%d (%s)", e, strerror(e));
    if (want < nblk * bs) memset(dst + want, 0, nblk * bs - want);  // zero-pad the last block
    return PP_OK;
  };
  const size_t nchunks = (N + chunk - 1) / chunk;
  CUDA_TRY(ctx, cudaEventRecord(ctx->start_ev, ctx->stream));  // scratch is free once earlier work is done
  CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy, ctx->start_ev, 0));
  if (int r = read_chunk(0, ctx->pinned)) return r;
  for (size_t c = 0; c < nchunks; c++) {
    const int slot = (int)(c & 1);
    const size_t c0 = c * chunk, nc = std::min(chunk, N - c0);
    uint8_t* h = ctx->pinned + slot * cbytes;
    uint8_t* d = dbuf + slot * cbytes;
    if (c >= 2) CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy, freed[slot], 0));
    CUDA_TRY(ctx, cudaMemcpyAsync(d, h, nc * bs, cudaMemcpyHostToDevice, ctx->copy));
    CUDA_TRY(ctx, cudaEventRecord(copied[slot], ctx->copy));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, copied[slot], 0));
    CUDA_TRY(ctx, gf64_region(ctx, (const uint64_t*)d, nullptr, B, nc, B, M + c0, N, R, drec, nullptr, B, c > 0,
                              aligned_rows64((const uint64_t*)d, B) && aligned_rows64(drec, B)));
    if (data_hashes) {
      CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->hash, copied[slot], 0));
      B3Job J = hj;
      J.data = d;
      J.n = nc;
      J.first_index = first_input + c0;
      J.hash_out = dh + 16 * c0;
      CUDA_TRY(ctx, launch_blake3_blocks(J, hcv, ctx->hash));
      CUDA_TRY(ctx, cudaEventRecord(ctx->hash_ev, ctx->hash));
      CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->hash_ev, 0));
    }
    CUDA_TRY(ctx, cudaEventRecord(freed[slot], ctx->stream));
    if (c + 1 < nchunks) {
      // the other pinned buffer is free once its copy (chunk c - 1) is done
      if (c >= 1) CUDA_TRY(ctx, cudaEventSynchronize(copied[slot ^ 1]));
      if (int r = read_chunk(c + 1, ctx->pinned + (slot ^ 1) * cbytes)) {
        cudaStreamSynchronize(ctx->stream);
        return r;
      }
    }
  }
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(recovery, drec, R * bs, cudaMemcpyDeviceToHost, ctx->stream));
  if (data_hashes && dh != data_hashes)
    CUDA_TRY(ctx, cudaMemcpyAsync(data_hashes, dh, 16 * N, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (stats) {
    stats->bytes_read = total;
    stats->num_inputs = N;
    stats->seconds = std::chrono::duration<double>(clk::now() - t_start).count();
    stats->read_seconds = read_s;
  }
  return device_status(ctx);
}

PP_API int pp_par2_recovery_packet_headers(pp_ctx* ctx, const void* slices, size_t slice_stride, size_t num_slices,
                                           size_t slice_bytes, const uint8_t* set_id, const uint16_t* exps,
                                           uint8_t* headers) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (num_slices == 0) return PP_OK;
  if (!slices || !set_id || !exps || !headers) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  if (slice_bytes % 4) return set_err(ctx, PP_ERR_INVALID_ARG, "PAR2 slice size must be a multiple of 4");
  if (num_slices > 1 && slice_stride < slice_bytes)
    return set_err(ctx, PP_ERR_INVALID_ARG, "slice_stride < slice_bytes");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  uint8_t sid[16];
  if (int r = host_bytes(ctx, set_id, 16, sid)) return r;
  uint32_t pre[8];
  for (int k = 0; k < 4; k++) pre[k] = le32(sid + 4 * k);
  static const uint8_t type[16] = {'P', 'A', 'R', ' ', '2', '.', '0', 0, 'R', 'e', 'c', 'v', 'S', 'l', 'i', 'c'};
  for (int k = 0; k < 4; k++) pre[4 + k] = le32(type + 4 * k);
  int st = PP_OK;
  size_t dstride = 0;
  const uint8_t* drows =
      rows_on_device(ctx, S_IN, slices, slice_stride, num_slices, slice_bytes, slice_bytes, true, &dstride, &st);
  if (!drows) return st;
  const uint16_t* dex = to_device(ctx, S_A, exps, num_slices, &st);
  if (st) return st;
  const bool out_dev = is_device_ptr(headers) && ((uintptr_t)headers % 4) == 0;
  uint8_t* dout = out_dev ? headers : (uint8_t*)scratch(ctx, S_OUT, 68 * num_slices);
  if (!dout) return set_err(ctx, PP_ERR_NO_MEMORY, "header output");
  CUDA_TRY(ctx, launch_par2_packet_headers(drows, dstride, num_slices, slice_bytes, pre, dex, dout, ctx->stream));
  if (!out_dev) CUDA_TRY(ctx, cudaMemcpyAsync(headers, dout, 68 * num_slices, cudaMemcpyDefault, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

PP_API int pp_xor_buffers(pp_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx) return PP_ERR_INVALID_ARG;
  if (!bytes) return PP_OK;
  if (!dst || !src) return set_err(ctx, PP_ERR_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int r = bind(ctx)) return r;
  const bool d_dev = is_device_ptr(dst), s_dev = is_device_ptr(src);
  uint8_t* dd = (uint8_t*)dst;
  const uint8_t* ds = (const uint8_t*)src;
  if (!d_dev) {
    dd = (uint8_t*)scratch(ctx, S_OUT, bytes);
    if (!dd) return set_err(ctx, PP_ERR_NO_MEMORY, "staging");
    CUDA_TRY(ctx, cudaMemcpyAsync(dd, dst, bytes, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (!s_dev) {
    uint8_t* t = (uint8_t*)scratch(ctx, S_IN, bytes);
    if (!t) return set_err(ctx, PP_ERR_NO_MEMORY, "staging");
    CUDA_TRY(ctx, cudaMemcpyAsync(t, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    ds = t;
  }
  CUDA_TRY(ctx, launch_xor_bytes(dd, ds, bytes, ctx->stream));
  if (!d_dev) CUDA_TRY(ctx, cudaMemcpyAsync(dst, dd, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (!d_dev || !s_dev) CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PP_OK;
}

}  // extern "C"

// ====================================================== one job, many GPUs
// A job's slices split by byte range over several contexts (one per GPU),
// each range computed by its own host thread on its own device: what
// PAR2Proc does with its backends (gf16/controller.cpp:42-84: every backend
// takes [offset, offset + size) of every slice) and what the Fenger path does
// with word ranges (src/par3_engine_fenger.cc:266-290).  No data crosses
// between devices: each context reads its range of the caller's buffers
// (host memory, or device memory of that context's own GPU) and writes the
// same range of the outputs.

// The reference's acceptance rule for a split (PAR2Proc::checkBackendAllocation):
// the non-empty ranges cover [0, slice) without gaps or overlaps, start on
// multiples of `unit`, and only the range that ends the slice may have a
// size that is not a multiple of `unit`.
static bool split_cover_ok(const size_t* b, const size_t* e, unsigned n, size_t slice, size_t unit) {
  std::vector<std::pair<size_t, size_t>> r;
  for (unsigned i = 0; i < n; i++) {
    if (e[i] < b[i] || e[i] > slice) return false;
    if (e[i] > b[i]) r.push_back({b[i], e[i]});
  }
  std::sort(r.begin(), r.end());
  size_t pos = 0;
  for (auto& x : r) {
    if (x.first != pos || x.first % unit) return false;
    if ((x.second - x.first) % unit && x.second != slice) return false;
    pos = x.second;
  }
  return pos == slice;
}

// a context may dereference `p` only if it is host memory or its own device's
static bool readable_by(const pp_ctx* ctx, const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;  // pageable host memory
  }
  if (a.type == cudaMemoryTypeDevice) return a.device == ctx->device;
  return true;
}

template <class Fn>
static int run_split(pp_ctx* const* ctxs, const size_t* b, const size_t* e, unsigned n, Fn fn) {
  std::vector<int> st(n, PP_OK);
  std::vector<std::thread> th;
  for (unsigned i = 0; i < n; i++) {
    if (e[i] == b[i]) continue;
    th.emplace_back([&, i] {
      st[i] = fn(ctxs[i], b[i], e[i]);
      if (st[i] == PP_OK) st[i] = pp_ctx_synchronize(ctxs[i]);  // device buffers: wait for the range
    });
  }
  for (auto& t : th) t.join();
  for (unsigned i = 0; i < n; i++)
    if (st[i] != PP_OK) return st[i];
  return PP_OK;
}

PP_API int pp_par2_create_split(pp_ctx* const* ctxs, const size_t* range_begin, const size_t* range_end,
                                unsigned n_ranges, const void* inputs, size_t input_stride, unsigned num_inputs,
                                size_t slice_bytes, const uint16_t* input_idx, const uint16_t* exps,
                                unsigned num_outputs, void* outputs, size_t output_stride) {
  if (!ctxs || !range_begin || !range_end || !n_ranges) return PP_ERR_INVALID_ARG;
  for (unsigned i = 0; i < n_ranges; i++)
    if (!ctxs[i]) return PP_ERR_INVALID_ARG;
  if (!split_cover_ok(range_begin, range_end, n_ranges, slice_bytes, 2))
    return set_err(ctxs[0], PP_ERR_INVALID_ARG, "ranges do not split the slice on 16-bit words");
  for (unsigned i = 0; i < n_ranges; i++)
    if ((num_inputs && !readable_by(ctxs[i], inputs)) || !readable_by(ctxs[i], outputs))
      return set_err(ctxs[i], PP_ERR_INVALID_ARG, "a device buffer of another GPU");
  return run_split(ctxs, range_begin, range_end, n_ranges, [&](pp_ctx* c, size_t b, size_t e) {
    return pp_par2_create(c, (const uint8_t*)inputs + b, input_stride, num_inputs, e - b, input_idx, exps,
                          num_outputs, (uint8_t*)outputs + b, output_stride);
  });
}

PP_API int pp_gf64_compute_recovery_split(pp_ctx* const* ctxs, const size_t* range_begin, const size_t* range_end,
                                          unsigned n_ranges, const uint64_t* inputs, size_t num_inputs,
                                          uint64_t* recovery, size_t num_recovery, size_t block_size64,
                                          uint64_t first_input, uint64_t first_recovery) {
  if (!ctxs || !range_begin || !range_end || !n_ranges) return PP_ERR_INVALID_ARG;
  for (unsigned i = 0; i < n_ranges; i++)
    if (!ctxs[i]) return PP_ERR_INVALID_ARG;
  if (num_inputs == 0 || num_recovery == 0 || block_size64 == 0) return PP_OK;
  if (!inputs || !recovery) return set_err(ctxs[0], PP_ERR_INVALID_ARG, "null buffer");
  // ranges in bytes of a block, on whole words
  if (!split_cover_ok(range_begin, range_end, n_ranges, block_size64 * 8, 8))
    return set_err(ctxs[0], PP_ERR_INVALID_ARG, "ranges do not split the block on 8-byte words");
  for (unsigned i = 0; i < n_ranges; i++)
    if (!readable_by(ctxs[i], inputs) || !readable_by(ctxs[i], recovery))
      return set_err(ctxs[i], PP_ERR_INVALID_ARG, "a device buffer of another GPU");
  return run_split(ctxs, range_begin, range_end, n_ranges, [&](pp_ctx* c, size_t b, size_t e) {
    std::lock_guard<std::mutex> g(c->mu);
    if (int r = bind(c)) return r;
    int st;
    uint64_t* M = cauchy_get(c, num_inputs, num_recovery, first_input, first_recovery, &st);
    if (!M) return st;
    return gf64_matvec_impl(c, inputs + b / 8, num_inputs, recovery + b / 8, num_recovery, (e - b) / 8, M, false,
                            nullptr, nullptr, block_size64, block_size64);
  });
}
