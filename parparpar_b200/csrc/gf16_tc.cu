// GF(2^16) region multiply-accumulate on the 5th-generation tensor cores
// (tcgen05, kind::i8), sm_100a.
//
// Multiplication by a constant c in GF(2^16) is a 16x16 matrix over GF(2):
// bit b of c*x = XOR_e bit_e(x) * bit_b(c * x^e).  The whole region product
//   out[o][w] = XOR_i c[o][i] * in_i[w]
// is therefore one GF(2) matrix product; here it is computed as the parity
// of an exact integer u8 MMA.
//
// Shift trick: with A entries in {0,1}, sum_k A_k * B_k is congruent mod 2 to
// sum_k A_k * (B_k mod 2), so only the lowest bit of each B byte matters.
// Feeding the RAW input bytes shifted right by j (a plain 32-bit shift: the
// bits that slide in from the neighbouring byte only add even amounts) makes
// the low bit of byte beta equal bit 8*beta + j of the word.  With
//   A[(o,b)][(j, i, beta)] = bit_b(c[o][i] * x^(8*beta + j))
//   B[w][(j, i, beta)]     = byte_beta(in_i[w]) >> j        (j = 0..7)
// the count D[(o,b)][w] = sum A*B has parity = bit b of out[o][w].  Counts
// stay below 255 * 16 * num_inputs < 2^31.
//
// CTA tile: 8 outputs (M = 128 rows = 8 x 16 bits) x 512 words (two MMAs of
// N = 256), looping over the inputs 8 at a time.  A stage's K is 128 bytes:
// eight 16-byte chunks j = 0..7, each holding the 2 bytes of the 8 inputs'
// words shifted right by j; four K = 32 MMA steps per stage.  The
// accumulator fills TMEM (128 lanes x 512 columns of int32).
//
//   warp 0      producer: cp.async.bulk of the stage's A tile (pre-expanded
//               coefficient bits, already in the swizzled smem layout) and
//               of the 8 raw input rows of the word tile
//   warp 1      TMEM allocation + one thread issuing tcgen05.mma
//   warps 2-9   build the B tile (byte-permute the 8 inputs' words of a word
//               pair into one 16-byte row, shift by j, 128-byte swizzle),
//               then the epilogue: tcgen05.ld of the counts, parity, warp
//               ballot -> two u16 outputs per lane
//
// Every mbarrier wait is bounded (about one second of %globaltimer); on a
// timeout the CTA records an error in *status, drains what it issued, frees
// TMEM and returns.
#include "pp_common.cuh"
#include "pp_internal.h"
#include "tc_batch.h"
#include "tc_common.cuh"
#include "tma_map.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>

namespace pp {

// Tensor maps of the jobs' input matrices, entry j for job j of the table: a
// second __grid_constant__ parameter (the TMA reads the map from parameter
// space), rows = the job's inputs, boxes of one stage's rows
struct alignas(64) Gf16TcMaps {
  CUtensorMap raw[kTcMaxJobs];
};

namespace tc16 {
using namespace pp::tc;

constexpr int kStageIn = 8;                 // inputs per stage
constexpr int kABytes = 128 * 128;          // A tile of one output group: 128 rows x 128 B
constexpr int kThreads = 320;
constexpr int kExp = 256;  // expander / epilogue threads (warps 2-9)

// Tile shape by output groups per CTA (KG): KG = 1 -> 8 outputs x 512 words;
// KG = 2 -> 16 outputs x 256 words, two MMA accumulators of N = 256 sharing
// each B tile, which halves the B tile built per output.  Either way the
// accumulator fills TMEM (128 lanes x 512 columns).
template <int KG>
struct Shape {
  static constexpr int kLd = 4;                       // load ring depth (A tiles + raw rows)
  static constexpr int kBs = 2;                       // B tile ring depth
  static constexpr int kWords = KG == 2 ? 256 : 512;  // words per CTA
  static constexpr int kAStage = KG * kABytes;        // A bytes per stage
  static constexpr int kBBytes = kWords * 128;        // B tile: kWords rows x 128 B
  static constexpr int kRawBytes = kStageIn * kWords * 2;
  static constexpr int kOffA = 0;
  static constexpr int kOffB = kLd * kAStage;
  static constexpr int kOffRaw = kOffB + kBs * kBBytes;
  static constexpr int kOffBar = kOffRaw + kLd * kRawBytes;
  static constexpr int kSmemBytes = kOffBar + 256 + 1024;  // + barriers + alignment slack
};
static_assert(Shape<1>::kSmemBytes <= 227 * 1024 && Shape<2>::kSmemBytes <= 227 * 1024, "shared memory");
// raw rows arrive as tensor-map boxes of kStageIn rows x kBox bytes: a word
// tile's 2 * kWords bytes are 2 (KG = 2) or 4 (KG = 1) boxes, box b of a ring
// slot at b * kBoxStage, row ii of a box at ii * kBox
constexpr int kBox = 256;
constexpr int kBoxStage = kStageIn * kBox;

// instruction descriptor: D int32, A/B unsigned 8-bit, both K-major,
// N = 256, M = 128
constexpr uint32_t kIdesc = (2u << 4) | ((256u >> 3) << 17) | ((128u >> 4) << 24);

// 4 bits -> 4 bytes of 0/1 (bit k of n lands in byte k)
PP_D uint32_t spread4(uint32_t n) { return (n * 0x00204081u) & 0x01010101u; }

// ----------------------------------------------------------------------------
// A tiles: for output group g (outputs 8g..8g+7) and input stage s (inputs
// 8s..8s+7) a 16 KiB tile in the smem canonical layout (K-major, 128-byte
// swizzle): row m = 16*oo + b; chunk j (shift); byte 2*ii + beta within the
// chunk holds bit b of c[8g+oo][8s+ii] * x^(8*beta + j).
//
// With Q_b(c) = the 16-bit mask whose bit e is bit b of c * x^e (row b of the
// multiplication matrix of c) and P = Q_b(c[2q]) | Q_b(c[2q+1]) << 16, the
// 32-bit word q of chunk j is (P >> j) & 0x01010101: byte (ii, beta) = bit
// 8*beta + j of Q_b(c[ii]).  Q_b is linear in c, so
//   Q_b(c) = XOR_q T[q][nibble q of c][b],   T[q][n][b] = Q_b(n << 4q),
// a 2 KiB table (b fastest: the 16 threads of one coefficient read 32
// consecutive bytes) filled once per device.
__device__ __align__(16) uint16_t g_gf16_qtab[4 * 16 * 16];
static std::atomic<uint64_t> g_qtab_ready{0};

__global__ void k_gf16_qtab_init() {
  for (unsigned t = threadIdx.x; t < 1024; t += blockDim.x) {
    const unsigned q = t >> 8, n = (t >> 4) & 15, b = t & 15;
    uint32_t c = n << (4 * q), v = 0;
    for (int e = 0; e < 16; e++) {
      v |= ((c >> b) & 1u) << e;
      c = gf16_dbl(c);
    }
    g_gf16_qtab[t] = (uint16_t)v;
  }
}

static cudaError_t qtab_on(cudaStream_t s) {
  if (device_done(g_qtab_ready)) return cudaSuccess;
  k_gf16_qtab_init<<<1, 256, 0, s>>>();
  note_launch();
  return cudaGetLastError();
}

// One CTA per tile (g, s), thread m builds row m; each warp store writes
// 512 contiguous bytes, so the 16 KiB tile leaves as whole lines.
__global__ void __launch_bounds__(128)
k_gf16_tc_expand_coeffs(const uint16_t* __restrict__ coeffs, size_t ldc, unsigned n_in, unsigned n_out,
                        unsigned n_stages, uint8_t* __restrict__ a_exp) {
  __shared__ __align__(16) uint16_t T[4 * 16 * 16];
  reinterpret_cast<uint4*>(T)[threadIdx.x] = reinterpret_cast<const uint4*>(g_gf16_qtab)[threadIdx.x];
  __syncthreads();
  const unsigned m = threadIdx.x, oo = m >> 4, b = m & 15;
  const size_t tiles = (size_t)((n_out + 7) / 8) * n_stages;
  for (size_t gs = blockIdx.x; gs < tiles; gs += gridDim.x) {  // gs = g * n_stages + s
    const unsigned s = (unsigned)(gs % n_stages), g = (unsigned)(gs / n_stages);
    const unsigned o = 8 * g + oo;
    uint32_t P[4] = {0, 0, 0, 0};
#pragma unroll
    for (int ii = 0; ii < 8; ii++) {
      const unsigned i = 8 * s + ii;
      const uint32_t c = (o < n_out && i < n_in) ? coeffs[(size_t)o * ldc + i] : 0;
      const uint32_t q = (uint32_t)T[((c & 15) << 4) + b] ^ T[256 + (((c >> 4) & 15) << 4) + b] ^
                         T[512 + (((c >> 8) & 15) << 4) + b] ^ T[768 + ((c >> 12) << 4) + b];  // Q_b(c)
      P[ii >> 1] |= q << (16 * (ii & 1));
    }
    // the warp's 32 rows are 4 KiB of contiguous memory; store k writes its
    // 512 bytes [512k, 512k + 512): lane L the 16-byte slot L of it, i.e. row
    // 4k + L/8 of the warp, physical chunk L%8 (logical chunk (L%8) ^ (row%8)),
    // from the words of the lane that built that row
    const unsigned lane = m & 31;
    uint8_t* wbase = a_exp + gs * kABytes + (m >> 5) * 4096;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const unsigned r = 4 * k + (lane >> 3), j = (lane & 7) ^ (r & 7);
      const uint32_t p0 = __shfl_sync(0xFFFFFFFFu, P[0], r), p1 = __shfl_sync(0xFFFFFFFFu, P[1], r),
                     p2 = __shfl_sync(0xFFFFFFFFu, P[2], r), p3 = __shfl_sync(0xFFFFFFFFu, P[3], r);
      *reinterpret_cast<uint4*>(wbase + 512 * k + 16 * lane) =
          make_uint4((p0 >> j) & 0x01010101u, (p1 >> j) & 0x01010101u, (p2 >> j) & 0x01010101u,
                     (p3 >> j) & 0x01010101u);
    }
  }
}

// One CTA per work item of the job table (tc_batch.h): the item fixes the
// job, the output group, the word tile and the stage range; mode 0 stores,
// 1 XORs into the output, 2 XORs atomically (the job is split over CTAs).
template <int KG>
__global__ void __launch_bounds__(kThreads, 1)
k_gf16_muladd_tc(const __grid_constant__ Gf16TcBatch batch, const __grid_constant__ Gf16TcMaps maps,
                 int* __restrict__ status) {
  using S = Shape<KG>;
  constexpr int kWords = S::kWords, kBBytes = S::kBBytes, kRawBytes = S::kRawBytes, kAStage = S::kAStage;
  constexpr int kOffA = S::kOffA, kOffB = S::kOffB, kOffRaw = S::kOffRaw, kOffBar = S::kOffBar;
  constexpr int kLd = S::kLd, kBs = S::kBs;
  const TcSeg sg = tc_item(&batch, blockIdx.x);
  const Gf16TcJob J = pinned_job(batch.job[sg.job]);
  const unsigned n_in = J.n_in;
  const size_t slice_bytes = J.slice_bytes;
  const uint8_t* __restrict__ a_exp = J.a_exp;
  const unsigned n_stages_total = J.a_stride;  // tile-buffer stride (the launcher defaults it to n_stages)
  const unsigned n_out = J.n_out;
  uint8_t* __restrict__ out = J.out;
  const size_t out_stride = J.out_stride;
  const int mode = sg.mode;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t base_s = smem_addr(smem_raw);
  const uint32_t pad = ((base_s + 1023) & ~1023u) - base_s;
  uint8_t* smem = smem_raw + pad;
  const uint32_t sA = base_s + pad + kOffA, sB = base_s + pad + kOffB, sRaw = base_s + pad + kOffRaw;
  uint8_t* raw_p = smem + kOffRaw;
  uint8_t* b_p = smem + kOffB;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
  const uint32_t bar0 = smem_addr(bars);
  // load ring: A_FULL, RAW_FULL, A_EMPTY, RAW_EMPTY  (kLd each)
  // B ring:    B_FULL, B_EMPTY                       (kBs each)
  enum {
    A_FULL = 0,
    RAW_FULL = A_FULL + kLd,
    A_EMPTY = RAW_FULL + kLd,
    RAW_EMPTY = A_EMPTY + kLd,
    B_FULL = RAW_EMPTY + kLd,
    B_EMPTY = B_FULL + kBs,
    D_FULL = B_EMPTY + kBs,
    DONE = D_FULL + 1,
    NBARS = DONE + 1
  };
  static_assert(8 * NBARS + 16 <= 256, "barrier area");
  auto BAR = [&](int k) { return bar0 + 8u * (uint32_t)k; };
  volatile uint32_t* tmem_holder = reinterpret_cast<volatile uint32_t*>(smem + kOffBar + 8 * NBARS);
  volatile int* err = reinterpret_cast<volatile int*>(smem + kOffBar + 8 * NBARS + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned g = (unsigned)(sg.tile % J.groups) * KG;  // first output group of the CTA
  const size_t w0 = (size_t)(sg.tile / J.groups) * kWords;
  const unsigned st_begin = sg.st0;
  const unsigned nst = sg.st1 - sg.st0;
  const size_t total_words = (slice_bytes + 1) / 2;
  const unsigned words_valid = (unsigned)min((size_t)kWords, total_words - w0);
  // bytes of the word tile inside the slice
  const size_t tile_bytes_valid = min((size_t)kWords * 2, slice_bytes - 2 * w0);
  const unsigned n_box = (unsigned)((tile_bytes_valid + kBox - 1) / kBox);
  const void* raw_map = &maps.raw[sg.job];

  if (threadIdx.x == 0) {
    for (int k = 0; k < NBARS; k++) {
      const bool by_expanders = (k >= RAW_EMPTY && k < RAW_EMPTY + kLd) || (k >= B_FULL && k < B_FULL + kBs);
      mbar_init(BAR(k), by_expanders ? (uint32_t)kExp : 1u);
    }
    *err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr((const void*)tmem_holder)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      tma_prefetch_map(raw_map);
      unsigned issued = 0;
      for (unsigned k = 0; k < nst && !*err; k++) {
        const unsigned sl = k % kLd, use = k / kLd;
        if (k >= kLd) {
          if (!mbar_wait(BAR(A_EMPTY + sl), (use - 1) & 1) || !mbar_wait(BAR(RAW_EMPTY + sl), (use - 1) & 1)) {
            *err = 1;
            break;
          }
        }
        const unsigned st = st_begin + k;
        mbar_expect_tx(BAR(A_FULL + sl), kAStage);
#pragma unroll
        for (int gg = 0; gg < KG; gg++)
          bulk_g2s(sA + sl * kAStage + gg * kABytes, a_exp + ((size_t)(g + gg) * n_stages_total + st) * kABytes,
                   kABytes, BAR(A_FULL + sl));
        // the stage's rows: one box per kBox bytes of the tile that start
        // inside the slice (rows past the last input arrive as zeros)
        mbar_expect_tx(BAR(RAW_FULL + sl), n_box * kBoxStage);
        for (unsigned b = 0; b < n_box; b++)
          tma_load_2d(sRaw + sl * kRawBytes + b * kBoxStage, raw_map, (int)(2 * w0) + (int)b * kBox,
                      (int)(st * kStageIn), BAR(RAW_FULL + sl));
        issued = k + 1;
      }
      // drain: every issued copy lands before the CTA exits
      if (*err) {
        for (unsigned k = issued > (unsigned)kLd ? issued - kLd : 0; k < issued; k++) {
          mbar_wait(BAR(A_FULL + k % kLd), (k / kLd) & 1);
          mbar_wait(BAR(RAW_FULL + k % kLd), (k / kLd) & 1);
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      for (unsigned k = 0; k < nst; k++) {
        const unsigned sl = k % kLd, bs = k % kBs;
        if (*err || !mbar_wait(BAR(A_FULL + sl), (k / kLd) & 1) || !mbar_wait(BAR(B_FULL + bs), (k / kBs) & 1)) {
          *err = 1;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
#pragma unroll
          for (int nn = 0; nn < 2; nn++) {
            // KG = 1: two word halves of one group; KG = 2: one word tile of two groups
            const uint32_t a_off = KG == 2 ? nn * kABytes : 0;
            const uint32_t b_off = KG == 2 ? 0 : nn * (256 * 128);
            mma_i8(tmem + nn * 256, sw128_desc(sA + sl * kAStage + a_off + 32 * kk),
                   sw128_desc(sB + bs * kBBytes + b_off + 32 * kk), kIdesc, (k > 0 || kk > 0) ? 1u : 0u);
          }
        }
        mma_commit(BAR(A_EMPTY + sl));
        mma_commit(BAR(B_EMPTY + bs));
      }
      if (!*err) mma_commit(BAR(D_FULL));
      // all MMAs issued by this thread complete before TMEM is released
      mma_commit(BAR(DONE));
      if (!mbar_wait(BAR(DONE), 0)) *err = 1;
    }
  } else {
    // ------------------------------------------------------------ expanders
    const int e = threadIdx.x - 64;  // 0..255
    if constexpr (KG == 2) {
      // one word row per thread: row n = e holds the 8 inputs' words, shifted by j
      const unsigned n = e;
      const bool odd_tail = (slice_bytes & 1) && (w0 + kWords >= total_words);
      const unsigned last_word = (unsigned)(total_words - 1 - w0);
      uint32_t mask = n < words_valid ? 0xFFFFu : 0u;
      if (odd_tail && n == last_word) mask &= 0x00FFu;
      const uint32_t rowA = (n >> 3) * 1024 + (n & 7) * 128, rA = n & 7;
      const unsigned rb = (2 * n / kBox) * kBoxStage + (2 * n) % kBox;  // word n of row 0 within a ring slot
      for (unsigned k = 0; k < nst; k++) {
        const unsigned sl = k % kLd, bs = k % kBs;
        if (*err || !mbar_wait(BAR(RAW_FULL + sl), (k / kLd) & 1)) {
          *err = 1;
          break;
        }
        const unsigned i0 = (st_begin + k) * kStageIn;
        const unsigned ni = min((unsigned)kStageIn, n_in - i0);
        const uint8_t* raw = raw_p + sl * kRawBytes;
        uint32_t v[kStageIn];
#pragma unroll
        for (int ii = 0; ii < kStageIn; ii++)
          v[ii] = (unsigned)ii < ni ? (*reinterpret_cast<const uint16_t*>(raw + ii * kBox + rb) & mask) : 0u;
        mbar_arrive(BAR(RAW_EMPTY + sl));
        if (k >= (unsigned)kBs && !mbar_wait(BAR(B_EMPTY + bs), (k / kBs - 1) & 1)) {
          *err = 1;
          break;
        }
        uint8_t* bt = b_p + bs * kBBytes;
        uint32_t pA[4];
#pragma unroll
        for (int q = 0; q < 4; q++) pA[q] = v[2 * q] | (v[2 * q + 1] << 16);
        // 8 consecutive threads store 8 rows of one swizzle atom at 8 distinct chunks: conflict-free
#pragma unroll
        for (int j = 0; j < 8; j++)
          *reinterpret_cast<uint4*>(bt + rowA + ((j ^ rA) << 4)) =
              make_uint4(pA[0] >> j, pA[1] >> j, pA[2] >> j, pA[3] >> j);
        fence_async_smem();
        mbar_arrive(BAR(B_FULL + bs));
      }
    } else {
    const unsigned n = 2 * e;  // word pair n, n + 1 of the tile
    const bool odd_tail = (slice_bytes & 1) && (w0 + kWords >= total_words);
    const unsigned last_word = (unsigned)(total_words - 1 - w0);
    uint32_t mask = 0;
    if (n < words_valid) mask = 0xFFFFu;
    if (n + 1 < words_valid) mask |= 0xFFFF0000u;
    if (odd_tail) {
      if (n == last_word) mask &= 0xFFFF00FFu;
      else if (n + 1 == last_word) mask &= 0x00FFFFFFu;
    }
    // A 128-bit store is serviced in phases of 8 consecutive threads; threads
    // with bit 2 set store the odd word of their pair first, so each phase
    // covers all eight rows of a swizzle atom (conflict-free).
    const unsigned sw = (e >> 2) & 1;
    const unsigned mA = n + sw, mB = n + 1 - sw;
    const uint32_t rowA = (mA >> 3) * 1024 + (mA & 7) * 128, rA = mA & 7;
    const uint32_t rowB = (mB >> 3) * 1024 + (mB & 7) * 128, rB = mB & 7;
    const unsigned rb = (2 * n / kBox) * kBoxStage + (2 * n) % kBox;  // words n, n+1 of row 0 within a ring slot
    for (unsigned k = 0; k < nst; k++) {
      const unsigned sl = k % kLd, bs = k % kBs;
      if (*err || !mbar_wait(BAR(RAW_FULL + sl), (k / kLd) & 1)) {
        *err = 1;
        break;
      }
      const unsigned i0 = (st_begin + k) * kStageIn;
      const unsigned ni = min((unsigned)kStageIn, n_in - i0);
      const uint8_t* raw = raw_p + sl * kRawBytes;
      uint32_t v[kStageIn];
#pragma unroll
      for (int ii = 0; ii < kStageIn; ii++)
        v[ii] = (unsigned)ii < ni ? (*reinterpret_cast<const uint32_t*>(raw + ii * kBox + rb) & mask) : 0u;
      mbar_arrive(BAR(RAW_EMPTY + sl));
      if (k >= (unsigned)kBs && !mbar_wait(BAR(B_EMPTY + bs), (k / kBs - 1) & 1)) {
        *err = 1;
        break;
      }
      uint8_t* bt = b_p + bs * kBBytes;
      // row of word n: low halves of the 8 inputs; word n+1: high halves
      uint32_t pA[4], pB[4];
      const uint32_t selA = sw ? 0x7632u : 0x5410u, selB = sw ? 0x5410u : 0x7632u;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        pA[q] = __byte_perm(v[2 * q], v[2 * q + 1], selA);
        pB[q] = __byte_perm(v[2 * q], v[2 * q + 1], selB);
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        *reinterpret_cast<uint4*>(bt + rowA + ((j ^ rA) << 4)) =
            make_uint4(pA[0] >> j, pA[1] >> j, pA[2] >> j, pA[3] >> j);
        *reinterpret_cast<uint4*>(bt + rowB + ((j ^ rB) << 4)) =
            make_uint4(pB[0] >> j, pB[1] >> j, pB[2] >> j, pB[3] >> j);
      }
      fence_async_smem();
      mbar_arrive(BAR(B_FULL + bs));
    }
    }
    // ------------------------------------------------------------ epilogue
    const bool have = nst > 0 && !*err && mbar_wait(BAR(D_FULL), 0);
    if (nst > 0 && !have) *err = 1;
    tc_fence_after();
    const int q = warp & 3;               // TMEM lane quarter of this warp
    const int chalf = (warp - 2) >> 2;    // columns [256*chalf, 256*chalf + 256)
    // KG = 1: the halves are words 0-255 / 256-511 of one group; KG = 2: two groups
    const unsigned o_lo = 8 * (g + (KG == 2 ? chalf : 0)) + 2 * q, o_hi = o_lo + 1;
    for (int c = 8 * chalf; c < 8 * chalf + 8; c++) {
      uint32_t r[32];
      if (have) {
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + 32 * c, r);
      } else {
#pragma unroll
        for (int j = 0; j < 32; j++) r[j] = 0;
      }
      uint32_t mine = 0;
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, r[j] & 1u);
        if (lane == j) mine = bal;
      }
      if (!have) continue;
      const unsigned widx = 32 * (KG == 2 ? c - 8 * chalf : c) + lane;  // word within the tile
      // pair lanes into 32-bit words: even lane holds words widx, widx+1
      const uint32_t nb = __shfl_down_sync(0xFFFFFFFFu, mine, 1);
      if ((lane & 1) || widx >= words_valid) continue;
      const size_t wbyte = 2 * (w0 + widx);
      const size_t nbytes = min((size_t)4, slice_bytes - wbyte);
#pragma unroll
      for (int hsel = 0; hsel < 2; hsel++) {
        const unsigned o = hsel ? o_hi : o_lo;
        if (o >= n_out) continue;
        uint32_t val = hsel ? ((mine >> 16) | (nb & 0xFFFF0000u)) : ((mine & 0xFFFFu) | (nb << 16));
        uint8_t* dst = out + (size_t)o * out_stride + wbyte;
        if (nbytes >= 4) {
          if (mode == 2) {
            if (val) atomicXor(reinterpret_cast<uint32_t*>(dst), val);
          } else if (mode == 1) {
            *reinterpret_cast<uint32_t*>(dst) ^= val;
          } else {
            *reinterpret_cast<uint32_t*>(dst) = val;
          }
        } else {
          if (mode == 2) {
            uint32_t m = nbytes >= 4 ? 0xFFFFFFFFu : ((1u << (8 * nbytes)) - 1u);
            if (val & m) atomicXor(reinterpret_cast<uint32_t*>(dst), val & m);
          } else {
            for (size_t bb = 0; bb < nbytes; bb++) {
              uint8_t nbv = (uint8_t)(val >> (8 * bb));
              dst[bb] = mode == 1 ? (uint8_t)(dst[bb] ^ nbv) : nbv;
            }
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
  if (threadIdx.x == 0 && *err) atomicOr(status, 1);
}

static uint64_t tiles16(const Gf16TcJob& j) { return (uint64_t)j.groups * j.wt; }

}  // namespace tc16

// ============================================================================
// The same product on the block-scaled FP4 path (tcgen05.mma kind::mxf4).
//
// A operands are e2m1 values 0 or 1.0 (nibbles 0x0 / 0x2), two per byte; B
// operands are 0 or a power of two, cancelled by the block scale factors
// (ue8m0), so each MMA adds exact integer counts into fp32 accumulators
// (counts stay below 16 * 32768 < 2^23).  The parity of a count is read by
// adding 2^23: the sum's lowest mantissa bit is the count's lowest bit.  Half
// the operand bytes of the int8 form per GF(2) product and the FP4 rate of
// the tensor pipe.
//
// Bit selection: e2m1 codes are not parities of their value, so a B element
// must be 0 or one fixed nonzero value per scale block.  Bit j of each nibble
// of a word, masked in place, is such a value: w & 0x1111 -> 0 / 0.5 (0x1),
// w & 0x2222 -> 0 / 1.0 (0x2), w & 0x4444 -> 0 / 2.0 (0x4); bit 3 (0x8 is
// -0) is shifted down first, (w >> 1) & 0x4444 -> 0 / 2.0.  The MMA step j
// reads only elements of selection j, so its B scale factor 1 / v_j makes
// every nonzero product exactly 1: 2.0 for j = 0, 1.0 for j = 1, 0.5 for j = 2
// and 3 (three sets of B scale columns, A scales 1.0).  With
//   A[(o,b)][(j, i, m)] = 1.0 * bit_b(c[o][i] * x^(4m + j))
//   B[w][(j, i, m)]     = v_j * bit_(4m + j)(in_i[w])     (v_j = 0.5, 1, 2, 2)
// D[(o,b)][w] counts the terms of bit b of out[o][w].  A stage is 16 inputs:
// K = 256 elements = one 128-byte (swizzled) row; the 64-element MMA step j
// covers 32 bytes: inputs 0-7 then 8-15, two u32 words (two inputs) each.
//
// CTA tile: KG = 2 -> 16 outputs x 240 words (two accumulators of N = 240,
// one per output group, sharing each B tile); KG = 1 -> 8 outputs x 480 words
// (two accumulators of N = 240 on the two halves of the B tile, sharing each
// A tile).  TMEM: accumulators at columns 0 and 256 (240 each); scale
// factors A 1.0 in columns 240-243, B 2.0 in 248-255, 1.0 in 496-503, 0.5 in
// 504-511 (8-column B sets on 8-column boundaries).  Warp roles and bounded
// waits as in the int8 kernel.
namespace tc16f4 {
using namespace pp::tc;

constexpr int kStageIn = 16;        // inputs per stage
constexpr int kABytes = 128 * 128;  // A tile of one output group: 128 rows x 128 B
constexpr int kThreads = 320;
constexpr int kExp = 256;
constexpr int kN = 240;             // words per accumulator
// scale-factor columns: A (4 columns), B for selections 0, 1 and 2-3 (8 columns each)
constexpr uint32_t kSfaCol = 240, kSfb0Col = 248, kSfb1Col = 496, kSfb2Col = 504;

// ring depths (A tiles + raw rows, B tiles); the two-group tile's can be set
// at build time for measurements
#ifndef PP_F4_LD2
#define PP_F4_LD2 4
#endif
#ifndef PP_F4_BS2
#define PP_F4_BS2 2
#endif
template <int KG>
struct Shape {
  static constexpr int kLd = KG == 2 ? PP_F4_LD2 : 3;
  static constexpr int kBs = KG == 2 ? PP_F4_BS2 : 2;
  static constexpr int kWords = KG == 2 ? kN : 2 * kN;
  static constexpr int kAStage = KG * kABytes;
  static constexpr int kBBytes = kWords * 128;
  static constexpr int kRawBytes = kStageIn * kWords * 2;
  static constexpr int kOffA = 0;
  static constexpr int kOffB = kLd * kAStage;
  static constexpr int kOffRaw = kOffB + kBs * kBBytes;
  static constexpr int kOffBar = kOffRaw + kLd * kRawBytes;
  static constexpr int kSmemBytes = kOffBar + 256 + 1024;
};
static_assert(Shape<1>::kSmemBytes <= 227 * 1024 && Shape<2>::kSmemBytes <= 227 * 1024, "shared memory");
static_assert(Shape<1>::kOffB % 1024 == 0 && Shape<2>::kOffB % 1024 == 0 && (kN * 128) % 1024 == 0,
              "operand tiles start on 1024-byte swizzle atoms");
// raw rows arrive as tensor-map boxes of kStageIn rows x kBox bytes: a word
// tile's 2 * kWords bytes are 2 (KG = 2) or 4 (KG = 1) boxes, box b of a ring
// slot at b * kBoxStage (a multiple of 128 bytes), row ii of a box at ii * kBox
constexpr int kBox = 240;
constexpr int kBoxStage = kStageIn * kBox;
static_assert(kBoxStage % 128 == 0 && Shape<1>::kOffRaw % 128 == 0 && Shape<2>::kOffRaw % 128 == 0 &&
                  Shape<1>::kRawBytes % 128 == 0 && Shape<2>::kRawBytes % 128 == 0,
              "box destinations on 128-byte boundaries");

// instruction descriptor, block-scaled kinds: A/B e2m1 (mxf4 format 1), both
// K-major, N = 240, scale factors ue8m0, M = 128, dense K = 64
constexpr uint32_t kIdesc = (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) | (1u << 23) | ((128u >> 4) << 24);

PP_D void mma_f4(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate, uint32_t sfa, uint32_t sfb) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %6, [%4], [%5], p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(accumulate), "r"(sfa), "r"(sfb), "r"(kIdesc)
      : "memory");
}

// A operand: nibbles 0x2 (1.0) where bit (4m + j) of each 16-bit half of p is set
PP_D uint32_t pick4(uint32_t p, int j) { return ((p >> j) & 0x11111111u) << 1; }
// selection j of the B operand: nibble m holds bit (4m + j) of p as 0 or v_j
// (0x1 = 0.5, 0x2 = 1.0, 0x4 = 2.0, 0x4 = 2.0 for j = 0..3)
PP_D uint32_t sel4(uint32_t p, int j) {
  return j == 3 ? (p >> 1) & 0x44444444u : p & (0x11111111u << j);
}

// A tiles: for output group g and stage s (inputs 16s..16s+15) a 16 KiB tile
// in the canonical K-major 128-byte-swizzled layout: row m = 16*oo + b; the
// 16-byte chunk 2j + h holds, for inputs 8h..8h+7 (two per 32-bit word), the
// nibbles 2*bit_(4m+j) of Q_b(c[8g+oo][16s+8h+ii]) (bit e of Q_b(c) = bit b of
// c * x^e, the nibble table of the int8 expansion).
__global__ void __launch_bounds__(128)
k_gf16_f4_expand_coeffs(const uint16_t* __restrict__ coeffs, size_t ldc, unsigned n_in, unsigned n_out,
                        unsigned n_stages, uint8_t* __restrict__ a_exp) {
  __shared__ __align__(16) uint16_t T[4 * 16 * 16];
  reinterpret_cast<uint4*>(T)[threadIdx.x] = reinterpret_cast<const uint4*>(tc16::g_gf16_qtab)[threadIdx.x];
  __syncthreads();
  const unsigned m = threadIdx.x, oo = m >> 4, b = m & 15;
  const size_t tiles = (size_t)((n_out + 7) / 8) * n_stages;
  for (size_t gs = blockIdx.x; gs < tiles; gs += gridDim.x) {  // gs = g * n_stages + s
    const unsigned s = (unsigned)(gs % n_stages), g = (unsigned)(gs / n_stages);
    const unsigned o = 8 * g + oo;
    uint32_t P[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int ii = 0; ii < kStageIn; ii++) {
      const unsigned i = kStageIn * s + ii;
      const uint32_t c = (o < n_out && i < n_in) ? coeffs[(size_t)o * ldc + i] : 0;
      const uint32_t q = (uint32_t)T[((c & 15) << 4) + b] ^ T[256 + (((c >> 4) & 15) << 4) + b] ^
                         T[512 + (((c >> 8) & 15) << 4) + b] ^ T[768 + ((c >> 12) << 4) + b];  // Q_b(c)
      P[ii >> 1] |= q << (16 * (ii & 1));
    }
    // warp stores of 512 contiguous bytes: lane L writes 16-byte slot L of
    // store k = row 4k + L/8 of the warp, physical chunk L%8 (logical chunk
    // (L%8) ^ (row%8) = 2j + h), from the words of the lane that built the row
    const unsigned lane = m & 31;
    uint8_t* wbase = a_exp + gs * kABytes + (m >> 5) * 4096;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const unsigned r = 4 * k + (lane >> 3), lc = (lane & 7) ^ (r & 7), j = lc >> 1, h = lc & 1;
      uint32_t w[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const uint32_t lo = __shfl_sync(0xFFFFFFFFu, P[t], r), hi = __shfl_sync(0xFFFFFFFFu, P[4 + t], r);
        w[t] = pick4(h ? hi : lo, (int)j);
      }
      *reinterpret_cast<uint4*>(wbase + 512 * k + 16 * lane) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

template <int KG>
__global__ void __launch_bounds__(kThreads, 1)
k_gf16_muladd_f4(const __grid_constant__ Gf16TcBatch batch, const __grid_constant__ Gf16TcMaps maps,
                 int* __restrict__ status) {
  using S = Shape<KG>;
  constexpr int kWords = S::kWords, kBBytes = S::kBBytes, kRawBytes = S::kRawBytes, kAStage = S::kAStage;
  constexpr int kOffA = S::kOffA, kOffB = S::kOffB, kOffRaw = S::kOffRaw, kOffBar = S::kOffBar;
  constexpr int kLd = S::kLd, kBs = S::kBs;
  const TcSeg sg = tc_item(&batch, blockIdx.x);
  const Gf16TcJob J = pinned_job(batch.job[sg.job]);
  const unsigned n_in = J.n_in;
  const size_t slice_bytes = J.slice_bytes;
  const uint8_t* __restrict__ a_exp = J.a_exp;
  const unsigned n_stages_total = J.a_stride;
  const unsigned n_out = J.n_out;
  uint8_t* __restrict__ out = J.out;
  const size_t out_stride = J.out_stride;
  const int mode = sg.mode;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t base_s = smem_addr(smem_raw);
  const uint32_t pad = ((base_s + 1023) & ~1023u) - base_s;
  uint8_t* smem = smem_raw + pad;
  const uint32_t sA = base_s + pad + kOffA, sB = base_s + pad + kOffB, sRaw = base_s + pad + kOffRaw;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
  const uint32_t bar0 = smem_addr(bars);
  enum {
    A_FULL = 0,
    RAW_FULL = A_FULL + kLd,
    A_EMPTY = RAW_FULL + kLd,
    RAW_EMPTY = A_EMPTY + kLd,
    B_FULL = RAW_EMPTY + kLd,
    B_EMPTY = B_FULL + kBs,
    D_FULL = B_EMPTY + kBs,
    DONE = D_FULL + 1,
    NBARS = DONE + 1
  };
  static_assert(8 * NBARS + 16 <= 256, "barrier area");
  auto BAR = [&](int k) { return bar0 + 8u * (uint32_t)k; };
  volatile uint32_t* tmem_holder = reinterpret_cast<volatile uint32_t*>(smem + kOffBar + 8 * NBARS);
  volatile int* err = reinterpret_cast<volatile int*>(smem + kOffBar + 8 * NBARS + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned g = (unsigned)(sg.tile % J.groups) * KG;  // first output group of the CTA
  const size_t w0 = (size_t)(sg.tile / J.groups) * kWords;
  const unsigned st_begin = sg.st0;
  const unsigned nst = sg.st1 - sg.st0;
  const size_t total_words = (slice_bytes + 1) / 2;
  const unsigned words_valid = (unsigned)min((size_t)kWords, total_words - w0);
  const size_t tile_bytes_valid = min((size_t)kWords * 2, slice_bytes - 2 * w0);
  const unsigned n_box = (unsigned)((tile_bytes_valid + kBox - 1) / kBox);
  const void* raw_map = &maps.raw[sg.job];

  if (threadIdx.x == 0) {
    for (int k = 0; k < NBARS; k++) {
      const bool by_expanders = (k >= RAW_EMPTY && k < RAW_EMPTY + kLd) || (k >= B_FULL && k < B_FULL + kBs);
      mbar_init(BAR(k), by_expanders ? (uint32_t)kExp : 1u);
    }
    *err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr((const void*)tmem_holder)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  if (warp >= 2 && warp < 6) {
    // scale factors (ue8m0: 0x80 = 2.0, 0x7F = 1.0, 0x7E = 0.5) in this warp's
    // lane quarter: columns 240-255 = A 1.0 (240-243), unused, B 2.0 (248-255);
    // columns 496-511 = B 1.0 (496-503), B 0.5 (504-511)
    const uint32_t q = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t two = 0x80808080u, one = 0x7F7F7F7Fu, half = 0x7E7E7E7Eu;
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%2,%2,%2,%2,%2,%2,%2,%2};" ::"r"(
            tmem + q + kSfaCol),
        "r"(one), "r"(two)
        : "memory");
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%2,%2,%2,%2,%2,%2,%2,%2};" ::"r"(
            tmem + q + kSfb1Col),
        "r"(one), "r"(half)
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      tma_prefetch_map(raw_map);
      unsigned issued = 0;
      for (unsigned k = 0; k < nst && !*err; k++) {
        const unsigned sl = k % kLd, use = k / kLd;
        if (k >= kLd) {
          if (!mbar_wait(BAR(A_EMPTY + sl), (use - 1) & 1) || !mbar_wait(BAR(RAW_EMPTY + sl), (use - 1) & 1)) {
            *err = 1;
            break;
          }
        }
        const unsigned st = st_begin + k;
        mbar_expect_tx(BAR(A_FULL + sl), kAStage);
#pragma unroll
        for (int gg = 0; gg < KG; gg++)
          bulk_g2s(sA + sl * kAStage + gg * kABytes, a_exp + ((size_t)(g + gg) * n_stages_total + st) * kABytes,
                   kABytes, BAR(A_FULL + sl));
        // the stage's rows: one box per kBox bytes of the tile that start
        // inside the slice (rows past the last input arrive as zeros)
        mbar_expect_tx(BAR(RAW_FULL + sl), n_box * kBoxStage);
        for (unsigned b = 0; b < n_box; b++)
          tma_load_2d(sRaw + sl * kRawBytes + b * kBoxStage, raw_map, (int)(2 * w0) + (int)b * kBox,
                      (int)(st * kStageIn), BAR(RAW_FULL + sl));
        issued = k + 1;
      }
      if (*err) {
        for (unsigned k = issued > (unsigned)kLd ? issued - kLd : 0; k < issued; k++) {
          mbar_wait(BAR(A_FULL + k % kLd), (k / kLd) & 1);
          mbar_wait(BAR(RAW_FULL + k % kLd), (k / kLd) & 1);
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t sfa = tmem + kSfaCol;
      for (unsigned k = 0; k < nst; k++) {
        const unsigned sl = k % kLd, bs = k % kBs;
        if (*err || !mbar_wait(BAR(A_FULL + sl), (k / kLd) & 1) || !mbar_wait(BAR(B_FULL + bs), (k / kBs) & 1)) {
          *err = 1;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
#pragma unroll
          for (int nn = 0; nn < 2; nn++) {
            // KG = 2: one word tile, two groups; KG = 1: one group, two word halves
            const uint32_t a_off = KG == 2 ? nn * kABytes : 0;
            const uint32_t b_off = KG == 2 ? 0 : nn * (kN * 128);
            mma_f4(tmem + nn * 256, sw128_desc(sA + sl * kAStage + a_off + 32 * kk),
                   sw128_desc(sB + bs * kBBytes + b_off + 32 * kk), (k > 0 || kk > 0) ? 1u : 0u, sfa,
                   tmem + (kk == 0 ? kSfb0Col : kk == 1 ? kSfb1Col : kSfb2Col));
          }
        }
        mma_commit(BAR(A_EMPTY + sl));
        mma_commit(BAR(B_EMPTY + bs));
      }
      if (!*err) mma_commit(BAR(D_FULL));
      mma_commit(BAR(DONE));
      if (!mbar_wait(BAR(DONE), 0)) *err = 1;
    }
  } else {
    // ------------------------------------------------------------ expanders
    const int e = threadIdx.x - 64;  // 0..255
    const bool odd_tail = (slice_bytes & 1) && (w0 + kWords >= total_words);
    const unsigned last_word = (unsigned)(total_words - 1 - w0);
    // KG = 2 (240 words): thread e < 240 builds word row e, 16-bit loads.
    // KG = 1 (480 words): thread e < 240 builds the adjacent rows 2e, 2e+1 from
    // one 32-bit load per input (byte permutes split the two words); threads
    // with bit 2 of e set store their odd row first, so each 128-bit store
    // phase of 8 threads covers eight distinct rows of a swizzle atom.
    const unsigned n0 = KG == 2 ? (unsigned)e : 2u * (unsigned)e;
    const unsigned sw = KG == 2 ? 0u : ((unsigned)e >> 2) & 1u;
    const bool active = e < kN;
    const unsigned rb = (2 * n0 / kBox) * kBoxStage + (2 * n0) % kBox;  // word n0 of row 0 within a ring slot
    uint32_t mask = 0;
    if (KG == 2) {
      if (n0 < words_valid) mask = 0xFFFFu;
      if (odd_tail && n0 == last_word) mask &= 0x00FFu;
    } else {
      if (n0 < words_valid) mask = 0xFFFFu;
      if (n0 + 1 < words_valid) mask |= 0xFFFF0000u;
      if (odd_tail) {
        if (n0 == last_word) mask &= 0xFFFF00FFu;
        else if (n0 + 1 == last_word) mask &= 0x00FFFFFFu;
      }
    }
    for (unsigned k = 0; k < nst; k++) {
      const unsigned sl = k % kLd, bs = k % kBs;
      if (*err || !mbar_wait(BAR(RAW_FULL + sl), (k / kLd) & 1)) {
        *err = 1;
        break;
      }
      const unsigned i0 = (st_begin + k) * kStageIn;
      const unsigned ni = min((unsigned)kStageIn, n_in - i0);
      // explicit shared-memory loads (a generic load would resolve its
      // address space at run time and wait on the long scoreboard)
      const uint32_t raw = sRaw + sl * kRawBytes;
      uint32_t P0[8], P1[8];  // row n0 (and n0 + 1): inputs (2q, 2q+1) as the halves of word q
#pragma unroll
      for (int q = 0; q < 8; q++) {
        if (KG == 2) {
          const uint32_t lo = (unsigned)(2 * q) < ni && active ? lds16(raw + (2 * q) * kBox + rb) : 0u;
          const uint32_t hi =
              (unsigned)(2 * q + 1) < ni && active ? lds16(raw + (2 * q + 1) * kBox + rb) : 0u;
          P0[q] = (lo & mask) | ((hi & mask) << 16);
          P1[q] = 0;
        } else {
          const uint32_t a = (unsigned)(2 * q) < ni && active ? lds32(raw + (2 * q) * kBox + rb) & mask : 0u;
          const uint32_t b =
              (unsigned)(2 * q + 1) < ni && active ? lds32(raw + (2 * q + 1) * kBox + rb) & mask : 0u;
          P0[q] = __byte_perm(a, b, 0x5410);  // word n0 of both inputs
          P1[q] = __byte_perm(a, b, 0x7632);  // word n0 + 1
        }
      }
      mbar_arrive(BAR(RAW_EMPTY + sl));
      if (k >= (unsigned)kBs && !mbar_wait(BAR(B_EMPTY + bs), (k / kBs - 1) & 1)) {
        *err = 1;
        break;
      }
      const uint32_t bt = sB + bs * kBBytes;
      if (active) {
#pragma unroll
        for (int rr = 0; rr < (KG == 2 ? 1 : 2); rr++) {
          const unsigned n = n0 + (rr ^ sw);
          const uint32_t* P = (rr ^ sw) ? P1 : P0;
          const uint32_t row = bt + (n >> 3) * 1024 + (n & 7) * 128, r7 = n & 7;
#pragma unroll
          for (int j = 0; j < 4; j++) {
            sts128(row + (((2 * j) ^ r7) << 4), sel4(P[0], j), sel4(P[1], j), sel4(P[2], j), sel4(P[3], j));
            sts128(row + (((2 * j + 1) ^ r7) << 4), sel4(P[4], j), sel4(P[5], j), sel4(P[6], j), sel4(P[7], j));
          }
        }
      }
      fence_async_smem();
      mbar_arrive(BAR(B_FULL + bs));
    }
    // ------------------------------------------------------------ epilogue
    const bool have = nst > 0 && !*err && mbar_wait(BAR(D_FULL), 0);
    if (nst > 0 && !have) *err = 1;
    tc_fence_after();
    const int q = warp & 3;             // TMEM lane quarter of this warp
    const int chalf = (warp - 2) >> 2;  // accumulator 0 (columns 0-239) or 1 (256-495)
    // KG = 2: accumulator = output group; KG = 1: accumulator = word half
    const unsigned o_lo = 8 * (g + (KG == 2 ? chalf : 0)) + 2 * q, o_hi = o_lo + 1;
    const unsigned wbase = KG == 2 ? 0u : (unsigned)chalf * kN;
    for (int c = 0; c < (kN + 31) / 32; c++) {
      uint32_t r[32];
      if (have) {
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + 256 * chalf + 32 * c, r);
      } else {
#pragma unroll
        for (int j = 0; j < 32; j++) r[j] = 0;
      }
      uint32_t mine = 0;
#pragma unroll
      for (int j = 0; j < 32; j++) {
        // exact count f < 2^23: the lowest mantissa bit of f + 2^23 is f's lowest bit
        const uint32_t bit = __float_as_uint(__fadd_rn(__uint_as_float(r[j]), 8388608.0f)) & 1u;
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, bit);
        if (lane == j) mine = bal;
      }
      if (!have) continue;
      const unsigned wcol = 32 * c + lane;   // column of the accumulator
      const unsigned widx = wbase + wcol;    // word within the tile
      const uint32_t nb = __shfl_down_sync(0xFFFFFFFFu, mine, 1);
      if ((lane & 1) || wcol >= (unsigned)kN || widx >= words_valid) continue;
      const size_t wbyte = 2 * (w0 + widx);
      const size_t nbytes = min((size_t)4, slice_bytes - wbyte);
#pragma unroll
      for (int hsel = 0; hsel < 2; hsel++) {
        const unsigned o = hsel ? o_hi : o_lo;
        if (o >= n_out) continue;
        uint32_t val = hsel ? ((mine >> 16) | (nb & 0xFFFF0000u)) : ((mine & 0xFFFFu) | (nb << 16));
        uint8_t* dst = out + (size_t)o * out_stride + wbyte;
        if (nbytes >= 4) {
          if (mode == 2) {
            if (val) atomicXor(reinterpret_cast<uint32_t*>(dst), val);
          } else if (mode == 1) {
            *reinterpret_cast<uint32_t*>(dst) ^= val;
          } else {
            *reinterpret_cast<uint32_t*>(dst) = val;
          }
        } else {
          if (mode == 2) {
            const uint32_t mm = (1u << (8 * nbytes)) - 1u;
            if (val & mm) atomicXor(reinterpret_cast<uint32_t*>(dst), val & mm);
          } else {
            for (size_t bb = 0; bb < nbytes; bb++) {
              const uint8_t nbv = (uint8_t)(val >> (8 * bb));
              dst[bb] = mode == 1 ? (uint8_t)(dst[bb] ^ nbv) : nbv;
            }
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
  if (threadIdx.x == 0 && *err) atomicOr(status, 1);
}

}  // namespace tc16f4

// Operand format of the GF(2^16) tensor-core path, fixed for the process at
// first use: block-scaled FP4 (kind::mxf4, 16 inputs per stage) unless
// PARPAR_B200_GF16_TC=i8 selects the int8 form (8 inputs per stage).  Every
// expansion and launch of the process uses the same format, so resident tiles
// always match the kernel that reads them.
static bool gf16_tc_use_f4() {
  static const bool f4 = [] {
    const char* e = getenv("PARPAR_B200_GF16_TC");
    return !(e && strcmp(e, "i8") == 0);
  }();
  return f4;
}

unsigned gf16_tc_stage_inputs() { return gf16_tc_use_f4() ? tc16f4::kStageIn : tc16::kStageIn; }

cudaError_t gf16_tc_tables_init(cudaStream_t s) {
  if (device_done(tc16::g_qtab_ready)) return cudaSuccess;
  cudaError_t e = tc16::qtab_on(s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) device_mark(tc16::g_qtab_ready);
  return e;
}

size_t gf16_tc_coeff_bytes(unsigned n_in, unsigned n_out) {
  const unsigned si = gf16_tc_stage_inputs();
  return (size_t)((n_out + 7) / 8) * ((n_in + si - 1) / si) * tc16::kABytes;
}

cudaError_t launch_gf16_tc_expand(const uint16_t* d_coeffs, size_t ldc, unsigned n_in, unsigned n_out,
                                  uint8_t* d_aexp, cudaStream_t s) {
  const unsigned si = gf16_tc_stage_inputs();
  const unsigned n_stages = (n_in + si - 1) / si;
  const size_t tiles = (size_t)((n_out + 7) / 8) * n_stages;
  if (!tiles) return cudaSuccess;
  if (cudaError_t e = tc16::qtab_on(s)) return e;
  unsigned blocks = (unsigned)std::min<size_t>(tiles, 148 * 32);
  if (gf16_tc_use_f4())
    tc16f4::k_gf16_f4_expand_coeffs<<<blocks, 128, 0, s>>>(d_coeffs, ldc, n_in, n_out, n_stages, d_aexp);
  else
    tc16::k_gf16_tc_expand_coeffs<<<blocks, 128, 0, s>>>(d_coeffs, ldc, n_in, n_out, n_stages, d_aexp);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_gf16_tc_batch(Gf16TcBatch& b, int sms, int* d_status, cudaStream_t s) {
  static std::atomic<uint64_t> attr{0};
  const bool f4 = gf16_tc_use_f4();
  if (!device_done(attr)) {
    cudaError_t e = f4 ? cudaFuncSetAttribute(tc16f4::k_gf16_muladd_f4<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              tc16f4::Shape<1>::kSmemBytes)
                       : cudaFuncSetAttribute(tc16::k_gf16_muladd_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              tc16::Shape<1>::kSmemBytes);
    if (e == cudaSuccess)
      e = f4 ? cudaFuncSetAttribute(tc16f4::k_gf16_muladd_f4<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    tc16f4::Shape<2>::kSmemBytes)
             : cudaFuncSetAttribute(tc16::k_gf16_muladd_tc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    tc16::Shape<2>::kSmemBytes);
    if (e != cudaSuccess) return e;
    device_mark(attr);
  }
  // two output groups per CTA when every job's outputs pair up into groups of 16
  int kg = 2;
  for (uint32_t j = 0; j < b.n_jobs; j++)
    if (b.job[j].n_out && b.job[j].slice_bytes && b.job[j].n_in && (b.job[j].n_out + 7) / 8 % 2) kg = 1;
  const size_t words = f4 ? (kg == 2 ? tc16f4::Shape<2>::kWords : tc16f4::Shape<1>::kWords)
                          : (kg == 2 ? tc16::Shape<2>::kWords : tc16::Shape<1>::kWords);
  const unsigned si = gf16_tc_stage_inputs();
  uint32_t m = 0;
  for (uint32_t j = 0; j < b.n_jobs; j++) {
    Gf16TcJob& J = b.job[j];
    if (!J.n_out || !J.slice_bytes) continue;
    J.n_stages = (J.n_in + si - 1) / si;
    if (!J.a_stride) J.a_stride = J.n_stages;
    J.groups = (J.n_out + 7) / 8 / (unsigned)kg;  // output tiles of a CTA: groups (kg = 1) or group pairs
    const size_t wt = ceil_div((J.slice_bytes + 1) / 2, words);
    if (wt > 0xFFFFFFFFu) return cudaErrorInvalidValue;
    J.wt = (uint32_t)wt;
    if (!J.n_in) {
      if (J.accumulate) continue;
      cudaError_t e = cudaMemset2DAsync(J.out, J.out_stride, 0, J.slice_bytes, J.n_out, s);
      note_launch();
      if (e != cudaSuccess) return e;
      continue;
    }
    b.job[m++] = J;
  }
  b.n_jobs = m;
  if (!m) return cudaGetLastError();
  // a box's byte column is a 32-bit coordinate: slices of 2 GiB and more run
  // as separate launches over column bands of 1 GiB (16-byte aligned starts)
  constexpr size_t kBand = size_t(1) << 30;
  m = 0;
  for (uint32_t j = 0; j < b.n_jobs; j++) {
    const Gf16TcJob J = b.job[j];
    if (J.slice_bytes < (size_t(1) << 31)) {
      b.job[m++] = J;
      continue;
    }
    for (size_t c0 = 0; c0 < J.slice_bytes; c0 += kBand) {
      Gf16TcBatch one{};
      one.n_jobs = 1;
      one.job[0] = J;
      one.job[0].in = J.in + c0;
      one.job[0].out = J.out + c0;
      one.job[0].slice_bytes = std::min(kBand, J.slice_bytes - c0);
      one.job[0].a_stride = J.a_stride;
      if (cudaError_t e = launch_gf16_tc_batch(one, sms, d_status, s)) return e;
    }
  }
  b.n_jobs = m;
  if (!m) return cudaGetLastError();
  Gf16TcMaps maps;
  for (uint32_t j = 0; j < m; j++) {
    const Gf16TcJob& J = b.job[j];
    if (cudaError_t e = tma_encode_rows(&maps.raw[j], J.in, J.slice_bytes, J.n_in, J.in_stride,
                                        f4 ? tc16f4::kBox : tc16::kBox, si))
      return e;
  }
  // FP4: at most 16,384 stages (262,144 inputs) per item, so a count stays below 16 * 2^18 < 2^23
  const uint64_t ctas = tc_batch_plan(b, tc16::tiles16, sms, f4 ? 16384u : 0u);
  if (ctas > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
  for (uint32_t j = 0; j < m; j++) {
    const Gf16TcJob& J = b.job[j];
    if (J.splits == 1 || J.accumulate) continue;
    cudaError_t e = cudaMemset2DAsync(J.out, J.out_stride, 0, J.slice_bytes, J.n_out, s);
    note_launch();
    if (e != cudaSuccess) return e;
  }
  if (f4 && kg == 2)
    tc16f4::k_gf16_muladd_f4<2><<<(unsigned)ctas, tc16f4::kThreads, tc16f4::Shape<2>::kSmemBytes, s>>>(b, maps, d_status);
  else if (f4)
    tc16f4::k_gf16_muladd_f4<1><<<(unsigned)ctas, tc16f4::kThreads, tc16f4::Shape<1>::kSmemBytes, s>>>(b, maps, d_status);
  else if (kg == 2)
    tc16::k_gf16_muladd_tc<2><<<(unsigned)ctas, tc16::kThreads, tc16::Shape<2>::kSmemBytes, s>>>(b, maps, d_status);
  else
    tc16::k_gf16_muladd_tc<1><<<(unsigned)ctas, tc16::kThreads, tc16::Shape<1>::kSmemBytes, s>>>(b, maps, d_status);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_gf16_muladd_tc(const uint8_t* d_in, size_t in_stride, unsigned n_in, size_t slice_bytes,
                                  const uint8_t* d_aexp, unsigned n_out, uint8_t* d_out, size_t out_stride,
                                  bool accumulate, int sms, int* d_status, cudaStream_t s, unsigned a_stride) {
  if (!n_out || !slice_bytes) return cudaSuccess;
  Gf16TcBatch b{};
  b.n_jobs = 1;
  Gf16TcJob& J = b.job[0];
  J.in = d_in;
  J.in_stride = in_stride;
  J.a_exp = d_aexp;
  J.out = d_out;
  J.out_stride = out_stride;
  J.slice_bytes = slice_bytes;
  J.n_in = n_in;
  J.n_out = n_out;
  J.accumulate = accumulate ? 1 : 0;
  J.a_stride = a_stride;
  return launch_gf16_tc_batch(b, sms, d_status, s);
}

}  // namespace pp
