// Block hashes on the device, over slices that are already resident in HBM.
//
//  * PAR2 input-slice checksums: MD5 then CRC32 (little-endian) of each slice
//    followed by zero padding up to the slice size -- the 20-byte IFSC entry
//    that HasherInput::getBlock(md5crc, zeroPad) produces
//    (hasher/hasher_input_base.h:104-117).  MD5 is a serial chain within a
//    message, so one thread owns one slice and runs MD5 and CRC32 side by side
//    on the same 64-byte block (one load of each byte, two independent
//    dependency chains for the scheduler to interleave).
//  * BLAKE3 of "prefix || block" messages: the PAR3 data-packet checksum of
//    lib/par3gen.js:1001-1017 (prefix = the packet's 24 post-checksum header
//    bytes + u64le block index) and the recovery packets of
//    src/gf64_addon.cc:2884-2934 (prefix also carries u64le block count 1).
//    One thread per 1 KiB chunk computes the chunk chaining value; the parent
//    nodes are merged level by level (pairing adjacent nodes, an odd last node
//    carried up), which is exactly BLAKE3's left-complete tree.
#include <cuda_runtime.h>

#include <cstdint>

#include "pp_internal.h"

namespace pp {
namespace {

// ----------------------------------------------------------------- MD5
// RFC 1321.  Step constants floor(|sin(i + 1)| * 2^32).
__constant__ uint32_t c_md5k[64] = {
    0xd76aa478u, 0xe8c7b756u, 0x242070dbu, 0xc1bdceeeu, 0xf57c0fafu, 0x4787c62au, 0xa8304613u, 0xfd469501u,
    0x698098d8u, 0x8b44f7afu, 0xffff5bb1u, 0x895cd7beu, 0x6b901122u, 0xfd987193u, 0xa679438eu, 0x49b40821u,
    0xf61e2562u, 0xc040b340u, 0x265e5a51u, 0xe9b6c7aau, 0xd62f105du, 0x02441453u, 0xd8a1e681u, 0xe7d3fbc8u,
    0x21e1cde6u, 0xc33707d6u, 0xf4d50d87u, 0x455a14edu, 0xa9e3e905u, 0xfcefa3f8u, 0x676f02d9u, 0x8d2a4c8au,
    0xfffa3942u, 0x8771f681u, 0x6d9d6122u, 0xfde5380cu, 0xa4beea44u, 0x4bdecfa9u, 0xf6bb4b60u, 0xbebfbc70u,
    0x289b7ec6u, 0xeaa127fau, 0xd4ef3085u, 0x04881d05u, 0xd9d4d039u, 0xe6db99e5u, 0x1fa27cf8u, 0xc4ac5665u,
    0xf4292244u, 0x432aff97u, 0xab9423a7u, 0xfc93a039u, 0x655b59c3u, 0x8f0ccc92u, 0xffeff47du, 0x85845dd1u,
    0x6fa87e4fu, 0xfe2ce6e0u, 0xa3014314u, 0x4e0811a1u, 0xf7537e82u, 0xbd3af235u, 0x2ad7d2bbu, 0xeb86d391u,
};

__device__ __forceinline__ uint32_t rotl(uint32_t x, int s) { return __funnelshift_l(x, x, s); }

// BLAKE3 is bound by the integer ALU pipe (its XORs, rotations and adds all
// issue there) while the FMA pipe idles.  madd is a + b issued as an integer
// multiply-add with a multiplier the compiler cannot see (`one`, a kernel
// argument equal to 1), so it executes on the FMA pipe and leaves the ALU pipe
// to the logic and rotate instructions.  (MD5's adds stay on the ALU: its
// serial chain is latency-bound and the multiply-add is slower there.)
__device__ __forceinline__ uint32_t madd(uint32_t a, uint32_t b, uint32_t one) {
  uint32_t r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(one), "r"(b));
  return r;
}

__device__ __forceinline__ int md5_shift(int i) {
  const int r = i >> 4, k = i & 3;
  if (r == 0) return k == 0 ? 7 : k == 1 ? 12 : k == 2 ? 17 : 22;
  if (r == 1) return k == 0 ? 5 : k == 1 ? 9 : k == 2 ? 14 : 20;
  if (r == 2) return k == 0 ? 4 : k == 1 ? 11 : k == 2 ? 16 : 23;
  return k == 0 ? 6 : k == 1 ? 10 : k == 2 ? 15 : 21;
}

__device__ __forceinline__ void md5_block(uint32_t st[4], const uint32_t m[16]) {
  uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
#pragma unroll
  for (int i = 0; i < 64; i++) {
    uint32_t f;
    int g;
    if (i < 16) {
      f = d ^ (b & (c ^ d));
      g = i;
    } else if (i < 32) {
      f = c ^ (d & (b ^ c));
      g = (5 * i + 1) & 15;
    } else if (i < 48) {
      f = b ^ c ^ d;
      g = (3 * i + 5) & 15;
    } else {
      f = c ^ (b | ~d);
      g = (7 * i) & 15;
    }
    const uint32_t t = d;
    const uint32_t x = a + c_md5k[i] + m[g];  // off the dependency chain
    d = c;
    c = b;
    b = b + rotl(x + f, md5_shift(i));
    a = t;
  }
  st[0] += a;
  st[1] += b;
  st[2] += c;
  st[3] += d;
}

// --------------------------------------------------------------- CRC32
// Reflected CRC-32 (0xEDB88320), slice-by-4.  T_t[e] is the register after
// byte e followed by t zero bytes, from a zero register.  Each table entry is
// stored kCrcCopies times, copy k holding it at word ((t*256 + e) * copies +
// k): lane L reads copy L % copies, so lanes whose indices collide on a bank
// are spread over different banks.
constexpr int kCrcCopies = 16;
constexpr int kCrcWords = 4 * 256 * kCrcCopies;  // 64 KiB
constexpr uint32_t kCrcPoly = 0xEDB88320u;

__device__ __forceinline__ void crc_tables_init(uint32_t* tab) {
  for (int idx = threadIdx.x; idx < 1024; idx += blockDim.x) {
    const int t = idx >> 8;
    uint32_t r = (uint32_t)(idx & 255);
    for (int j = 0; j < 8 * (t + 1); j++) r = (r >> 1) ^ (kCrcPoly & (0u - (r & 1u)));
#pragma unroll
    for (int k = 0; k < kCrcCopies; k++) tab[idx * kCrcCopies + k] = r;
  }
}

__device__ __forceinline__ uint32_t crc_word(uint32_t r, uint32_t w, const uint32_t* tk) {
  const uint32_t x = r ^ w;
  return tk[(3 * 256 + (x & 255u)) * kCrcCopies] ^ tk[(2 * 256 + ((x >> 8) & 255u)) * kCrcCopies] ^
         tk[(1 * 256 + ((x >> 16) & 255u)) * kCrcCopies] ^ tk[(x >> 24) * kCrcCopies];
}

__device__ __forceinline__ uint32_t crc_byte(uint32_t r, uint32_t byte, const uint32_t* tk) {
  return (r >> 8) ^ tk[((r ^ byte) & 255u) * kCrcCopies];
}

// word w of the message: bytes [4w, 4w+4) of the row, zero at and past len
__device__ __forceinline__ uint32_t masked_word(const uint8_t* row, uint64_t o, uint64_t len) {
  if (o + 4 <= len) return *reinterpret_cast<const uint32_t*>(row + o);
  uint32_t v = 0;
  for (uint64_t j = o; j < len && j < o + 4; j++) v |= (uint32_t)row[j] << (8 * (j - o));
  return v;
}

// One thread per slice.  Rows are 16-byte aligned (data and stride).  The
// message is L bytes: the row's first len bytes, then zeros.
// MD5 and / or CRC32 over the whole 64-byte blocks [b0, b1) of a row (all
// inside the data): 16-byte loads, one block prefetched.
template <bool kMd5, bool kCrc>
__device__ __forceinline__ void hash_full_blocks(const uint8_t* row, uint64_t b0, uint64_t b1, uint32_t st[4],
                                                 uint32_t& crc, const uint32_t* tk) {
  uint32_t m[16];
  uint4 nx[4];
  if (b0 < b1) {
#pragma unroll
    for (int q = 0; q < 4; q++) nx[q] = __ldg(reinterpret_cast<const uint4*>(row + 64 * b0) + q);
  }
  for (uint64_t b = b0; b < b1; b++) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      m[4 * q] = nx[q].x;
      m[4 * q + 1] = nx[q].y;
      m[4 * q + 2] = nx[q].z;
      m[4 * q + 3] = nx[q].w;
    }
    if (b + 1 < b1) {
#pragma unroll
      for (int q = 0; q < 4; q++) nx[q] = __ldg(reinterpret_cast<const uint4*>(row + 64 * (b + 1)) + q);
    }
    if constexpr (kCrc) {
#pragma unroll
      for (int w = 0; w < 16; w++) crc = crc_word(crc, m[w], tk);
    }
    if constexpr (kMd5) md5_block(st, m);
  }
}

// The rest of the message after its first `nfull` whole data blocks: the
// remaining L / 64 blocks (data tail, then zero padding), the final partial
// block with the MD5 padding, and the IFSC entry: MD5 to o20[0..16), CRC32
// to o20[16..20).
template <bool kMd5, bool kCrc>
__device__ __forceinline__ void hash_finish(const uint8_t* row, uint64_t len, uint64_t L, uint64_t nfull,
                                            uint32_t st[4], uint32_t crc, const uint32_t* tk, uint8_t* o20) {
  uint32_t m[16];
  const uint64_t nblk = L / 64;
  for (uint64_t b = nfull; b < nblk; b++) {
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = masked_word(row, 64 * b + 4 * w, len);
    if constexpr (kCrc) {
#pragma unroll
      for (int w = 0; w < 16; w++) crc = crc_word(crc, m[w], tk);
    }
    if constexpr (kMd5) md5_block(st, m);
  }
  // final partial block (L % 64 bytes) with the MD5 padding
  const uint32_t tail = (uint32_t)(L % 64);
  const uint64_t t0 = 64 * nblk;
#pragma unroll
  for (int w = 0; w < 16; w++) m[w] = (4u * w < tail) ? masked_word(row, t0 + 4 * w, len) : 0u;
  if constexpr (kCrc) {
#pragma unroll
    for (uint32_t w = 0; w < 16; w++) {
      if (4 * w + 4 <= tail) {
        crc = crc_word(crc, m[w], tk);
      } else if (4 * w < tail) {
#pragma unroll
        for (uint32_t j = 0; j < 3; j++)
          if (4 * w + j < tail) crc = crc_byte(crc, (m[w] >> (8 * j)) & 255u, tk);
      }
    }
    reinterpret_cast<uint32_t*>(o20)[4] = crc ^ 0xFFFFFFFFu;
  }
  if constexpr (kMd5) {
    // clear the bytes at and past `tail` in the last partial word, then 0x80
#pragma unroll
    for (int w = 0; w < 16; w++) {
      const uint32_t lo = 4u * w;
      if (lo < tail && tail < lo + 4) m[w] &= (1u << (8 * (tail - lo))) - 1u;
      if (lo <= tail && tail < lo + 4) m[w] |= 0x80u << (8 * (tail - lo));
    }
    if (tail >= 56) {
      md5_block(st, m);
#pragma unroll
      for (int w = 0; w < 16; w++) m[w] = 0;
    }
    m[14] = (uint32_t)(L << 3);
    m[15] = (uint32_t)(L >> 29);
    md5_block(st, m);
    uint32_t* o = reinterpret_cast<uint32_t*>(o20);
    o[0] = st[0];
    o[1] = st[1];
    o[2] = st[2];
    o[3] = st[3];
  }
}

// MD5 and / or CRC32 of one slice's message (the whole-slice kernels keep
// this single body: the band kernel below uses the split helpers above).
// MD5 and / or CRC32 of one slice's message (the row's first len bytes,
// then zeros up to L bytes); MD5 goes to o20[0..16), CRC32 to o20[16..20).
template <bool kMd5, bool kCrc>
__device__ __forceinline__ void par2_slice_hash(const uint8_t* row, uint64_t len, uint64_t L, const uint32_t* tk,
                                                uint8_t* o20) {
  uint32_t st[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
  uint32_t crc = 0xFFFFFFFFu;
  uint32_t m[16];

  // blocks wholly inside the data: 16-byte loads, one block prefetched
  const uint64_t nfull = len / 64;
  uint4 nx[4];
  if (nfull) {
#pragma unroll
    for (int q = 0; q < 4; q++) nx[q] = __ldg(reinterpret_cast<const uint4*>(row) + q);
  }
  for (uint64_t b = 0; b < nfull; b++) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      m[4 * q] = nx[q].x;
      m[4 * q + 1] = nx[q].y;
      m[4 * q + 2] = nx[q].z;
      m[4 * q + 3] = nx[q].w;
    }
    if (b + 1 < nfull) {
#pragma unroll
      for (int q = 0; q < 4; q++) nx[q] = __ldg(reinterpret_cast<const uint4*>(row + 64 * (b + 1)) + q);
    }
    if constexpr (kCrc) {
#pragma unroll
      for (int w = 0; w < 16; w++) crc = crc_word(crc, m[w], tk);
    }
    if constexpr (kMd5) md5_block(st, m);
  }
  // the rest of the L / 64 whole message blocks: data tail, then zero padding
  const uint64_t nblk = L / 64;
  for (uint64_t b = nfull; b < nblk; b++) {
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = masked_word(row, 64 * b + 4 * w, len);
    if constexpr (kCrc) {
#pragma unroll
      for (int w = 0; w < 16; w++) crc = crc_word(crc, m[w], tk);
    }
    if constexpr (kMd5) md5_block(st, m);
  }
  // final partial block (L % 64 bytes) with the MD5 padding
  const uint32_t tail = (uint32_t)(L % 64);
  const uint64_t t0 = 64 * nblk;
#pragma unroll
  for (int w = 0; w < 16; w++) m[w] = (4u * w < tail) ? masked_word(row, t0 + 4 * w, len) : 0u;
  if constexpr (kCrc) {
#pragma unroll
    for (uint32_t w = 0; w < 16; w++) {
      if (4 * w + 4 <= tail) {
        crc = crc_word(crc, m[w], tk);
      } else if (4 * w < tail) {
#pragma unroll
        for (uint32_t j = 0; j < 3; j++)
          if (4 * w + j < tail) crc = crc_byte(crc, (m[w] >> (8 * j)) & 255u, tk);
      }
    }
    reinterpret_cast<uint32_t*>(o20)[4] = crc ^ 0xFFFFFFFFu;
  }
  if constexpr (kMd5) {
    // clear the bytes at and past `tail` in the last partial word, then 0x80
#pragma unroll
    for (int w = 0; w < 16; w++) {
      const uint32_t lo = 4u * w;
      if (lo < tail && tail < lo + 4) m[w] &= (1u << (8 * (tail - lo))) - 1u;
      if (lo <= tail && tail < lo + 4) m[w] |= 0x80u << (8 * (tail - lo));
    }
    if (tail >= 56) {
      md5_block(st, m);
#pragma unroll
      for (int w = 0; w < 16; w++) m[w] = 0;
    }
    m[14] = (uint32_t)(L << 3);
    m[15] = (uint32_t)(L >> 29);
    md5_block(st, m);
    uint32_t* o = reinterpret_cast<uint32_t*>(o20);
    o[0] = st[0];
    o[1] = st[1];
    o[2] = st[2];
    o[3] = st[3];
  }
}

// kIdx: row i's entry goes to out + 20 * idx[i] (0xFFFF: not hashed); the
// variant without it is the plain whole-slice kernel
template <bool kIdx>
__global__ void __launch_bounds__(128) k_par2_block_hash(const uint8_t* __restrict__ data, size_t stride,
                                                         size_t n, uint64_t L,
                                                         const uint64_t* __restrict__ lengths,
                                                         uint8_t* __restrict__ out,
                                                         const uint16_t* __restrict__ idx) {
  extern __shared__ uint32_t crc_tab[];
  crc_tables_init(crc_tab);
  __syncthreads();
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  size_t o = i;
  if constexpr (kIdx) {
    o = idx[i];
    if (o == 0xFFFF) return;
  }
  const uint64_t len = lengths ? (lengths[i] < L ? lengths[i] : L) : L;
  par2_slice_hash<true, true>(data + i * stride, len, L, crc_tab + (threadIdx.x % kCrcCopies), out + 20 * o);
}

// Few slices (too few threads to fill the GPU): MD5 and CRC32 of a slice in
// two threads of different warps, so each serial chain runs alone instead of
// sharing one thread's in-order instruction stream.  The MD5 chain itself
// (about 2,000 cycles per 64-byte block) then sets the time.  Threads 0-63 of a CTA
// hash slices 64b .. 64b+63 with MD5, threads 64-127 the same slices with
// CRC32 (they read the same bytes at about the same time, served by L1/L2).
template <bool kIdx>
__global__ void __launch_bounds__(128) k_par2_block_hash_split(const uint8_t* __restrict__ data, size_t stride,
                                                               size_t n, uint64_t L,
                                                               const uint64_t* __restrict__ lengths,
                                                               uint8_t* __restrict__ out,
                                                               const uint16_t* __restrict__ idx) {
  extern __shared__ uint32_t crc_tab[];
  crc_tables_init(crc_tab);
  __syncthreads();
  const size_t i = (size_t)blockIdx.x * 64 + (threadIdx.x & 63);
  if (i >= n) return;
  size_t o = i;
  if constexpr (kIdx) {
    o = idx[i];
    if (o == 0xFFFF) return;
  }
  const uint64_t len = lengths ? (lengths[i] < L ? lengths[i] : L) : L;
  if (threadIdx.x < 64)
    par2_slice_hash<true, false>(data + i * stride, len, L, nullptr, out + 20 * o);
  else
    par2_slice_hash<false, true>(data + i * stride, len, L, crc_tab + (threadIdx.x % kCrcCopies), out + 20 * o);
}

// Resumable form over column bands (every row L bytes of data): blocks
// [k0, k1) of every slice, with MD5 and CRC32 in separate warps as above.
// state[5 i ..] holds slice i's MD5 words and CRC32 register between bands;
// the first band starts them, the last one (k1 = L / 64) also hashes the
// final partial block and padding and writes the IFSC entry.  Slices whose
// bytes arrive band by band are hashed as they land: a band's launch takes
// as long as its own blocks, not the whole chain of the slice.
__global__ void __launch_bounds__(128) k_par2_block_hash_band(const uint8_t* __restrict__ data, size_t stride,
                                                              size_t n, uint64_t L, uint64_t k0, uint64_t k1,
                                                              uint32_t* __restrict__ state, uint8_t* __restrict__ out,
                                                              int first, int last) {
  extern __shared__ uint32_t crc_tab[];
  crc_tables_init(crc_tab);
  __syncthreads();
  const size_t i = (size_t)blockIdx.x * 64 + (threadIdx.x & 63);
  if (i >= n) return;
  const uint8_t* row = data + i * stride;
  uint32_t* S = state + 5 * i;
  uint32_t st[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
  uint32_t crc = 0xFFFFFFFFu;
  if (threadIdx.x < 64) {
    if (!first) {
#pragma unroll
      for (int w = 0; w < 4; w++) st[w] = S[w];
    }
    hash_full_blocks<true, false>(row, k0, k1, st, crc, nullptr);
    if (last) {
      hash_finish<true, false>(row, L, L, k1, st, crc, nullptr, out + 20 * i);
    } else {
#pragma unroll
      for (int w = 0; w < 4; w++) S[w] = st[w];
    }
  } else {
    const uint32_t* tk = crc_tab + (threadIdx.x % kCrcCopies);
    if (!first) crc = S[4];
    hash_full_blocks<false, true>(row, k0, k1, st, crc, tk);
    if (last)
      hash_finish<false, true>(row, L, L, k1, st, crc, tk, out + 20 * i);
    else
      S[4] = crc;
  }
}

// PAR2 recovery-slice packet headers (lib/par2.js:517-530 getRecoveryHeader;
// the MD5 fed as in :255-330): 68 bytes per slice -- "PAR2\0PKT", u64le
// packet length (68 + L), MD5 of packet bytes [32, 68 + L) (set id, type
// "PAR 2.0\0RecvSlic", u32le exponent, slice data), set id, type, exponent.
// One thread per slice; the message is 36 prefix bytes then the L data bytes.
struct Par2PktArgs {
  const uint8_t* data;
  size_t stride;
  size_t n;
  uint64_t L;           // slice bytes (multiple of 4)
  uint32_t pre[8];      // set id (4 words), type (4 words)
  const uint16_t* exps;
  uint8_t* out;         // n x 68 bytes
};

__device__ __forceinline__ uint32_t pkt_word(const Par2PktArgs& A, const uint8_t* row, uint32_t ex, uint64_t w) {
  if (w < 8) {  // select with constant indices: the parameter array stays in the constant bank
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < 8; k++)
      if (w == (uint64_t)k) v = A.pre[k];
    return v;
  }
  if (w == 8) return ex;
  const uint64_t o = 4 * (w - 9);
  return o < A.L ? __ldg(reinterpret_cast<const uint32_t*>(row + o)) : 0u;
}

__global__ void __launch_bounds__(64) k_par2_packet_headers(const Par2PktArgs A) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint8_t* row = A.data + i * A.stride;
  const uint32_t ex = A.exps[i];
  const uint64_t T = 36 + A.L;
  uint32_t st[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
  uint32_t m[16];
  const uint64_t nblk = T / 64;
  // blocks after the first are whole data words (message byte 64b + 4w is
  // data byte 64b + 4w - 36); the next block is loaded while this one is
  // compressed
  uint32_t nx[16];
  if (nblk > 1) {
    const uint32_t* p = reinterpret_cast<const uint32_t*>(row + 64 - 36);
#pragma unroll
    for (int w = 0; w < 16; w++) nx[w] = __ldg(p + w);
  }
  for (uint64_t b = 0; b < nblk; b++) {
    if (b == 0) {
#pragma unroll
      for (int w = 0; w < 16; w++) m[w] = pkt_word(A, row, ex, w);
    } else {
#pragma unroll
      for (int w = 0; w < 16; w++) m[w] = nx[w];
      if (b + 1 < nblk) {
        const uint32_t* p = reinterpret_cast<const uint32_t*>(row + 64 * (b + 1) - 36);
#pragma unroll
        for (int w = 0; w < 16; w++) nx[w] = __ldg(p + w);
      }
    }
    md5_block(st, m);
  }
  const uint32_t tail = (uint32_t)(T % 64);  // a multiple of 4
#pragma unroll
  for (int w = 0; w < 16; w++) m[w] = (4u * w < tail) ? pkt_word(A, row, ex, 16 * nblk + w) : 0u;
#pragma unroll
  for (int w = 0; w < 16; w++)
    if (4u * w == tail) m[w] = 0x80u;
  if (tail >= 56) {
    md5_block(st, m);
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = 0;
  }
  m[14] = (uint32_t)(T << 3);
  m[15] = (uint32_t)(T >> 29);
  md5_block(st, m);
  uint32_t* h = reinterpret_cast<uint32_t*>(A.out + 68 * i);
  const uint64_t len = 68 + A.L;
  h[0] = 0x32524150u;  // "PAR2"
  h[1] = 0x544B5000u;  // "\0PKT"
  h[2] = (uint32_t)len;
  h[3] = (uint32_t)(len >> 32);
#pragma unroll
  for (int q = 0; q < 4; q++) h[4 + q] = st[q];
#pragma unroll
  for (int q = 0; q < 8; q++) h[8 + q] = A.pre[q];
  h[16] = ex;
}

// -------------------------------------------------------------- BLAKE3
__constant__ uint32_t c_b3iv[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                   0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
constexpr uint32_t kB3ChunkStart = 1, kB3ChunkEnd = 2, kB3Parent = 4, kB3Root = 8;

__device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

// the additions on the FMA pipe (madd), the XORs and rotations on the ALU pipe
__device__ __forceinline__ void b3_g(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d, uint32_t x, uint32_t y,
                                     uint32_t one) {
  a = madd(madd(a, x, one), b, one);
  d = __byte_perm(d ^ a, 0, 0x1032);  // rotr 16
  c = madd(c, d, one);
  b = rotr(b ^ c, 12);
  a = madd(madd(a, y, one), b, one);
  d = __byte_perm(d ^ a, 0, 0x0321);  // rotr 8
  c = madd(c, d, one);
  b = rotr(b ^ c, 7);
}

// cv <- first half of compress(cv, m, counter, len, flags)
__device__ __forceinline__ void b3_compress(uint32_t cv[8], const uint32_t m_in[16], uint64_t counter,
                                            uint32_t len, uint32_t flags, uint32_t one) {
  uint32_t v[16], m[16];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = cv[i];
#pragma unroll
  for (int i = 0; i < 4; i++) v[8 + i] = c_b3iv[i];
  v[12] = (uint32_t)counter;
  v[13] = (uint32_t)(counter >> 32);
  v[14] = len;
  v[15] = flags;
#pragma unroll
  for (int i = 0; i < 16; i++) m[i] = m_in[i];
  const int perm[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
#pragma unroll
  for (int r = 0; r < 7; r++) {
    b3_g(v[0], v[4], v[8], v[12], m[0], m[1], one);
    b3_g(v[1], v[5], v[9], v[13], m[2], m[3], one);
    b3_g(v[2], v[6], v[10], v[14], m[4], m[5], one);
    b3_g(v[3], v[7], v[11], v[15], m[6], m[7], one);
    b3_g(v[0], v[5], v[10], v[15], m[8], m[9], one);
    b3_g(v[1], v[6], v[11], v[12], m[10], m[11], one);
    b3_g(v[2], v[7], v[8], v[13], m[12], m[13], one);
    b3_g(v[3], v[4], v[9], v[14], m[14], m[15], one);
    if (r < 6) {
      uint32_t t[16];
#pragma unroll
      for (int i = 0; i < 16; i++) t[i] = m[perm[i]];
#pragma unroll
      for (int i = 0; i < 16; i++) m[i] = t[i];
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) cv[i] = v[i] ^ v[i + 8];
}

__device__ __forceinline__ void store_digest16(uint8_t* p, const uint32_t cv[8], bool aligned) {
  if (aligned) {
    reinterpret_cast<uint2*>(p)[0] = make_uint2(cv[0], cv[1]);
    reinterpret_cast<uint2*>(p)[1] = make_uint2(cv[2], cv[3]);
  } else {
#pragma unroll
    for (int j = 0; j < 16; j++) p[j] = (uint8_t)(cv[j >> 2] >> (8 * (j & 3)));
  }
}

// u64 word at message offset mo (a multiple of 8) of message i
template <bool kAligned>
__device__ __forceinline__ uint64_t b3_word(const B3Job& J, const uint8_t* src, uint8_t* dst, uint64_t i,
                                            uint64_t mo, uint64_t T) {
  if (mo < J.P) {
    const uint32_t k = (uint32_t)(mo >> 3);
    if (k < 3) return (uint64_t)J.pre[2 * k] | (uint64_t)J.pre[2 * k + 1] << 32;
    return k == 3 ? J.first_index + i : J.extra;
  }
  if (mo >= T) return 0;
  const uint64_t o = mo - J.P;
  if (kAligned) {
    const uint64_t v = __ldg(reinterpret_cast<const unsigned long long*>(src + o));
    if (dst) *reinterpret_cast<uint64_t*>(dst + o) = v;
    return v;
  }
  uint64_t v = 0;
  const uint64_t e = (T - mo) < 8 ? (T - mo) : 8;
  for (uint64_t j = 0; j < e; j++) {
    const uint8_t b = src[o + j];
    if (dst) dst[o + j] = b;
    v |= (uint64_t)b << (8 * j);
  }
  return v;
}

// One thread per (message, 1 KiB chunk).
template <bool kAligned>
__global__ void __launch_bounds__(128) k_b3_chunks(const B3Job J, uint32_t* __restrict__ cvs) {
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= J.n * J.C) return;
  const uint64_t i = g / J.C, c = g % J.C;
  const uint64_t T = J.P + J.D;
  const uint8_t* src = J.data + i * J.stride;
  uint8_t* dst = J.copy_to ? J.copy_to + i * J.copy_stride : nullptr;
  const uint64_t c0 = 1024 * c;
  const uint64_t bytes = (T - c0) < 1024 ? (T - c0) : 1024;
  const uint32_t nb = (uint32_t)((bytes + 63) / 64);
  uint32_t cv[8];
#pragma unroll
  for (int k = 0; k < 8; k++) cv[k] = c_b3iv[k];
  for (uint32_t b = 0; b < nb; b++) {
    const uint64_t m0 = c0 + 64 * b;
    uint32_t m[16];
    if (kAligned && m0 >= J.P && m0 + 64 <= T) {
      const uint64_t o = m0 - J.P;
#pragma unroll
      for (int w = 0; w < 8; w++) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(src + o) + w);
        m[2 * w] = v.x;
        m[2 * w + 1] = v.y;
        if (dst) reinterpret_cast<uint2*>(dst + o)[w] = v;
      }
    } else {
#pragma unroll
      for (int w = 0; w < 8; w++) {
        const uint64_t v = b3_word<kAligned>(J, src, dst, i, m0 + 8 * w, T);
        m[2 * w] = (uint32_t)v;
        m[2 * w + 1] = (uint32_t)(v >> 32);
      }
    }
    const uint32_t blen = (uint32_t)((T - m0) < 64 ? (T - m0) : 64);
    uint32_t flags = (b == 0 ? kB3ChunkStart : 0u);
    if (b == nb - 1) flags |= kB3ChunkEnd | (J.C == 1 ? kB3Root : 0u);
    b3_compress(cv, m, c, blen, flags, J.one);
  }
  if (J.C == 1) {
    store_digest16(J.hash_out + i * J.hash_stride, cv, kAligned);
  } else {
    uint4* o = reinterpret_cast<uint4*>(cvs + 8 * (i * J.C + c));
    o[0] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
    o[1] = make_uint4(cv[4], cv[5], cv[6], cv[7]);
  }
}

// One level of parent nodes: m nodes per message (slot stride C) -> ceil(m/2).
template <bool kAligned>
__global__ void __launch_bounds__(128) k_b3_merge(const B3Job J, const uint32_t* __restrict__ src,
                                                  uint32_t* __restrict__ dst, uint64_t m) {
  const uint64_t half = (m + 1) / 2;
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= J.n * half) return;
  const uint64_t i = g / half, j = g % half;
  const uint4* s = reinterpret_cast<const uint4*>(src + 8 * (i * J.C + 2 * j));
  uint4* d = reinterpret_cast<uint4*>(dst + 8 * (i * J.C + j));
  if (2 * j + 1 == m) {  // odd node carried up
    d[0] = s[0];
    d[1] = s[1];
    return;
  }
  uint32_t blk[16];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const uint4 v = s[q];
    blk[4 * q] = v.x;
    blk[4 * q + 1] = v.y;
    blk[4 * q + 2] = v.z;
    blk[4 * q + 3] = v.w;
  }
  uint32_t cv[8];
#pragma unroll
  for (int k = 0; k < 8; k++) cv[k] = c_b3iv[k];
  const bool root = (m == 2);
  b3_compress(cv, blk, 0, 64, kB3Parent | (root ? kB3Root : 0u), J.one);
  if (root) {
    store_digest16(J.hash_out + i * J.hash_stride, cv, kAligned);
  } else {
    d[0] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
    d[1] = make_uint4(cv[4], cv[5], cv[6], cv[7]);
  }
}

// PAR3 recovery-packet headers (src/gf64_addon.cc:2895-2921) except the
// checksum: magic, total length, input-set id, type, block index, count 1.
__global__ void k_par3_packet_headers(uint8_t* __restrict__ pkts, size_t n, uint64_t pkt_bytes, uint64_t set_id,
                                      uint64_t first) {
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n * 6) return;
  const uint64_t i = g / 6, f = g % 6;
  // words 0, 3..7 of the 8-word header (word 1-2 = checksum)
  const uint64_t word = f == 0 ? 0 : f + 2;
  uint64_t v;
  switch (word) {
    case 0: v = 0x544B500033524150ull; break;  // "PAR3\0PKT"
    case 3: v = pkt_bytes; break;
    case 4: v = set_id; break;
    case 5: v = 0x0043455220524150ull; break;  // "PAR REC\0"
    case 6: v = first + i; break;
    default: v = 1; break;
  }
  uint8_t* p = pkts + i * pkt_bytes + 8 * word;
  if ((((uintptr_t)p) & 7) == 0) {
    *reinterpret_cast<uint64_t*>(p) = v;
  } else {
    for (int j = 0; j < 8; j++) p[j] = (uint8_t)(v >> (8 * j));
  }
}

// ---------------------------------------------------- PAR2 memory checksum
// The staging checksum of the reference's PAR2 processors
// (gf16/gf16_checksum_generic.h gf16_multi_mul2, gf16/gf16_cksum_base.h:40-55):
// a row is read as nb 16-byte blocks B_j of 8 little-endian GF(2^16) lanes
// and C = 2*C ^ B_j over the blocks, i.e. C = sum_j 2^(nb-1-j) * B_j lane-wise.
// It is linear, so the region product of the inputs' checksums is the
// checksum of the product: carried through the multiply-accumulate as one
// more block per row, it checks the outputs.
__device__ __forceinline__ uint32_t gf16x2_dbl(uint32_t v) {
  return ((v << 1) & 0xFFFEFFFEu) ^ (((v >> 15) & 0x00010001u) * 0x100Bu);
}

__device__ __forceinline__ uint32_t gf16x2_mul(uint32_t v, uint32_t g) {
  uint32_t r = 0;
  for (int b = 15; b >= 0; b--) {
    r = gf16x2_dbl(r);
    if ((g >> b) & 1u) r ^= v;
  }
  return r;
}

struct CksumArgs {
  const uint8_t* rows;
  size_t stride;
  size_t n;
  uint64_t len;     // bytes of data per row (later bytes read as zero)
  uint64_t nb;      // 16-byte blocks per row: ceil(len / 16)
  uint64_t k;       // blocks per lane: ceil(nb / 32)
  uint32_t g[5];    // 2^(k * 2^L), the weight of the right-hand group at tree level L
  uint8_t* out;     // make: checksum of row i at out + i * out_stride
  size_t out_stride;
  int* valid;       // check: valid[i] = (checksum == the 16 bytes at out + i * out_stride)
};

// One warp per row.  The blocks are dealt to the lanes end-aligned, k per
// lane (lane t ends at block nb - (31 - t) k; blocks before 0 are zeros, which
// Horner from zero ignores), so every right-hand group at tree level L is
// 2^L k blocks long and the combine weights are uniform.
__global__ void __launch_bounds__(256) k_par2_cksum(const CksumArgs A) {
  const size_t r = (size_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (r >= A.n) return;
  const unsigned lane = threadIdx.x & 31;
  const uint8_t* row = A.rows + r * A.stride;
  const int64_t s1 = (int64_t)A.nb - (int64_t)(31 - lane) * (int64_t)A.k;
  int64_t j = s1 - (int64_t)A.k;
  if (j < 0) j = 0;
  uint32_t c[4] = {0, 0, 0, 0};
  for (; j < s1; j++) {
    uint32_t w[4];
    const uint64_t o = 16 * (uint64_t)j;
    if (o + 16 <= A.len) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(row + o));
      w[0] = v.x;
      w[1] = v.y;
      w[2] = v.z;
      w[3] = v.w;
    } else {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        uint32_t x = 0;
        for (int b = 0; b < 4; b++)
          if (o + 4 * q + b < A.len) x |= (uint32_t)row[o + 4 * q + b] << (8 * b);
        w[q] = x;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) c[q] = gf16x2_dbl(c[q]) ^ w[q];
  }
#pragma unroll
  for (int L = 0; L < 5; L++) {
    const unsigned d = 1u << L;
    uint32_t left[4];
#pragma unroll
    for (int q = 0; q < 4; q++) left[q] = __shfl_up_sync(0xFFFFFFFFu, c[q], d);
    if ((lane & (2 * d - 1)) == 2 * d - 1) {
#pragma unroll
      for (int q = 0; q < 4; q++) c[q] ^= gf16x2_mul(left[q], A.g[L]);
    }
  }
  if (lane == 31) {
    uint32_t* o = reinterpret_cast<uint32_t*>(A.out + r * A.out_stride);
    if (A.valid) {
      A.valid[r] = (o[0] == c[0] && o[1] == c[1] && o[2] == c[2] && o[3] == c[3]) ? 1 : 0;
    } else {
#pragma unroll
      for (int q = 0; q < 4; q++) o[q] = c[q];
    }
  }
}

// host: 2^e in GF(2^16)
uint32_t gf16_pow2(uint64_t e) {
  e %= 65535;
  uint32_t r = 1, b = 2;
  auto mul = [](uint32_t a, uint32_t x) {
    uint32_t p = 0;
    for (int i = 15; i >= 0; i--) {
      p <<= 1;
      if (p & 0x10000u) p ^= 0x1100Bu;
      if ((x >> i) & 1u) p ^= a;
    }
    return p;
  };
  while (e) {
    if (e & 1) r = mul(r, b);
    b = mul(b, b);
    e >>= 1;
  }
  return r;
}

}  // namespace

cudaError_t launch_par2_block_hash(const uint8_t* d_data, size_t stride, size_t n, uint64_t slice,
                                   const uint64_t* d_lengths, uint8_t* d_out, cudaStream_t s, const uint16_t* d_idx) {
  if (n == 0) return cudaSuccess;
  const int smem = kCrcWords * 4;
  static std::atomic<uint64_t> attr{0};
  if (!device_done(attr)) {
    cudaError_t e = cudaSuccess;
    for (auto f : {k_par2_block_hash<false>, k_par2_block_hash<true>, k_par2_block_hash_split<false>,
                   k_par2_block_hash_split<true>})
      if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    device_mark(attr);
  }
  // split MD5 / CRC32 threads for up to 8,192 slices (1 GiB of device data:
  // 1,024 x 1 MiB 17.40 -> 17.17 ms, 4,096 x 256 KiB 4.36 -> 4.17 ms, 8,192 x
  // 128 KiB 2.18 -> 1.96 ms; at 32,768 x 32 KiB the one-thread form is
  // faster, 0.68 vs 1.22 ms, as the ALU pipe is then the limit)
  const unsigned gs = (unsigned)((n + 63) / 64), g1 = (unsigned)((n + 127) / 128);
  if (n <= 8192 && d_idx)
    k_par2_block_hash_split<true><<<gs, 128, smem, s>>>(d_data, stride, n, slice, d_lengths, d_out, d_idx);
  else if (n <= 8192)
    k_par2_block_hash_split<false><<<gs, 128, smem, s>>>(d_data, stride, n, slice, d_lengths, d_out, nullptr);
  else if (d_idx)
    k_par2_block_hash<true><<<g1, 128, smem, s>>>(d_data, stride, n, slice, d_lengths, d_out, d_idx);
  else
    k_par2_block_hash<false><<<g1, 128, smem, s>>>(d_data, stride, n, slice, d_lengths, d_out, nullptr);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_par2_block_hash_band(const uint8_t* d_data, size_t stride, size_t n, uint64_t slice,
                                        uint64_t k0, uint64_t k1, uint32_t* d_state, uint8_t* d_out, bool first,
                                        bool last, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int smem = kCrcWords * 4;
  static std::atomic<uint64_t> attr{0};
  if (!device_done(attr)) {
    cudaError_t e = cudaFuncSetAttribute(k_par2_block_hash_band, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    device_mark(attr);
  }
  k_par2_block_hash_band<<<(unsigned)((n + 63) / 64), 128, smem, s>>>(d_data, stride, n, slice, k0, k1, d_state,
                                                                      d_out, first ? 1 : 0, last ? 1 : 0);
  note_launch();
  return cudaGetLastError();
}

size_t blake3_scratch_words(size_t n, uint64_t message_bytes) {
  const uint64_t C = (message_bytes + 1023) / 1024;
  return C > 1 ? (size_t)(2 * n * C * 8) : 0;
}

cudaError_t launch_blake3_blocks(const B3Job& job, uint32_t* d_scratch, cudaStream_t s) {
  if (job.n == 0) return cudaSuccess;
  B3Job J = job;
  J.C = (J.P + J.D + 1023) / 1024;
  J.one = 1;
  const bool al = ((uintptr_t)J.data % 8) == 0 && J.stride % 8 == 0 && J.D % 8 == 0 && J.P % 8 == 0 &&
                  ((uintptr_t)J.copy_to % 8) == 0 && J.copy_stride % 8 == 0 &&
                  ((uintptr_t)J.hash_out % 8) == 0 && J.hash_stride % 8 == 0;
  const unsigned threads = 128;
  const uint64_t tot = J.n * J.C;
  if (al)
    k_b3_chunks<true><<<(unsigned)((tot + threads - 1) / threads), threads, 0, s>>>(J, d_scratch);
  else
    k_b3_chunks<false><<<(unsigned)((tot + threads - 1) / threads), threads, 0, s>>>(J, d_scratch);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  uint32_t* a = d_scratch;
  uint32_t* b = d_scratch + J.n * J.C * 8;
  for (uint64_t m = J.C; m > 1; m = (m + 1) / 2) {
    const uint64_t t = J.n * ((m + 1) / 2);
    if (al)
      k_b3_merge<true><<<(unsigned)((t + threads - 1) / threads), threads, 0, s>>>(J, a, b, m);
    else
      k_b3_merge<false><<<(unsigned)((t + threads - 1) / threads), threads, 0, s>>>(J, a, b, m);
    note_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    uint32_t* tmp = a;
    a = b;
    b = tmp;
  }
  return cudaSuccess;
}

cudaError_t launch_par3_packet_headers(uint8_t* d_pkts, size_t n, size_t block_size, uint64_t set_id_le,
                                       uint64_t first, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const uint64_t t = (uint64_t)n * 6;
  k_par3_packet_headers<<<(unsigned)((t + 255) / 256), 256, 0, s>>>(d_pkts, n, 64 + (uint64_t)block_size,
                                                                    set_id_le, first);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_par2_cksum(const uint8_t* d_rows, size_t stride, size_t n, uint64_t len, uint8_t* d_out,
                              size_t out_stride, int* d_valid, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  CksumArgs A;
  A.rows = d_rows;
  A.stride = stride;
  A.n = n;
  A.len = len;
  A.nb = (len + 15) / 16;
  A.k = (A.nb + 31) / 32;
  for (int L = 0; L < 5; L++) A.g[L] = gf16_pow2(A.k << L);
  A.out = d_out;
  A.out_stride = out_stride;
  A.valid = d_valid;
  k_par2_cksum<<<(unsigned)((n + 7) / 8), 256, 0, s>>>(A);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_par2_packet_headers(const uint8_t* d_data, size_t stride, size_t n, uint64_t slice,
                                       const uint32_t pre[8], const uint16_t* d_exps, uint8_t* d_out,
                                       cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  Par2PktArgs A;
  A.data = d_data;
  A.stride = stride;
  A.n = n;
  A.L = slice;
  for (int k = 0; k < 8; k++) A.pre[k] = pre[k];
  A.exps = d_exps;
  A.out = d_out;
  k_par2_packet_headers<<<(unsigned)((n + 63) / 64), 64, 0, s>>>(A);
  note_launch();
  return cudaGetLastError();
}

}  // namespace pp
