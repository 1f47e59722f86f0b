// Additive FFT over GF(2^64) in the novel-polynomial basis on the Cantor
// basis (sm_100a), batched.
//
// Semantics: gf64_addfft64_{fwd,inv}_recursive_scratch
// (reference gf64/gf64_additive_fft_hqc2026.c:1656-1705):
//   forward = monomial -> novel-polynomial basis conversion (hqc_cvt, an
//             XOR-only network, :1011-1017) followed by radix-2 butterflies
//             (butterfly_fwd, :1068-1086) with affine shift v_{n/2};
//   inverse = inverse butterflies (:1088-1108), then the inverse conversion.
//
// Layout: `batch` polynomials of n coefficients, coefficient c of polynomial
// b at data[c * ld + b].  The batch index is the fast axis, so every step is
// a row operation over contiguous memory (one polynomial per word position
// is how the PAR3 FFT path uses it).
//
// Level-synchronous restatement of the recursions:
//   * conversion phase (polylen, sh, sl), dd = sh - sl, inside every aligned
//     block of polylen rows, rows r in [sl, polylen - dd):
//       forward  new[r] = d[r] ^ d[r+dd] ^ (r+2dd < polylen ? d[r+2dd] : 0)
//       inverse  new[r] = d[r] ^ d[r+dd]
//     (the reference's descending / ascending in-place loops; dd >= sh/2, so
//     a forward chain has at most two links);
//   * butterfly depth d, block t (block size n >> d, half h): twiddle
//     w = v_{2^d XOR 2t}, v_j = XOR of Cantor basis vectors at the set bits
//     of j;  forward lo = f[k] ^ w*f[k+h], f[k+h] ^= lo, f[k] = lo;
//     inverse fh = f[k] ^ f[k+h], f[k] ^= w*fh, f[k+h] = fh.
#include <vector>

#include "pp_common.cuh"
#include "pp_internal.h"

namespace pp {

// Cantor basis of GF(2^64) for x^64+x^4+x^3+x+1: v_0 = 1,
// v_{i+1}^2 + v_{i+1} = v_i (the reference's table, gf64/gf64_cantor_basis.h:23-44).
__constant__ uint64_t c_cantor[20] = {
    0x0000000000000001ULL, 0x19c9369f278adc02ULL, 0xa181e7d66f5ff794ULL, 0x5db84357ce785d08ULL,
    0xb973d466f5c9d0caULL, 0x521ac889831a075eULL, 0x033ce8beddc8a656ULL, 0xb5846c4e07b91010ULL,
    0x4087b8cbb37a32ecULL, 0x00d0d3888c0ae17cULL, 0xafd5ac70237f2222ULL, 0xe3f5af99cc3aaaf8ULL,
    0x5a1db3b16a0b58b8ULL, 0x09947c54fe7ee248ULL, 0x0e8eaf0e0068f544ULL, 0xa2a113500b4b4f5aULL,
    0xe96f9805d6ce0bb0ULL, 0x53496f8b5c9edd4cULL, 0xad325cb6f4ac2a9eULL, 0x4a8dcf8bd7ede826ULL,
};

PP_D uint64_t cantor_v(uint32_t j) {
  uint64_t v = 0;
#pragma unroll
  for (int k = 0; k < 20; k++)
    if ((j >> k) & 1) v ^= c_cantor[k];
  return v;
}

// one conversion phase, out of place
__global__ void k_fft_cvt_phase(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst, size_t n, size_t batch,
                                size_t ld, uint32_t polylen, uint32_t sh, uint32_t sl, int inverse) {
  const size_t total = n * batch;
  const uint32_t dd = sh - sl;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    size_t row = e / batch, col = e % batch;
    uint32_t r = (uint32_t)(row & (polylen - 1));
    uint64_t v = src[row * ld + col];
    if (r >= sl && r < polylen - dd) {
      v ^= src[(row + dd) * ld + col];
      if (!inverse && r + 2 * dd < polylen) v ^= src[(row + 2 * dd) * ld + col];
    }
    dst[row * ld + col] = v;
  }
}

// one butterfly depth, in place; each element pair is owned by one thread
__global__ void k_fft_butterfly(uint64_t* __restrict__ f, size_t n, size_t batch, size_t ld, int depth,
                                int inverse) {
  const size_t h = n >> (depth + 1);
  const size_t pairs = (n >> 1) * batch;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < pairs; e += (size_t)gridDim.x * blockDim.x) {
    size_t p = e / batch, col = e % batch;
    size_t t = p / h, k = p % h;
    size_t ra = t * 2 * h + k, rb = ra + h;
    uint64_t w = cantor_v((uint32_t)((1u << depth) ^ (2 * t)));
    uint64_t a = f[ra * ld + col], b = f[rb * ld + col];
    if (!inverse) {
      uint64_t lo = a ^ gf64_mul(w, b);
      f[ra * ld + col] = lo;
      f[rb * ld + col] = b ^ lo;
    } else {
      uint64_t fh = a ^ b;
      f[ra * ld + col] = a ^ gf64_mul(w, fh);
      f[rb * ld + col] = fh;
    }
  }
}

struct CvtPhase {
  uint32_t polylen, sh, sl;
};

static int choose_si(int pl) {
  int si = 1;
  for (int i = 1; (1 << i) < pl; i++) si = 1 << i;
  return si;
}
// hqc_cvt recursion order (reference :1011-1017)
static void sched_fwd(int lb, int pl, std::vector<CvtPhase>& out) {
  if (pl <= 1) return;
  int si = choose_si(pl);
  for (int i = pl - 1; i >= si; i--)
    out.push_back({1u << (i + lb + 1), 1u << (i + lb), 1u << (i + lb - si)});
  sched_fwd(lb, si, out);
  sched_fwd(lb + si, pl - si, out);
}
// hqc_icvt recursion order (reference :1020-1026)
static void sched_inv(int lb, int pl, std::vector<CvtPhase>& out) {
  if (pl <= 1) return;
  int si = choose_si(pl);
  sched_inv(lb, si, out);
  sched_inv(lb + si, pl - si, out);
  for (int i = si; i < pl; i++) out.push_back({1u << (i + lb + 1), 1u << (i + lb), 1u << (i + lb - si)});
}

static unsigned grid_for(size_t work) {
  size_t b = ceil_div(work, 256);
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)(b ? b : 1);
}

// d_tmp: n*ld words of scratch (ping-pong partner of d_data).
cudaError_t launch_gf64_fft(uint64_t* d_data, uint64_t* d_tmp, size_t n, size_t batch, size_t ld, bool inverse,
                            cudaStream_t s) {
  if (n <= 1 || !batch) return cudaSuccess;
  int L = 0;
  while (((size_t)1 << L) < n) L++;
  std::vector<CvtPhase> ph;
  if (!inverse) sched_fwd(0, L, ph);
  else sched_inv(0, L, ph);
  const unsigned g_el = grid_for(n * batch), g_pair = grid_for((n >> 1) * batch);
  uint64_t* cur = d_data;
  uint64_t* oth = d_tmp;
  auto run_cvt = [&]() {
    for (const auto& p : ph) {
      k_fft_cvt_phase<<<g_el, 256, 0, s>>>(cur, oth, n, batch, ld, p.polylen, p.sh, p.sl, inverse ? 1 : 0);
      note_launch();
      uint64_t* t = cur;
      cur = oth;
      oth = t;
    }
  };
  if (!inverse) {
    run_cvt();
    for (int d = 0; d < L; d++) {
      k_fft_butterfly<<<g_pair, 256, 0, s>>>(cur, n, batch, ld, d, 0);
      note_launch();
    }
  } else {
    for (int d = L - 1; d >= 0; d--) {
      k_fft_butterfly<<<g_pair, 256, 0, s>>>(cur, n, batch, ld, d, 1);
      note_launch();
    }
    run_cvt();
  }
  if (cur != d_data) {
    cudaError_t e = cudaMemcpy2DAsync(d_data, ld * 8, cur, ld * 8, batch * 8, n, cudaMemcpyDeviceToDevice, s);
    note_launch();
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

}  // namespace pp
