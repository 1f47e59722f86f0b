/* Test infrastructure only: the oracle (see gf_oracle.h).
 *
 * Plain C, written from the field definitions and the reference's documented
 * semantics; no SIMD, no reference code.  Never linked into the product.
 */
#include "gf_oracle.h"
#include <stdlib.h>
#include <string.h>

/* ======================================================================= */
/* GF(2^16)                                                                 */
/* ======================================================================= */
/* Field: GF(2)[x]/(x^16+x^12+x^3+x+1), the PAR2 field (gf16/gfmat_coeff.c:28,
 * polynomial 0x1100B), generator 2 (= x).  Log/antilog tables are built by
 * repeated doubling, as the PAR2 specification defines the field. */
static uint16_t g16_exp[65535 * 2];
static uint16_t g16_log[65536];
static int g16_ready = 0;

static void g16_init(void) {
	if (g16_ready) return;
	uint32_t n = 1;
	for (uint32_t e = 0; e < 65535; e++) {
		g16_exp[e] = (uint16_t)n;
		g16_exp[e + 65535] = (uint16_t)n;
		g16_log[n] = (uint16_t)e;
		n <<= 1;
		if (n & 0x10000) n ^= 0x1100B;
	}
	g16_log[0] = 0;
	g16_ready = 1;
}

uint16_t or_gf16_mul(uint16_t a, uint16_t b) {
	g16_init();
	if (!a || !b) return 0;
	return g16_exp[(uint32_t)g16_log[a] + g16_log[b]];
}

uint16_t or_gf16_exp(uint32_t e) {
	g16_init();
	return g16_exp[e % 65535];
}

uint16_t or_gf16_inv(uint16_t a) {
	g16_init();
	if (!a) return 0;
	return g16_exp[(65535 - g16_log[a]) % 65535];
}

/* PAR2 input constant log: the (i+1)-th positive integer coprime to 65535
 * (= 3*5*17*257).  Restates gfmat_init's table walk (gf16/gfmat_coeff.c:21-32)
 * and gfmat_input_log (gf16/gfmat_coeff.c:80-82). */
static uint16_t g16_ilog[32768];
static int g16_ilog_ready = 0;
uint16_t or_par2_input_log(uint16_t inputBlock) {
	if (!g16_ilog_ready) {
		uint32_t e = 0;
		for (uint32_t i = 0; i < 32768; i++) {
			do { e++; } while (!(e % 3) || !(e % 5) || !(e % 17) || !(e % 257));
			g16_ilog[i] = (uint16_t)e;
		}
		g16_ilog_ready = 1;
	}
	return g16_ilog[inputBlock & 32767];
}

/* coeff(i, e) = 2^(L_i * e mod 65535) (gf16/gfmat_coeff.c:84-101). */
uint16_t or_par2_coeff(uint16_t inputBlock, uint16_t recoveryExp) {
	uint32_t l = or_par2_input_log(inputBlock);
	return or_gf16_exp((uint32_t)(((uint64_t)l * recoveryExp) % 65535));
}

/* Region multiply-accumulate of the PAR2 controller, as its tests define the
 * result (test/gf16/test-ctrl.cpp:185-199): words are little-endian u16; a
 * source shorter than the slice contributes zeros past its end; an odd final
 * byte is a word whose high byte is zero. */
void or_par2_muladd(const uint8_t* const* src, const size_t* sizes, unsigned numInputs,
                    size_t sliceSize, const uint16_t* coeffs, unsigned numOutputs,
                    uint8_t* dst) {
	g16_init();
	size_t words = (sliceSize + 1) / 2;
	uint16_t* acc = (uint16_t*)calloc(words ? words : 1, sizeof(uint16_t));
	uint16_t* x = (uint16_t*)calloc(words ? words : 1, sizeof(uint16_t));
	for (unsigned o = 0; o < numOutputs; o++) {
		memset(acc, 0, words * sizeof(uint16_t));
		for (unsigned i = 0; i < numInputs; i++) {
			uint16_t c = coeffs[(size_t)o * numInputs + i];
			if (!c) continue;
			size_t sz = sizes[i] < sliceSize ? sizes[i] : sliceSize;
			size_t nw = (sz + 1) / 2;
			for (size_t w = 0; w < nw; w++) {
				uint16_t lo = src[i][2 * w];
				uint16_t hi = (2 * w + 1 < sz) ? src[i][2 * w + 1] : 0;
				x[w] = (uint16_t)(lo | (hi << 8));
			}
			if (c == 1) {
				for (size_t w = 0; w < nw; w++) acc[w] ^= x[w];
			} else {
				uint32_t lc = g16_log[c];
				for (size_t w = 0; w < nw; w++)
					if (x[w]) acc[w] ^= g16_exp[lc + g16_log[x[w]]];
			}
		}
		uint8_t* d = dst + (size_t)o * sliceSize;
		for (size_t b = 0; b < sliceSize; b++)
			d[b] = (uint8_t)(b & 1 ? acc[b / 2] >> 8 : acc[b / 2] & 0xff);
	}
	free(acc);
	free(x);
}

static int cmp_u16(const void* a, const void* b) {
	return (int)*(const uint16_t*)a - (int)*(const uint16_t*)b;
}

/* PAR2 repair matrix inversion, restating Galois16RecMatrix::Compute
 * (gf16/gfmat_inv.cpp:560-690) and Construct (:462-558):
 *   - recovery exponents are sorted; the first m = #missing are the rows;
 *   - columns: valid inputs in index order, then missing inputs in index order;
 *   - Gauss-Jordan WITHOUT pivoting, row k pivots on column (validCount + k);
 *     the eliminated column is replaced in place by the identity column, so the
 *     result row k is GetFactor(col, k) (gf16/gfmat_inv.h:40-45);
 *   - a zero pivot drops that recovery row and restarts (:631-668, "PAR2 flaw");
 *     too few rows left -> not invertible. */
int or_par2_invert(const uint8_t* valid, unsigned numInputs, uint16_t* recovery,
                   unsigned* numRec, uint16_t* factors) {
	g16_init();
	unsigned validCount = 0;
	for (unsigned i = 0; i < numInputs; i++) validCount += valid[i] ? 1 : 0;
	unsigned m = numInputs - validCount;
	unsigned nrec = *numRec;
	if (m == 0 || m > nrec) return 0;
	uint16_t* rec = (uint16_t*)malloc(nrec * sizeof(uint16_t));
	memcpy(rec, recovery, nrec * sizeof(uint16_t));
	qsort(rec, nrec, sizeof(uint16_t), cmp_u16);
	unsigned* colOf = (unsigned*)malloc(numInputs * sizeof(unsigned));
	unsigned vc = 0, mc = validCount;
	for (unsigned i = 0; i < numInputs; i++) colOf[i] = valid[i] ? vc++ : mc++;
	uint16_t* M = factors; /* m x numInputs, row-major */
	int ok = 0;
	for (;;) {
		if (nrec < m) break;
		for (unsigned r = 0; r < m; r++)
			for (unsigned i = 0; i < numInputs; i++)
				M[(size_t)r * numInputs + colOf[i]] = or_par2_coeff((uint16_t)i, rec[r]);
		int bad = -1;
		for (unsigned k = 0; k < m && bad < 0; k++) {
			uint16_t* rowk = M + (size_t)k * numInputs;
			uint16_t p = rowk[validCount + k];
			rowk[validCount + k] = 1;
			if (!p) { bad = (int)k; break; }
			if (p != 1) {
				uint16_t ip = or_gf16_inv(p);
				for (unsigned c = 0; c < numInputs; c++) rowk[c] = or_gf16_mul(rowk[c], ip);
			}
			for (unsigned r = 0; r < m; r++) {
				if (r == k) continue;
				uint16_t* rowr = M + (size_t)r * numInputs;
				uint16_t f = rowr[validCount + k];
				rowr[validCount + k] = 0;
				if (!f) continue;
				for (unsigned c = 0; c < numInputs; c++) rowr[c] ^= or_gf16_mul(f, rowk[c]);
			}
		}
		if (bad < 0) { ok = 1; break; }
		memmove(rec + bad, rec + bad + 1, (nrec - bad - 1) * sizeof(uint16_t));
		nrec--;
	}
	if (ok) {
		memcpy(recovery, rec, m * sizeof(uint16_t));
		*numRec = m;
	}
	free(rec);
	free(colOf);
	return ok;
}

/* ======================================================================= */
/* GF(2^64)                                                                 */
/* ======================================================================= */
/* Field: GF(2)[x]/(x^64+x^4+x^3+x+1) (gf64/gf64_global.h:8), multiplication
 * as gf64_mul_reference defines it (gf64/gf64_single.c:6-53): the 128-bit
 * carry-less product reduced modulo the polynomial.  Written here as a plain
 * shift-and-add carry-less multiply followed by a two-step fold. */
uint64_t or_gf64_mul(uint64_t a, uint64_t b) {
	uint64_t lo = 0, hi = 0;
	for (int i = 0; i < 64; i++) {
		if ((b >> i) & 1) {
			lo ^= a << i;
			if (i) hi ^= a >> (64 - i);
		}
	}
	/* x^64 == x^4+x^3+x+1 (0x1B): fold hi twice. */
	uint64_t t = hi ^ (hi >> 60) ^ (hi >> 61) ^ (hi >> 63);
	return lo ^ t ^ (t << 1) ^ (t << 3) ^ (t << 4);
}

/* Multiplicative inverse, inverse(0) = 0 (gf64/gf64_invert.c:29-67 computes
 * it by the extended Euclidean algorithm; the inverse is unique, so it is
 * restated here as a^(2^64-2) by square-and-multiply). */
uint64_t or_gf64_inv(uint64_t a) {
	if (a == 0) return 0;
	uint64_t r = 1, s = a;
	/* exponent 2^64 - 2 = 0xFFFF...FE: bits 1..63 set */
	for (int i = 1; i < 64; i++) {
		s = or_gf64_mul(s, s);
		r = or_gf64_mul(r, s);
	}
	return r;
}

/* Cauchy matrix (src/par3_engine.cc:358-425):
 * M[r][c] = inv((firstInput + c) XOR (firstRecovery + r)), with a zero
 * denominator replaced by 1; row-major numRecovery x numInputs. */
void or_gf64_build_cauchy(uint64_t* m, size_t numInputs, size_t numRecovery,
                          uint64_t firstInput, uint64_t firstRecovery) {
	for (size_t r = 0; r < numRecovery; r++) {
		uint64_t y = firstRecovery + r;
		for (size_t c = 0; c < numInputs; c++) {
			uint64_t d = (firstInput + c) ^ y;
			m[r * numInputs + c] = or_gf64_inv(d ? d : 1);
		}
	}
}

/* out[r][w] (^)= XOR_c coeff[r][c] * in[c][w]
 * (ComputeRecoveryBlocksWithCoeff, src/par3_engine.cc:1165-1387; zero-init
 * unless accumulate). */
void or_gf64_matvec(const uint64_t* in, size_t numInputs, uint64_t* out, size_t numRecovery,
                    size_t blockSize64, const uint64_t* coeff, int accumulate) {
	for (size_t r = 0; r < numRecovery; r++) {
		uint64_t* o = out + r * blockSize64;
		if (!accumulate) memset(o, 0, blockSize64 * sizeof(uint64_t));
		for (size_t c = 0; c < numInputs; c++) {
			uint64_t k = coeff[r * numInputs + c];
			const uint64_t* x = in + c * blockSize64;
			for (size_t w = 0; w < blockSize64; w++) o[w] ^= or_gf64_mul(x[w], k);
		}
	}
}

/* ComputeRecoveryBlocks (src/par3_engine.cc:1061-1114): Cauchy build + matvec.
 * Empty problems return without touching the output. */
void or_gf64_compute_recovery(const uint64_t* in, size_t numInputs, uint64_t* out,
                              size_t numRecovery, size_t blockSize64, uint64_t firstInput,
                              uint64_t firstRecovery, int accumulate) {
	if (!numInputs || !numRecovery) return;
	uint64_t* m = (uint64_t*)malloc(numInputs * numRecovery * sizeof(uint64_t));
	or_gf64_build_cauchy(m, numInputs, numRecovery, firstInput, firstRecovery);
	or_gf64_matvec(in, numInputs, out, numRecovery, blockSize64, m, accumulate);
	free(m);
}

/* SolveAndReconstruct (src/par3_engine.cc:980-1053): in-place Gauss-Jordan
 * on A (n x n) with the same row operations applied to the RHS blocks;
 * pivot = first nonzero at or below the diagonal; returns -1 if singular. */
int or_gf64_solve_and_reconstruct(uint64_t* A, uint64_t* rhs, size_t n, size_t B) {
	for (size_t col = 0; col < n; col++) {
		size_t piv = col;
		while (piv < n && A[piv * n + col] == 0) piv++;
		if (piv == n) return -1;
		if (piv != col) {
			for (size_t j = 0; j < n; j++) {
				uint64_t t = A[col * n + j]; A[col * n + j] = A[piv * n + j]; A[piv * n + j] = t;
			}
			for (size_t w = 0; w < B; w++) {
				uint64_t t = rhs[col * B + w]; rhs[col * B + w] = rhs[piv * B + w]; rhs[piv * B + w] = t;
			}
		}
		uint64_t pv = A[col * n + col];
		if (pv != 1) {
			uint64_t pi = or_gf64_inv(pv);
			for (size_t j = 0; j < n; j++) A[col * n + j] = or_gf64_mul(A[col * n + j], pi);
			for (size_t w = 0; w < B; w++) rhs[col * B + w] = or_gf64_mul(rhs[col * B + w], pi);
		}
		for (size_t row = 0; row < n; row++) {
			if (row == col) continue;
			uint64_t f = A[row * n + col];
			if (!f) continue;
			for (size_t j = 0; j < n; j++) A[row * n + j] ^= or_gf64_mul(f, A[col * n + j]);
			for (size_t w = 0; w < B; w++) rhs[row * B + w] ^= or_gf64_mul(rhs[col * B + w], f);
		}
	}
	return 0;
}

/* Region primitives (gf64/gf64_region_scalar.c:8-28). */
void or_gf64_region_mul(uint64_t* out, const uint64_t* in, size_t len, uint64_t c) {
	for (size_t i = 0; i < len; i++) out[i] = or_gf64_mul(in[i], c);
}
/* mul_arr cycles the coefficients: out[i] = in[i] * coeff[i % nCoeff]. */
void or_gf64_region_mul_arr(uint64_t* out, const uint64_t* in, const uint64_t* coeff,
                            size_t len, size_t nCoeff) {
	for (size_t i = 0; i < len; i++) out[i] = or_gf64_mul(in[i], coeff[i % nCoeff]);
}
/* muladd_arr XORs the products of ALL coefficients into every word. */
void or_gf64_region_muladd_arr(uint64_t* out, const uint64_t* in, const uint64_t* coeff,
                               size_t len, size_t nCoeff) {
	for (size_t i = 0; i < len; i++) {
		uint64_t s = 0;
		for (size_t c = 0; c < nCoeff; c++) s ^= or_gf64_mul(in[i], coeff[c]);
		out[i] ^= s;
	}
}

/* ======================================================================= */
/* Additive FFT over GF(2^64), novel-polynomial basis on the Cantor basis   */
/* ======================================================================= */
/* Restates gf64_addfft64_{fwd,inv}_recursive_scratch
 * (gf64/gf64_additive_fft_hqc2026.c:1656-1705):
 *   forward = monomial -> novel-polynomial basis conversion (hqc_cvt,
 *             :1011-1017, an XOR-only network), then the radix-2 butterflies
 *             (butterfly_fwd, :1068-1086) with affine shift v_{n/2};
 *   inverse = inverse butterflies (:1088-1108), then the inverse conversion.
 * The Cantor basis v_0..v_19 (gf64/gf64_cantor_basis.h:20-44) satisfies
 * v_0 = 1 and v_{i+1}^2 + v_{i+1} = v_i; it is regenerated here from that
 * recurrence (below) and checked against the reference's fixtures.  With
 * v_j = XOR of basis vectors at the set bits of j, the butterfly twiddle of
 * block t at depth d (block size n >> d) is v_{2^d XOR 2t}: the recursion's
 * s_{logn-1}(v_j) = v_{j >> (logn-1)} evaluated on the shift index
 * 2^(L-1) XOR (t << (L-d)). */
static uint64_t cantor[20];
static int cantor_ready = 0;

/* Solve y^2 + y = c over GF(2^64): the map y -> y^2 + y is GF(2)-linear with
 * kernel {0, 1}; solve by Gaussian elimination over GF(2) and return the
 * solution with bit 0 clear.  Returns 0 when c has no solution. */
static int solve_artin_schreier(uint64_t c, uint64_t* out) {
	uint64_t col[64];
	for (int j = 0; j < 64; j++) {
		uint64_t e = 1ull << j;
		col[j] = or_gf64_mul(e, e) ^ e; /* image of basis vector x^j */
	}
	/* augmented system rows: row i = bit i of the images; solve L y = c */
	uint64_t rows[64];
	uint64_t rhs = 0;
	for (int i = 0; i < 64; i++) {
		uint64_t r = 0;
		for (int j = 0; j < 64; j++) r |= ((col[j] >> i) & 1ull) << j;
		rows[i] = r;
		rhs |= ((c >> i) & 1ull) << i;
	}
	int pivcol[64];
	int rank = 0;
	for (int j = 0; j < 64 && rank < 64; j++) {
		int p = -1;
		for (int i = rank; i < 64; i++) if ((rows[i] >> j) & 1) { p = i; break; }
		if (p < 0) continue;
		uint64_t t = rows[p]; rows[p] = rows[rank]; rows[rank] = t;
		uint64_t b1 = (rhs >> p) & 1, b2 = (rhs >> rank) & 1;
		rhs &= ~((1ull << p) | (1ull << rank));
		rhs |= (b1 << rank) | (b2 << p);
		for (int i = 0; i < 64; i++) {
			if (i != rank && ((rows[i] >> j) & 1)) {
				rows[i] ^= rows[rank];
				rhs ^= ((rhs >> rank) & 1ull) << i;
			}
		}
		pivcol[rank++] = j;
	}
	for (int i = rank; i < 64; i++) if ((rhs >> i) & 1) return 0;
	uint64_t y = 0;
	for (int i = 0; i < rank; i++) if ((rhs >> i) & 1) y |= 1ull << pivcol[i];
	if (y & 1) y ^= 1; /* pick the root with bit 0 clear (y and y+1 both solve) */
	*out = y;
	return 1;
}

uint64_t or_gf64_cantor(int i) {
	if (!cantor_ready) {
		cantor[0] = 1;
		for (int k = 1; k < 20; k++) solve_artin_schreier(cantor[k - 1], &cantor[k]);
		cantor_ready = 1;
	}
	return cantor[i];
}

static uint64_t vj(uint64_t j) {
	uint64_t v = 0;
	for (int k = 0; k < 20; k++) if ((j >> k) & 1) v ^= or_gf64_cantor(k);
	return v;
}

static int ilog2(size_t n) { int l = 0; while (((size_t)1 << l) < n) l++; return l; }

/* hqc_cvt: recursive XOR network, monomial -> novel polynomial basis */
static int choose_si(int n) { int si = 1; for (int i = 1; (1 << i) < n; i++) si = 1 << i; return si; }
static void cvt(uint64_t* d, int len, int lb, int pl) {
	if (pl <= 1) return;
	int si = choose_si(pl);
	for (int i = pl - 1; i >= si; i--) {
		int polylen = 1 << (i + lb + 1), sh = 1 << (i + lb), sl = 1 << (i + lb - si), dd = sh - sl;
		for (int j = 0; j < len; j += polylen)
			for (int k = polylen - 1; k >= sh; k--) d[j + k - dd] ^= d[j + k];
	}
	cvt(d, len, lb, si);
	cvt(d, len, lb + si, pl - si);
}
static void icvt(uint64_t* d, int len, int lb, int pl) {
	if (pl <= 1) return;
	int si = choose_si(pl);
	icvt(d, len, lb, si);
	icvt(d, len, lb + si, pl - si);
	for (int i = si; i < pl; i++) {
		int polylen = 1 << (i + lb + 1), sh = 1 << (i + lb), sl = 1 << (i + lb - si), dd = sh - sl;
		for (int j = 0; j < len; j += polylen)
			for (int k = sh; k < polylen; k++) d[j + k - dd] ^= d[j + k];
	}
}

void or_gf64_fft_fwd(uint64_t* a, size_t n) {
	if (n <= 1) return;
	int L = ilog2(n);
	cvt(a, (int)n, 0, L);
	for (int d = 0; d < L; d++) {
		size_t h = n >> (d + 1);
		for (size_t t = 0; t < ((size_t)1 << d); t++) {
			uint64_t w = vj(((uint64_t)1 << d) ^ (2 * t));
			uint64_t* f = a + t * 2 * h;
			for (size_t k = 0; k < h; k++) {
				uint64_t lo = f[k] ^ or_gf64_mul(w, f[k + h]);
				f[k + h] ^= lo;
				f[k] = lo;
			}
		}
	}
}

void or_gf64_fft_inv(uint64_t* a, size_t n) {
	if (n <= 1) return;
	int L = ilog2(n);
	for (int d = L - 1; d >= 0; d--) {
		size_t h = n >> (d + 1);
		for (size_t t = 0; t < ((size_t)1 << d); t++) {
			uint64_t w = vj(((uint64_t)1 << d) ^ (2 * t));
			uint64_t* f = a + t * 2 * h;
			for (size_t k = 0; k < h; k++) {
				uint64_t fh = f[k] ^ f[k + h];
				f[k] ^= or_gf64_mul(w, fh);
				f[k + h] = fh;
			}
		}
	}
	icvt(a, (int)n, 0, L);
}

/* ------------------------------------------------------------- BLAKE3 */
/* BLAKE3 in its default hash mode, written from the published
 * specification's recursive definition: the message is cut into 1024-byte
 * chunks, each a chain of 64-byte block compressions keyed by the IV; a
 * message of more than one chunk is split so that the left subtree holds the
 * largest power-of-two number of chunks that leaves the right subtree
 * non-empty, and each parent compresses its children's chaining values.  The
 * reference hashes PAR3 blocks with the npm `blake3` package
 * (lib/par3gen.js:1001-1017) and packet checksums with its port of BLAKE3
 * v1.8.7 (hasher/hasher_blake3.c, called at src/gf64_addon.cc:2925-2932). */
static const uint32_t B3_IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                  0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
static const uint8_t B3_PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
enum { B3_CHUNK_START = 1, B3_CHUNK_END = 2, B3_PARENT = 4, B3_ROOT = 8 };

static uint32_t b3_rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

static void b3_g(uint32_t* v, int a, int b, int c, int d, uint32_t x, uint32_t y) {
	v[a] = v[a] + v[b] + x;
	v[d] = b3_rotr(v[d] ^ v[a], 16);
	v[c] = v[c] + v[d];
	v[b] = b3_rotr(v[b] ^ v[c], 12);
	v[a] = v[a] + v[b] + y;
	v[d] = b3_rotr(v[d] ^ v[a], 8);
	v[c] = v[c] + v[d];
	v[b] = b3_rotr(v[b] ^ v[c], 7);
}

static void b3_compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter, uint32_t len,
                        uint32_t flags, uint32_t out[8]) {
	uint32_t v[16], m[16], t[16];
	for (int i = 0; i < 8; i++) v[i] = cv[i];
	for (int i = 0; i < 4; i++) v[8 + i] = B3_IV[i];
	v[12] = (uint32_t)counter;
	v[13] = (uint32_t)(counter >> 32);
	v[14] = len;
	v[15] = flags;
	memcpy(m, block, sizeof m);
	for (int r = 0; r < 7; r++) {
		b3_g(v, 0, 4, 8, 12, m[0], m[1]);
		b3_g(v, 1, 5, 9, 13, m[2], m[3]);
		b3_g(v, 2, 6, 10, 14, m[4], m[5]);
		b3_g(v, 3, 7, 11, 15, m[6], m[7]);
		b3_g(v, 0, 5, 10, 15, m[8], m[9]);
		b3_g(v, 1, 6, 11, 12, m[10], m[11]);
		b3_g(v, 2, 7, 8, 13, m[12], m[13]);
		b3_g(v, 3, 4, 9, 14, m[14], m[15]);
		for (int i = 0; i < 16; i++) t[i] = m[B3_PERM[i]];
		memcpy(m, t, sizeof m);
	}
	for (int i = 0; i < 8; i++) out[i] = v[i] ^ v[i + 8];
}

static void b3_block_words(const uint8_t* p, size_t n, uint32_t m[16]) {
	uint8_t buf[64] = {0};
	memcpy(buf, p, n);
	for (int i = 0; i < 16; i++)
		m[i] = (uint32_t)buf[4 * i] | (uint32_t)buf[4 * i + 1] << 8 | (uint32_t)buf[4 * i + 2] << 16 |
		       (uint32_t)buf[4 * i + 3] << 24;
}

/* chaining value of chunk `counter` (n <= 1024 bytes); `extra` = ROOT for a
 * one-chunk message */
static void b3_chunk(const uint8_t* p, size_t n, uint64_t counter, uint32_t extra, uint32_t out[8]) {
	uint32_t cv[8], m[16];
	memcpy(cv, B3_IV, sizeof cv);
	size_t nb = n ? (n + 63) / 64 : 1;
	for (size_t b = 0; b < nb; b++) {
		size_t len = n - 64 * b < 64 ? n - 64 * b : 64;
		uint32_t flags = (b == 0 ? B3_CHUNK_START : 0) | (b == nb - 1 ? B3_CHUNK_END | extra : 0);
		b3_block_words(p + 64 * b, len, m);
		b3_compress(cv, m, counter, (uint32_t)len, flags, cv);
	}
	memcpy(out, cv, sizeof cv);
}

static void b3_node(const uint8_t* p, size_t n, uint64_t counter, uint32_t extra, uint32_t out[8]) {
	if (n <= 1024) {
		b3_chunk(p, n, counter, extra, out);
		return;
	}
	size_t chunks = (n + 1023) / 1024, left = 1;
	while (2 * left < chunks) left *= 2;
	uint32_t m[16];
	b3_node(p, left * 1024, counter, 0, m);
	b3_node(p + left * 1024, n - left * 1024, counter + left, 0, m + 8);
	b3_compress(B3_IV, m, 0, 64, B3_PARENT | extra, out);
}

void or_blake3(const uint8_t* in, size_t len, uint8_t* out, size_t out_len) {
	uint32_t h[8];
	b3_node(in, len, 0, B3_ROOT, h);
	for (size_t i = 0; i < out_len && i < 32; i++) out[i] = (uint8_t)(h[i / 4] >> (8 * (i % 4)));
}

static void put_le64(uint8_t* p, uint64_t v) {
	for (int b = 0; b < 8; b++) p[b] = (uint8_t)(v >> (8 * b));
}

/* lib/par3gen.js:1001-1017 (_inlineHashBlock): the data-packet checksum of
 * block `first_index + i`, the packet's 24 post-checksum header bytes
 * followed by the body (u64le block index, block data). */
void or_par3_block_hashes(const uint8_t* blocks, size_t stride, size_t n, size_t block_size,
                          uint64_t first_index, const uint8_t* after_checksum, uint8_t* out16) {
	uint8_t* msg = (uint8_t*)malloc(32 + block_size);
	memcpy(msg, after_checksum, 24);
	for (size_t i = 0; i < n; i++) {
		put_le64(msg + 24, first_index + i);
		memcpy(msg + 32, blocks + i * stride, block_size);
		or_blake3(msg, 32 + block_size, out16 + 16 * i, 16);
	}
	free(msg);
}

/* src/gf64_addon.cc:2884-2934 (AssembleRecoveryPackets_NAPI): per packet the
 * magic "PAR3\0PKT", the 16-byte checksum, u64le total length, the 8-byte
 * input-set id, the type "PAR REC\0", then the body u64le(first_index + i),
 * u64le(1) and the block; checksum = BLAKE3(packet[24 .. 64 + block_size))[0:16]. */
void or_par3_recovery_packets(const uint8_t* recovery, size_t n, size_t block_size,
                              const uint8_t* input_set_id, uint64_t first_index, uint8_t* packets) {
	static const uint8_t magic[8] = {'P', 'A', 'R', '3', 0, 'P', 'K', 'T'};
	static const uint8_t type[8] = {'P', 'A', 'R', ' ', 'R', 'E', 'C', 0};
	size_t pkt = 64 + block_size;
	for (size_t i = 0; i < n; i++) {
		uint8_t* p = packets + i * pkt;
		memcpy(p, magic, 8);
		memset(p + 8, 0, 16);
		put_le64(p + 24, pkt);
		memcpy(p + 32, input_set_id, 8);
		memcpy(p + 40, type, 8);
		put_le64(p + 48, first_index + i);
		put_le64(p + 56, 1);
		memcpy(p + 64, recovery + i * block_size, block_size);
		or_blake3(p + 24, 40 + block_size, p + 8, 16);
	}
}

/* ------------------------------------------------- PAR2 memory checksum */
/* The staging checksum of the reference's PAR2 processors: each block is
 * folded in as ck = ck * 2 ^ block, lane-wise over GF(2^16) (gf16_multi_mul2,
 * gf16/gf16_checksum_generic.h; the copy loop of gf16/gf16_cksum_base.h:20-55).
 * The reference's block width is its SIMD width; this restatement and the
 * device both use 16 bytes. */
void or_par2_mem_cksum(const uint8_t* data, size_t len, uint8_t* out) {
	uint16_t c[8] = {0};
	for (size_t o = 0; o < len; o += 16) {
		for (int l = 0; l < 8; l++) {
			uint16_t w = 0;
			for (int b = 0; b < 2; b++)
				if (o + 2 * l + b < len) w |= (uint16_t)(data[o + 2 * l + b] << (8 * b));
			c[l] = (uint16_t)(or_gf16_mul(c[l], 2) ^ w);
		}
	}
	for (int l = 0; l < 8; l++) {
		out[2 * l] = (uint8_t)c[l];
		out[2 * l + 1] = (uint8_t)(c[l] >> 8);
	}
}
