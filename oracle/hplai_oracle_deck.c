/*
 * hplai_oracle_deck.c -- CPU oracle for the reference's lazy-initialised,
 * double-decker LU (`driver.out ... -d`, dd_layout = 1).
 *
 * TEST INFRASTRUCTURE ONLY, like hplai_oracle.c: the CUDA library never
 * links, loads or calls it.
 *
 * With `-d` the reference never stores A.  The FP32 panel storage starts at
 * zero (pmatgen0, matgen.hpp:81-105) and the trailing updates go to an FP16
 * "deck" (the lower deck of the double-decker layout, panel.hpp:48-61,89-109)
 * through an FP16-accumulating GEMM; a block's FP32 value is formed only when
 * the block joins a panel, as  downscale * deck + a_ij  with a_ij regenerated
 * from the LCG (lazy_init.hpp:92-227).  The L panel is down-cast with the
 * scale scalea = n^0.75 (hpl_rand.hpp:154, panel_trf.hpp:717-719) and
 * downscale = 1 / scalea brings the deck back.
 *
 * The FP16 GEMM is the x86 build's hgemm_opt (kernels/avx2.cpp:82-189,
 * fp16sim.hpp:185-213): per element, over k-chunks of 100, an FP16
 * accumulator t <- fp16(fp32(a*b + t)) (the FP16 x FP16 product is exact in
 * FP32, so fused or not gives the same FP32 value) and after each chunk
 * deck <- fp16(fp32(deck - t)); every FP32 -> FP16 conversion rounds to
 * nearest even (_mm256_cvtps_ph(.., 0), _cvtss_sh(.., 0)).
 *
 * The lazy-init sum scale * deck + a_ij is one FMA in the reference's x86
 * build (g++ -O2 contracts it), written here as fmaf().  Compiled with
 * -ffp-contract=off, like hplai_oracle.c.
 *
 * The back buffer (`--back_buffer`, dd_layout = 2, back_buffer.hpp:81-170,
 * back_buffer.cpp:53-191): a second FP16 array per element.  At the end of
 * step k with (k - 1) % 32 == 31 (BB_NCYCLE = 32) every element of the
 * trailing blocks (rows and columns from (k+1) b on; panel k's update not yet
 * applied) moves its deck value into the back buffer with a compensated sum,
 * in FP16 arithmetic (each operation rounded to FP16 through FP32, the x86
 * build's emulation of the SVE FP16 instructions, svesim.hpp:190-262):
 *     p = h(y / 32),  t2 = h(x + p),  t3 = h(t2 - x),  t4 = h(p - t3),
 *     back = t2,  deck = h(32 t4);
 * the lazy initialisation then forms fma(scale, deck + 32 back, a_ij)
 * (lazy_init_omp.cpp:600-630, 704-760).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* from hplai_oracle.c */
void orc_getrf_nopiv(int n, float *a, int64_t lda);
void orc_trsm_right_upper(int m, int n, const float *u, int64_t ldu, float *b, int64_t ldb);
void orc_trsm_left_lower_unit(int m, int n, const float *l, int64_t ldl, float *b, int64_t ldb);
void orc_coeff_pow(uint64_t m, uint64_t *a, uint64_t *c);
uint64_t orc_state_at(int n, int64_t i, int64_t j, uint64_t seed);

static inline uint16_t to_f16(float x)
{
	_Float16 h = (_Float16)x;
	uint16_t r;
	memcpy(&r, &h, 2);
	return r;
}

static inline float from_f16(uint16_t b)
{
	_Float16 h;
	memcpy(&h, &b, 2);
	return (float)h;
}

/* RandStat -> double -> FHigh (hpl_rand.hpp:50-56) */
static inline float lcg_float(uint64_t x) { return (float)((double)(int64_t)x * 0x1.fffffffffffffP-65); }

/* scalea = n^0.75 as the reference computes it (double sqrt(n * sqrt(n)),
 * then FHigh), and downscale = FHigh(1 / (scalea * scaleb)), scaleb = 1. */
ORC_EXPORT void orc_deck_scales(int n, float *scalea, float *downscale)
{
	const float sa = (float)sqrt(n * sqrt((double)n));
	const float sb = 1.0f;
	*scalea = sa;
	*downscale = (float)(1. / (double)(sa * sb));
}

/* LazyInitializer<FLow,1,true>::update / update_diag over the rectangle
 * rows r0..r1, cols c0..c1 (block-aligned): A = fma(downscale, deck, a_ij),
 * a_ii = diag_f[i]. */
static void lazy_init(int n, uint64_t seed, const float *diag_f, float downscale, const uint16_t *deck,
	const uint16_t *back, float *a, int64_t lda, int r0, int r1, int c0, int c1)
{
	uint64_t ia, ic;
	orc_coeff_pow(1, &ia, &ic);
	#pragma omp parallel for schedule(static)
	for (int j = c0; j < c1; j++) {
		uint64_t s = orc_state_at(n, r0, j, seed);
		for (int i = r0; i < r1; i++) {
			const float aij = i == j ? diag_f[i] : lcg_float(s);
			const int64_t o = (int64_t)j * lda + i;
			/* with the back buffer: deck + 32 back in FP32 (exact scaling, one rounding) */
			const float x = back ? fmaf(32.0f, from_f16(back[o]), from_f16(deck[o])) : from_f16(deck[o]);
			a[o] = fmaf(downscale, x, aij);
			s = ia * s + ic;
		}
	}
}

/* hgemm_opt with alpha = -1, beta = 1 on the deck:
 * D(m x n) -= L(m x k) U(k x n), L and U FP16 column-major. */
static void hgemm_deck(int m, int n, int k, const uint16_t *l, int64_t ldl, const uint16_t *u, int64_t ldu,
	uint16_t *d, int64_t ldd)
{
	const int bk = 100;
	#pragma omp parallel
	{
		float *ucol = (float *)malloc(sizeof(float) * (size_t)k);
		#pragma omp for schedule(static)
		for (int j = 0; j < n; j++) {
			for (int q = 0; q < k; q++) ucol[q] = from_f16(u[(int64_t)j * ldu + q]);
			for (int i = 0; i < m; i++) {
				uint16_t dij = d[(int64_t)j * ldd + i];
				for (int q0 = 0; q0 < k; q0 += bk) {
					const int q1 = q0 + bk < k ? q0 + bk : k;
					uint16_t t = 0;
					for (int q = q0; q < q1; q++)
						t = to_f16(fmaf(from_f16(l[(int64_t)q * ldl + i]), ucol[q], from_f16(t)));
					dij = to_f16(fmaf(-1.0f, from_f16(t), from_f16(dij)));
				}
				d[(int64_t)j * ldd + i] = dij;
			}
		}
		free(ucol);
	}
}

/* bb_writeback_b_impl_fp16 over rows and columns [r0, n) */
static void back_buffer_writeback(int n, int r0, uint16_t *deck, uint16_t *back, int64_t ld)
{
	#pragma omp parallel for schedule(static)
	for (int j = r0; j < n; j++)
		for (int i = r0; i < n; i++) {
			const int64_t o = (int64_t)j * ld + i;
			const float x = from_f16(back[o]);
			const float p = from_f16(to_f16(from_f16(deck[o]) * (1.0f / 32.0f)));
			const float t2 = from_f16(to_f16(x + p));
			const float t3 = from_f16(to_f16(t2 - x));
			const float t4 = from_f16(to_f16(p - t3));
			back[o] = to_f16(t2);
			deck[o] = to_f16(t4 * 32.0f);
		}
}

/* The first kend block steps of RDMAPanelLU::run<Matgen, 1, true, false>
 * (panel_trf.hpp:703-856) collapsed onto one process.  On return `a` holds
 * the FP32 factors of the factored blocks (unit L below the diagonal, U on
 * and above) and, when kend < n/b, the not-yet-factored blocks hold zero
 * (their value lives in the deck, returned in `deck_out` if not NULL, n x n
 * FP16 with leading dimension lda).  diag_f is the FP32 diagonal (pdiaggen,
 * then FHigh).  back_buffer: the `--back_buffer` form (RDMAPanelLU::run
 * <Matgen, 2, true, false>).  Returns 0, or -1 on bad sizes, -2 on
 * allocation failure. */
ORC_EXPORT int orc_lu_deck_steps(int n, int b, uint64_t seed, const float *diag_f, float *a, int64_t lda, int kend,
	uint16_t *deck_out, int back_buffer)
{
	if (n <= 0 || b <= 0 || n % b || lda < n) return -1;
	int nb = n / b;
	if (kend < nb) nb = kend;
	float scalea, downscale;
	orc_deck_scales(n, &scalea, &downscale);
	uint16_t *deck = (uint16_t *)calloc((size_t)lda * n, sizeof(uint16_t));
	uint16_t *back = back_buffer ? (uint16_t *)calloc((size_t)lda * n, sizeof(uint16_t)) : NULL;
	uint16_t *lh = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)n * b);
	uint16_t *uh = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)n * b);
	if (!deck || !lh || !uh || (back_buffer && !back)) {
		free(back);
		free(deck);
		free(lh);
		free(uh);
		return -2;
	}
	for (int64_t j = 0; j < n; j++) memset(a + j * lda, 0, sizeof(float) * (size_t)n);   /* pmatgen0 */
	for (int k = 0; k < nb; k++) {
		const int kb = k * b;
		float *lu = a + (int64_t)kb * lda + kb;
		lazy_init(n, seed, diag_f, downscale, deck, back, a, lda, kb, kb + b, kb, kb + b);
		orc_getrf_nopiv(b, lu, lda);
		if (kb + b == n) break;
		const int rem = n - kb - b;
		/* column panel: lazy init, TRSM, down-cast with scalea */
		lazy_init(n, seed, diag_f, downscale, deck, back, a, lda, kb + b, n, kb, kb + b);
		orc_trsm_right_upper(rem, b, lu, lda, lu + b, lda);
		for (int j = 0; j < b; j++)
			for (int i = 0; i < rem; i++) lh[(size_t)j * rem + i] = to_f16(scalea * lu[b + (int64_t)j * lda + i]);
		/* row panel: lazy init, TRSM, down-cast with scaleb = 1 */
		lazy_init(n, seed, diag_f, downscale, deck, back, a, lda, kb, kb + b, kb + b, n);
		orc_trsm_left_lower_unit(b, rem, lu, lda, lu + (int64_t)b * lda, lda);
		for (int j = 0; j < rem; j++)
			for (int i = 0; i < b; i++) uh[(size_t)j * b + i] = to_f16(1.0f * lu[(int64_t)(b + j) * lda + i]);
		if (k == kend - 1 && kend < n / b) break;   /* warm-up: the last panel's update is not applied */
		/* BackBuffer::write_back at the end of the reference's iteration k,
		 * before panel k's update (applied in its iteration k+1) */
		if (back && k >= 1 && (k - 1) % 32 == 31) back_buffer_writeback(n, kb + b, deck, back, lda);
		hgemm_deck(rem, rem, b, lh, rem, uh, b, deck + (int64_t)(kb + b) * lda + kb + b, lda);
	}
	if (deck_out) memcpy(deck_out, deck, sizeof(uint16_t) * (size_t)lda * n);
	free(back);
	free(deck);
	free(lh);
	free(uh);
	return 0;
}

ORC_EXPORT int orc_lu_deck(int n, int b, uint64_t seed, const float *diag_f, float *a, int64_t lda)
{
	return orc_lu_deck_steps(n, b, seed, diag_f, a, lda, n / (b > 0 ? b : 1), NULL, 0);
}
