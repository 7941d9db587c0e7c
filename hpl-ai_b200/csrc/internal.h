// internal.h -- launch functions shared between the translation units of
// libhplai.  Every function enqueues work on `st` and returns an
// hplai_status; none of them allocates device memory.
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

namespace hplai {

// Number of kernel launches the library has enqueued (all launch paths
// below add to it); read through hplai_launch_count().
void count_launches(int k = 1);

// gen.cu
int launch_fill(int n, int i0, int j0, int nrow, int ncol, float *a, int64_t lda, uint64_t seed, int calc_diag,
	cudaStream_t st);
int launch_diag(int n, int i0, int count, double *d, float *adiag, int64_t lda, uint64_t seed, cudaStream_t st);
int launch_rhs(int n, double *rhs, uint64_t seed, cudaStream_t st);
// columns n + col0 .. n + col0 + ncols - 1 of the stream, column-major with ld n
int launch_rhs_cols(int n, int col0, int ncols, double *out, uint64_t seed, cudaStream_t st);
// pmatl1est: strictly lower part of A (n x n, lda) times float(1/d_j) per column
int launch_l1est(int n, float *a, int64_t lda, const double *d, cudaStream_t st);
// Higham's HPL-AI matrix: beta for cond(A, inf) = kappa and alpha = rho beta
// (NaN if the bisection fails), the FP32 matrix and the FP64 diagonal.
double higham_beta(int n, double kappa, double rho);
// With `factors`, the exact factors instead (-beta above, 1 on and -alpha
// below the diagonal; d untouched).
int launch_higham_fill(int n, double alpha, double beta, float *a, int64_t lda, double *d, bool factors, cudaStream_t st);
double higham_norm(int n, double alpha, double beta);
// The `-d` lazy initialisation a = fma(downscale, deck, a0) on rows [r0, r1)
// x columns [c0, c1), a0 regenerated (regen) or read from a; the deck's
// element (i, j) at deck[(j - dc0) * ldd + (i - dr0)].
int launch_lazy_init(int n, int r0, int r1, int c0, int c1, float *a, int64_t lda, const uint16_t *deck,
	const uint16_t *back, int64_t ldd, int dr0, int dc0, float downscale, uint64_t seed, const double *d, bool regen,
	cudaStream_t st);
// The back buffer's write-back of the deck over rows and columns [r0, n)
// (bb_writeback_b_impl_fp16, back_buffer.cpp:53-100).
int launch_backbuf_writeback(int n, int r0, uint16_t *deck, uint16_t *back, int64_t ld, cudaStream_t st);
// The reference's FP16-accumulating Schur update of the deck (hgemm_opt,
// alpha = -1): D(m x n) -= L(m x k) U(k x n) with an FP16 accumulator per
// element over k-chunks of 100.  L row i at l + i ldl, U column j at
// u + j ldu (both K-major), D column-major.
int launch_hgemm_deck(int m, int n, int k, const uint16_t *l, int64_t ldl, const uint16_t *u, int64_t ldu,
	uint16_t *d, int64_t ldd, cudaStream_t st);

// panel.cu
// getrf.cu: tile-parallel diagonal block LU (bit-exact with the sequential
// order).  `work` holds getrf_workspace() bytes, zeroed once; `epoch` is
// the host-side launch counter that goes with it.  launch_getrf is the
// leaf entry point's form on a library-owned workspace (it waits for the
// result and returns the kernel's status).
size_t getrf_workspace();
int launch_getrf_tiles(int b, float *a, int64_t lda, void *work, uint32_t *epoch, int max_ctas, cudaStream_t st);
int getrf_status(void *work, cudaStream_t st, int *status);
int launch_getrf(int b, float *a, int64_t lda, cudaStream_t st);
int launch_trsm_right_upper(int m, int b, const float *u, int64_t ldu, float *a, int64_t lda, uint16_t *lh,
	int64_t ldh, float scale, cudaStream_t st);
int launch_trsm_left_lower(int b, int ncols, const float *l, int64_t ldl, float *a, int64_t lda, uint16_t *uh,
	int64_t ldh, float scale, cudaStream_t st);

// schur.cu
// Tensor maps for the FP16 panel buffers are built once per buffer and
// reused for every step; `SchurMaps` is opaque storage for two CUtensorMap.
struct SchurMaps {
	alignas(64) unsigned char lmap[128];
	alignas(64) unsigned char umap[128];
	alignas(64) unsigned char umap2[128];   // U with 128-row boxes (CTA-pair kernel)
	int k;         // inner dimension (panel width)
	// FP32 matrix holding C, for the TMA reduce-add epilogue (a map clipped to
	// each launch's region is encoded per launch).
	float *cbase = nullptr;
	int64_t cld = 0, crows = 0, ccols = 0;
	bool has_cmap = false;
	unsigned *status = nullptr;   // device word set on a wait timeout (null: the library's own)
	// FP16 deck (trailing-matrix updates of the lazy form): base and leading
	// dimension in halves
	void *deck_base = nullptr;
	int64_t deck_ld = 0;
	// tile rows per group of the persistent kernel's tile order (0: the
	// default, 32); hplai_set_tile_group / hplai_autotune set it
	int group_m = 0;
	// deck updates on CTA pairs (256 x 256 tiles, tcgen05 cta_group::2):
	// 1 on, 0 off, -1 the library default (hplai_set_cta_pairs)
	int pairs = -1;
};
// L: lrows x k FP16, row-major with ldl; U: urows x k FP16 (row j = column j
// of U), ldu.  Rows beyond lrows/urows read as zero.
int schur_make_maps(SchurMaps *m, const uint16_t *lh, int lrows, int64_t ldl, const uint16_t *uh, int urows,
	int64_t ldu, int k);
// The library default for deck updates on CTA pairs (SchurMaps::pairs < 0).
void schur_set_pairs_default(bool on);
// Matrix holding C for the TMA reduce-add epilogue; left unset (plain
// epilogue) when c or ldc is not 16-byte aligned.
int schur_set_cmap(SchurMaps *m, const float *c, int rows, int cols, int64_t ldc);
// C (m x n, ldc) -= L[lrow0 : lrow0+m, 0:k] * U[urow0 : urow0+n, 0:k]^T.  C(0,0)
// sits at (crow0, ccol0) of the matrix given to schur_set_cmap.  At most
// max_ctas persistent CTAs (0 = one per SM), so that concurrent work on
// another stream keeps some SMs.
int launch_schur(const SchurMaps &maps, int lrow0, int urow0, int m, int n, float *c, int64_t ldc, int crow0,
	int ccol0, int max_ctas, cudaStream_t st);
// FP8 (e4m3) panels: L8 lrows x k bytes (row-major, ldl), U8 urows x k; maps
// for the same kernel with kind::f8f6f4.  The C matrix is set with
// schur_set_cmap as for FP16.
int schur_make_maps_fp8(SchurMaps *m, const uint8_t *l8, int lrows, int64_t ldl, const uint8_t *u8, int urows,
	int64_t ldu, int k);
// C -= (sl x L8)(su x U8)^T with one power-of-two factor per 128 rows of L8
// (sl[(row - sl0) / 128]) and per 128 rows of U8 (su[(row - su0) / 128]).
int launch_schur_fp8(const SchurMaps &maps8, const float *sl, int sl0, const float *su, int su0, int lrow0, int urow0,
	int m, int n, float *c, int64_t ldc, int crow0, int ccol0, int max_ctas, cudaStream_t st);
// deck -= dscale * L U on the FP16 deck of `maps` (rows crow0.., cols ccol0..;
// crow0 a multiple of 8), FP16 (fp8 = false) or e4m3 operands.
// Block maxima of a panel written by the store form, for its e4m3 copies:
// atomicMax of |value| bits into bits[t][(index - base[t]) / 128] for the
// region's rows (dim 0: an L panel, blocks of 128 rows) or columns (dim 1: a
// U panel, blocks of 128 columns) from base[t] on (region-relative, a
// multiple of 128); a null bits[t] is skipped.
struct AmaxTargets {
	unsigned *bits[2] = {nullptr, nullptr};
	int base[2] = {0, 0};
	int dim = 0;
};
// C (m x n FP32 region of the map's matrix) = (L U) * *oscale, written by TMA
// store (FP16 operands; crow0 and m multiples of 4); with amax, the written
// values' block maxima as well.
int launch_schur_store(const SchurMaps &maps, int lrow0, int urow0, int m, int n, float *c, int64_t ldc, int crow0,
	int ccol0, const float *oscale, int max_ctas, cudaStream_t st, const AmaxTargets *amax = nullptr);
int launch_schur_deck(const SchurMaps &maps, bool fp8, const float *sl, int sl0, const float *su, int su0, int lrow0,
	int urow0, int m, int n, int crow0, int ccol0, float dscale, int max_ctas, cudaStream_t st);
// The batched form: `ntiles` 128 x 256 tiles, tile t updating C rows
// tiles[t].z.. and columns tiles[t].w.. of the matrix given to
// schur_set_cmap with L rows tiles[t].x.. and U rows tiles[t].y.. (FP16
// maps); a tile may reach past the columns of its system into columns nobody
// reads (or past the matrix, where it is clipped).
int launch_schur_tiles(const SchurMaps &maps, const int4 *tiles, int ntiles, int max_ctas, cudaStream_t st);
int schur_status();          // the library's word: HPLAI_ETIMEOUT if a device wait ran out since the last reset
void schur_status_reset();

// tcpanel.cu
// Panel TRSMs on tensor cores (3xTF32): triangular inverses of the diagonal
// block and the two panel products.  Buffers are caller-owned; the tensor
// maps are built once per context.
struct TcPanels {
	alignas(64) unsigned char m_phi[128];
	alignas(64) unsigned char m_plo[128];
	alignas(64) unsigned char m_uhi[128];
	alignas(64) unsigned char m_ulo[128];
	alignas(64) unsigned char m_lhi[128];
	alignas(64) unsigned char m_llo[128];
	int n, b;
	int64_t ldp;                     // row pitch of every buffer below, a multiple of 32 floats
	float *phi, *plo;                // n x ldp: K-major hi/lo copy of the current panel
	float *uhi, *ulo, *lhi, *llo;    // b x ldp: hi/lo of U11^{-1} and L11^{-1}
	float *xu, *xl, *wu, *wl;        // ldp x ldp FP32 work of the inversion (zeroed once)
	unsigned *status = nullptr;      // device word set on a wait timeout (null: the library's own)
	int terms = 3;                   // 3xTF32 (FP32 accuracy) or 1 (TF32, for the precision form)
	unsigned *f16_amax = nullptr;    // FP16 panel products: 2 words of triangle maxima
	float *f16_oscale = nullptr;     // and the 2 inverse scales of the FP16 triangles
};
// `work` holds tc_inverse_work_elems(ldp) floats, zeroed before first use.
inline size_t tc_inverse_work_elems(int64_t ldp) { return 4 * static_cast<size_t>(ldp) * static_cast<size_t>(ldp); }
int tc_panels_make(TcPanels *t, int n, int b, float *phi, float *plo, int64_t ldp, float *uhi, float *ulo,
	float *lhi, float *llo, float *work);
int launch_tri_inverses(const TcPanels &t, const float *lu, int64_t lda, cudaStream_t st, bool split = true);
// The precision form's panel products on FP16 tensor cores (after
// launch_tri_inverses without the split): the triangles are scaled by powers
// of two into rows kb..kb+b-1 of the FP16 panel buffers lh/uh, the panels are
// copied to FP16 (rows kb+b..), and A_col <- A_col U11^{-1},
// A_row <- L11^{-1} A_row are written back into A by the Schur kernel's store
// form.  `maps` are the FP16 maps over lh/uh with the C map over A.  With
// the FP16 deck (element (i, j) at deck[j*ldd + i]; null if none) the panels
// are read as A + deck * inv_dscale, so only the diagonal block needs
// deck_apply.  src (null: A itself) holds the panel's A values instead of A
// (column-major, leading dimension lds; element (r, k) of A_col at
// src[k*lds + r], of A_row at src[r*lds + k]) -- the matrix regenerated into
// a scratch panel when A is not stored.
// amax: the block maxima of the panel written (AmaxTargets, dim 0 for
// the L panel, 1 for the U panel), for its e4m3 copies.
int launch_lpanel_f16(const TcPanels &t, const SchurMaps &maps, int kb, int rem, float *a, int64_t lda,
	uint16_t *lh, uint16_t *uh, int64_t ldh, const uint16_t *deck, int64_t ldd, float inv_dscale, int max_ctas,
	cudaStream_t st, const float *src = nullptr, int64_t lds = 0, const AmaxTargets *amax = nullptr);
int launch_upanel_f16(const TcPanels &t, const SchurMaps &maps, int kb, int rem, float *a, int64_t lda,
	uint16_t *uh, int64_t ldh, const uint16_t *deck, int64_t ldd, float inv_dscale, int max_ctas, cudaStream_t st,
	const float *src = nullptr, int64_t lds = 0, const AmaxTargets *amax = nullptr);
// A_col (rem x b) <- A_col U11^{-1}; lh row i = half(scale * A_col row i)
int launch_lpanel_tc(const TcPanels &t, int rem, float *acol, int64_t lda, uint16_t *lh, int64_t ldh, float scale,
	int max_ctas, cudaStream_t st);
// A_row (b x rem) <- L11^{-1} A_row; uh row j = half(scale * A_row column j)
int launch_upanel_tc(const TcPanels &t, int rem, float *arow, int64_t lda, uint16_t *uh, int64_t ldh, float scale,
	int max_ctas, cudaStream_t st);
int tc_status();
void tc_status_reset();

// fp8.cu
// e4m3 copies of the L panel (rows x b, column-major FP32 source) and of the
// U panel (read by columns), row-major with K contiguous (ld8 a multiple of
// 128 bytes), and one power-of-two factor per 128 rows/columns in `scale`
// (block 0 = the first row).  `bits` is rows/128 + 1 words of scratch.
// Row bytes past b are zero up to the next multiple of 128 (the Schur
// kernel's K chunk), or up to ld8 with pad_row.  bits_ready: `bits` already
// holds the blocks' maxima (the store form's AmaxTargets), so no pass of its own.
int launch_quantize_lpanel(int rows, int b, const float *acol, int64_t lda, unsigned *bits, uint8_t *l8, int64_t ld8,
	float *scale, cudaStream_t st, bool pad_row = false, bool bits_ready = false);
int launch_quantize_upanel(int cols, int b, const float *arow, int64_t lda, unsigned *bits, uint8_t *u8, int64_t ld8,
	float *scale, cudaStream_t st, bool pad_row = false, bool bits_ready = false);

// A[i][j] += deck[i][j] * inv_scale on rows [r0, r1) x cols [c0, c1) (FP16 deck, ld ldd)
int launch_deck_apply(int r0, int r1, int c0, int c1, float *a, int64_t lda, const void *deck, int64_t ldd,
	float inv_scale, cudaStream_t st);

// refine.cu
size_t otf_gemv_workspace(int n);
// trans: y <- beta*y + alpha*A^T x
int launch_otf_gemv(int n, double alpha, const double *x, double beta, double *y, uint64_t seed,
	const double *diag, void *work, size_t work_bytes, cudaStream_t st, bool trans = false);
// y <- beta y + alpha A x (A^T x with trans) over Higham's matrix with
// parameters (halpha, hbeta), entries computed on the fly in FP64.
int launch_higham_gemv(int n, double alpha, const double *x, double beta, double *y, double halpha, double hbeta,
	const double *diag, void *work, size_t work_bytes, cudaStream_t st, bool trans);
int launch_otf_gemv_block(int64_t n, int mb, int nb, double alpha, const double *x, double *y, uint64_t state00,
	void *work, size_t work_bytes, cudaStream_t st);
size_t trsv_workspace(int n);
// trans: solve with the transpose of the stored triangle (lower = U^T non-unit,
// upper = L^T unit); otherwise lower = L (unit), upper = U (non-unit).
// dinv (optional): FP64 inverses of the 128 x 128 diagonal blocks of both
// factors (launch_trsv_dinv), applied as products instead of substitution.
int launch_trsv(bool lower, int n, const float *a, int64_t lda, double *x, void *work, size_t work_bytes,
	cudaStream_t st, bool trans = false, const double *dinv = nullptr);
size_t trsv_dinv_doubles(int n);
// blocks blk0 .. blk0 + nblk - 1 of 128 rows (nblk < 0: to the last)
int launch_trsv_dinv(int n, const float *a, int64_t lda, double *dinv, cudaStream_t st, int blk0 = 0, int nblk = -1);
int trsv_status(void *work, cudaStream_t st, int *status);
int launch_infnorm(int n, const double *x, double *out, cudaStream_t st);
// panel_check: sigs (device, 3 doubles) = FP64 sums of |a_ij| over the
// diagonal, strict upper and strict lower triangle of a (n x n, lda).
size_t panel_check_workspace(int n);
int launch_panel_check(int n, const float *a, int64_t lda, double *sigs, void *work, size_t work_bytes,
	cudaStream_t st);
int launch_div(int n, const double *num, const double *den, double *out, cudaStream_t st);
int launch_axpy1(int n, const double *x, double *y, cudaStream_t st);

// krylov.cu -- GMRES vector kernels.  `part` holds kDotBlocks x kMaxBasis
// doubles.  V is column-major n x nv with leading dimension ldv.
constexpr int kMaxBasis = 32;
constexpr int kDotBlocks = 296;
// out[0..nv) (op 0: =, 1: +=) V^T w
int launch_dots(int n, int nv, const double *v, int64_t ldv, const double *w, double *part, double *out, int op,
	cudaStream_t st);
// w -= V h; if norm_out, *norm_out = ||w||_2 afterwards
int launch_gs_update(int n, int nv, const double *v, int64_t ldv, const double *h, double *w, double *part,
	double *norm_out, cudaStream_t st);
int launch_add_small(int nv, const double *a, double *b, cudaStream_t st);
int launch_scale(int n, const double *w, const double *den, double *out, cudaStream_t st);
// x += V y
int launch_combine(int n, int nv, const double *v, int64_t ldv, const double *y, double *x, cudaStream_t st);

// batched.cu: the step-synchronous batched engine (plain form, IR)
struct BatchEngine;
int batched_create(BatchEngine **out, int count, const int *n, const int *nrhs, const uint64_t *seeds);
void batched_destroy(BatchEngine *e);
int batched_solve(BatchEngine *e, int maxit, unsigned long long *launches);
int batched_result(BatchEngine *e, int orig, hplai_ir_errors *worst, int *iters, int *status);
int batched_get_x(BatchEngine *e, int orig, double *x, int64_t ldx);
int batched_get_lu(BatchEngine *e, int orig, float *a, int64_t lda);
int batched_pad(BatchEngine *e, int orig);
unsigned long long batched_launches(const BatchEngine *e);

} // namespace hplai

// api.cu, for the batched solver: right-hand side column n + col of the
// context's stream, solved with its factors into host memory.
struct hplai_ctx;
struct hplai_ir_errors;
int hplai_ctx_solve_stream_rhs(hplai_ctx *c, int col, double *x, int maxit, hplai_ir_errors *err, int *iters);
