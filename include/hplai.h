/*
 * hplai.h -- C ABI of libhplai, a single-GPU B200 (sm_100a) HPL-AI solver.
 *
 * The library solves A x = b for the HPL-AI matrix (the 64-bit LCG matrix of
 * RIKEN-RCCS/hpl-ai with a row-sum diagonal) by a no-pivot blocked LU with
 * FP32 panels and an FP16-input / FP32-accumulate Schur update on tcgen05
 * tensor cores, followed by FP64 iterative refinement that regenerates A on
 * the fly.  Every entry point is extern "C" with plain pointers and sizes.
 *
 * Conventions (the reference's, panel.hpp:20-35 and otf_gemv.cpp:5-7):
 *   - matrices are column-major with an explicit leading dimension;
 *   - caller-owned buffers: the leaf kernels below never allocate device
 *     memory, they take a caller-provided workspace where they need one;
 *   - every function returns an hplai_status (0 = success), never aborts;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy stream);
 *     leaf kernels are asynchronous on that stream;
 *   - a context is not thread-safe; distinct contexts are independent.
 */
#ifndef HPLAI_H
#define HPLAI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; everything declared here is
 * exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define HPLAI_VERSION 100

typedef enum hplai_status {
	HPLAI_OK = 0,
	HPLAI_EINVAL = 1,        /* bad argument (e.g. n % b != 0, main.cpp:181 / panel.hpp:142) */
	HPLAI_ENOMEM = 2,        /* device or pinned-host allocation failed */
	HPLAI_ECUDA = 3,         /* a CUDA runtime call failed */
	HPLAI_ENOTCONV = 4,      /* refinement did not reach hpl-harness < 16 (IRErrors {-1,-1}) */
	HPLAI_ETIMEOUT = 5,      /* a device-side bounded wait ran out; the context stays usable */
	HPLAI_ESTATE = 6,        /* call out of order (e.g. refine before factor) */
	HPLAI_EUNSUPPORTED = 7   /* configuration outside what this build implements */
} hplai_status;

/* FHIGH / FLOW precision pair (main.cpp:27-31): the panel precision is FP32,
 * the Schur-update input precision is FP16 (the reference default) or FP8. */
typedef enum hplai_precision {
	HPLAI_F32_F16 = 0,
	HPLAI_F32_F8 = 1
} hplai_precision;

/* Refinement flavour. */
typedef enum hplai_refine_mode {
	HPLAI_IR = 0,            /* classical refinement, iterative_refinement.hpp:18-57 */
	HPLAI_GMRES = 1          /* FP64 GMRES-IR preconditioned by the LU (no reference counterpart) */
} hplai_refine_mode;

/* IRErrors (iterative_refinement.hpp:13-16): {residual, hpl_harness}, or
 * {-1, -1} when refinement fails to converge. */
typedef struct hplai_ir_errors {
	double residual;
	double hpl_harness;
} hplai_ir_errors;

/* Phase timers, named after the reference's Timer items (timer.hpp:58-84). */
typedef enum hplai_phase {
	HPLAI_PH_DIAG_LU = 0,
	HPLAI_PH_TRSM_L = 1,
	HPLAI_PH_TRSM_R = 2,
	HPLAI_PH_GEMM_UPDATE = 3,
	HPLAI_PH_IR_GEMV = 4,
	HPLAI_PH_IR_TRSV = 5,
	HPLAI_PH_TOTAL = 6,      /* sum of the other items (overlapping side-stream items included) */
	HPLAI_PH_LAZY_INIT = 7,  /* FP16 deck folded into the next block column/row (lazy_init.hpp:92-227) */
	HPLAI_PH_WRITE_BACK = 8, /* the back buffer's write-backs (back_buffer.hpp:125-169) */
	HPLAI_PH_COUNT = 9
} hplai_phase;

/* hplai_create flags. */
/* Panel TRSMs on CUDA cores in netlib strsm order -- bit-exact with the
 * reference's substitution -- instead of the default tensor-core path
 * (triangular inverses of the diagonal block applied in 3xTF32). */
#define HPLAI_FLAG_SIMT_PANELS 1u
/* One-step look-ahead on two streams: the next diagonal block and panels are
 * formed on a high-priority side stream while the main stream applies the
 * rest of the trailing update, leaving the side stream a fixed SM count or a
 * share that grows as the trailing matrix shrinks (hplai_set_schedule;
 * hplai_autotune picks one).  Results are bit-identical to the one-stream
 * schedule. */
#define HPLAI_FLAG_LOOKAHEAD 2u
/* The trailing matrix's updates accumulate in an FP16 "deck" (the
 * double-decker lazy form, lazy_init.hpp:92-227): each step adds
 * -s L U (FP32 accumulation, one FP16 rounding per step, s a power of two
 * near n^0.75 as scalea, lazy_init.hpp / hpl_rand.hpp:154), and a block
 * column/row becomes A + deck / s just before it is factored.  Halves the
 * Schur update's memory traffic; the FP32 matrix keeps the original
 * entries and receives the factors.  Requires b % 8 == 0. */
#define HPLAI_FLAG_FP16_DECK 4u
/* Two-panel groups: the trailing matrix is updated once per two panels,
 * C -= [L_k L_k+1] [U_k; U_k+1] (K = 2b), after the group's second block has
 * received the first panel's update alone -- the aggregated form of
 * GemmControl's split update (schur_updator.hpp:108-269), which halves the
 * passes over the trailing matrix.  With HPLAI_FLAG_LOOKAHEAD both panels of
 * the next group are formed on the side stream.  Requires b % 128 == 0
 * (hplai_create returns HPLAI_EINVAL otherwise); hplai_autotune may switch
 * it on or off for contexts whose b allows it. */
#define HPLAI_FLAG_GROUP2 8u
/* Four-panel groups: as HPLAI_FLAG_GROUP2 with K = 4b -- the group's block
 * e + j receives the updates of the group's panels e .. e + j - 1 (each
 * alone) before it is factored, and the trailing matrix is updated once per
 * four panels, which quarters the passes over it (at the 1000 W cap of a
 * B200 the e4m3 deck update sustains 11 % more at K = 4096 than at 2048).
 * At creation it also sizes the group buffers for four panels (28 n b bytes
 * more than two-panel buffers with HPLAI_F32_F8, 16 n b with HPLAI_F32_F16),
 * which hplai_autotune and hplai_set_schedule need to choose it later.  Requires b % 128 == 0; not with HPLAI_FLAG_GROUP2. */
#define HPLAI_FLAG_GROUP4 128u
/* The reference's `-d` arithmetic bit for bit (a parity mode, CUDA cores):
 * A is never stored -- a block is formed when it joins a panel as
 * fma(downscale, deck, a_ij) with a_ij regenerated from the LCG
 * (lazy_init.hpp:92-227; read from the matrix instead after hplai_upload);
 * the L panel's FP16 copy is scaled by scalea = n^0.75 (hpl_rand.hpp:154) and
 * downscale = 1 / scalea; the trailing updates go to an FP16 deck through the
 * reference's FP16-accumulating GEMM (hgemm_opt, kernels/avx2.cpp:82-189: an
 * FP16 accumulator rounded after every product, folded into the deck every
 * 100 products); panels in netlib order (as HPLAI_FLAG_SIMT_PANELS), one
 * stream.  Only with HPLAI_F32_F16 and without HPLAI_FLAG_FP16_DECK,
 * HPLAI_FLAG_GROUP2, HPLAI_FLAG_GROUP4 and HPLAI_FLAG_LOOKAHEAD (HPLAI_EINVAL
 * otherwise). */
#define HPLAI_FLAG_REF_DECK 16u
/* With HPLAI_FLAG_REF_DECK: the reference's `--back_buffer` form bit for bit
 * (dd_layout = 2, back_buffer.hpp:81-170): every 32 steps the deck is written
 * back into a second FP16 array with a compensated FP16 sum (deck / 32 moved
 * into it, the remainder kept), and the lazy initialisation forms
 * fma(downscale, deck + 32 back, a_ij).  HPLAI_EINVAL without
 * HPLAI_FLAG_REF_DECK. */
#define HPLAI_FLAG_REF_BACKBUF 32u
/* With HPLAI_FLAG_FP16_DECK and HPLAI_F32_F8: A is never stored.  A block's
 * entries are regenerated from the LCG when it joins a panel (the reference's
 * lazy initialisation, lazy_init.hpp:92-227), and the FP16 deck shares the
 * factors' storage -- it lives in the upper half of each FP32 column, where
 * the factors arrive only after the deck entries there are consumed -- so a
 * solve holds 4 n^2 bytes of matrix instead of 6 n^2 (n = 196608 fits in
 * 180 GB).  The factors are bit-identical to the stored-A deck form.
 * hplai_upload and hplai_solve_host return HPLAI_EUNSUPPORTED (nothing to
 * regenerate a caller's matrix from).  HPLAI_EINVAL without
 * HPLAI_FLAG_FP16_DECK, with another precision, b % 4 != 0,
 * HPLAI_FLAG_SIMT_PANELS or HPLAI_FLAG_REF_DECK. */
#define HPLAI_FLAG_LAZY_A 64u

typedef struct hplai_ctx hplai_ctx;

/* ---------------------------------------------------------------------- */
/* Whole-solve context: the single-GPU collapse of main.cpp:185-488.       */
/* ---------------------------------------------------------------------- */

const char *hplai_status_string(int status);
/* Text of the last CUDA error the library saw (thread-shared). */
int hplai_last_error(char *buf, size_t len);
int hplai_version(void);
/* Kernel launches enqueued by this library since it was loaded (all
 * contexts and leaf calls). */
unsigned long long hplai_launch_count(void);

/* build_panels (panel.hpp:135-268) + the driver's vector allocations
 * (main.cpp:196-213).  Requires n % b == 0 and 16 <= b <= 1024.  Allocates
 * every device buffer of the solve on the current CUDA device.  `flags` is a
 * combination of HPLAI_FLAG_* (0 for the defaults). */
int hplai_create(hplai_ctx **ctx, int n, int b, int precision, unsigned flags);
int hplai_destroy(hplai_ctx *ctx);

/* Matrix, right-hand side and diagonal from the LCG seed on the device:
 * pmatgen + pcolvgen + pdiaggen (matgen.hpp:7-22,193-225, main.cpp:255-270)
 * and the norms (main.cpp:273-276).  Bit-exact with the reference.  The
 * reference driver uses seed 42 (main.cpp:174). */
int hplai_generate(hplai_ctx *ctx, uint64_t seed);

/* Matrix families.  HPLAI_MATRIX_LCG: the HPL-AI benchmark matrix (LCG
 * entries, row-sum diagonal; the default).  HPLAI_MATRIX_HIGHAM: Higham's
 * HPL-AI matrix (the reference's --highammat, HMGen, highammgen.hpp:5-28,
 * higham_mat_impl.cpp:116-128): A = L U with L unit lower triangular, every
 * strictly lower entry -alpha, and U unit upper triangular, every strictly
 * upper entry -beta, i.e. a_ij = -beta + alpha beta i above the diagonal,
 * 1 + alpha beta i on it, -alpha + alpha beta j below it; beta is chosen by
 * bisection so that an estimate of cond(A, inf) equals `cond` and
 * alpha = rho beta (the reference's driver: cond 1000, rho 0.5). */
#define HPLAI_MATRIX_LCG 0
#define HPLAI_MATRIX_HIGHAM 1
/* The matrix that hplai_generate produces and that the refinement's FP64
 * GEMV regenerates (also after hplai_upload): kind HPLAI_MATRIX_LCG (cond and
 * rho ignored) or HPLAI_MATRIX_HIGHAM with its condition number and ratio.
 * The right-hand side stays column n of the LCG stream (main.cpp:266).
 * hplai_l1est on Higham's matrix writes its exact factors (pmatl1est with
 * HMGen, matgen.hpp:147-192).  Clears the inputs (call hplai_generate or
 * hplai_upload next).  HPLAI_EUNSUPPORTED for Higham's matrix with
 * HPLAI_FLAG_REF_DECK; HPLAI_EINVAL when the bisection finds no beta. */
int hplai_set_matrix(hplai_ctx *ctx, int kind, double cond, double rho);
/* alpha and beta of Higham's matrix of order n (higham_mat_comp_beta,
 * higham_mat_impl.cpp:87-113; the estimate's integer terms in 32-bit int as
 * the reference computes them, so that the values are the reference's for
 * every n). */
int hplai_higham_params(int n, double cond, double rho, double *alpha, double *beta);

/* Host-supplied inputs: FP32 matrix (lda >= n), FP64 right-hand side and
 * FP64 diagonal, plus the LCG seed they came from (refinement regenerates
 * A in FP64 from it, as Matgen<double> does, main.cpp:257).  Copies
 * host -> device on the context stream and waits. */
int hplai_upload(hplai_ctx *ctx, const float *a, int64_t lda, const double *rhs,
	const double *diag, uint64_t seed);

/* The LU in place: RDMAPanelLU::run / panel_lu_async (panel_trf.hpp:434-858)
 * collapsed to one GPU.  Unit-L below and U on/above the diagonal, FP32. */
int hplai_factor(hplai_ctx *ctx);

/* The benchmark warm-up of the reference's driver (`-w`, main.cpp:57,
 * RDMAPanelLU::run / panel_lu_async with warmup, panel_trf.hpp:458,726:
 * kend = nrow + 2): only panels 0 .. steps-1 are factored, and -- as the
 * reference's loop applies panel k-1's update in iteration k -- the updates
 * of panels 0 .. steps-2 applied; the rest of the matrix is left partly
 * updated.  steps >= n/b is hplai_factor.  One-panel trailing updates. */
int hplai_factor_steps(hplai_ctx *ctx, int steps);

/* Approximate factors without a decomposition (`--l1est`, pmatl1est,
 * matgen.hpp:108-144, main.cpp:282-301): the strictly lower part of the
 * generated matrix scaled column by column by float(1 / d_j), the upper part
 * and the diagonal kept, then marked factored for the refinement. */
int hplai_l1est(hplai_ctx *ctx);

/* Schedule tuner in place of lda_tuner (lda_tuner.hpp:9-45): times
 * hplai_factor on this context (regenerated from seed before each trial)
 * under each schedule -- one-, two- or four-panel groups (HPLAI_FLAG_GROUP2
 * when b % 128 == 0, HPLAI_FLAG_GROUP4 when the context was created with
 * it), serial or with HPLAI_FLAG_LOOKAHEAD at fixed side-stream SM
 * counts (16, 32) or at shares growing as the trailing matrix shrinks
 * (negative side_sms, see hplai_set_schedule: c = 8, 16, 24; 16, 20, 24,
 * 28, 32 for four-panel groups, whose optimum is sharper) -- after one discarded warm-up
 * factorisation, re-times the two
 * fastest twice more, keeps the one with the lowest median as the context's
 * schedule, then times that schedule twice under each of two other tile
 * orders of the Schur kernel (groups of 16 and 64 tile rows instead of 32,
 * hplai_set_tile_group) and keeps one only if both of its trials beat the
 * median by 0.5 %, then -- for the FP16 deck with groups of K >= 2048 --
 * the deck update's 256 x 256 tiles on CTA pairs instead of 128 x 256
 * (hplai_set_cta_pairs) by the same rule; leaves the context generated and
 * unfactored.  Outputs
 * (may be NULL): the chosen flags, the side-stream SM count and the chosen
 * configuration's factorisation time in ms. */
int hplai_autotune(hplai_ctx *ctx, uint64_t seed, unsigned *flags, int *side_sms, double *ms);
/* In the flags of hplai_get_autotune_trials / hplai_get_autotune_log: the
 * trial ran the deck update on CTA pairs. */
#define HPLAI_TRIAL_CTA_PAIRS 0x80000000u
/* Sets the schedule by hand, as hplai_autotune would: `flags` a combination
 * of HPLAI_FLAG_LOOKAHEAD and HPLAI_FLAG_GROUP2 or HPLAI_FLAG_GROUP4 (the
 * latter for contexts created with it; the other flags of the
 * context are kept), side_sms the SMs left to the side stream with
 * look-ahead: a fixed count (1 .. 64), or, negative, a share growing as the
 * trailing matrix shrinks -- with c = -side_sms (1 .. 256) the group whose
 * trailing matrix has r block columns left gets sms * c / (r + c) SMs, and
 * forms its panels on the whole GPU, without overlap, once that is more
 * than half of them.  The reference's schedule is fixed at build time
 * (panel_lu_async / RDMAPanelLU::run, panel_trf.hpp:434-858). */
int hplai_set_schedule(hplai_ctx *ctx, unsigned flags, int side_sms);
/* The trials of the last hplai_autotune in the order they ran (the warm-up
 * first): flags, side-stream SMs and factorisation ms of each; *count is
 * the number of trials (at most cap are written).  No counterpart in the
 * reference (lda_tuner prints its choice only). */
int hplai_get_autotune_log(hplai_ctx *ctx, unsigned *flags, int *side_sms, double *ms, int cap, int *count);
/* The same trials with the tile group each ran with (any output may be NULL). */
int hplai_get_autotune_trials(hplai_ctx *ctx, unsigned *flags, int *side_sms, int *tile_group, double *ms, int cap,
	int *count);
/* Tile order of the context's Schur launches: the persistent kernel sweeps
 * its tiles in groups of group_m tile rows (1 .. 1024; 0 restores the
 * default, 32), each group column by column, so that a group's L rows stay
 * in L2 while it crosses the trailing matrix.  Results do not depend on it. */
int hplai_set_tile_group(hplai_ctx *ctx, int group_m);
int hplai_get_tile_group(hplai_ctx *ctx, int *group_m);

/* The FP16-deck trailing update on CTA pairs: a cluster of two CTAs per
 * 256 x 256 tile, the leader issuing tcgen05 MMAs of M = 256 (cta_group::2)
 * over both CTAs' shared memory, so that each SM streams 32 KB of operands per
 * stage instead of 48 KB.  on = 1 or 0 for the context (-1: follow the
 * library default); with ctx = NULL, sets the library default (off at start),
 * which the leaf calls (hplai_f8gemm_deck_minus, hplai_shgemm_deck_minus)
 * follow.  Replaces nothing in the reference (its GEMM is a CPU kernel,
 * kernels/avx2.cpp:82-302); a performance setting, results are unchanged. */
int hplai_set_cta_pairs(hplai_ctx *ctx, int on);
/* The context's setting: 1, 0 or -1 (the library default). */
int hplai_get_cta_pairs(hplai_ctx *ctx, int *on);

/* iterative_refinement (iterative_refinement.hpp:18-57) with maxit steps
 * (the driver uses 50).  Fills *err ({-1,-1} on failure) and *iters (the
 * number of residual evaluations).  Returns HPLAI_ENOTCONV on failure.
 * mode HPLAI_IR corrects with x += U^{-1} L^{-1} r as the reference does;
 * HPLAI_GMRES corrects with one cycle of FP64 GMRES(restart) on
 * (LU)^{-1} A d = (LU)^{-1} r, same residual, harness and stopping test. */
int hplai_refine(hplai_ctx *ctx, int mode, int maxit, hplai_ir_errors *err, int *iters);
/* Solves with the context's factors for a caller's right-hand side (host
 * vectors of n doubles): A x = b, or the adjoint system A^T lambda = g
 * (U^T and L^T solves, A^T regenerated as element (j, i) = state j + n*i).
 * Same refinement, harness and stopping test as hplai_refine (the harness
 * is scaled by ||A||_inf and ||b||_inf); HPLAI_GMRES corrections for an
 * HPLAI_F32_F8 context, HPLAI_IR otherwise.  The context's own rhs and x
 * are left untouched; the refinement log is replaced.  No reference
 * counterpart: these serve the adjoint (gradient) of the solve. */
int hplai_solve_rhs(hplai_ctx *ctx, const double *b, double *x, int maxit, hplai_ir_errors *err, int *iters);
int hplai_solve_transpose(hplai_ctx *ctx, const double *g, double *lambda, int maxit, hplai_ir_errors *err,
	int *iters);
/* GMRES parameters: restart length (1..31, default 30) and the relative
 * reduction of the preconditioned residual that ends a cycle (default 1e-12). */
int hplai_set_gmres(hplai_ctx *ctx, int restart, double tol);
/* GMRES preconditioning side: 1 (default) right / flexible -- the basis of
 * A M^{-1} with the vectors z_j = M^{-1} v_j kept and the correction Z y, one
 * application of M^{-1} = (L U)^{-1} per inner step; 0 left -- the basis of
 * M^{-1} A, one more application (M^{-1} r) per cycle.  Both end a cycle
 * when the residual of their own system has fallen by the tolerance. */
int hplai_set_gmres_side(hplai_ctx *ctx, int right);
/* Residual evaluations and GMRES inner steps of the last hplai_refine. */
int hplai_get_refine_counts(hplai_ctx *ctx, int *outer, int *inner);

/* Copies of the results. */
int hplai_get_x(hplai_ctx *ctx, double *x);                      /* n doubles */
int hplai_get_lu(hplai_ctx *ctx, float *a, int64_t lda);           /* n x n FP32 */
int hplai_get_rhs(hplai_ctx *ctx, double *rhs);
int hplai_get_diag(hplai_ctx *ctx, double *diag);
/* panel_check (panel_check.hpp:9-65, `--checksum` at main.cpp:298-302):
 * sigs[0..2] (host) = FP64 sums of |a_ij| over the diagonal, the strict
 * upper and the strict lower triangle of the context's matrix -- the
 * factors after hplai_factor.  Deterministic for a given matrix; agrees with
 * the reference's sequential sums to rounding (the summation order differs). */
int hplai_checksum(hplai_ctx *ctx, double *sigs);
/* The per-step refinement log the reference prints (iterative_refinement.hpp:45):
 * up to `cap` entries; returns the number of steps through *count. */
int hplai_get_ir_log(hplai_ctx *ctx, double *residual, double *harness, int cap, int *count);
/* Accumulated milliseconds per hplai_phase since the last hplai_factor. */
int hplai_get_phase_ms(hplai_ctx *ctx, double *ms, int count);
/* The CUDA stream (cudaStream_t) every operation of this context runs on,
 * for callers that time or order work against it. */
void *hplai_get_stream(hplai_ctx *ctx);
/* ||A||_inf (= 2 max diag, panel_norm.hpp:78-84) and ||b||_inf. */
int hplai_get_norms(hplai_ctx *ctx, double *norma, double *normb);

/* One end-to-end solve through host buffers: upload, factor, refine and
 * copy x back (the whole of main.cpp's timed region plus the transfers).
 * Refines with HPLAI_IR, or HPLAI_GMRES for an HPLAI_F32_F8 context.  With
 * HPLAI_FLAG_FP16_DECK and a page-locked `a` (cudaHostAlloc / registered),
 * the matrix is copied panel by panel on a copy stream behind the
 * factorisation -- block column and row j arrive before panel j is formed,
 * which is the first time the deck form reads them -- so the transfer
 * overlaps the trailing updates; results are identical to the device path. */
int hplai_solve_host(hplai_ctx *ctx, const float *a, int64_t lda, const double *rhs,
	const double *diag, uint64_t seed, int maxit, double *x, hplai_ir_errors *err, int *iters);

/* The reference's report line (main.cpp:451-452) into buf:
 * "%.9f sec. %.9f GFlop/s resid = %20.15e hpl-harness = %.9f". */
int hplai_format_report(int n, double seconds, hplai_ir_errors err, char *buf, size_t len);

/* ---------------------------------------------------------------------- */
/* Batched solver (no reference counterpart: the reference solves one      */
/* system per run).                                                        */
/* ---------------------------------------------------------------------- */
typedef struct hplai_batch hplai_batch;

/* `count` independent systems: system s is the HPL-AI matrix of order n[s]
 * from seeds[s] (as hplai_generate) with nrhs[s] >= 1 right-hand sides,
 * columns n[s], n[s]+1, ... of its stream -- the reference's one-system
 * driver (main.cpp:144-492) over a batch.  The plain form (HPLAI_F32_F16,
 * flags 0, at most 8 right-hand sides per system) runs on the batched
 * engine: any n[s] >= 1 (padded with the identity to a multiple of 128,
 * 128-wide panels), every kernel over all systems at once, generation and
 * factorisation captured in one CUDA graph; `workers` is unused.  Other
 * forms give every system its own context (block size: the largest multiple
 * of 16 up to 512 dividing n[s]) fed by `workers` host threads (0: 8). */
int hplai_batch_create(hplai_batch **batch, int count, const int *n, const int *nrhs, const uint64_t *seeds,
	int precision, unsigned flags, int workers);
int hplai_batch_destroy(hplai_batch *batch);
/* Generate, factor and refine every right-hand side of every system
 * (largest systems first).  HPLAI_ENOTCONV if any right-hand side missed
 * hpl-harness < 16 within maxit steps. */
int hplai_batch_solve(hplai_batch *batch, int maxit);
/* System s: the largest hpl-harness over its right-hand sides ({-1,-1} on
 * failure), the most refinement steps any took, and its status. */
int hplai_batch_result(hplai_batch *batch, int s, hplai_ir_errors *worst, int *iters, int *status);
/* System s's solutions, n[s] x nrhs[s] column-major with leading dimension ldx. */
int hplai_batch_get_x(hplai_batch *batch, int s, double *x, int64_t ldx);
/* The block size chosen for system s. */
int hplai_batch_block(hplai_batch *batch, int s);
/* System s's factors after hplai_batch_solve: n[s] x n[s] FP32,
 * column-major with leading dimension lda (unit L below the diagonal, U on
 * and above) -- the reference's Panels after the LU (panel.hpp:20-60). */
int hplai_batch_get_lu(hplai_batch *batch, int s, float *a, int64_t lda);
/* Kernel launches per hplai_batch_solve of the batched engine's graph
 * (generation and factorisation; 0 for per-system contexts).  No
 * counterpart in the reference. */
unsigned long long hplai_batch_launches(hplai_batch *batch);

/* ---------------------------------------------------------------------- */
/* Leaf kernels on caller-owned device buffers.                            */
/* ---------------------------------------------------------------------- */

/* fill_one_panel_with_rand<float> (hpl_rand.hpp:59-106): the sub-matrix
 * (i0:i0+nrow, j0:j0+ncol) of the n x n HPL-AI matrix into `a` (FP32,
 * column-major, lda).  With calc_diag on a square diagonal block the
 * diagonal is float(sum_{j != i} |a_ij|) summed sequentially in FP64. */
int hplai_fill_panel(int n, int i0, int j0, int nrow, int ncol, float *a, int64_t lda,
	uint64_t seed, int calc_diag, void *stream);

/* pcolvgen (matgen.hpp:193-207): rhs_i = element (i, n) in FP64, i < n. */
int hplai_gen_rhs(int n, uint64_t seed, double *rhs, void *stream);
/* pcolvgen extended: out[i + r*n] = element (i, n + first + r), r < count. */
int hplai_gen_rhs_cols(int n, uint64_t seed, int first, int count, double *out, void *stream);

/* pdiaggen / calc_diag (matgen.hpp:209-225, hpl_rand.hpp:108-123):
 * d_i for i in [i0, i0+count). */
int hplai_gen_diag(int n, uint64_t seed, int i0, int count, double *d, void *stream);

/* getrf_nopiv<float> (getrf_nopiv.hpp:124-141): b x b no-pivot LU in place,
 * b <= 1024. */
int hplai_getrf_nopiv(int b, float *a, int64_t lda, void *stream);

/* update_left_panels + convert_left_panels (panel_trf.hpp:143-157,182-207):
 * a (m x b, lda) <- a * U^{-1} with U the upper triangle of u (b x b, ldu,
 * non-unit), then lh[i*ldh + k] = half(scale * a[i, k]) (row-major FP16
 * copy, the layout the Schur GEMM reads).  lh may be NULL. */
int hplai_trsm_right_upper(int m, int b, const float *u, int64_t ldu, float *a, int64_t lda,
	uint16_t *lh, int64_t ldh, float scale, void *stream);

/* update_right_panels + convert_right_panels (panel_trf.hpp:158-171,208-233):
 * a (b x ncols, lda) <- L^{-1} a with L the unit lower triangle of l
 * (b x b, ldl), then uh[j*ldh + k] = half(scale * a[k, j]).  uh may be NULL. */
int hplai_trsm_left_lower(int b, int ncols, const float *l, int64_t ldl, float *a, int64_t lda,
	uint16_t *uh, int64_t ldh, float scale, void *stream);

/* gemmschur -> shgemm with alpha = -1, beta = 1 (schur_updator.hpp:24-31,
 * fp16sim.hpp:216-233):  C (m x n FP32, ldc) -= L * U, FP32 accumulation,
 * on tcgen05 tensor cores.  L is m x k FP16 stored row-major
 * (lh[i*ldlh + p]), U is k x n FP16 stored column-major (uh[j*lduh + p]);
 * ldlh and lduh are multiples of 8 and the buffers 16-byte aligned. */
int hplai_shgemm_minus(int m, int n, int k, const uint16_t *lh, int64_t ldlh,
	const uint16_t *uh, int64_t lduh, float *c, int64_t ldc, void *stream);

/* Precision form (no reference counterpart; the down-cast follows
 * convert_left/right_panels, panel_trf.hpp:173-233, with one factor per 128
 * rows instead of one global factor).  X is rows x k FP32, element (r, p) at
 * src[r + p*lds] (col_major, an L panel) or src[p + r*lds] (a U panel read
 * by columns).  For each block of 128 rows, e = the exponent with
 * max|X_blk| = f 2^e, f in [0.5, 1) after dividing by 448; then
 * dst[r*ld8 + p] = e4m3_rn(X[r,p] 2^(-e)) (bytes k..ld8 of a row zero) and
 * scale[r/128] = 2^e.  ld8 is a multiple of 128; `bits` is scratch for
 * rows/128 + 1 words. */
int hplai_quantize_e4m3(int rows, int k, const float *src, int64_t lds, int col_major, uint8_t *dst,
	int64_t ld8, float *scale, unsigned *bits, void *stream);

/* C (m x n FP32, ldc) -= diag(sl) L8 U8^T diag(su): e4m3 operands row-major
 * with K contiguous (l8[i*ldl + p], u8[j*ldu + p]), exact products
 * accumulated in FP32 on tcgen05 (kind::f8f6f4) and scaled by the
 * power-of-two factors sl[i/128] su[j/128] before the update. */
int hplai_f8gemm_minus(int m, int n, int k, const uint8_t *l8, int64_t ldl, const float *sl,
	const uint8_t *u8, int64_t ldu, const float *su, float *c, int64_t ldc, void *stream);

/* The FP16-deck form of the two updates above (the double-decker lower
 * deck, lazy_init.hpp:92-227): deck (m x n FP16, column-major, ldd) <-
 * half_rn(deck - dscale * L U) (FP16 operands) or
 * half_rn(deck - dscale * diag(sl) L8 U8^T diag(su)) (e4m3 operands), the
 * product accumulated in FP32 and each deck element rounded once.  m and ldd
 * are multiples of 8 (the deck is stored in 16-byte units) and deck is
 * 16-byte aligned. */
int hplai_shgemm_deck_minus(int m, int n, int k, const uint16_t *lh, int64_t ldlh,
	const uint16_t *uh, int64_t lduh, uint16_t *deck, int64_t ldd, float dscale, void *stream);
int hplai_f8gemm_deck_minus(int m, int n, int k, const uint8_t *l8, int64_t ldl, const float *sl,
	const uint8_t *u8, int64_t ldu, const float *su, uint16_t *deck, int64_t ldd, float dscale,
	void *stream);

/* Workspace bytes for hplai_otf_gemv at order n. */
size_t hplai_otf_gemv_workspace(int n);

/* panel_gemv / otf_gemv (panel_gemv.hpp:57-180, otf_gemv.cpp:5-131) over the
 * whole matrix:  y <- beta*y + alpha * A x, A(i,j) regenerated in FP64 from
 * the LCG (seed) for i != j and A(i,i) = diag[i].  `work` holds at least
 * hplai_otf_gemv_workspace(n) bytes. */
int hplai_otf_gemv(int n, double alpha, const double *x, double beta, double *y,
	uint64_t seed, const double *diag, void *work, size_t work_bytes, void *stream);

/* otf_gemv_kernel (otf_gemv.cpp:5-7) on one off-diagonal sub-block:
 * y(0:mb) += alpha * A_sub x(0:nb) where `state00` is the LCG state of the
 * sub-block's (0,0) element and n the order of the whole matrix.  The
 * sub-block must not contain diagonal elements (otf_gemv.cpp:12-13).
 * `work` holds at least hplai_otf_gemv_workspace(max(mb,nb)) bytes. */
int hplai_otf_gemv_block(int64_t n, int mb, int nb, double alpha, const double *x, double *y,
	uint64_t state00, void *work, size_t work_bytes, void *stream);

/* Allocation-free variant of hplai_otf_gemv (no counterpart in the
 * reference): same arguments and result, minus the workspace.  For callers
 * that cannot allocate device memory -- code that only receives device
 * buffers from another runtime's allocator, or a solve loop that must not
 * call cudaMalloc because it can synchronise the device.  The partial sums go
 * to a scratch array compiled into the library (4 MiB on every GPU that
 * loads it, held until the process exits), so n <= HPLAI_OTF_GEMV_NOALLOC_MAX_N;
 * larger n returns HPLAI_EINVAL.  It allocates nothing.  The first call on
 * each device looks the array's device address up with that device current;
 * make that first call before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU (other streams, other host threads on
 * the same device) race on it -- serialise them. */
#define HPLAI_OTF_GEMV_NOALLOC_MAX_N 32768
int hplai_otf_gemv_noalloc(int n, double alpha, const double *x, double beta, double *y,
	uint64_t seed, const double *diag, void *stream);

/* Workspace bytes for the triangular solves at order n. */
size_t hplai_trsv_workspace(int n);

/* panel_trsvL / panel_trsvU (panel_trsv.hpp:310-758): x <- L^{-1} x with L
 * the unit lower triangle of a, or x <- U^{-1} x with U the upper triangle
 * of a (FP32 factors, FP64 vector).  `work` holds at least
 * hplai_trsv_workspace(n) bytes and must be zeroed before its first use. */
int hplai_trsv_lower(int n, const float *a, int64_t lda, double *x, void *work, size_t work_bytes, void *stream);
int hplai_trsv_upper(int n, const float *a, int64_t lda, double *x, void *work, size_t work_bytes, void *stream);

/* Workspace bytes for hplai_panel_check at order n (at most 28416). */
size_t hplai_panel_check_workspace(int n);
/* panel_check (panel_check.hpp:9-65) on caller buffers: sigs (device, 3
 * doubles) = FP64 sums of |a_ij| over the diagonal, strict upper and strict
 * lower triangle of a (n x n FP32, column-major, lda >= n).  `work` holds at
 * least hplai_panel_check_workspace(n) bytes; no clearing needed. */
int hplai_panel_check(int n, const float *a, int64_t lda, double *sigs, void *work, size_t work_bytes,
	void *stream);

/* colv_infnorm / calc_infnorm (panel_norm.hpp:8-41): *out = max_i |x_i|
 * written to device memory. */
int hplai_infnorm(int n, const double *x, double *out, void *stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* HPLAI_H */
