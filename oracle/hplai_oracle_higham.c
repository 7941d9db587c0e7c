/*
 * hplai_oracle_higham.c -- CPU oracle for Higham's HPL-AI matrix
 * (`driver.out ... --highammat`).
 *
 * TEST INFRASTRUCTURE ONLY, like hplai_oracle.c: the CUDA library never
 * links, loads or calls it.
 *
 * The matrix (higham_mat_impl.cpp:116-128, from Higham's hpl-ai-matrix) is
 * A = L U with L unit lower triangular, every strictly lower entry -alpha,
 * and U unit upper triangular, every strictly upper entry -beta:
 *     a_ij = -beta  + alpha beta i   (i < j)
 *     a_ii =  1     + alpha beta i
 *     a_ij = -alpha + alpha beta j   (i > j)
 * with beta chosen by bisection so that the estimate of cond(A, inf)
 * equals kappa (1000 in the reference's driver) and alpha = rho beta
 * (rho = 1/2): higham_mat_comp_beta, fhpl and zero_find,
 * higham_mat_impl.cpp:38-113, restated below.  The reference evaluates the
 * integer parts of the estimate in 32-bit int, which wraps from about
 * n = 46341 on (at n = 65536 it moves beta by 1 %); the restatement
 * reproduces that wrap so that alpha and beta are the reference's for every n.
 *
 * Values as the reference forms them: the FP32 matrix element
 * fmaf(alpha_f beta_f, (float)idx, c_f) with c = -beta or -alpha in FP32
 * (the lazy initialisation's float arithmetic, lazy_init.hpp:331-440, one
 * fused multiply-add in its x86 build), the FP64 element
 * fma(alpha beta, idx, c) (otf_gemv.cpp:133-314, svmla), the FP64 diagonal
 * fma(alpha beta, i, 1) (pdiaggen, matgen.hpp:227-243).  The right-hand side
 * stays column n of the LCG stream (pcolvgen with Matgen, main.cpp:266).
 *
 * Compiled with -ffp-contract=off, like hplai_oracle.c.
 */
#include <stdint.h>
#include <stdlib.h>
#include <math.h>
#include <float.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* 32-bit int arithmetic with wrap-around, as the reference's int
 * expressions compute on x86 */
static int32_t w32(int64_t v) { return (int32_t)(uint32_t)(uint64_t)v; }
static int32_t mul32(int32_t a, int32_t b) { return w32((int64_t)a * b); }
static int32_t add32(int32_t a, int32_t b) { return w32((int64_t)a + b); }
static int32_t sub32(int32_t a, int32_t b) { return w32((int64_t)a - b); }

/* fhpl: the estimate of cond(A, inf) for parameters (alpha, beta),
 * higham_mat_impl.cpp:38-61 */
static double cond_estimate(int n, double a, double b)
{
	if (isnan(a)) a = b / 2;
	const double lambda_1 = 1 + (n - 1) * b;
	int idash = (int)floor(1. / a);
	if (idash > n) idash = n;
	int k = (int)floor((1 + b) / b);
	if (k > n - 1) k = n - 1;
	/* -k*k + k + 3*idash*(idash-1)/2 - n*idash + n, in int */
	int32_t t = add32(mul32(-k, k), k);
	t = add32(t, mul32(mul32(3, idash), idash - 1) / 2);
	t = sub32(t, mul32(n, idash));
	t = add32(t, n);
	const double lambda_idash = 1 + (2 * k - idash + 1) * a + (n - idash) * b + (double)t * a * b;
	/* -k*k + k + n*(n-1)/2, in int */
	int32_t u = add32(add32(mul32(-k, k), k), mul32(n, n - 1) / 2);
	const double lambda_n = 1 + (2 * k - n + 1) * a + (double)u * a * b;
	double na = lambda_1 > lambda_idash ? lambda_1 : lambda_idash;
	if (lambda_n > na) na = lambda_n;
	const double r = (1 + a) * (1 + b);
	const double delta1 = (1 + a) * (1. / (1 + a) + (r == 0. ? 0. : b * (1 - pow(r, n - 1)) / (1 - r)));
	const double deltan = pow(1 + a, n) * (1. / (1 + a));
	const double ninv = delta1 > deltan ? delta1 : deltan;
	const double ret = na * ninv;
	return isinf(ret) ? DBL_MAX : ret;
}

/* zero_find: bisection on cond_estimate(n, rho x, x) - kappa over
 * [left, right], higham_mat_impl.cpp:63-84 */
static double bisect(int n, double kappa, double rho, double left, double right)
{
	const double fl = cond_estimate(n, rho * left, left) - kappa;
	const double fr = cond_estimate(n, rho * right, right) - kappa;
	if (fl > 0. || fr < 0.) return NAN;
	for (;;) {
		const double tol = (2. * fabs(right) + 0.5) * DBL_EPSILON;
		if (right - left < tol) break;
		const double mid = (left + right) / 2;
		if (mid == left || mid == right) break;
		const double fm = cond_estimate(n, rho * mid, mid) - kappa;
		if (fm == 0.) return mid;
		if (fm < 0.) left = mid;
		else right = mid;
	}
	return right;
}

/* higham_mat_comp_beta, higham_mat_impl.cpp:87-113 */
ORC_EXPORT double orc_higham_beta(int n, double kappa, double rho)
{
	const double left = DBL_EPSILON;
	double right = 1. / rho;
	for (int k = 1;;) {
		const double v = cond_estimate(n, rho * right, right) - kappa;
		if (isfinite(v) && v > 0.) break;
		right *= 0.5;
		if (++k == 100) break;
	}
	double beta = bisect(n, kappa, rho, left, right);
	while (rho * beta > 1.) {
		right *= 0.5;
		right = right / 2;
		beta = bisect(n, kappa, rho, left, right);
	}
	return beta;
}

/* FP32 sub-matrix (i0:i0+nrow, j0:j0+ncol), column-major with lda */
ORC_EXPORT void orc_higham_fill(int i0, int j0, int nrow, int ncol, double alpha, double beta, float *a, int64_t lda)
{
	const float af = (float)alpha, bf = (float)beta;
	const float abf = af * bf, ma = -af, mb = -bf;
	for (int jj = 0; jj < ncol; jj++) {
		const int j = j0 + jj;
		for (int ii = 0; ii < nrow; ii++) {
			const int i = i0 + ii;
			float v;
			if (i < j) v = fmaf(abf, (float)i, mb);
			else if (i > j) v = fmaf(abf, (float)j, ma);
			else v = fmaf(abf, (float)j, 1.0f);
			a[(int64_t)jj * lda + ii] = v;
		}
	}
}

/* the FP64 element and diagonal */
ORC_EXPORT double orc_higham_elem(int64_t i, int64_t j, double alpha, double beta)
{
	const double ab = alpha * beta;
	if (i < j) return fma(ab, (double)i, -beta);
	if (i > j) return fma(ab, (double)j, -alpha);
	return fma(ab, (double)i, 1.0);
}

ORC_EXPORT void orc_higham_diag(int n, double alpha, double beta, double *d)
{
	for (int i = 0; i < n; i++) d[i] = orc_higham_elem(i, i, alpha, beta);
}

/* ||A||_inf: the largest row sum of |a_ij| (long double, then FP64) */
ORC_EXPORT double orc_higham_norm(int n, double alpha, double beta)
{
	long double best = 0, lower = 0;   /* lower = sum_{j<i} |a_ij| */
	for (int i = 0; i < n; i++) {
		const long double row = lower + fabsl((long double)orc_higham_elem(i, i, alpha, beta)) +
			(long double)(n - 1 - i) * fabsl((long double)orc_higham_elem(i, i + 1, alpha, beta));
		if (row > best) best = row;
		lower += fabsl((long double)orc_higham_elem(i + 1, i, alpha, beta));
	}
	return (double)best;
}

/* r_t = b_t - sum_j a(rows[t], j) x_j in long double over the FP64
 * elements: the independent residual check */
ORC_EXPORT void orc_higham_residual_rows(int n, double alpha, double beta, const double *x, const int64_t *rows,
	int count, const double *rhs, double *r)
{
	for (int t = 0; t < count; t++) {
		const int64_t i = rows[t];
		long double acc = 0;
		for (int64_t j = 0; j < n; j++) acc += (long double)orc_higham_elem(i, j, alpha, beta) * (long double)x[j];
		r[t] = (double)((long double)rhs[i] - acc);
	}
}
