// gen.cu -- on-device HPL-AI matrix generator, bit-exact with the reference.
//
// Element (i, j) of the n x n matrix is the LCG state at linear index
// i + n*j after state_0 = a*seed + c, mapped to int64(x) * (1-2^-53)*2^-64
// (hpl_rand.hpp:35-106).  The diagonal is replaced by the sequential FP64
// sum of |a_ij| over j != i (hpl_rand.hpp:108-123); the right-hand side is
// column n of the same stream (matgen.hpp:193-207).  All arithmetic here is
// integer or explicitly rounded (__dmul_rn, __dadd_rn) so no contraction
// can change a bit.
#include "common.cuh"
#include "internal.h"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace hplai {

// inc1^(2^k) for k < 64, passed by value as a kernel parameter.
struct JumpTable {
	Coeff p[64];
};

static JumpTable make_jump_table()
{
	JumpTable t;
	Coeff p{kLcgA, kLcgC};
	for (int k = 0; k < 64; ++k) {
		t.p[k] = p;
		p = coeff_mul(p, p);
	}
	return t;
}

static const JumpTable &jump_table()
{
	static const JumpTable t = make_jump_table();
	return t;
}

__device__ __forceinline__ Coeff jump_of(const JumpTable &t, uint64_t m)
{
	Coeff r{1ULL, 0ULL};
	for (int k = 0; m; ++k, m >>= 1)
		if (m & 1ULL) r = coeff_mul(r, t.p[k]);
	return r;
}

constexpr int kFillRows = 256;  // rows per CTA (one per thread)
constexpr int kFillCols = 32;   // columns per CTA

// a(i, j) for i in [0,nrow), j in [0,ncol) of the sub-matrix at (i0, j0).
__global__ void __launch_bounds__(kFillRows) fill_kernel(int n, int i0, int j0, int nrow, int ncol, float *a,
	int64_t lda, uint64_t seed, JumpTable tab)
{
	const int r = blockIdx.x * kFillRows + threadIdx.x;
	const int c0 = blockIdx.y * kFillCols;
	if (r >= nrow) return;
	const Coeff jn = jump_of(tab, static_cast<uint64_t>(n));
	uint64_t s = coeff_apply(jump_of(tab, static_cast<uint64_t>(i0 + r) +
	                                          static_cast<uint64_t>(n) * static_cast<uint64_t>(j0 + c0)),
		state_initial(seed));
	const int c1 = min(c0 + kFillCols, ncol);
	float *col = a + static_cast<int64_t>(c0) * lda + r;
	for (int c = c0; c < c1; ++c) {
		*col = __double2float_rn(state_value(s));
		col += lda;
		s = coeff_apply(jn, s);
	}
}

// d_k = sum_{j != i} |a_ij| for i = i0 + k, summed in j order in FP64.
// Four interleaved LCG chains break the state dependency; the sum stays one
// sequential chain so the rounding matches hpl_rand.hpp:117-121 exactly.
// Writes the FP64 value to d (if non-null) and/or its FP32 rounding to the
// matrix diagonal a[(i - i0)*(lda+1)] (if non-null).
__global__ void __launch_bounds__(128) diag_kernel(int n, int i0, int count, double *d, float *adiag, int64_t lda,
	uint64_t seed, JumpTable tab)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= count) return;
	const int i = i0 + k;
	const Coeff jn = jump_of(tab, static_cast<uint64_t>(n));
	const Coeff jn4 = coeff_mul(coeff_mul(jn, jn), coeff_mul(jn, jn));
	uint64_t s0 = coeff_apply(jump_of(tab, static_cast<uint64_t>(i)), state_initial(seed));
	uint64_t s1 = coeff_apply(jn, s0);
	uint64_t s2 = coeff_apply(jn, s1);
	uint64_t s3 = coeff_apply(jn, s2);
	double sum = 0.0;
	int j = 0;
	for (; j + 3 < n; j += 4) {
		const double v0 = fabs(state_value(s0));
		const double v1 = fabs(state_value(s1));
		const double v2 = fabs(state_value(s2));
		const double v3 = fabs(state_value(s3));
		if (j != i) sum = __dadd_rn(sum, v0);
		if (j + 1 != i) sum = __dadd_rn(sum, v1);
		if (j + 2 != i) sum = __dadd_rn(sum, v2);
		if (j + 3 != i) sum = __dadd_rn(sum, v3);
		s0 = coeff_apply(jn4, s0);
		s1 = coeff_apply(jn4, s1);
		s2 = coeff_apply(jn4, s2);
		s3 = coeff_apply(jn4, s3);
	}
	for (; j < n; ++j) {
		if (j != i) sum = __dadd_rn(sum, fabs(state_value(s0)));
		s0 = coeff_apply(jn, s0);
	}
	if (d) d[k] = sum;
	if (adiag) adiag[static_cast<int64_t>(k) * (lda + 1)] = __double2float_rn(sum);
}

// out[k + r*n] = element (k, n + col0 + r) in FP64: column n of the stream is
// the right-hand side (pcolvgen), columns n+1, n+2, ... further ones.
__global__ void rhs_kernel(int n, int col0, int ncols, double *out, uint64_t seed, JumpTable tab)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= n) return;
	const Coeff jn = jump_of(tab, static_cast<uint64_t>(n));
	uint64_t s = coeff_apply(jump_of(tab, static_cast<uint64_t>(k) +
	                                          static_cast<uint64_t>(n) * (static_cast<uint64_t>(n) + col0)),
		state_initial(seed));
	for (int r = 0; r < ncols; ++r) {
		out[k + static_cast<int64_t>(r) * n] = state_value(s);
		s = coeff_apply(jn, s);
	}
}

// pmatl1est (matgen.hpp:108-144): approximate factors without a
// decomposition -- the strictly lower part scaled column by column,
// a_ij <- a_ij * float(1 / d_j) for i > j (d_j the FP64 row sum, rounded to
// FP32 after the division, as the reference's FHIGH d = buf[jj]), the upper
// part and the diagonal kept.
__global__ void __launch_bounds__(256) l1est_kernel(int n, float *__restrict__ a, int64_t lda,
	const double *__restrict__ d)
{
	for (int j = blockIdx.y; j < n; j += gridDim.y) {
		const float inv = static_cast<float>(1.0 / d[j]);
		float *col = a + static_cast<int64_t>(j) * lda;
		for (int i = j + 1 + blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) col[i] *= inv;
	}
}

int launch_l1est(int n, float *a, int64_t lda, const double *d, cudaStream_t st)
{
	if (n <= 1) return HPLAI_OK;
	// grid.y is limited to 65535: columns beyond it are taken in a grid stride
	l1est_kernel<<<dim3(static_cast<unsigned>((n + 255) / 256 < 8 ? (n + 255) / 256 : 8),
		static_cast<unsigned>(n < 65535 ? n : 65535)), 256, 0, st>>>(n, a, lda, d);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

// Lazy initialisation of the double-decker LU (`-d`,
// LazyInitializer<FLow,1,true>::update/update_diag, lazy_init.hpp:92-227):
// a block's FP32 value is formed only when it joins a panel, as
//     a(i, j) = fma(downscale, deck(i, j), a0(i, j)),
// one fused multiply-add like the reference's x86 build, with the initial
// value a0 regenerated from the LCG (float(d_i) on the diagonal, d the FP64
// row sums) when `regen`, or read from a (an uploaded matrix) otherwise;
// with a back buffer the deck value is deck + 32 back.  Rows [r0, r1) x
// columns [c0, c1), one thread per row; deck (and back) element (i, j) at
// [(j - dc0) * ldd + (i - dr0)].
__global__ void __launch_bounds__(kFillRows) lazy_init_kernel(int n, int r0, int r1, int c0, int c1,
	float *__restrict__ a, int64_t lda, const __half *__restrict__ deck, const __half *__restrict__ back, int64_t ldd,
	int dr0, int dc0, float downscale, uint64_t seed, const double *__restrict__ d, int regen, JumpTable tab)
{
	const int i = r0 + blockIdx.x * kFillRows + threadIdx.x;
	const int j0 = c0 + blockIdx.y * kFillCols;
	if (i >= r1) return;
	const Coeff jn = jump_of(tab, static_cast<uint64_t>(n));
	uint64_t s = regen ? coeff_apply(jump_of(tab, static_cast<uint64_t>(i) +
	                                               static_cast<uint64_t>(n) * static_cast<uint64_t>(j0)),
	                         state_initial(seed))
	                   : 0;
	const int j1 = min(j0 + kFillCols, c1);
	for (int j = j0; j < j1; ++j) {
		const int64_t o = static_cast<int64_t>(j) * lda + i;
		float a0;
		if (regen) {
			a0 = (i == j) ? __double2float_rn(d[i]) : __double2float_rn(state_value(s));
			s = coeff_apply(jn, s);
		} else {
			a0 = a[o];
		}
		const int64_t od = static_cast<int64_t>(j - dc0) * ldd + (i - dr0);
		// with the back buffer: deck + 32 back (lazy_init_omp.cpp:704-760)
		const float x = back ? __fmaf_rn(32.0f, __half2float(back[od]), __half2float(deck[od])) : __half2float(deck[od]);
		a[o] = __fmaf_rn(downscale, x, a0);
	}
}

int launch_lazy_init(int n, int r0, int r1, int c0, int c1, float *a, int64_t lda, const uint16_t *deck,
	const uint16_t *back, int64_t ldd, int dr0, int dc0, float downscale, uint64_t seed, const double *d, bool regen,
	cudaStream_t st)
{
	if (r1 <= r0 || c1 <= c0) return HPLAI_OK;
	dim3 grid((r1 - r0 + kFillRows - 1) / kFillRows, (c1 - c0 + kFillCols - 1) / kFillCols);
	lazy_init_kernel<<<grid, kFillRows, 0, st>>>(n, r0, r1, c0, c1, a, lda, reinterpret_cast<const __half *>(deck),
		reinterpret_cast<const __half *>(back), ldd, dr0, dc0, downscale, seed, d, regen ? 1 : 0, jump_table());
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

// ---------------------------------------------------------------------------
// Higham's HPL-AI matrix (--highammat; higham_mat_impl.cpp, from Higham's
// hpl-ai-matrix): A = L U with L unit lower triangular with every strictly
// lower entry -alpha and U unit upper triangular with every strictly upper
// entry -beta, so a_ij = -beta + ab i above the diagonal, 1 + ab i on it and
// -alpha + ab j below it (ab = alpha beta).  beta is found by bisection so
// that an estimate of cond(A, inf) equals kappa, alpha = rho beta.
// ---------------------------------------------------------------------------
namespace {

// 32-bit int arithmetic with wrap-around: the reference evaluates the
// estimate's integer terms in int, which wraps from about n = 46341 on, and
// alpha and beta are kept identical to its values for every n.
int32_t wrap32(int64_t v) { return static_cast<int32_t>(static_cast<uint32_t>(static_cast<uint64_t>(v))); }
int32_t imul(int32_t a, int32_t b) { return wrap32(static_cast<int64_t>(a) * b); }

// the condition-number estimate for (a, b) (fhpl, higham_mat_impl.cpp:38-61)
double cond_estimate(int n, double a, double b)
{
	if (std::isnan(a)) a = b / 2;
	const double l1 = 1 + (n - 1) * b;
	const int id = std::min(static_cast<int>(std::floor(1. / a)), n);
	const int k = std::min(static_cast<int>(std::floor((1 + b) / b)), n - 1);
	int32_t t = wrap32(static_cast<int64_t>(imul(-k, k)) + k);
	t = wrap32(static_cast<int64_t>(t) + imul(imul(3, id), id - 1) / 2);
	t = wrap32(static_cast<int64_t>(t) - imul(n, id));
	t = wrap32(static_cast<int64_t>(t) + n);
	const double lid = 1 + (2 * k - id + 1) * a + (n - id) * b + static_cast<double>(t) * a * b;
	const int32_t u = wrap32(static_cast<int64_t>(wrap32(static_cast<int64_t>(imul(-k, k)) + k)) + imul(n, n - 1) / 2);
	const double ln = 1 + (2 * k - n + 1) * a + static_cast<double>(u) * a * b;
	const double na = std::max(std::max(l1, lid), ln);
	const double r = (1 + a) * (1 + b);
	const double d1 = (1 + a) * (1. / (1 + a) + (r == 0. ? 0. : b * (1 - std::pow(r, n - 1)) / (1 - r)));
	const double dn = std::pow(1 + a, n) * (1. / (1 + a));
	const double ret = na * std::max(d1, dn);
	return std::isinf(ret) ? DBL_MAX : ret;
}

// bisection on cond_estimate(rho x, x) - kappa (zero_find, higham_mat_impl.cpp:63-84)
double bisect_beta(int n, double kappa, double rho, double lo, double hi)
{
	auto f = [&](double x) { return cond_estimate(n, rho * x, x) - kappa; };
	if (f(lo) > 0. || f(hi) < 0.) return std::nan("");
	for (;;) {
		if (hi - lo < (2. * std::fabs(hi) + 0.5) * DBL_EPSILON) break;
		const double mid = (lo + hi) / 2;
		if (mid == lo || mid == hi) break;
		const double fm = f(mid);
		if (fm == 0.) return mid;
		(fm < 0. ? lo : hi) = mid;
	}
	return hi;
}

// The FP32 matrix as the reference forms it in float (lazy_init.hpp:331-440:
// one fused multiply-add of alpha_f beta_f, the index and -beta_f / -alpha_f
// / 1) and the FP64 diagonal fma(ab, i, 1) (pdiaggen, matgen.hpp:227-243).
__global__ void __launch_bounds__(kFillRows) higham_fill_kernel(int n, float abf, float mb, float ma,
	float *__restrict__ a, int64_t lda, double ab, double *__restrict__ d)
{
	const int i = blockIdx.x * kFillRows + threadIdx.x;
	const int j0 = blockIdx.y * kFillCols;
	if (i >= n) return;
	const float fi = static_cast<float>(i);
	const float up = __fmaf_rn(abf, fi, mb);
	const int j1 = min(j0 + kFillCols, n);
	for (int j = j0; j < j1; ++j) {
		const float v = i < j ? up : (i > j ? __fmaf_rn(abf, static_cast<float>(j), ma) : __fmaf_rn(abf, fi, 1.0f));
		a[static_cast<int64_t>(j) * lda + i] = v;
	}
	if (blockIdx.y == 0 && d) d[i] = fma(ab, static_cast<double>(i), 1.0);
}

} // namespace

double higham_beta(int n, double kappa, double rho)
{
	if (n < 2 || !(kappa > 1.) || !(rho > 0.)) return std::nan("");
	// higham_mat_comp_beta (higham_mat_impl.cpp:87-113)
	const double lo = DBL_EPSILON;
	double hi = 1. / rho;
	for (int k = 1;;) {
		const double v = cond_estimate(n, rho * hi, hi) - kappa;
		if (std::isfinite(v) && v > 0.) break;
		hi *= 0.5;
		if (++k == 100) break;
	}
	double beta = bisect_beta(n, kappa, rho, lo, hi);
	while (rho * beta > 1.) {
		hi *= 0.25;
		beta = bisect_beta(n, kappa, rho, lo, hi);
	}
	return beta;
}

double higham_norm(int n, double alpha, double beta)
{
	// largest row sum of |a_ij|: the lower constants of the columns before the
	// row, the diagonal, the row's upper constant n - 1 - i times
	const double ab = alpha * beta;
	long double best = 0, lower = 0;
	for (int i = 0; i < n; ++i) {
		const long double row = lower + std::fabs(std::fma(ab, static_cast<double>(i), 1.0)) +
			static_cast<long double>(n - 1 - i) * std::fabs(std::fma(ab, static_cast<double>(i), -beta));
		best = std::max(best, row);
		lower += std::fabs(std::fma(ab, static_cast<double>(i), -alpha));
	}
	return static_cast<double>(best);
}

int launch_higham_fill(int n, double alpha, double beta, float *a, int64_t lda, double *d, bool factors, cudaStream_t st)
{
	if (n <= 0) return HPLAI_OK;
	const float af = static_cast<float>(alpha), bf = static_cast<float>(beta);
	dim3 grid((n + kFillRows - 1) / kFillRows, (n + kFillCols - 1) / kFillCols);
	// factors: ab = 0 leaves -beta above, 1 on and -alpha below the diagonal,
	// the exact unit-L / U factors in the one-array layout
	higham_fill_kernel<<<grid, kFillRows, 0, st>>>(n, factors ? 0.0f : af * bf, -bf, -af, a, lda, alpha * beta,
		factors ? nullptr : d);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_fill(int n, int i0, int j0, int nrow, int ncol, float *a, int64_t lda, uint64_t seed, int calc_diag,
	cudaStream_t st)
{
	if (nrow <= 0 || ncol <= 0) return HPLAI_OK;
	dim3 grid((nrow + kFillRows - 1) / kFillRows, (ncol + kFillCols - 1) / kFillCols);
	fill_kernel<<<grid, kFillRows, 0, st>>>(n, i0, j0, nrow, ncol, a, lda, seed, jump_table());
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	if (calc_diag && i0 == j0 && nrow == ncol) {
		diag_kernel<<<(nrow + 127) / 128, 128, 0, st>>>(n, i0, nrow, nullptr, a, lda, seed, jump_table());
		count_launches();
		HPLAI_CUDA_TRY(cudaGetLastError());
	}
	return HPLAI_OK;
}

int launch_diag(int n, int i0, int count, double *d, float *adiag, int64_t lda, uint64_t seed, cudaStream_t st)
{
	if (count <= 0) return HPLAI_OK;
	diag_kernel<<<(count + 127) / 128, 128, 0, st>>>(n, i0, count, d, adiag, lda, seed, jump_table());
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_rhs(int n, double *rhs, uint64_t seed, cudaStream_t st)
{
	return launch_rhs_cols(n, 0, 1, rhs, seed, st);
}

int launch_rhs_cols(int n, int col0, int ncols, double *out, uint64_t seed, cudaStream_t st)
{
	if (n <= 0 || ncols <= 0) return HPLAI_OK;
	rhs_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, col0, ncols, out, seed, jump_table());
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

} // namespace hplai

extern "C" int hplai_fill_panel(int n, int i0, int j0, int nrow, int ncol, float *a, int64_t lda, uint64_t seed,
	int calc_diag, void *stream)
{
	if (n <= 0 || i0 < 0 || j0 < 0 || nrow < 0 || ncol < 0 || !a || lda < nrow) return HPLAI_EINVAL;
	return hplai::launch_fill(n, i0, j0, nrow, ncol, a, lda, seed, calc_diag, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_gen_rhs(int n, uint64_t seed, double *rhs, void *stream)
{
	if (n <= 0 || !rhs) return HPLAI_EINVAL;
	return hplai::launch_rhs(n, rhs, seed, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_gen_rhs_cols(int n, uint64_t seed, int first, int count, double *out, void *stream)
{
	if (n <= 0 || first < 0 || count < 0 || !out) return HPLAI_EINVAL;
	return hplai::launch_rhs_cols(n, first, count, out, seed, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_gen_diag(int n, uint64_t seed, int i0, int count, double *d, void *stream)
{
	if (n <= 0 || i0 < 0 || count < 0 || i0 + count > n || !d) return HPLAI_EINVAL;
	return hplai::launch_diag(n, i0, count, d, nullptr, 0, seed, static_cast<cudaStream_t>(stream));
}
