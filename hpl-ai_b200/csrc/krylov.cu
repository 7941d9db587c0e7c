// krylov.cu -- FP64 vector kernels of the GMRES correction (refinement mode
// HPLAI_GMRES).
//
// GMRES-IR replaces the correction x += U^{-1} L^{-1} r of the classical
// refinement (iterative_refinement.hpp:50-53) by a restarted GMRES solve of
// A d = r, left-preconditioned by the same LU factors, so that a factor of
// lower quality (e4m3 Schur updates) still yields an FP64 solution in few
// outer steps.  The basis V (n x (m+1), column-major) stays in HBM; the
// orthogonalisation is classical Gram-Schmidt applied twice (CGS2), whose
// projections are one pass over V per sweep instead of j passes.
//
// Every reduction is deterministic: a fixed grid of kDotBlocks CTAs, each
// owning a fixed contiguous slice of rows, writes per-CTA partial sums that
// a single thread per output then folds in CTA order.
#include "common.cuh"
#include "internal.h"

namespace hplai {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void slice_of(int n, int &r0, int &r1)
{
	const int chunk = (n + kDotBlocks - 1) / kDotBlocks;
	r0 = min(n, static_cast<int>(blockIdx.x) * chunk);
	r1 = min(n, r0 + chunk);
}

// Sum over the CTA of one value per thread, in a fixed order; result valid in
// thread 0.
__device__ __forceinline__ double block_sum(double v, double *sh)
{
	for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	__syncthreads();
	if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
	__syncthreads();
	double s = 0.0;
	if (threadIdx.x == 0)
		for (int w = 0; w < kThreads / 32; ++w) s += sh[w];
	return s;
}

// part[cta * kMaxBasis + i] = sum over the CTA's rows of V_i[r] * w[r], i < nv.
__global__ void __launch_bounds__(kThreads) dots_kernel(int n, int nv, const double *__restrict__ v, int64_t ldv,
	const double *__restrict__ w, double *__restrict__ part)
{
	__shared__ double sh[kThreads / 32];
	int r0, r1;
	slice_of(n, r0, r1);
	double acc[kMaxBasis];
#pragma unroll
	for (int i = 0; i < kMaxBasis; ++i) acc[i] = 0.0;
	for (int r = r0 + threadIdx.x; r < r1; r += kThreads) {
		const double wr = w[r];
#pragma unroll
		for (int i = 0; i < kMaxBasis; ++i)
			if (i < nv) acc[i] = fma(v[static_cast<int64_t>(i) * ldv + r], wr, acc[i]);
	}
#pragma unroll
	for (int i = 0; i < kMaxBasis; ++i) {
		if (i >= nv) break;
		const double s = block_sum(acc[i], sh);
		if (threadIdx.x == 0) part[static_cast<int64_t>(blockIdx.x) * kMaxBasis + i] = s;
	}
}

// w -= V h (h on the device, nv entries); optionally the CTA's partial sum of
// the updated w[r]^2 into part[cta * kMaxBasis].
__global__ void __launch_bounds__(kThreads) gs_update_kernel(int n, int nv, const double *__restrict__ v, int64_t ldv,
	const double *__restrict__ h, double *__restrict__ w, double *__restrict__ part)
{
	__shared__ double sh[kThreads / 32];
	__shared__ double hs[kMaxBasis];
	if (threadIdx.x < nv) hs[threadIdx.x] = h[threadIdx.x];
	__syncthreads();
	int r0, r1;
	slice_of(n, r0, r1);
	double sq = 0.0;
	for (int r = r0 + threadIdx.x; r < r1; r += kThreads) {
		double wr = w[r];
		for (int i = 0; i < nv; ++i) wr = fma(-hs[i], v[static_cast<int64_t>(i) * ldv + r], wr);
		w[r] = wr;
		sq = fma(wr, wr, sq);
	}
	if (part) {
		const double s = block_sum(sq, sh);
		if (threadIdx.x == 0) part[static_cast<int64_t>(blockIdx.x) * kMaxBasis] = s;
	}
}

// out[i] (op) sum over CTAs of part[cta * kMaxBasis + i], CTAs in order.
// op 0: out = s; 1: out += s; 2: out = sqrt(s).
__global__ void fold_kernel(int nv, const double *__restrict__ part, double *out, int op)
{
	const int i = threadIdx.x;
	if (i >= nv) return;
	double s = 0.0;
	for (int c = 0; c < kDotBlocks; ++c) s += part[static_cast<int64_t>(c) * kMaxBasis + i];
	out[i] = op == 0 ? s : op == 1 ? out[i] + s : sqrt(s);
}

__global__ void add_small_kernel(int nv, const double *__restrict__ a, double *b)
{
	if (threadIdx.x < nv) b[threadIdx.x] += a[threadIdx.x];
}

// out = w / *den
__global__ void scale_kernel(int n, const double *__restrict__ w, const double *__restrict__ den, double *out)
{
	const double d = *den;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = w[i] / d;
}

// x += V y (y on the device, nv entries), terms summed in basis order.
__global__ void combine_kernel(int n, int nv, const double *__restrict__ v, int64_t ldv, const double *__restrict__ y,
	double *x)
{
	__shared__ double ys[kMaxBasis];
	if (threadIdx.x < nv) ys[threadIdx.x] = y[threadIdx.x];
	__syncthreads();
	for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
		double d = 0.0;
		for (int i = 0; i < nv; ++i) d = fma(ys[i], v[static_cast<int64_t>(i) * ldv + r], d);
		x[r] += d;
	}
}

int grid_for(int n)
{
	int g = (n + kThreads - 1) / kThreads;
	return g > 4 * 148 ? 4 * 148 : (g < 1 ? 1 : g);
}

} // namespace

int launch_dots(int n, int nv, const double *v, int64_t ldv, const double *w, double *part, double *out, int op,
	cudaStream_t st)
{
	if (nv <= 0 || nv > kMaxBasis || n <= 0) return HPLAI_EINVAL;
	dots_kernel<<<kDotBlocks, kThreads, 0, st>>>(n, nv, v, ldv, w, part);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	fold_kernel<<<1, 32, 0, st>>>(nv, part, out, op);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_gs_update(int n, int nv, const double *v, int64_t ldv, const double *h, double *w, double *part,
	double *norm_out, cudaStream_t st)
{
	if (nv <= 0 || nv > kMaxBasis || n <= 0) return HPLAI_EINVAL;
	gs_update_kernel<<<kDotBlocks, kThreads, 0, st>>>(n, nv, v, ldv, h, w, norm_out ? part : nullptr);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	if (norm_out) {
		fold_kernel<<<1, 32, 0, st>>>(1, part, norm_out, 2);
		count_launches();
		HPLAI_CUDA_TRY(cudaGetLastError());
	}
	return HPLAI_OK;
}

int launch_add_small(int nv, const double *a, double *b, cudaStream_t st)
{
	add_small_kernel<<<1, 32, 0, st>>>(nv, a, b);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_scale(int n, const double *w, const double *den, double *out, cudaStream_t st)
{
	scale_kernel<<<grid_for(n), kThreads, 0, st>>>(n, w, den, out);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_combine(int n, int nv, const double *v, int64_t ldv, const double *y, double *x, cudaStream_t st)
{
	if (nv <= 0) return HPLAI_OK;
	if (nv > kMaxBasis) return HPLAI_EINVAL;
	combine_kernel<<<grid_for(n), kThreads, 0, st>>>(n, nv, v, ldv, y, x);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

} // namespace hplai
