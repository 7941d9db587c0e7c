// panel.cu -- FP32 panel factorisation kernels for the blocked no-pivot LU.
//
//  getrf_kernel     : b x b diagonal block LU in one CTA (getrf_nopiv.hpp:30-141)
//  trsm_ru_kernel   : L panel  A_col <- A_col * U^{-1}, plus its FP16 copy
//                     (update_left_panels + convert_left_panels, panel_trf.hpp:143-157,182-207)
//  trsm_ll_kernel   : U panel  A_row <- L^{-1} * A_row, plus its FP16 copy
//                     (update_right_panels + convert_right_panels, panel_trf.hpp:158-171,208-233)
//
// Every element receives its updates a_ij <- fma(-l_ik, u_kj, a_ij) in
// increasing k, and the multipliers are formed as a_ik * (1/u_kk), which
// is exactly the operation sequence of the reference's unblocked kernel and
// of netlib strsm (getrf_nopiv.hpp:33-44), so these kernels reproduce a
// sequential FP32 factorisation bit for bit whatever their blocking.
#include "common.cuh"
#include "internal.h"

namespace hplai {

// ---------------------------------------------------------------------------
// Diagonal block LU.
// ---------------------------------------------------------------------------
constexpr int kGetrfThreads = 1024;

template <int NB>
__global__ void __launch_bounds__(kGetrfThreads, 1) getrf_kernel(int b, float *__restrict__ a, int64_t lda)
{
	extern __shared__ float sm[];
	float *Lp = sm;                // panel, column-major: Lp[c*b + r], r relative to kb
	float *Up = sm + b * NB;       // U12 rows: Up[i*b + c], c relative to kb+w
	float *prow = Up + NB * b;     // two pivot-row buffers of NB floats
	const int t = threadIdx.x;

	for (int kb = 0; kb < b; kb += NB) {
		const int w = min(NB, b - kb);
		const int mrows = b - kb;
		const int rem = mrows - w;

		// Phase 1: factor the (b-kb) x w column panel, one row per thread.
		float p[NB];
		const bool own = t < mrows;
#pragma unroll
		for (int c = 0; c < NB; ++c)
			p[c] = (own && c < w) ? a[static_cast<int64_t>(kb + c) * lda + kb + t] : 0.f;
#pragma unroll
		for (int j = 0; j < NB; ++j) {
			if (j < w) {
				float *pr = prow + (j & 1) * NB;
				if (t == j) {
#pragma unroll
					for (int c = 0; c < NB; ++c) pr[c] = p[c];
				}
				__syncthreads();
				if (own && t > j) {
					const float inv = 1.0f / pr[j];
					const float l = p[j] * inv;
					p[j] = l;
#pragma unroll
					for (int c = j + 1; c < NB; ++c)
						if (c < w) p[c] = fmaf(-l, pr[c], p[c]);
				}
			}
		}
		if (own) {
#pragma unroll
			for (int c = 0; c < NB; ++c) {
				if (c < w) {
					a[static_cast<int64_t>(kb + c) * lda + kb + t] = p[c];
					Lp[c * b + t] = p[c];
				}
			}
		}
		__syncthreads();
		if (rem <= 0) break;

		// Phase 2: U12 = L11^{-1} A12 (unit lower), one column per thread.
		if (t < rem) {
			float q[NB];
			float *colp = a + static_cast<int64_t>(kb + w + t) * lda + kb;
#pragma unroll
			for (int i = 0; i < NB; ++i) q[i] = (i < w) ? colp[i] : 0.f;
#pragma unroll
			for (int k = 0; k < NB; ++k) {
#pragma unroll
				for (int i = k + 1; i < NB; ++i)
					if (i < w) q[i] = fmaf(-q[k], Lp[k * b + i], q[i]);
			}
#pragma unroll
			for (int i = 0; i < NB; ++i) {
				if (i < w) {
					colp[i] = q[i];
					Up[i * b + t] = q[i];
				}
			}
		}
		__syncthreads();

		// Phase 3: A22 -= L21 * U12.  Warp items of 256 rows x 4 columns;
		// lane owns rows lane + 32*i.  Each element is updated in increasing p.
		{
			const int warp = t >> 5, lane = t & 31;
			const int rblocks = (rem + 255) / 256;
			const int cblocks = (rem + 3) / 4;
			for (int item = warp; item < rblocks * cblocks; item += kGetrfThreads / 32) {
				const int rb = item % rblocks, cbk = item / rblocks;
				const int r0 = rb * 256 + lane, c0 = cbk * 4;
				float acc[8][4];
#pragma unroll
				for (int i = 0; i < 8; ++i)
#pragma unroll
					for (int j = 0; j < 4; ++j) {
						const int r = r0 + 32 * i, c = c0 + j;
						acc[i][j] = (r < rem && c < rem)
							? a[static_cast<int64_t>(kb + w + c) * lda + kb + w + r] : 0.f;
					}
				for (int pp = 0; pp < w; ++pp) {
					float lv[8], uv[4];
#pragma unroll
					for (int i = 0; i < 8; ++i) {
						const int r = r0 + 32 * i;
						lv[i] = (r < rem) ? Lp[pp * b + w + r] : 0.f;
					}
#pragma unroll
					for (int j = 0; j < 4; ++j) uv[j] = (c0 + j < rem) ? Up[pp * b + c0 + j] : 0.f;
#pragma unroll
					for (int i = 0; i < 8; ++i)
#pragma unroll
						for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(-lv[i], uv[j], acc[i][j]);
				}
#pragma unroll
				for (int i = 0; i < 8; ++i)
#pragma unroll
					for (int j = 0; j < 4; ++j) {
						const int r = r0 + 32 * i, c = c0 + j;
						if (r < rem && c < rem) a[static_cast<int64_t>(kb + w + c) * lda + kb + w + r] = acc[i][j];
					}
			}
		}
		__syncthreads();
	}
}

template <int NB>
static int getrf_launch(int b, float *a, int64_t lda, cudaStream_t st)
{
	const size_t smem = (static_cast<size_t>(2) * b * NB + 2 * NB) * sizeof(float);
	HPLAI_CUDA_TRY(cudaFuncSetAttribute(getrf_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(smem)));
	getrf_kernel<NB><<<1, kGetrfThreads, smem, st>>>(b, a, lda);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_getrf(int b, float *a, int64_t lda, cudaStream_t st)
{
	if (b <= 0 || b > 1024) return HPLAI_EINVAL;
	if (b <= 640) return getrf_launch<32>(b, a, lda, st);
	return getrf_launch<16>(b, a, lda, st);
}

// ---------------------------------------------------------------------------
// L panel: X (m x b) <- X * U^{-1}, U upper non-unit; lh = half(scale * X),
// row-major.  A CTA owns R rows of X in shared memory (Xs[j*R + r]).
// ---------------------------------------------------------------------------
constexpr int kTrsmThreads = 256;

template <int R>
__global__ void __launch_bounds__(kTrsmThreads) trsm_ru_kernel(int m, int b, const float *__restrict__ u,
	int64_t ldu, float *__restrict__ a, int64_t lda, __half *__restrict__ lh, int64_t ldh, float scale)
{
	constexpr int CW = 4 * 4 * kTrsmThreads / R;   // update chunk width (4x4 tiles, one per thread)
	constexpr int LDX = R + 4;                     // padded so row-wise reads spread over banks
	constexpr int LDU = CW + 1;
	extern __shared__ float sm[];
	float *Xs = sm;                                  // b x LDX, Xs[j*LDX + r]
	float *Us = Xs + static_cast<size_t>(b) * LDX;   // 32 x LDU, Us[p*LDU + cc] = U[jb+p][c0+cc]
	float *Ud = Us + 32 * LDU;                       // 32 x 33,  Ud[p*33 + j]  = U[jb+p][jb+j]
	float *inv = Ud + 32 * 33;                       // 32 reciprocals
	const int t = threadIdx.x;
	const int row0 = blockIdx.x * R;
	const int rows = min(R, m - row0);

	for (int idx = t; idx < R * b; idx += kTrsmThreads) {
		const int r = idx % R, j = idx / R;
		Xs[j * LDX + r] = (r < rows) ? a[static_cast<int64_t>(j) * lda + row0 + r] : 0.f;
	}

	for (int jb = 0; jb < b; jb += 32) {
		const int jw = min(32, b - jb);
		for (int idx = t; idx < 32 * 32; idx += kTrsmThreads) {
			const int p = idx & 31, j = idx >> 5;
			Ud[p * 33 + j] = (p < jw && j < jw) ? u[static_cast<int64_t>(jb + j) * ldu + jb + p] : 0.f;
		}
		if (t < jw) inv[t] = 1.0f / u[static_cast<int64_t>(jb + t) * ldu + jb + t];
		__syncthreads();
		// Triangular 32-column block: one row per thread.
		if (t < R) {
			float x[32];
#pragma unroll
			for (int j = 0; j < 32; ++j) x[j] = (j < jw) ? Xs[(jb + j) * LDX + t] : 0.f;
#pragma unroll
			for (int j = 0; j < 32; ++j) {
				if (j < jw) {
#pragma unroll
					for (int p = 0; p < j; ++p) x[j] = fmaf(-Ud[p * 33 + j], x[p], x[j]);
					x[j] *= inv[j];
				}
			}
#pragma unroll
			for (int j = 0; j < 32; ++j)
				if (j < jw) Xs[(jb + j) * LDX + t] = x[j];
		}
		__syncthreads();
		// Update the columns right of the block, CW at a time.
		for (int c0 = jb + jw; c0 < b; c0 += CW) {
			const int cw = min(CW, b - c0);
			for (int idx = t; idx < 32 * CW; idx += kTrsmThreads) {
				const int p = idx & 31, cc = idx >> 5;
				Us[p * LDU + cc] = (p < jw && cc < cw) ? u[static_cast<int64_t>(c0 + cc) * ldu + jb + p] : 0.f;
			}
			__syncthreads();
			const int rt = t % (R / 4), ct = t / (R / 4);
			const int r0 = rt * 4, cc0 = ct * 4;
			if (cc0 < cw) {
				float acc[4][4];
#pragma unroll
				for (int i = 0; i < 4; ++i)
#pragma unroll
					for (int j = 0; j < 4; ++j)
						acc[i][j] = (cc0 + j < cw) ? Xs[(c0 + cc0 + j) * LDX + r0 + i] : 0.f;
				for (int p = 0; p < jw; ++p) {
					const float4 xv = *reinterpret_cast<const float4 *>(&Xs[(jb + p) * LDX + r0]);
					const float xr[4] = {xv.x, xv.y, xv.z, xv.w};
					float ur[4];
#pragma unroll
					for (int j = 0; j < 4; ++j) ur[j] = Us[p * LDU + cc0 + j];
#pragma unroll
					for (int i = 0; i < 4; ++i)
#pragma unroll
						for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(-ur[j], xr[i], acc[i][j]);
				}
#pragma unroll
				for (int i = 0; i < 4; ++i)
#pragma unroll
					for (int j = 0; j < 4; ++j)
						if (cc0 + j < cw) Xs[(c0 + cc0 + j) * LDX + r0 + i] = acc[i][j];
			}
			__syncthreads();
		}
	}

	for (int idx = t; idx < R * b; idx += kTrsmThreads) {
		const int r = idx % R, j = idx / R;
		if (r < rows) a[static_cast<int64_t>(j) * lda + row0 + r] = Xs[j * LDX + r];
	}
	if (lh) {
		for (int idx = t; idx < R * b; idx += kTrsmThreads) {
			const int r = idx / b, j = idx % b;
			if (r < rows) lh[static_cast<int64_t>(row0 + r) * ldh + j] = __float2half_rn(scale * Xs[j * LDX + r]);
		}
	}
}

template <int R>
static int trsm_ru_launch(int m, int b, const float *u, int64_t ldu, float *a, int64_t lda, uint16_t *lh,
	int64_t ldh, float scale, cudaStream_t st)
{
	constexpr int CW = 4 * 4 * kTrsmThreads / R;
	const size_t smem = (static_cast<size_t>(b) * (R + 4) + 32 * (CW + 1) + 32 * 33 + 32) * sizeof(float);
	HPLAI_CUDA_TRY(cudaFuncSetAttribute(trsm_ru_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(smem)));
	trsm_ru_kernel<R><<<(m + R - 1) / R, kTrsmThreads, smem, st>>>(m, b, u, ldu, a, lda,
		reinterpret_cast<__half *>(lh), ldh, scale);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_trsm_right_upper(int m, int b, const float *u, int64_t ldu, float *a, int64_t lda, uint16_t *lh,
	int64_t ldh, float scale, cudaStream_t st)
{
	if (m <= 0) return HPLAI_OK;
	if (b <= 0 || b > 1024) return HPLAI_EINVAL;
	if (b <= 512) return trsm_ru_launch<64>(m, b, u, ldu, a, lda, lh, ldh, scale, st);
	return trsm_ru_launch<32>(m, b, u, ldu, a, lda, lh, ldh, scale, st);
}

// ---------------------------------------------------------------------------
// U panel: Y (b x ncols) <- L^{-1} Y, L unit lower; uh[j*ldh + k] =
// half(scale * Y[k][j]).  A CTA owns C columns (Ys[i*LDY + c]).
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(kTrsmThreads) trsm_ll_kernel(int b, int ncols, const float *__restrict__ l,
	int64_t ldl, float *__restrict__ a, int64_t lda, __half *__restrict__ uh, int64_t ldh, float scale)
{
	constexpr int LDY = C + 1;
	constexpr int RW = 4 * 4 * kTrsmThreads / C;   // update chunk height (rows)
	extern __shared__ float sm[];
	float *Ys = sm;                                  // b x LDY
	float *Ls = Ys + static_cast<size_t>(b) * LDY;   // RW x 33  (rows of L, 32 columns)
	float *Ld = Ls + RW * 33;                        // 32 x 33 diagonal block Ld[i*33 + k]
	const int t = threadIdx.x;
	const int col0 = blockIdx.x * C;
	const int cols = min(C, ncols - col0);

	for (int idx = t; idx < C * b; idx += kTrsmThreads) {
		const int i = idx % b, c = idx / b;
		Ys[i * LDY + c] = (c < cols) ? a[static_cast<int64_t>(col0 + c) * lda + i] : 0.f;
	}

	for (int kb = 0; kb < b; kb += 32) {
		const int kw = min(32, b - kb);
		for (int idx = t; idx < 32 * 32; idx += kTrsmThreads) {
			const int i = idx & 31, k = idx >> 5;
			Ld[i * 33 + k] = (i < kw && k < kw) ? l[static_cast<int64_t>(kb + k) * ldl + kb + i] : 0.f;
		}
		__syncthreads();
		if (t < C) {
			float y[32];
#pragma unroll
			for (int i = 0; i < 32; ++i) y[i] = (i < kw) ? Ys[(kb + i) * LDY + t] : 0.f;
#pragma unroll
			for (int k = 0; k < 32; ++k) {
#pragma unroll
				for (int i = k + 1; i < 32; ++i)
					if (i < kw) y[i] = fmaf(-y[k], Ld[i * 33 + k], y[i]);
			}
#pragma unroll
			for (int i = 0; i < 32; ++i)
				if (i < kw) Ys[(kb + i) * LDY + t] = y[i];
		}
		__syncthreads();
		for (int i0 = kb + kw; i0 < b; i0 += RW) {
			const int rw = min(RW, b - i0);
			for (int idx = t; idx < RW * 32; idx += kTrsmThreads) {
				const int ii = idx % RW, k = idx / RW;
				Ls[ii * 33 + k] = (ii < rw && k < kw) ? l[static_cast<int64_t>(kb + k) * ldl + i0 + ii] : 0.f;
			}
			__syncthreads();
			const int ct = t % (C / 4), rt = t / (C / 4);
			const int cc0 = ct * 4, ii0 = rt * 4;
			if (ii0 < rw) {
				float acc[4][4];
#pragma unroll
				for (int i = 0; i < 4; ++i)
#pragma unroll
					for (int j = 0; j < 4; ++j) acc[i][j] = (ii0 + i < rw) ? Ys[(i0 + ii0 + i) * LDY + cc0 + j] : 0.f;
				for (int k = 0; k < kw; ++k) {
					float yv[4], lv[4];
#pragma unroll
					for (int j = 0; j < 4; ++j) yv[j] = Ys[(kb + k) * LDY + cc0 + j];
#pragma unroll
					for (int i = 0; i < 4; ++i) lv[i] = Ls[(ii0 + i) * 33 + k];
#pragma unroll
					for (int i = 0; i < 4; ++i)
#pragma unroll
						for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(-yv[j], lv[i], acc[i][j]);
				}
#pragma unroll
				for (int i = 0; i < 4; ++i)
#pragma unroll
					for (int j = 0; j < 4; ++j)
						if (ii0 + i < rw) Ys[(i0 + ii0 + i) * LDY + cc0 + j] = acc[i][j];
			}
			__syncthreads();
		}
	}

	for (int idx = t; idx < C * b; idx += kTrsmThreads) {
		const int i = idx % b, c = idx / b;
		if (c < cols) {
			const float v = Ys[i * LDY + c];
			a[static_cast<int64_t>(col0 + c) * lda + i] = v;
			if (uh) uh[static_cast<int64_t>(col0 + c) * ldh + i] = __float2half_rn(scale * v);
		}
	}
}

template <int C>
static int trsm_ll_launch(int b, int ncols, const float *l, int64_t ldl, float *a, int64_t lda, uint16_t *uh,
	int64_t ldh, float scale, cudaStream_t st)
{
	constexpr int RW = 4 * 4 * kTrsmThreads / C;
	const size_t smem = (static_cast<size_t>(b) * (C + 1) + RW * 33 + 32 * 33) * sizeof(float);
	HPLAI_CUDA_TRY(cudaFuncSetAttribute(trsm_ll_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(smem)));
	trsm_ll_kernel<C><<<(ncols + C - 1) / C, kTrsmThreads, smem, st>>>(b, ncols, l, ldl, a, lda,
		reinterpret_cast<__half *>(uh), ldh, scale);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_trsm_left_lower(int b, int ncols, const float *l, int64_t ldl, float *a, int64_t lda, uint16_t *uh,
	int64_t ldh, float scale, cudaStream_t st)
{
	if (ncols <= 0) return HPLAI_OK;
	if (b <= 0 || b > 1024) return HPLAI_EINVAL;
	if (b <= 512) return trsm_ll_launch<64>(b, ncols, l, ldl, a, lda, uh, ldh, scale, st);
	return trsm_ll_launch<32>(b, ncols, l, ldl, a, lda, uh, ldh, scale, st);
}

} // namespace hplai

extern "C" int hplai_getrf_nopiv(int b, float *a, int64_t lda, void *stream)
{
	if (!a || lda < b) return HPLAI_EINVAL;
	return hplai::launch_getrf(b, a, lda, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_trsm_right_upper(int m, int b, const float *u, int64_t ldu, float *a, int64_t lda,
	uint16_t *lh, int64_t ldh, float scale, void *stream)
{
	if (m < 0 || !u || !a || ldu < b || lda < m || (lh && ldh < b)) return HPLAI_EINVAL;
	return hplai::launch_trsm_right_upper(m, b, u, ldu, a, lda, lh, ldh, scale, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_trsm_left_lower(int b, int ncols, const float *l, int64_t ldl, float *a, int64_t lda,
	uint16_t *uh, int64_t ldh, float scale, void *stream)
{
	if (ncols < 0 || !l || !a || ldl < b || lda < b || (uh && ldh < b)) return HPLAI_EINVAL;
	return hplai::launch_trsm_left_lower(b, ncols, l, ldl, a, lda, uh, ldh, scale, static_cast<cudaStream_t>(stream));
}
