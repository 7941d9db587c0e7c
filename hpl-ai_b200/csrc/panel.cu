// panel.cu -- FP32 panel factorisation kernels for the blocked no-pivot LU.
//
//  trsm_kernel      : L panel  A_col <- A_col * U^{-1}, plus its FP16 copy
//                     (update_left_panels + convert_left_panels, panel_trf.hpp:143-157,182-207)
//                     U panel  A_row <- L^{-1} * A_row, plus its FP16 copy, as the
//                     same solve on the transpose
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
// Panel TRSM + FP16 copy, one kernel for both panels.
//
// X (m x b) <- X * T^{-1} with T upper triangular (b x b).  A CTA owns R rows
// of X in shared memory (Xs[j*LDX + r]).
//   L panel (update_left_panels):  X = A_col (column-major, X[r][j] at
//            a[j*lda + r]), T = U11 (T[p][j] at t[j*ldt + p]), non-unit.
//   U panel (update_right_panels): L^{-1} A_row = (A_row^T L^{-T})^T, so
//            X = A_row^T (row-major, X[r][j] at a[r*lda + j]) and T = L11^T
//            (T[p][j] = L[j][p] at t[p*ldt + j]), unit diagonal.
// Element (r, j) receives x -= T[p][j] * x[r][p] for p = 0..j-1 in
// increasing p, then x *= 1/T[j][j] when non-unit: netlib strsm's order for
// both (R,U,N,N) and (L,L,N,U), so the result is bit-exact with it.
// hc[(row0 + r)*ldh + j] = half(scale * X[r][j]) in both cases (the L copy is
// row-major; the U copy stores column j of U as row j).
// ---------------------------------------------------------------------------
constexpr int kTrsmThreads = 256;

template <int R, bool ROWX, bool TRANS_T>
__global__ void __launch_bounds__(kTrsmThreads) trsm_kernel(int m, int b, const float *__restrict__ t,
	int64_t ldt, float *__restrict__ a, int64_t lda, __half *__restrict__ hc, int64_t ldh, float scale)
{
	constexpr int CW = 4 * 4 * kTrsmThreads / R;   // update chunk width (4x4 tiles, one per thread)
	constexpr int LDX = R + 4;                     // padded so row-wise reads spread over banks
	constexpr int LDU = CW + 1;
	constexpr bool UNIT = TRANS_T;                 // L11^T has a unit diagonal
	extern __shared__ float sm[];
	float *Xs = sm;                                  // b x LDX
	float *Us = Xs + static_cast<size_t>(b) * LDX;   // 32 x LDU, Us[p*LDU + cc] = T[jb+p][c0+cc]
	float *Ud = Us + 32 * LDU;                       // 32 x 33,  Ud[p*33 + j]  = T[jb+p][jb+j]
	float *inv = Ud + 32 * 33;                       // 32 reciprocals
	const int tid = threadIdx.x;
	const int row0 = blockIdx.x * R;
	const int rows = min(R, m - row0);
	auto tval = [&](int p, int j) -> float {
		return TRANS_T ? t[static_cast<int64_t>(p) * ldt + j] : t[static_cast<int64_t>(j) * ldt + p];
	};

	if (ROWX) {
		for (int idx = tid; idx < R * b; idx += kTrsmThreads) {
			const int r = idx / b, j = idx - r * b;
			Xs[j * LDX + r] = (r < rows) ? a[static_cast<int64_t>(row0 + r) * lda + j] : 0.f;
		}
	} else {
		for (int idx = tid; idx < R * b; idx += kTrsmThreads) {
			const int r = idx % R, j = idx / R;
			Xs[j * LDX + r] = (r < rows) ? a[static_cast<int64_t>(j) * lda + row0 + r] : 0.f;
		}
	}

	for (int jb = 0; jb < b; jb += 32) {
		const int jw = min(32, b - jb);
		for (int idx = tid; idx < 32 * 32; idx += kTrsmThreads) {
			const int p = TRANS_T ? (idx >> 5) : (idx & 31), j = TRANS_T ? (idx & 31) : (idx >> 5);
			Ud[p * 33 + j] = (p < jw && j < jw) ? tval(jb + p, jb + j) : 0.f;
		}
		if (!UNIT && tid < jw) inv[tid] = 1.0f / tval(jb + tid, jb + tid);
		__syncthreads();
		// Triangular 32-column block: one row per thread.
		if (tid < R) {
			float x[32];
#pragma unroll
			for (int j = 0; j < 32; ++j) x[j] = (j < jw) ? Xs[(jb + j) * LDX + tid] : 0.f;
#pragma unroll
			for (int j = 0; j < 32; ++j) {
				if (j < jw) {
#pragma unroll
					for (int p = 0; p < j; ++p) x[j] = fmaf(-Ud[p * 33 + j], x[p], x[j]);
					if (!UNIT) x[j] *= inv[j];
				}
			}
#pragma unroll
			for (int j = 0; j < 32; ++j)
				if (j < jw) Xs[(jb + j) * LDX + tid] = x[j];
		}
		__syncthreads();
		// Update the columns right of the block, CW at a time.
		for (int c0 = jb + jw; c0 < b; c0 += CW) {
			const int cw = min(CW, b - c0);
			for (int idx = tid; idx < 32 * CW; idx += kTrsmThreads) {
				// coalesced along the contiguous index of T's storage
				const int p = TRANS_T ? (idx / CW) : (idx & 31), cc = TRANS_T ? (idx % CW) : (idx >> 5);
				Us[p * LDU + cc] = (p < jw && cc < cw) ? tval(jb + p, c0 + cc) : 0.f;
			}
			__syncthreads();
			const int rt = tid % (R / 4), ct = tid / (R / 4);
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

	if (ROWX) {
		for (int idx = tid; idx < R * b; idx += kTrsmThreads) {
			const int r = idx / b, j = idx - r * b;
			if (r < rows) a[static_cast<int64_t>(row0 + r) * lda + j] = Xs[j * LDX + r];
		}
	} else {
		for (int idx = tid; idx < R * b; idx += kTrsmThreads) {
			const int r = idx % R, j = idx / R;
			if (r < rows) a[static_cast<int64_t>(j) * lda + row0 + r] = Xs[j * LDX + r];
		}
	}
	if (hc) {
		// 8 consecutive halves per thread (16-byte store), rows across lanes.
		const int b8 = b / 8;
		for (int idx = tid; idx < R * b8; idx += kTrsmThreads) {
			const int r = idx % R, q = idx / R;
			if (r < rows) {
				__align__(16) __half h[8];
#pragma unroll
				for (int e = 0; e < 8; ++e) h[e] = __float2half_rn(scale * Xs[(8 * q + e) * LDX + r]);
				*reinterpret_cast<uint4 *>(hc + static_cast<int64_t>(row0 + r) * ldh + 8 * q) =
					*reinterpret_cast<const uint4 *>(h);
			}
		}
		for (int idx = tid; idx < R * (b - 8 * b8); idx += kTrsmThreads) {
			const int r = idx % R, j = 8 * b8 + idx / R;
			if (r < rows) hc[static_cast<int64_t>(row0 + r) * ldh + j] = __float2half_rn(scale * Xs[j * LDX + r]);
		}
	}
}

template <int R, bool ROWX, bool TRANS_T>
static int trsm_launch(int m, int b, const float *t, int64_t ldt, float *a, int64_t lda, uint16_t *hc, int64_t ldh,
	float scale, cudaStream_t st)
{
	constexpr int CW = 4 * 4 * kTrsmThreads / R;
	const size_t smem = (static_cast<size_t>(b) * (R + 4) + 32 * (CW + 1) + 32 * 33 + 32) * sizeof(float);
	HPLAI_CUDA_TRY(cudaFuncSetAttribute(trsm_kernel<R, ROWX, TRANS_T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(smem)));
	trsm_kernel<R, ROWX, TRANS_T><<<(m + R - 1) / R, kTrsmThreads, smem, st>>>(m, b, t, ldt, a, lda,
		reinterpret_cast<__half *>(hc), ldh, scale);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

static bool vec_ok(const uint16_t *hc, int64_t ldh)
{
	return !hc || ((reinterpret_cast<uintptr_t>(hc) & 15u) == 0 && ldh % 8 == 0);
}

int launch_trsm_right_upper(int m, int b, const float *u, int64_t ldu, float *a, int64_t lda, uint16_t *lh,
	int64_t ldh, float scale, cudaStream_t st)
{
	if (m <= 0) return HPLAI_OK;
	if (b <= 0 || b > 1024 || !vec_ok(lh, ldh)) return HPLAI_EINVAL;
	if (b <= 512) return trsm_launch<64, false, false>(m, b, u, ldu, a, lda, lh, ldh, scale, st);
	return trsm_launch<32, false, false>(m, b, u, ldu, a, lda, lh, ldh, scale, st);
}

int launch_trsm_left_lower(int b, int ncols, const float *l, int64_t ldl, float *a, int64_t lda, uint16_t *uh,
	int64_t ldh, float scale, cudaStream_t st)
{
	if (ncols <= 0) return HPLAI_OK;
	if (b <= 0 || b > 1024 || !vec_ok(uh, ldh)) return HPLAI_EINVAL;
	if (b <= 512) return trsm_launch<64, true, true>(ncols, b, l, ldl, a, lda, uh, ldh, scale, st);
	return trsm_launch<32, true, true>(ncols, b, l, ldl, a, lda, uh, ldh, scale, st);
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
