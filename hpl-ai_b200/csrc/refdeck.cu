// refdeck.cu -- the reference's FP16-accumulating Schur update of the `-d`
// (lazy-init, double-decker) LU, bit for bit.
//
// The reference's x86 build updates its FP16 deck with hgemm_opt
// (kernels/avx2.cpp:82-189, fp16sim.hpp:185-213) with alpha = -1: for every
// element, over k-chunks of 100 (bk), an FP16 accumulator
//     t <- fp16(fp32(l_iq * u_qj + t))
// (the FP16 x FP16 product is exact in FP32, so the FP32 FMA and the
// reference's FMA give the same value), and after each chunk
//     d_ij <- fp16(fp32(d_ij - t)),
// every FP32 -> FP16 conversion rounding to nearest even.  Tensor cores
// cannot round an accumulator to FP16 after every product, so this parity
// mode runs on CUDA cores: a 64 x 64 tile per CTA, 4 x 4 elements per thread,
// FP16 operand slabs converted to FP32 in shared memory.  It is a numerics
// mode (the reference's `-d` arithmetic), not the fast path: the fast deck
// form accumulates in FP32 on tcgen05 and rounds once per update.
#include "common.cuh"
#include "internal.h"

#include <algorithm>

namespace hplai {
namespace {

constexpr int kHt = 64;       // tile rows and columns
constexpr int kHk = 20;       // k-slab staged per pass (divides the chunk of 100)
constexpr int kChunk = 100;   // hgemm_opt's bk

__device__ __forceinline__ float round_f16(float x) { return __half2float(__float2half_rn(x)); }

__global__ void __launch_bounds__(256) hgemm_deck_kernel(int m, int n, int k, const __half *__restrict__ l,
	int64_t ldl, const __half *__restrict__ u, int64_t ldu, __half *__restrict__ d, int64_t ldd)
{
	__shared__ float ls[kHk][kHt + 4];
	__shared__ float us[kHk][kHt + 4];
	const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
	const int row0 = blockIdx.x * kHt, col0 = blockIdx.y * kHt;
	float acc[4][4], dv[4][4];
#pragma unroll
	for (int r = 0; r < 4; ++r)
#pragma unroll
		for (int c = 0; c < 4; ++c) {
			const int i = row0 + tx + 16 * r, j = col0 + ty + 16 * c;
			dv[r][c] = (i < m && j < n) ? __half2float(d[static_cast<int64_t>(j) * ldd + i]) : 0.f;
			acc[r][c] = 0.f;
		}
	for (int q0 = 0; q0 < k; q0 += kHk) {
		__syncthreads();
		for (int e = threadIdx.x; e < kHt * kHk; e += 256) {
			const int r = e / kHk, qq = e % kHk, q = q0 + qq;
			const int i = row0 + r, j = col0 + r;
			ls[qq][r] = (i < m && q < k) ? __half2float(l[static_cast<int64_t>(i) * ldl + q]) : 0.f;
			us[qq][r] = (j < n && q < k) ? __half2float(u[static_cast<int64_t>(j) * ldu + q]) : 0.f;
		}
		__syncthreads();
		const int qn = min(kHk, k - q0);
		for (int qq = 0; qq < qn; ++qq) {
			float a[4], bq[4];
#pragma unroll
			for (int r = 0; r < 4; ++r) a[r] = ls[qq][tx + 16 * r];
#pragma unroll
			for (int c = 0; c < 4; ++c) bq[c] = us[qq][ty + 16 * c];
#pragma unroll
			for (int r = 0; r < 4; ++r)
#pragma unroll
				for (int c = 0; c < 4; ++c) acc[r][c] = round_f16(__fmaf_rn(a[r], bq[c], acc[r][c]));
			const int q = q0 + qq;
			if ((q + 1) % kChunk == 0 || q + 1 == k) {
#pragma unroll
				for (int r = 0; r < 4; ++r)
#pragma unroll
					for (int c = 0; c < 4; ++c) {
						dv[r][c] = round_f16(__fsub_rn(dv[r][c], acc[r][c]));
						acc[r][c] = 0.f;
					}
			}
		}
	}
#pragma unroll
	for (int r = 0; r < 4; ++r)
#pragma unroll
		for (int c = 0; c < 4; ++c) {
			const int i = row0 + tx + 16 * r, j = col0 + ty + 16 * c;
			if (i < m && j < n) d[static_cast<int64_t>(j) * ldd + i] = __float2half_rn(dv[r][c]);
		}
}

// The back buffer (`--back_buffer`, back_buffer.hpp:81-170): every 32 steps
// the deck's value moves into a second FP16 array with a compensated sum,
// each operation rounded to FP16 through FP32 (the reference's FP16
// arithmetic, svesim.hpp:190-262):
//     p = h(y / 32), t2 = h(x + p), t3 = h(t2 - x), t4 = h(p - t3),
//     back = t2, deck = h(32 t4).
__global__ void __launch_bounds__(256) backbuf_kernel(int n, int r0, __half *__restrict__ deck,
	__half *__restrict__ back, int64_t ld)
{
	const int i = r0 + blockIdx.x * 256 + threadIdx.x;
	if (i >= n) return;
	for (int j = r0 + blockIdx.y; j < n; j += gridDim.y) {
		const int64_t o = static_cast<int64_t>(j) * ld + i;
		const float x = __half2float(back[o]);
		const float p = round_f16(__fmul_rn(__half2float(deck[o]), 0.03125f));
		const float t2 = round_f16(__fadd_rn(x, p));
		const float t3 = round_f16(__fsub_rn(t2, x));
		const float t4 = round_f16(__fsub_rn(p, t3));
		back[o] = __float2half_rn(t2);
		deck[o] = __float2half_rn(__fmul_rn(t4, 32.0f));
	}
}

} // namespace

int launch_backbuf_writeback(int n, int r0, uint16_t *deck, uint16_t *back, int64_t ld, cudaStream_t st)
{
	if (r0 >= n) return HPLAI_OK;
	if (!deck || !back || ld < n) return HPLAI_EINVAL;
	const dim3 grid((n - r0 + 255) / 256, std::min(n - r0, 4096));
	backbuf_kernel<<<grid, 256, 0, st>>>(n, r0, reinterpret_cast<__half *>(deck), reinterpret_cast<__half *>(back), ld);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_hgemm_deck(int m, int n, int k, const uint16_t *l, int64_t ldl, const uint16_t *u, int64_t ldu,
	uint16_t *d, int64_t ldd, cudaStream_t st)
{
	if (m <= 0 || n <= 0 || k <= 0) return HPLAI_OK;
	if (!l || !u || !d || ldl < k || ldu < k || ldd < m) return HPLAI_EINVAL;
	const dim3 grid((m + kHt - 1) / kHt, (n + kHt - 1) / kHt);
	if (grid.y > 65535) return HPLAI_EINVAL;
	hgemm_deck_kernel<<<grid, 256, 0, st>>>(m, n, k, reinterpret_cast<const __half *>(l), ldl,
		reinterpret_cast<const __half *>(u), ldu, reinterpret_cast<__half *>(d), ldd);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

} // namespace hplai
