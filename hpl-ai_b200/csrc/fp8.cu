// fp8.cu -- FP8 (e4m3) copies of the L and U panels for the precision form.
//
// The reference down-casts its FP32 panels to FLOW with one scale factor
// (convert_left/right_panels, panel_trf.hpp:173-233, scalea = n^0.75 under
// lazy init).  With e4m3 (3 mantissa bits, |x| <= 448) one global factor
// cannot cover the panels' dynamic range, so here every block of 128 panel
// rows (128 rows of L, 128 columns of U) gets its own power-of-two factor
// 2^e chosen so that the block's largest magnitude maps just below 448.  The
// Schur GEMM multiplies each accumulator element by the two blocks' factors
// (exact, powers of two) before the update.
//
// amax_kernel: per-block max |x| (atomicMax on the float bits, which order
// like the values for x >= 0).  cast8_cols_kernel / cast8_rows_kernel: x *
// 2^-e rounded to e4m3 (RN, saturating), row-major with K contiguous, plus
// the factor 2^e per block.
#include "common.cuh"
#include "internal.h"

#include <cuda_fp8.h>

#include <algorithm>

namespace hplai {

namespace {

constexpr float kE4M3Max = 448.f;

// X (rows x kdim), element (r, k) at src[r + k*ld] (RCONTIG, column-major L
// panel) or at src[k + r*ld] (the U panel read by columns).  A CTA covers
// 128 rows x 64 k with 16-byte loads along the contiguous index when vec
// (src 16-byte aligned, ld and the contiguous extent multiples of 4).
template <bool RCONTIG>
__global__ void __launch_bounds__(256) amax_kernel(int rows, int kdim, const float *__restrict__ src, int64_t ld,
	unsigned *__restrict__ bits, int vec)
{
	const int r0 = blockIdx.x * 128, k0 = blockIdx.y * 64;
	float m = 0.f;
	if (vec) {
#pragma unroll
		for (int q = 0; q < 8; ++q) {
			const int e = threadIdx.x + 256 * q;
			// RCONTIG: 32 float4 along r per k; else 16 float4 along k per r
			const int r = RCONTIG ? 4 * (e & 31) : (e >> 4), k = RCONTIG ? (e >> 5) : 4 * (e & 15);
			if (r0 + r < rows && k0 + k < kdim) {
				const float4 v = __ldg(reinterpret_cast<const float4 *>(
					RCONTIG ? src + static_cast<int64_t>(k0 + k) * ld + r0 + r
					        : src + static_cast<int64_t>(r0 + r) * ld + k0 + k));
				m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
			}
		}
	} else {
		for (int e = threadIdx.x; e < 128 * 64; e += 256) {
			const int r = RCONTIG ? (e & 127) : (e >> 6), k = RCONTIG ? (e >> 7) : (e & 63);
			if (r0 + r < rows && k0 + k < kdim) {
				const float v = RCONTIG ? src[static_cast<int64_t>(k0 + k) * ld + r0 + r]
				                        : src[static_cast<int64_t>(r0 + r) * ld + k0 + k];
				m = fmaxf(m, fabsf(v));
			}
		}
	}
	for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
	__shared__ float wm[8];
	if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int w = 1; w < 8; ++w) m = fmaxf(m, wm[w]);
		atomicMax(&bits[blockIdx.x], __float_as_uint(m));
	}
}

__device__ __forceinline__ int block_exponent(unsigned amax_bits)
{
	const float amax = __uint_as_float(amax_bits);
	if (!(amax > 0.f)) return 0;
	int e;
	frexpf(amax / kE4M3Max, &e);   // amax/448 = f 2^e, f in [0.5, 1): amax 2^-e < 448
	return e;
}

// Four values times the block factor to e4m3 (RN, saturating), packed little-endian.
__device__ __forceinline__ uint32_t pack_e4m3(float v0, float v1, float v2, float v3, float inv)
{
	const uint32_t lo = __nv_cvt_float2_to_fp8x2(make_float2(v0 * inv, v1 * inv), __NV_SATFINITE, __NV_E4M3);
	const uint32_t hi = __nv_cvt_float2_to_fp8x2(make_float2(v2 * inv, v3 * inv), __NV_SATFINITE, __NV_E4M3);
	return lo | (hi << 16);
}

// L panel (element (r, k) at src[r + k*ld]): a CTA converts 64 rows (inside
// one 128-row factor block: one factor per CTA) x 128 k.  The tile is read
// along r, 256 bytes per column (16-byte loads when src, ld and rows allow
// them), staged in shared memory and written along k, one warp per row's 128
// bytes.  (32-row tiles, 128 bytes per column, ran at a quarter of the copy
// bandwidth.)  Bytes past kdim up to kend are written as zeros.
constexpr int kC8Rows = 64, kC8K = 128;
__global__ void __launch_bounds__(256) cast8_cols_kernel(int rows, int kdim, int kend, const float *__restrict__ src,
	int64_t ld, const unsigned *__restrict__ bits, uint8_t *__restrict__ dst, int64_t ld8, float *__restrict__ scale,
	int vec)
{
	__shared__ float tile[kC8K][kC8Rows + 1];   // tile[k][r]
	const int r0 = blockIdx.x * kC8Rows, k0 = blockIdx.y * kC8K;
	const int ex = block_exponent(bits[r0 >> 7]);
	const float inv = ldexpf(1.f, -ex);
	if (threadIdx.x == 0 && (r0 & 127) == 0 && k0 == 0) scale[r0 >> 7] = ldexpf(1.f, ex);
#pragma unroll
	for (int q = 0; q < (kC8K * kC8Rows / 4) / 256; ++q) {
		const int idx = threadIdx.x + 256 * q, kk = idx >> 4, rr = (idx & 15) * 4;
		const int k = k0 + kk, r = r0 + rr;
		float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
		if (k < kdim) {
			const float *col = src + static_cast<int64_t>(k) * ld + r;
			if (vec) {
				if (r < rows) v = __ldg(reinterpret_cast<const float4 *>(col));
			} else {
				if (r < rows) v.x = col[0];
				if (r + 1 < rows) v.y = col[1];
				if (r + 2 < rows) v.z = col[2];
				if (r + 3 < rows) v.w = col[3];
			}
		}
		tile[kk][rr] = v.x;
		tile[kk][rr + 1] = v.y;
		tile[kk][rr + 2] = v.z;
		tile[kk][rr + 3] = v.w;
	}
	__syncthreads();
#pragma unroll
	for (int q = 0; q < (kC8K / 4 * kC8Rows) / 256; ++q) {
		const int idx = threadIdx.x + 256 * q, rr = idx >> 5, w = idx & 31;
		const int row = r0 + rr, k = k0 + 4 * w;
		if (row < rows && k < kend)
			*reinterpret_cast<uint32_t *>(dst + static_cast<int64_t>(row) * ld8 + k) =
				pack_e4m3(tile[4 * w][rr], tile[4 * w + 1][rr], tile[4 * w + 2][rr], tile[4 * w + 3][rr], inv);
	}
}

// U panel (element (r, k) at src[r*ld + k]): source and copy are both
// contiguous along k, so each thread converts four consecutive k of a row
// with no staging (16-byte loads when src and ld allow them).
__global__ void __launch_bounds__(256) cast8_rows_kernel(int rows, int kdim, int kend, const float *__restrict__ src,
	int64_t ld, const unsigned *__restrict__ bits, uint8_t *__restrict__ dst, int64_t ld8, float *__restrict__ scale,
	int vec)
{
	const int k = 4 * (blockIdx.x * 256 + threadIdx.x);
	if (k >= kend) return;
	for (int r = blockIdx.y; r < rows; r += gridDim.y) {
		const int ex = block_exponent(bits[r >> 7]);
		const float inv = ldexpf(1.f, -ex);
		const float *row = src + static_cast<int64_t>(r) * ld;
		float v0, v1, v2, v3;
		if (vec && k + 3 < kdim) {
			const float4 q = __ldg(reinterpret_cast<const float4 *>(row + k));
			v0 = q.x;
			v1 = q.y;
			v2 = q.z;
			v3 = q.w;
		} else {
			v0 = (k < kdim) ? row[k] : 0.f;
			v1 = (k + 1 < kdim) ? row[k + 1] : 0.f;
			v2 = (k + 2 < kdim) ? row[k + 2] : 0.f;
			v3 = (k + 3 < kdim) ? row[k + 3] : 0.f;
		}
		*reinterpret_cast<uint32_t *>(dst + static_cast<int64_t>(r) * ld8 + k) = pack_e4m3(v0, v1, v2, v3, inv);
		if ((r & 127) == 0 && k == 0) scale[r >> 7] = ldexpf(1.f, ex);
	}
}

template <bool RCONTIG>
int quantize(int rows, int kdim, const float *src, int64_t ld, unsigned *bits, uint8_t *dst, int64_t ld8,
	float *scale, cudaStream_t st, bool pad_row, bool bits_ready)
{
	if (rows <= 0) return HPLAI_OK;
	const int nblk = (rows + 127) / 128;
	const bool aligned = (reinterpret_cast<uintptr_t>(src) & 15u) == 0 && (ld & 3) == 0;
	if (!bits_ready) {
		HPLAI_CUDA_TRY(cudaMemsetAsync(bits, 0, sizeof(unsigned) * nblk, st));
		amax_kernel<RCONTIG><<<dim3(nblk, (kdim + 63) / 64), 256, 0, st>>>(rows, kdim, src, ld, bits,
			(aligned && (RCONTIG ? rows : kdim) % 4 == 0) ? 1 : 0);
		count_launches();
		HPLAI_CUDA_TRY(cudaGetLastError());
	}
	// the Schur kernel reads the copy in 128-byte K chunks: zeros up to the
	// chunk's end (pad_row: up to ld8)
	const int kend = pad_row ? static_cast<int>(ld8) : static_cast<int>(std::min<int64_t>(ld8, (kdim + 127) / 128 * 128));
	if (RCONTIG) {
		const int vec = (aligned && rows % 4 == 0) ? 1 : 0;
		cast8_cols_kernel<<<dim3((rows + kC8Rows - 1) / kC8Rows, static_cast<unsigned>((kend + kC8K - 1) / kC8K)), 256, 0,
			st>>>(rows, kdim, kend, src, ld, bits, dst, ld8, scale, vec);
	} else {
		cast8_rows_kernel<<<dim3(static_cast<unsigned>((kend / 4 + 255) / 256), static_cast<unsigned>(rows < 8192 ? rows : 8192)),
			256, 0, st>>>(rows, kdim, kend, src, ld, bits, dst, ld8, scale, aligned ? 1 : 0);
	}
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

} // namespace

int launch_quantize_lpanel(int rows, int b, const float *acol, int64_t lda, unsigned *bits, uint8_t *l8, int64_t ld8,
	float *scale, cudaStream_t st, bool pad_row, bool bits_ready)
{
	if (ld8 % 128) return HPLAI_EINVAL;
	return quantize<true>(rows, b, acol, lda, bits, l8, ld8, scale, st, pad_row, bits_ready);
}

int launch_quantize_upanel(int cols, int b, const float *arow, int64_t lda, unsigned *bits, uint8_t *u8, int64_t ld8,
	float *scale, cudaStream_t st, bool pad_row, bool bits_ready)
{
	if (ld8 % 128) return HPLAI_EINVAL;
	return quantize<false>(cols, b, arow, lda, bits, u8, ld8, scale, st, pad_row, bits_ready);
}

namespace {

// A[i][j] += deck[i][j] * inv_scale over rows [r0, r1) x cols [c0, c1).
__global__ void __launch_bounds__(256) deck_apply_kernel(int r0, int r1, int c0, int c1, float *__restrict__ a,
	int64_t lda, const __half *__restrict__ deck, int64_t ldd, float inv_scale)
{
	const int rows = r1 - r0;
	const int64_t total = static_cast<int64_t>(rows) * (c1 - c0);
	for (int64_t e = static_cast<int64_t>(blockIdx.x) * 256 + threadIdx.x; e < total;
		e += static_cast<int64_t>(gridDim.x) * 256) {
		const int i = r0 + static_cast<int>(e % rows), j = c0 + static_cast<int>(e / rows);
		const int64_t ia = static_cast<int64_t>(j) * lda + i, id = static_cast<int64_t>(j) * ldd + i;
		a[ia] = fmaf(__half2float(deck[id]), inv_scale, a[ia]);
	}
}

} // namespace

int launch_deck_apply(int r0, int r1, int c0, int c1, float *a, int64_t lda, const void *deck, int64_t ldd,
	float inv_scale, cudaStream_t st)
{
	if (r1 <= r0 || c1 <= c0) return HPLAI_OK;
	const int64_t total = static_cast<int64_t>(r1 - r0) * (c1 - c0);
	int64_t blocks = (total + 255) / 256;
	if (blocks > 148 * 16) blocks = 148 * 16;
	deck_apply_kernel<<<static_cast<unsigned>(blocks), 256, 0, st>>>(r0, r1, c0, c1, a, lda,
		static_cast<const __half *>(deck), ldd, inv_scale);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

} // namespace hplai

extern "C" int hplai_quantize_e4m3(int rows, int k, const float *src, int64_t lds, int col_major, uint8_t *dst,
	int64_t ld8, float *scale, unsigned *bits, void *stream)
{
	if (rows < 0 || k <= 0 || k > ld8 || !src || !dst || !scale || !bits || (ld8 % 128)) return HPLAI_EINVAL;
	if (reinterpret_cast<uintptr_t>(dst) % 16) return HPLAI_EINVAL;   // rows are written as 4-byte words
	if (col_major ? lds < rows : lds < k) return HPLAI_EINVAL;
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	return col_major ? hplai::launch_quantize_lpanel(rows, k, src, lds, bits, dst, ld8, scale, st, true)
	                 : hplai::launch_quantize_upanel(rows, k, src, lds, bits, dst, ld8, scale, st, true);
}
