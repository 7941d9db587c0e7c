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

namespace hplai {

namespace {

constexpr float kE4M3Max = 448.f;

// X (rows x kdim), element (r, k) at src[r + k*ld] (RCONTIG, column-major L
// panel) or at src[k + r*ld] (the U panel read by columns).
template <bool RCONTIG>
__global__ void __launch_bounds__(256) amax_kernel(int rows, int kdim, const float *__restrict__ src, int64_t ld,
	unsigned *__restrict__ bits)
{
	const int r0 = blockIdx.x * 128, k0 = blockIdx.y * 64;
	float m = 0.f;
	for (int e = threadIdx.x; e < 128 * 64; e += 256) {
		const int r = RCONTIG ? (e & 127) : (e >> 6), k = RCONTIG ? (e >> 7) : (e & 63);
		if (r0 + r < rows && k0 + k < kdim) {
			const float v = RCONTIG ? src[static_cast<int64_t>(k0 + k) * ld + r0 + r]
			                        : src[static_cast<int64_t>(r0 + r) * ld + k0 + k];
			m = fmaxf(m, fabsf(v));
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

// L panel (element (r, k) at src[r + k*ld]): tile of 32 rows x 128 k loaded
// coalesced along r, then 4 e4m3 bytes per thread written along k.  The 32
// rows lie in one 128-row block: one factor per CTA.
__global__ void __launch_bounds__(256) cast8_cols_kernel(int rows, int kdim, const float *__restrict__ src, int64_t ld,
	const unsigned *__restrict__ bits, uint8_t *__restrict__ dst, int64_t ld8, float *__restrict__ scale)
{
	__shared__ float tile[32][129];
	__shared__ float s_inv;
	const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 128;
	if (threadIdx.x == 0) {
		const int ex = block_exponent(bits[r0 >> 7]);
		s_inv = ldexpf(1.f, -ex);
		if ((r0 & 127) == 0 && k0 == 0) scale[r0 >> 7] = ldexpf(1.f, ex);
	}
	for (int e = threadIdx.x; e < 32 * 128; e += 256) {
		const int r = e & 31, k = e >> 5;
		tile[r][k] = (r0 + r < rows && k0 + k < kdim) ? src[static_cast<int64_t>(k0 + k) * ld + r0 + r] : 0.f;
	}
	__syncthreads();
	const float inv = s_inv;
	for (int e = threadIdx.x; e < 32 * 32; e += 256) {
		const int r = e >> 5, w = e & 31;
		const int row = r0 + r;
		if (row >= rows || k0 + 4 * w >= ld8) continue;
		*reinterpret_cast<uint32_t *>(dst + static_cast<int64_t>(row) * ld8 + k0 + 4 * w) =
			pack_e4m3(tile[r][4 * w], tile[r][4 * w + 1], tile[r][4 * w + 2], tile[r][4 * w + 3], inv);
	}
}

// U panel (element (r, k) at src[r*ld + k]): source and copy are both
// contiguous along k, so each thread converts four consecutive k of a row
// with no staging (16-byte loads when src and ld allow them).
__global__ void __launch_bounds__(256) cast8_rows_kernel(int rows, int kdim, const float *__restrict__ src, int64_t ld,
	const unsigned *__restrict__ bits, uint8_t *__restrict__ dst, int64_t ld8, float *__restrict__ scale, int vec)
{
	const int k = 4 * (blockIdx.x * 256 + threadIdx.x);
	if (k >= ld8) return;
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
	float *scale, cudaStream_t st)
{
	if (rows <= 0) return HPLAI_OK;
	const int nblk = (rows + 127) / 128;
	HPLAI_CUDA_TRY(cudaMemsetAsync(bits, 0, sizeof(unsigned) * nblk, st));
	amax_kernel<RCONTIG><<<dim3(nblk, (kdim + 63) / 64), 256, 0, st>>>(rows, kdim, src, ld, bits);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	if (RCONTIG) {
		cast8_cols_kernel<<<dim3((rows + 31) / 32, static_cast<unsigned>((ld8 + 127) / 128)), 256, 0, st>>>(rows, kdim,
			src, ld, bits, dst, ld8, scale);
	} else {
		const int vec = ((reinterpret_cast<uintptr_t>(src) & 15u) == 0 && (ld & 3) == 0) ? 1 : 0;
		cast8_rows_kernel<<<dim3(static_cast<unsigned>((ld8 / 4 + 255) / 256), static_cast<unsigned>(rows < 8192 ? rows : 8192)),
			256, 0, st>>>(rows, kdim, src, ld, bits, dst, ld8, scale, vec);
	}
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

} // namespace

int launch_quantize_lpanel(int rows, int b, const float *acol, int64_t lda, unsigned *bits, uint8_t *l8, int64_t ld8,
	float *scale, cudaStream_t st)
{
	if (ld8 % 128) return HPLAI_EINVAL;
	return quantize<true>(rows, b, acol, lda, bits, l8, ld8, scale, st);
}

int launch_quantize_upanel(int cols, int b, const float *arow, int64_t lda, unsigned *bits, uint8_t *u8, int64_t ld8,
	float *scale, cudaStream_t st)
{
	if (ld8 % 128) return HPLAI_EINVAL;
	return quantize<false>(cols, b, arow, lda, bits, u8, ld8, scale, st);
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
	return col_major ? hplai::launch_quantize_lpanel(rows, k, src, lds, bits, dst, ld8, scale, st)
	                 : hplai::launch_quantize_upanel(rows, k, src, lds, bits, dst, ld8, scale, st);
}
