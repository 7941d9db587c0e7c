// tcpanel.cu -- panel TRSMs of the blocked LU on tensor cores.
//
// update_left_panels / update_right_panels (panel_trf.hpp:143-171) solve
// A_col <- A_col U11^{-1} and A_row <- L11^{-1} A_row with the b x b
// triangles of the freshly factored diagonal block.  Here the two triangles
// are inverted once per step (tri_inv_kernel, FP32) and the panels are
// multiplied by the inverses on tcgen05 in "3xTF32": each FP32 operand x is
// split into hi = x with the low 13 mantissa bits cleared (exact in TF32)
// and lo = x - hi (exact in FP32), and
//     X = A_hi B_hi + A_hi B_lo + A_lo B_hi
// is accumulated in FP32 in TMEM (the dropped A_lo B_lo and the TF32
// rounding of the lo parts are ~2^-21 relative), so the panels keep FP32
// accuracy.  The epilogue writes the FP32 panel back into A and its FP16
// copy (convert_left/right_panels, panel_trf.hpp:173-233) for the Schur GEMM.
//
// Kernels: split_kernel (FP32 panel -> K-major hi/lo copies), tri_inv_kernel
// (triangular inverse, hi/lo), tf32x3_kernel (persistent, warp-specialised:
// TMA producer, one MMA-issuing thread, four epilogue warps; bounded waits).
#include "common.cuh"
#include "internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <cstring>

namespace hplai {

namespace {

// ---------------------------------------------------------------------------
// hi/lo split
// ---------------------------------------------------------------------------
__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// Row-major K-major copies P[r*ldp + k] (hi and lo) of an FP32 panel.
//   TRANS = true : source element (r, k) at src[k*lds + r] (column-major A_col)
//   TRANS = false: source element (r, k) at src[r*lds + k] (A_row seen by columns)
// k in [0, kdim), r in [0, rows); columns kdim..ldp-1 are zeroed.
// plo == nullptr: the hi part only (single-term TF32 products).
template <bool TRANS>
__global__ void __launch_bounds__(256) split_kernel(int rows, int kdim, const float *__restrict__ src, int64_t lds,
	float *__restrict__ phi, float *__restrict__ plo, int64_t ldp)
{
	__shared__ float tile[32][33];
	const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
	const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
	if (TRANS) {
		for (int i = ty; i < 32; i += 8) {
			const int k = k0 + i, r = r0 + tx;
			tile[i][tx] = (k < kdim && r < rows) ? src[static_cast<int64_t>(k) * lds + r] : 0.f;
		}
		__syncthreads();
		for (int i = ty; i < 32; i += 8) {
			const int r = r0 + i, k = k0 + tx;
			if (r < rows && k < ldp) {
				const float x = tile[tx][i];
				const float h = tf32_hi(x);
				phi[static_cast<int64_t>(r) * ldp + k] = h;
				if (plo) plo[static_cast<int64_t>(r) * ldp + k] = x - h;
			}
		}
	} else {
		for (int i = ty; i < 32; i += 8) {
			const int r = r0 + i, k = k0 + tx;
			if (r < rows && k < ldp) {
				const float x = (k < kdim) ? src[static_cast<int64_t>(r) * lds + k] : 0.f;
				const float h = tf32_hi(x);
				phi[static_cast<int64_t>(r) * ldp + k] = h;
				if (plo) plo[static_cast<int64_t>(r) * ldp + k] = x - h;
			}
		}
	}
}

// Vectorised forms of split_kernel for panels whose rows, width and offsets
// are multiples of 4 (b % 4 == 0): float4 loads, 8- or 16-byte stores.
// TRANS (A_col, element (r, k) at src[k*lds + r]): 64 x 64 transpose tiles.
__global__ void __launch_bounds__(256) split_t_kernel(int rows, int kdim, const float *__restrict__ src, int64_t lds,
	float *__restrict__ phi, float *__restrict__ plo, int64_t ldp)
{
	__shared__ float tile[64][65];   // tile[k][r]
	const int r0 = blockIdx.x * 64, k0 = blockIdx.y * 64;
	const int t = threadIdx.x;
#pragma unroll
	for (int q = 0; q < 4; ++q) {
		const int idx = t + 256 * q, kk = idx >> 4, rr = (idx & 15) * 4;
		const int k = k0 + kk, r = r0 + rr;
		float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
		if (k < kdim && r < rows) v = *reinterpret_cast<const float4 *>(src + static_cast<int64_t>(k) * lds + r);
		tile[kk][rr] = v.x;
		tile[kk][rr + 1] = v.y;
		tile[kk][rr + 2] = v.z;
		tile[kk][rr + 3] = v.w;
	}
	__syncthreads();
#pragma unroll
	for (int q = 0; q < 8; ++q) {
		const int idx = t + 256 * q, rr = idx >> 5, kp = (idx & 31) * 2;
		const int r = r0 + rr, k = k0 + kp;
		if (r < rows && k < ldp) {
			const float x0 = tile[kp][rr], x1 = tile[kp + 1][rr];
			const float h0 = tf32_hi(x0), h1 = tf32_hi(x1);
			*reinterpret_cast<float2 *>(phi + static_cast<int64_t>(r) * ldp + k) = make_float2(h0, h1);
			if (plo) *reinterpret_cast<float2 *>(plo + static_cast<int64_t>(r) * ldp + k) = make_float2(x0 - h0, x1 - h1);
		}
	}
}

// not TRANS (A_row seen by columns, element (r, k) at src[r*lds + k]).
__global__ void __launch_bounds__(256) split_n_kernel(int rows, int kdim, const float *__restrict__ src, int64_t lds,
	float *__restrict__ phi, float *__restrict__ plo, int64_t ldp)
{
	const int groups = static_cast<int>(ldp / 4);
	const int64_t total = static_cast<int64_t>(rows) * groups;
	for (int64_t e = static_cast<int64_t>(blockIdx.x) * 256 + threadIdx.x; e < total;
		e += static_cast<int64_t>(gridDim.x) * 256) {
		const int r = static_cast<int>(e / groups), k = static_cast<int>(e % groups) * 4;
		float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
		if (k < kdim) v = *reinterpret_cast<const float4 *>(src + static_cast<int64_t>(r) * lds + k);
		const float4 h = make_float4(tf32_hi(v.x), tf32_hi(v.y), tf32_hi(v.z), tf32_hi(v.w));
		*reinterpret_cast<float4 *>(phi + static_cast<int64_t>(r) * ldp + k) = h;
		if (plo)
			*reinterpret_cast<float4 *>(plo + static_cast<int64_t>(r) * ldp + k) =
				make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
	}
}

// FP16 K-major copies of a panel for the precision form's panel products:
// out[r*pitch + k] = half_rn(x(r, k)) for k < kdim, zero for kdim <= k < width
// (width <= pitch: a panel may be one slot of a wider group buffer).
// (The precision form's Schur operands are e4m3, so FP16 operands, 11
// significant bits, lose nothing that matters and run the panel products at
// the FP16 tensor rate with half the bytes of TF32.)  With the FP16 deck,
// x = fmaf(deck, inv_scale, a) as deck_apply_kernel forms it, the deck element
// at the same offset from `deck` (leading dimension ldd) as the panel element
// from `src`.  rows, kdim, the offsets and the leading dimensions are
// multiples of 4 (float4 loads, 4-half deck loads).
__device__ __forceinline__ float4 load4_deck(const float *src, const __half *deck, float inv_scale)
{
	float4 v = *reinterpret_cast<const float4 *>(src);
	if (deck) {
		const uint2 d = *reinterpret_cast<const uint2 *>(deck);
		const float2 d01 = __half22float2(*reinterpret_cast<const __half2 *>(&d.x));
		const float2 d23 = __half22float2(*reinterpret_cast<const __half2 *>(&d.y));
		v.x = fmaf(d01.x, inv_scale, v.x);
		v.y = fmaf(d01.y, inv_scale, v.y);
		v.z = fmaf(d23.x, inv_scale, v.z);
		v.w = fmaf(d23.y, inv_scale, v.w);
	}
	return v;
}

// A_col: element (r, k) at src[k*lds + r] (column-major).  64 x 64 tiles
// through shared memory: float4 loads along r, half2 stores along k.
__global__ void __launch_bounds__(256) panel_f16_t_kernel(int rows, int kdim, const float *__restrict__ src,
	int64_t lds, const __half *__restrict__ deck, int64_t ldd, float inv_scale, __half *__restrict__ out,
	int64_t pitch, int width)
{
	__shared__ float tile[64][65];   // tile[k][r]
	const int r0 = blockIdx.x * 64, k0 = blockIdx.y * 64;
	const int t = threadIdx.x;
#pragma unroll
	for (int q = 0; q < 4; ++q) {
		const int idx = t + 256 * q, kk = idx >> 4, rr = (idx & 15) * 4;
		const int k = k0 + kk, r = r0 + rr;
		float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
		if (k < kdim && r < rows)
			v = load4_deck(src + static_cast<int64_t>(k) * lds + r,
				deck ? deck + static_cast<int64_t>(k) * ldd + r : nullptr, inv_scale);
		tile[kk][rr] = v.x;
		tile[kk][rr + 1] = v.y;
		tile[kk][rr + 2] = v.z;
		tile[kk][rr + 3] = v.w;
	}
	__syncthreads();
#pragma unroll
	for (int q = 0; q < 8; ++q) {
		const int idx = t + 256 * q, rr = idx >> 5, kp = (idx & 31) * 2;
		const int r = r0 + rr, k = k0 + kp;
		if (r < rows && k < width)
			*reinterpret_cast<__half2 *>(out + static_cast<int64_t>(r) * pitch + k) =
				__floats2half2_rn(tile[kp][rr], tile[kp + 1][rr]);
	}
}

// A_row seen by columns: element (r, k) at src[r*lds + k]; no transpose.
__global__ void __launch_bounds__(256) panel_f16_n_kernel(int rows, int kdim, const float *__restrict__ src,
	int64_t lds, const __half *__restrict__ deck, int64_t ldd, float inv_scale, __half *__restrict__ out,
	int64_t pitch, int width)
{
	const int groups = width / 4;
	const int64_t total = static_cast<int64_t>(rows) * groups;
	for (int64_t e = static_cast<int64_t>(blockIdx.x) * 256 + threadIdx.x; e < total;
		e += static_cast<int64_t>(gridDim.x) * 256) {
		const int r = static_cast<int>(e / groups), k = static_cast<int>(e % groups) * 4;
		float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
		if (k < kdim)
			v = load4_deck(src + static_cast<int64_t>(r) * lds + k,
				deck ? deck + static_cast<int64_t>(r) * ldd + k : nullptr, inv_scale);
		const __half2 h01 = __floats2half2_rn(v.x, v.y), h23 = __floats2half2_rn(v.z, v.w);
		uint2 w;
		w.x = *reinterpret_cast<const uint32_t *>(&h01);
		w.y = *reinterpret_cast<const uint32_t *>(&h23);
		*reinterpret_cast<uint2 *>(out + static_cast<int64_t>(r) * pitch + k) = w;
	}
}

// Largest |entry| of the two inverted triangles (blockIdx.y: 0 = U11^{-1},
// 1 = L11^{-1}), as the bits of a non-negative float (ordered like unsigned).
__global__ void __launch_bounds__(256) tri_amax_kernel(int b, const float *__restrict__ xu,
	const float *__restrict__ xl, int64_t ldp, unsigned *amax)
{
	const float *x = blockIdx.y ? xl : xu;
	float m = 0.f;
	const int64_t total = static_cast<int64_t>(b) * ldp;
	for (int64_t e = blockIdx.x * 256 + threadIdx.x; e < total; e += static_cast<int64_t>(gridDim.x) * 256) {
		const int pp = static_cast<int>(e % ldp), j = static_cast<int>(e / ldp);
		if (pp <= j && pp < b) m = fmaxf(m, fabsf(x[e]));
	}
	for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
	__shared__ float wm[8];
	if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
	__syncthreads();
	if (threadIdx.x == 0) {
		float r = wm[0];
		for (int w = 1; w < 8; ++w) r = fmaxf(r, wm[w]);
		atomicMax(&amax[blockIdx.y], __float_as_uint(r));
	}
}

// 2^(14 - e) for amax = f 2^e, f in [0.5, 1): the scaled triangle stays below
// 2^14 (FP16 holds up to 65504) and its small entries stay normal longer.
__device__ __forceinline__ float f16_tri_scale(unsigned bits)
{
	const float a = __uint_as_float(bits);
	if (!(a > 0.f) || !isfinite(a)) return 1.f;
	int e = 0;
	(void)frexpf(a, &e);
	return ldexpf(1.f, 14 - e);
}

// The inverted triangles as FP16 Schur operands, scaled by a power of two:
//   uh[j*pitch + p] = half(s_u U11^{-1}(p, j))   (U operand of A_col U11^{-1})
//   lh[i*pitch + p] = half(s_l L11^{-1}(i, p))   (L operand of L11^{-1} A_row)
// for p < width (zero for b <= p), and oscale[0..1] = 1/s_u, 1/s_l (exact)
// for the products' epilogues.
__global__ void __launch_bounds__(256) tri_f16_kernel(int b, const float *__restrict__ xu,
	const float *__restrict__ xl, int64_t ldp, const unsigned *__restrict__ amax, __half *__restrict__ uh,
	__half *__restrict__ lh, int64_t pitch, int width, float *__restrict__ oscale)
{
	const bool lower = blockIdx.y != 0;
	const float *x = lower ? xl : xu;
	__half *o = lower ? lh : uh;
	const float sc = f16_tri_scale(amax[blockIdx.y]);
	if (blockIdx.x == 0 && threadIdx.x == 0) oscale[blockIdx.y] = 1.f / sc;
	const int64_t total = static_cast<int64_t>(b) * width;
	for (int64_t e = blockIdx.x * 256 + threadIdx.x; e < total; e += static_cast<int64_t>(gridDim.x) * 256) {
		const int pp = static_cast<int>(e % width), j = static_cast<int>(e / width);
		const float v = (pp <= j && pp < b) ? x[static_cast<int64_t>(j) * ldp + pp] * sc : 0.f;
		o[static_cast<int64_t>(j) * pitch + pp] = __float2half_rn(v);
	}
}

// ---------------------------------------------------------------------------
// Triangular inverses by recursive doubling.  X = T^{-1}, T upper triangular
// and padded with the identity to bp = ldp rows/columns:
//   TRANS_T = false: T = U11, T[p][j] at lu[j*lda + p], non-unit diagonal
//   TRANS_T = true : T = L11^T, T[p][j] = L[j][p] at lu[p*lda + j], unit diagonal
// Level 0 inverts the 32 x 32 diagonal tiles (one warp each, back
// substitution).  Level l joins pairs of inverted blocks of h = 32 * 2^(l-1):
//   [A B; 0 C]^{-1} = [A^{-1}, -A^{-1} (B C^{-1}); 0, C^{-1}]
// as two FP32 products W = B C^{-1}, then -A^{-1} W, each an upper-triangular
// operand whose zero blocks the tiles skip.  X (work, column-major, ld = ldp)
// is built in place; its strictly lower part is never written and stays zero.
// A final pass writes the hi/lo TF32 split of X for the tensor-core panels.
// ---------------------------------------------------------------------------
template <bool TRANS_T>
__device__ __forceinline__ float tri_t(const float *lu, int64_t lda, int b, int p, int j)
{
	if (p >= b || j >= b) return (p == j) ? 1.f : 0.f;
	if (p > j) return 0.f;
	if (TRANS_T) return (p == j) ? 1.f : lu[static_cast<int64_t>(p) * lda + j];
	return lu[static_cast<int64_t>(j) * lda + p];
}

// grid (tiles, 2): blockIdx.y = 0 -> U11, 1 -> L11^T; one warp per tile.
__global__ void __launch_bounds__(32) tri_diag_kernel(int b, const float *__restrict__ lu, int64_t lda,
	float *__restrict__ xu, float *__restrict__ xl, int64_t ldp)
{
	__shared__ float Tb[32][33];
	const bool lower = blockIdx.y != 0;
	float *x = lower ? xl : xu;
	const int o = blockIdx.x * 32, lane = threadIdx.x;
	for (int i = 0; i < 32; ++i)
		Tb[i][lane] = lower ? tri_t<true>(lu, lda, b, o + i, o + lane) : tri_t<false>(lu, lda, b, o + i, o + lane);
	__syncwarp();
	// column `lane` of the tile's inverse
	float v[32];
#pragma unroll
	for (int i = 31; i >= 0; --i) {
		float a = (i == lane) ? 1.f : 0.f;
#pragma unroll
		for (int p = i + 1; p < 32; ++p) a = fmaf(-Tb[i][p], v[p], a);
		v[i] = lower ? a : a / Tb[i][i];
	}
#pragma unroll
	for (int i = 0; i < 32; ++i) x[static_cast<int64_t>(o + lane) * ldp + o + i] = v[i];
}

// One level's products for every pair and both triangles.  grid.x = 32 x 32
// output tiles of an h x h block (clipped), grid.y = pair, grid.z = triangle.
//   STEP 0: W[o:o+h, o+h:o+h+h2] = T[o:o+h, o+h:..] X[o+h:.., o+h:..]
//   STEP 1: X[o:o+h, o+h:..]     = -X[o:o+h, o:o+h] W[o:o+h, o+h:..]
// K runs in chunks of 32; the next chunk is loaded into registers while the
// current one is multiplied from shared memory.
template <int STEP>
__global__ void __launch_bounds__(128) tri_level_kernel(int b, int bp, int h, const float *__restrict__ lu, int64_t lda,
	float *__restrict__ xu, float *__restrict__ xl, float *__restrict__ wu, float *__restrict__ wl, int64_t ldp)
{
	__shared__ float As[2][32][33];   // [buffer][k][row]
	__shared__ float Bs[2][32][33];   // [buffer][k][col]
	const bool lower = blockIdx.z != 0;
	float *x = lower ? xl : xu;
	float *w = lower ? wl : wu;
	const int o = blockIdx.y * 2 * h;
	const int h2 = min(h, bp - o - h);   // width of the second half
	if (h2 <= 0) return;
	const int tiles_n = (h2 + 31) / 32;
	const int tm = blockIdx.x / tiles_n, tn = blockIdx.x % tiles_n;
	if (tm * 32 >= h) return;
	const int row0 = o + tm * 32, col0 = o + h + tn * 32;   // output tile position in X / W
	const int rend = o + h, cend = o + h + h2;
	const int tid = threadIdx.x;
	// K range with nonzero contributions: STEP 0 rows of X_C up to the
	// tile's last column; STEP 1 columns of X_A from the tile's first row
	const int k_begin = (STEP == 0) ? o + h : row0;
	const int k_end = (STEP == 0) ? min(cend, col0 + 32) : rend;
	// A element (row, k) is contiguous along rows except for L11^T (along k);
	// B element (k, col) is contiguous along k.  Consecutive threads take the
	// contiguous index so every load is coalesced.
	const bool a_k_fast = (STEP == 0) && lower;
	float ra[8], rb[8];
	auto load = [&](int k0) {
#pragma unroll
		for (int q = 0; q < 8; ++q) {
			const int e = tid + 128 * q;
			const int r = a_k_fast ? (e >> 5) : (e & 31), kk = a_k_fast ? (e & 31) : (e >> 5);
			const int k = k0 + kk, row = row0 + r;
			float av = 0.f;
			if (k < k_end && row < rend) {
				if (STEP == 0)
					av = lower ? tri_t<true>(lu, lda, b, row, k) : tri_t<false>(lu, lda, b, row, k);
				else
					av = x[static_cast<int64_t>(k) * ldp + row];
			}
			ra[q] = av;
			const int kb = e & 31, cc = e >> 5;
			const int kq = k0 + kb, col = col0 + cc;
			float bv = 0.f;
			if (kq < k_end && col < cend)
				bv = (STEP == 0) ? x[static_cast<int64_t>(col) * ldp + kq] : w[static_cast<int64_t>(col) * ldp + kq];
			rb[q] = bv;
		}
	};
	auto stash = [&](int buf) {
#pragma unroll
		for (int q = 0; q < 8; ++q) {
			const int e = tid + 128 * q;
			const int r = a_k_fast ? (e >> 5) : (e & 31), kk = a_k_fast ? (e & 31) : (e >> 5);
			As[buf][kk][r] = ra[q];
			Bs[buf][e & 31][e >> 5] = rb[q];
		}
	};
	// thread: output column `c`, rows 8g .. 8g+7
	const int c = tid & 31, g = tid >> 5;
	float acc[8] = {};
	int buf = 0;
	if (k_begin < k_end) {
		load(k_begin);
		stash(0);
	}
	__syncthreads();
	for (int k0 = k_begin; k0 < k_end; k0 += 32) {
		const bool more = k0 + 32 < k_end;
		if (more) load(k0 + 32);
#pragma unroll
		for (int kk = 0; kk < 32; ++kk) {
			const float bv = Bs[buf][kk][c];
#pragma unroll
			for (int i = 0; i < 8; ++i) acc[i] = fmaf(As[buf][kk][8 * g + i], bv, acc[i]);
		}
		if (more) stash(buf ^ 1);
		__syncthreads();
		buf ^= 1;
	}
	// write through shared memory so the stores run along the rows
	float *out = (STEP == 0) ? w : x;
	const float sgn = (STEP == 0) ? 1.f : -1.f;
#pragma unroll
	for (int i = 0; i < 8; ++i) As[0][c][8 * g + i] = sgn * acc[i];
	__syncthreads();
#pragma unroll
	for (int q = 0; q < 8; ++q) {
		const int e = tid + 128 * q;
		const int r = e & 31, cc = e >> 5;
		const int row = row0 + r, col = col0 + cc;
		if (row < rend && col < cend) out[static_cast<int64_t>(col) * ldp + row] = As[0][cc][r];
	}
}

// X (work, ldp x ldp) -> hi/lo copies: column col < b is map row col of
// the K-major operand, rows 0..ldp-1 with zeros below the diagonal.
__global__ void __launch_bounds__(256) tri_split_kernel(int b, const float *__restrict__ xu,
	const float *__restrict__ xl, float *__restrict__ uhi, float *__restrict__ ulo, float *__restrict__ lhi,
	float *__restrict__ llo, int64_t ldp)
{
	const bool lower = blockIdx.y != 0;
	const float *x = lower ? xl : xu;
	float *hi = lower ? lhi : uhi, *lo = lower ? llo : ulo;
	const int64_t total = static_cast<int64_t>(b) * ldp;
	for (int64_t e = blockIdx.x * 256 + threadIdx.x; e < total; e += static_cast<int64_t>(gridDim.x) * 256) {
		const int row = static_cast<int>(e % ldp), col = static_cast<int>(e / ldp);
		const float v = (row <= col) ? x[e] : 0.f;
		const float hv = tf32_hi(v);
		hi[e] = hv;
		lo[e] = v - hv;
	}
}

// ---------------------------------------------------------------------------
// 3xTF32 GEMM: D (M x N) = A (M x K) B (N x K)^T, K-major hi/lo operands.
// Output: out32[m*s32m + n*s32n] = D, out16[m*s16m + n*s16n] = half(scale*D).
// ---------------------------------------------------------------------------
constexpr int TBM = 128, TBN = 128, TBK = 32;          // TBK FP32 = one 128-byte swizzle row
constexpr int TSTAGES = 3;
constexpr int TILE_BYTES = TBM * TBK * 4;              // 16 KB per operand tile (M and N both 128)
constexpr int TSTAGE_BYTES = 4 * TILE_BYTES;           // A hi/lo, B hi/lo
constexpr int TEPI_WARPS = 4;
constexpr int TTHREADS = (2 + TEPI_WARPS) * 32;
constexpr uint32_t TTMEM_COLS = 2 * TBN;
constexpr size_t TSMEM_BYTES = static_cast<size_t>(TSTAGES) * TSTAGE_BYTES + 1024 + 256;

struct TParams {
	int m, n, num_kc, tiles_m, tiles_n;
	int arow0, brow0;   // first rows of A and B in their maps
	float *out32;
	int64_t s32m, s32n;
	__half *out16;
	int64_t s16m, s16n;
	float scale;
	unsigned *status;   // set to 1 on a wait timeout
	int terms;          // 3: hi*hi + hi*lo + lo*hi (FP32 accuracy); 1: hi*hi only (TF32)
};

__device__ unsigned int g_tstatus;

// kind::tf32 instruction descriptor: FP32 accumulator, A/B TF32 (format 2), K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n)
{
	return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
	       (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
	uint32_t accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
		::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
		: "memory");
}

__global__ void __launch_bounds__(TTHREADS, 1) tf32x3_kernel(const __grid_constant__ CUtensorMap ahi,
	const __grid_constant__ CUtensorMap alo, const __grid_constant__ CUtensorMap bhi,
	const __grid_constant__ CUtensorMap blo, const TParams p)
{
	extern __shared__ uint8_t smem_raw[];
	const uint32_t raw_addr = smem_u32(smem_raw);
	uint8_t *smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
	uint64_t *bars = reinterpret_cast<uint64_t *>(smem + TSTAGES * TSTAGE_BYTES);
	uint64_t *full = bars;
	uint64_t *empty = bars + TSTAGES;
	uint64_t *accf = bars + 2 * TSTAGES;
	uint64_t *acce = accf + 2;
	uint64_t *drain = acce + 2;
	uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(drain + 1);
	int *consumed = reinterpret_cast<int *>(tmem_holder + 1);

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (threadIdx.x == 0) {
		for (int s = 0; s < TSTAGES; ++s) {
			mbar_init(&full[s], 1);
			mbar_init(&empty[s], 1);
		}
		for (int a = 0; a < 2; ++a) {
			mbar_init(&accf[a], 1);
			mbar_init(&acce[a], TEPI_WARPS * 32);
		}
		mbar_init(drain, 1);
		*consumed = 0;
		fence_mbar_init();
	}
	if (warp == 1) {
		tmem_alloc(tmem_holder, TTMEM_COLS);
		tmem_relinquish();
	}
	if (warp == 0 && lane == 0) {
		tma_prefetch_desc(&ahi);
		tma_prefetch_desc(&alo);
		tma_prefetch_desc(&bhi);
		tma_prefetch_desc(&blo);
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem_base = *tmem_holder;
	const int total = p.tiles_m * p.tiles_n;
	int issued = 0;

	if (warp == 0) {
		if (lane == 0) {
			bool ok = true;
			int stage = 0;
			uint32_t phase = 0;
			for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
				const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
				for (int kc = 0; kc < p.num_kc; ++kc) {
					if (!mbar_wait(&empty[stage], phase ^ 1u)) { ok = false; break; }
					mbar_arrive_expect_tx(&full[stage], p.terms == 1 ? 2 * TILE_BYTES : TSTAGE_BYTES);
					uint8_t *st = smem + stage * TSTAGE_BYTES;
					tma_load_2d(st, &ahi, &full[stage], kc * TBK, p.arow0 + tm * TBM);
					if (p.terms != 1) tma_load_2d(st + TILE_BYTES, &alo, &full[stage], kc * TBK, p.arow0 + tm * TBM);
					tma_load_2d(st + 2 * TILE_BYTES, &bhi, &full[stage], kc * TBK, p.brow0 + tn * TBN);
					if (p.terms != 1) tma_load_2d(st + 3 * TILE_BYTES, &blo, &full[stage], kc * TBK, p.brow0 + tn * TBN);
					++issued;
					if (++stage == TSTAGES) { stage = 0; phase ^= 1u; }
				}
			}
			if (!ok) atomicOr(p.status, 1u);
		}
	} else if (warp == 1) {
		if (lane == 0) {
			bool ok = true;
			int stage = 0, acc = 0, used = 0;
			uint32_t phase = 0, acc_phase = 0;
			const uint32_t idesc = idesc_tf32(TBM, TBN);
			for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
				if (!mbar_wait(&acce[acc], acc_phase ^ 1u)) { ok = false; break; }
				tc_fence_after();
				const uint32_t d = tmem_base + static_cast<uint32_t>(acc * TBN);
				for (int kc = 0; kc < p.num_kc; ++kc) {
					if (!mbar_wait(&full[stage], phase)) { ok = false; break; }
					tc_fence_after();
					const uint32_t st = smem_u32(smem + stage * TSTAGE_BYTES);
					const uint64_t dah = umma_desc_k_sw128(st), dal = umma_desc_k_sw128(st + TILE_BYTES);
					const uint64_t dbh = umma_desc_k_sw128(st + 2 * TILE_BYTES), dbl = umma_desc_k_sw128(st + 3 * TILE_BYTES);
#pragma unroll
					for (int kk = 0; kk < TBK / 8; ++kk) {
						// 8 FP32 = 32 bytes = 2 units of 16 B along K inside the swizzle row
						const uint32_t o = 2u * kk;
						umma_tf32(d, dah + o, dbh + o, idesc, (kc | kk) != 0 ? 1u : 0u);
						if (p.terms != 1) {
							umma_tf32(d, dah + o, dbl + o, idesc, 1u);
							umma_tf32(d, dal + o, dbh + o, idesc, 1u);
						}
					}
					umma_commit(&empty[stage]);
					++used;
					if (++stage == TSTAGES) { stage = 0; phase ^= 1u; }
				}
				if (!ok) break;
				umma_commit(&accf[acc]);
				if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
			}
			umma_commit(drain);
			if (!mbar_wait(drain, 0)) ok = false;
			*consumed = used;
			if (!ok) atomicOr(p.status, 1u);
		}
	} else {
		const int q = warp & 3;
		bool ok = true;
		int acc = 0;
		uint32_t acc_phase = 0;
		for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
			const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
			const bool mine = mbar_wait(&accf[acc], acc_phase);
			ok = __all_sync(0xffffffffu, mine) != 0;
			if (!ok) break;
			tc_fence_after();
			const int row = tm * TBM + q * 32 + lane;
			const bool rok = row < p.m;
			const uint32_t tbase = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * TBN);
#pragma unroll 1
			for (int ch = 0; ch < TBN / 32; ++ch) {
				uint32_t r[32];
				tmem_ld_32x32b_x32(tbase + static_cast<uint32_t>(ch * 32), r);
				tmem_ld_wait();
				const int col0 = tn * TBN + ch * 32;
				if (rok) {
					__half *o16 = p.out16 ? p.out16 + row * p.s16m + col0 * p.s16n : nullptr;
					// a row-major FP16 copy gets this thread's 32 columns as four 16-byte stores
					const bool vec16 = o16 && p.s16n == 1 && col0 + 32 <= p.n && (reinterpret_cast<uintptr_t>(o16) & 15u) == 0;
#pragma unroll
					for (int j = 0; j < 32; ++j) {
						const int col = col0 + j;
						if (col < p.n) {
							const float v = __uint_as_float(r[j]);
							p.out32[row * p.s32m + col * p.s32n] = v;
							if (o16 && !vec16) p.out16[row * p.s16m + col * p.s16n] = __float2half_rn(p.scale * v);
						}
					}
					if (vec16) {
#pragma unroll
						for (int q = 0; q < 4; ++q) {
							uint32_t w4[4];
#pragma unroll
							for (int e = 0; e < 4; ++e) {
								const __half2 h2 = __floats2half2_rn(p.scale * __uint_as_float(r[8 * q + 2 * e]),
									p.scale * __uint_as_float(r[8 * q + 2 * e + 1]));
								w4[e] = *reinterpret_cast<const uint32_t *>(&h2);
							}
							*reinterpret_cast<uint4 *>(o16 + 8 * q) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
						}
					}
				}
			}
			tc_fence_before();
			mbar_arrive(&acce[acc]);
			if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
		}
		if (lane == 0 && !ok) atomicOr(p.status, 1u);
	}

	tc_fence_before();
	__syncthreads();
	if (warp == 0 && lane == 0) {
		int left = issued - *consumed;
		for (int s = 0; left > 0 && s < TSTAGES; ++s, --left)
			(void)mbar_wait(&full[(*consumed + s) % TSTAGES], static_cast<uint32_t>(((*consumed + s) / TSTAGES) & 1));
	}
	if (warp == 1) {
		tc_fence_after();
		tmem_dealloc(tmem_base, TTMEM_COLS);
	}
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn_tc()
{
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	if (!fn) {
		void *ptr = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
			q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
	}
	return fn;
}

// FP32 K-major operand map: rows x kdim, row pitch ldp floats, box TBK x 128, 128B swizzle.
int make_f32_kmajor(void *out, const float *base, int rows, int kdim, int64_t ldp)
{
	auto fn = encode_fn_tc();
	if (!fn) return HPLAI_ECUDA;
	if ((reinterpret_cast<uintptr_t>(base) & 15u) || ((ldp * 4) & 15u)) return HPLAI_EINVAL;
	CUtensorMap m;
	cuuint64_t dims[2] = {static_cast<cuuint64_t>(kdim), static_cast<cuuint64_t>(rows)};
	cuuint64_t strides[1] = {static_cast<cuuint64_t>(ldp * 4)};
	cuuint32_t box[2] = {TBK, 128};
	cuuint32_t estr[2] = {1, 1};
	CUresult r = fn(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, estr,
		CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
		CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS) return HPLAI_EINVAL;
	std::memcpy(out, &m, sizeof(m));
	return HPLAI_OK;
}

int sm_count()
{
	int dev = 0, sms = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return 148;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return 148;
	return sms;
}

int launch_tf32x3(const unsigned char *m_ahi, const unsigned char *m_alo, const unsigned char *m_bhi,
	const unsigned char *m_blo, int arow0, int brow0, int M, int N, int K, float *out32, int64_t s32m, int64_t s32n,
	__half *out16, int64_t s16m, int64_t s16n, float scale, int max_ctas, cudaStream_t st, unsigned *status, int terms)
{
	if (M <= 0 || N <= 0) return HPLAI_OK;
	TParams p;
	p.terms = terms;
	p.status = status;
	if (!p.status) {
		void *g = nullptr;
		HPLAI_CUDA_TRY(cudaGetSymbolAddress(&g, g_tstatus));
		p.status = static_cast<unsigned *>(g);
	}
	p.m = M;
	p.n = N;
	p.num_kc = (K + TBK - 1) / TBK;
	p.tiles_m = (M + TBM - 1) / TBM;
	p.tiles_n = (N + TBN - 1) / TBN;
	p.arow0 = arow0;
	p.brow0 = brow0;
	p.out32 = out32;
	p.s32m = s32m;
	p.s32n = s32n;
	p.out16 = out16;
	p.s16m = s16m;
	p.s16n = s16n;
	p.scale = scale;
	static DeviceOnce attr;
	HPLAI_TRY(attr.get([](int, int *) -> int {
		HPLAI_CUDA_TRY(cudaFuncSetAttribute(tf32x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			static_cast<int>(TSMEM_BYTES)));
		return HPLAI_OK;
	}));
	const int total = p.tiles_m * p.tiles_n;
	int grid = max_ctas > 0 ? max_ctas : sm_count();
	if (grid > total) grid = total;
	CUtensorMap a0, a1, b0, b1;
	std::memcpy(&a0, m_ahi, sizeof(a0));
	std::memcpy(&a1, m_alo, sizeof(a1));
	std::memcpy(&b0, m_bhi, sizeof(b0));
	std::memcpy(&b1, m_blo, sizeof(b1));
	tf32x3_kernel<<<grid, TTHREADS, TSMEM_BYTES, st>>>(a0, a1, b0, b1, p);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

} // namespace

static_assert(sizeof(CUtensorMap) <= 128, "tensor map storage");

int tc_panels_make(TcPanels *t, int n, int b, float *phi, float *plo, int64_t ldp, float *uhi, float *ulo,
	float *lhi, float *llo, float *work)
{
	if (!t || n <= 0 || b <= 0 || ldp < b || (ldp % 32) || !work) return HPLAI_EINVAL;
	const size_t sq = static_cast<size_t>(ldp) * ldp;
	t->xu = work;
	t->xl = work + sq;
	t->wu = work + 2 * sq;
	t->wl = work + 3 * sq;
	t->n = n;
	t->b = b;
	t->ldp = ldp;
	t->phi = phi;
	t->plo = plo;
	t->uhi = uhi;
	t->ulo = ulo;
	t->lhi = lhi;
	t->llo = llo;
	HPLAI_TRY(make_f32_kmajor(t->m_phi, phi, n, b, ldp));
	HPLAI_TRY(make_f32_kmajor(t->m_plo, plo, n, b, ldp));
	HPLAI_TRY(make_f32_kmajor(t->m_uhi, uhi, b, b, ldp));
	HPLAI_TRY(make_f32_kmajor(t->m_ulo, ulo, b, b, ldp));
	HPLAI_TRY(make_f32_kmajor(t->m_lhi, lhi, b, b, ldp));
	HPLAI_TRY(make_f32_kmajor(t->m_llo, llo, b, b, ldp));
	return HPLAI_OK;
}

int launch_tri_inverses(const TcPanels &t, const float *lu, int64_t lda, cudaStream_t st, bool split)
{
	const int b = t.b;
	const int bp = static_cast<int>(t.ldp);
	const int nt = bp / 32;
	tri_diag_kernel<<<dim3(nt, 2), 32, 0, st>>>(b, lu, lda, t.xu, t.xl, t.ldp);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	for (int h = 32; h < bp; h *= 2) {
		const int pairs = (bp + 2 * h - 1) / (2 * h);
		const int tiles = ((h + 31) / 32) * ((h + 31) / 32);
		const dim3 g(tiles, pairs, 2);
		tri_level_kernel<0><<<g, 128, 0, st>>>(b, bp, h, lu, lda, t.xu, t.xl, t.wu, t.wl, t.ldp);
		count_launches();
		HPLAI_CUDA_TRY(cudaGetLastError());
		tri_level_kernel<1><<<g, 128, 0, st>>>(b, bp, h, lu, lda, t.xu, t.xl, t.wu, t.wl, t.ldp);
		count_launches();
		HPLAI_CUDA_TRY(cudaGetLastError());
	}
	if (!split) return HPLAI_OK;
	// U11^{-1} column-major = the B operand of the L-panel product (row n = column n of U^{-1});
	// (L11^T)^{-1} column-major = L11^{-1} row-major = the A operand of the U-panel product.
	tri_split_kernel<<<dim3((b * bp + 255) / 256 < 1184 ? (b * bp + 255) / 256 : 1184, 2), 256, 0, st>>>(b, t.xu,
		t.xl, t.uhi, t.ulo, t.lhi, t.llo, t.ldp);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_lpanel_tc(const TcPanels &t, int rem, float *acol, int64_t lda, uint16_t *lh, int64_t ldh, float scale,
	int max_ctas, cudaStream_t st)
{
	if (rem <= 0) return HPLAI_OK;
	const int b = t.b;
	float *plo = t.terms == 1 ? nullptr : t.plo;
	const bool vec = b % 4 == 0 && rem % 4 == 0 && lda % 4 == 0 && (reinterpret_cast<uintptr_t>(acol) & 15) == 0;
	if (vec) {
		split_t_kernel<<<dim3((rem + 63) / 64, static_cast<unsigned>((t.ldp + 63) / 64)), 256, 0, st>>>(rem, b, acol,
			lda, t.phi, plo, t.ldp);
	} else {
		dim3 g((rem + 31) / 32, static_cast<unsigned>(t.ldp / 32));
		split_kernel<true><<<g, 256, 0, st>>>(rem, b, acol, lda, t.phi, plo, t.ldp);
	}
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	// X (rem x b) = A_col U^{-1}: out32 column-major in A, out16 row-major (Lh row = panel row)
	return launch_tf32x3(t.m_phi, t.m_plo, t.m_uhi, t.m_ulo, 0, 0, rem, b, b, acol, 1, lda,
		reinterpret_cast<__half *>(lh), ldh, 1, scale, max_ctas, st, t.status, t.terms);
}

int launch_upanel_tc(const TcPanels &t, int rem, float *arow, int64_t lda, uint16_t *uh, int64_t ldh, float scale,
	int max_ctas, cudaStream_t st)
{
	if (rem <= 0) return HPLAI_OK;
	const int b = t.b;
	// B operand row j = column j of A_row (b contiguous floats, stride lda)
	float *plo = t.terms == 1 ? nullptr : t.plo;
	const bool vec = b % 4 == 0 && lda % 4 == 0 && (reinterpret_cast<uintptr_t>(arow) & 15) == 0;
	if (vec) {
		const int64_t work = static_cast<int64_t>(rem) * (t.ldp / 4);
		const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((work + 255) / 256, 148 * 16));
		split_n_kernel<<<blocks, 256, 0, st>>>(rem, b, arow, lda, t.phi, plo, t.ldp);
	} else {
		dim3 g((rem + 31) / 32, static_cast<unsigned>(t.ldp / 32));
		split_kernel<false><<<g, 256, 0, st>>>(rem, b, arow, lda, t.phi, plo, t.ldp);
	}
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	// Y (b x rem) = L^{-1} A_row: out32 column-major in A, out16 with column j of U as row j of Uh
	return launch_tf32x3(t.m_lhi, t.m_llo, t.m_phi, t.m_plo, 0, 0, b, rem, b, arow, 1, lda,
		reinterpret_cast<__half *>(uh), 1, ldh, scale, max_ctas, st, t.status, t.terms);
}

int launch_lpanel_f16(const TcPanels &t, const SchurMaps &maps, int kb, int rem, float *a, int64_t lda,
	uint16_t *lh, uint16_t *uh, int64_t ldh, const uint16_t *deck, int64_t ldd, float inv_dscale, int max_ctas,
	cudaStream_t st, const float *src, int64_t lds, const AmaxTargets *amax)
{
	if (rem <= 0) return HPLAI_OK;
	const int width = (t.b + 63) / 64 * 64;   // the panel's slot in a buffer of row pitch ldh
	if (!t.f16_amax || !t.f16_oscale || ldh % 64 || ldh < width || t.b % 4 || kb % 4 || rem % 4 || lda % 4 ||
		ldd % 4 || (src && (lds % 4 || lds < rem || reinterpret_cast<uintptr_t>(src) % 16)))
		return HPLAI_EINVAL;
	const int b = t.b;
	// the inverted triangles into rows kb .. kb+b-1 of the FP16 panel buffers
	// (rows the step's Schur update never reads)
	HPLAI_CUDA_TRY(cudaMemsetAsync(t.f16_amax, 0, 2 * sizeof(unsigned), st));
	const int tb = static_cast<int>(std::min<int64_t>((static_cast<int64_t>(b) * t.ldp + 255) / 256, 592));
	tri_amax_kernel<<<dim3(tb, 2), 256, 0, st>>>(b, t.xu, t.xl, t.ldp, t.f16_amax);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	tri_f16_kernel<<<dim3(tb, 2), 256, 0, st>>>(b, t.xu, t.xl, t.ldp, t.f16_amax,
		reinterpret_cast<__half *>(uh) + static_cast<int64_t>(kb) * ldh,
		reinterpret_cast<__half *>(lh) + static_cast<int64_t>(kb) * ldh, ldh, width, t.f16_oscale);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	// A_col (rows kb+b.., columns kb..kb+b-1) -> FP16 K-major rows kb+b.. of lh
	const int64_t kbl = kb;
	const float *acol = src ? src : a + (kbl + b) + kbl * lda;
	const __half *dcol = deck ? reinterpret_cast<const __half *>(deck) + (kbl + b) + kbl * ldd : nullptr;
	panel_f16_t_kernel<<<dim3((rem + 63) / 64, static_cast<unsigned>(width / 64)), 256, 0, st>>>(rem, b, acol,
		src ? lds : lda, dcol, ldd, inv_dscale, reinterpret_cast<__half *>(lh) + (kbl + b) * ldh, ldh, width);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	// A_col = (A_col (s_u U11^{-1})) / s_u
	return launch_schur_store(maps, kb + b, kb, rem, b, a, lda, kb + b, kb, t.f16_oscale, max_ctas, st, amax);
}

int launch_upanel_f16(const TcPanels &t, const SchurMaps &maps, int kb, int rem, float *a, int64_t lda,
	uint16_t *uh, int64_t ldh, const uint16_t *deck, int64_t ldd, float inv_dscale, int max_ctas, cudaStream_t st,
	const float *src, int64_t lds, const AmaxTargets *amax)
{
	if (rem <= 0) return HPLAI_OK;
	const int width = (t.b + 63) / 64 * 64;
	if (!t.f16_oscale || ldh % 64 || ldh < width || t.b % 4 || kb % 4 || rem % 4 || lda % 4 || ldd % 4 ||
		(src && (lds % 4 || lds < t.b || reinterpret_cast<uintptr_t>(src) % 16)))
		return HPLAI_EINVAL;
	const int b = t.b;
	const int64_t kbl = kb;
	// A_row (rows kb..kb+b-1, columns kb+b..): column j -> FP16 row kb+b+j of uh
	const float *arow = src ? src : a + kbl + (kbl + b) * lda;
	const __half *drow = deck ? reinterpret_cast<const __half *>(deck) + kbl + (kbl + b) * ldd : nullptr;
	{
		const int64_t work = static_cast<int64_t>(rem) * (width / 4);
		const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((work + 255) / 256, 148 * 16));
		panel_f16_n_kernel<<<blocks, 256, 0, st>>>(rem, b, arow, src ? lds : lda, drow, ldd, inv_dscale,
			reinterpret_cast<__half *>(uh) + (kbl + b) * ldh, ldh, width);
	}
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	// A_row = ((s_l L11^{-1}) A_row) / s_l, the triangle in rows kb.. of the L buffer
	return launch_schur_store(maps, kb, kb + b, b, rem, a, lda, kb, kb + b, t.f16_oscale + 1, max_ctas, st, amax);
}

int tc_status()
{
	unsigned int v = 0;
	if (cudaMemcpyFromSymbol(&v, g_tstatus, sizeof(v)) != cudaSuccess) return HPLAI_ECUDA;
	return v ? HPLAI_ETIMEOUT : HPLAI_OK;
}

void tc_status_reset()
{
	unsigned int z = 0;
	(void)cudaMemcpyToSymbol(g_tstatus, &z, sizeof(z));
}

} // namespace hplai
