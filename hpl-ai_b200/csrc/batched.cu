// batched.cu -- many independent HPL-AI systems in one step-synchronous
// pass: every kernel of the factorisation and of the refinement covers all
// systems at once, and the generation plus the whole factorisation are one
// CUDA graph replayed per solve.
//
// The reference solves one system per run (main.cpp:144-492); per system
// this is the same method: the HPL-AI matrix of order n from its seed
// (hpl_rand.hpp:35-123), right-hand sides from columns n, n+1, ... of the
// stream (pcolvgen, matgen.hpp:193-207), the no-pivot blocked LU with FP32
// panels and an FP16 Schur update (panel_trf.hpp:434-633), and FP64
// iterative refinement with the matrix regenerated on the fly
// (iterative_refinement.hpp:18-57).
//
// Layout.  System s is padded with the identity to P_s = roundup(n_s, 128)
// (the LU of [[A, 0], [0, I]] is [[L, 0], [0, I]] [[U, 0], [0, I]], exactly:
// the padding receives only zero updates), and the systems sit side by side
// in one FP32 matrix of P_max rows (ld = P_max): system s's A(i, j) is at
// row i, column C_s + j, with 128 unused columns after each system (the
// last 256-column Schur tile of a step may reach past a system's columns).
// A system's columns are contiguous in memory, so a 128-column block spans a
// few pages.  Its L and U panels of step k are FP16 copies in two stacked
// K-major buffers (row R_s + i of L16 = row i of L, row R_s + j of U16 =
// column j of U).  Systems are ordered by decreasing P_s, so the systems
// still factoring at step k are a prefix.
//
// Step k (128-wide panels):
//   getrf   one CTA per system, the 128 x 128 diagonal block in shared
//           memory, unblocked right-looking LU with fmaf(-l_ik, u_kj, a_ij)
//           and multipliers a_ik * (1 / u_kk): the operation sequence of
//           getrf_nopiv (getrf_nopiv.hpp:30-46, 124-160), bit for bit;
//   trsm    one CTA per 128-row (128-column) chunk of every system's L (U)
//           panel, netlib strsm order (panel_trf.hpp:143-171), writing the
//           FP32 panel and its FP16 copy;
//   schur   one persistent tcgen05 launch over the tiles of every system's
//           trailing update (a tile table; TMA reduce-add into A).
// Refinement, per (system, right-hand side): x_0 = b ./ d, then residuals
// with the matrix regenerated in FP64, the hpl-harness on the device, and
// corrections x += U^-1 L^-1 r for the pairs still above 16; the host reads
// one counter per step.
#include "common.cuh"
#include "internal.h"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

namespace hplai {

namespace {

constexpr int kBB = 128;          // panel width
constexpr int kGemvRows = 256;    // GEMV rows per CTA
constexpr int kGemvCols = 512;    // GEMV columns per CTA (one partial-sum chunk)
constexpr int kMaxRhs = 8;

struct JumpT {
	Coeff p[64];
};

JumpT make_jump()
{
	JumpT t;
	Coeff p{kLcgA, kLcgC};
	for (int k = 0; k < 64; ++k) {
		t.p[k] = p;
		p = coeff_mul(p, p);
	}
	return t;
}

__device__ __forceinline__ Coeff jump(const JumpT &t, uint64_t m)
{
	Coeff r{1ULL, 0ULL};
	for (int k = 0; m; ++k, m >>= 1)
		if (m & 1ULL) r = coeff_mul(r, t.p[k]);
	return r;
}

} // namespace

// Per-system descriptor (device copy), in factorisation order.
struct BSys {
	int n, P, nrhs, orig;   // order, padded order, right-hand sides, index in the caller's arrays
	int64_t R;              // its first row in the stacked FP16 panel buffers
	int64_t C;              // its first column in A (ld P_max; 128 unused columns after each system)
	int64_t voff;           // its n x nrhs vectors (rhs, x, r), column-major with ld n
	int64_t doff;           // its n diagonal entries
	int64_t poff;           // its GEMV partial sums: ceil(n / kGemvCols) x nrhs x n
	int pair0;              // index of its first (system, right-hand side) pair
	int pad_;
	uint64_t state0;        // a * seed + c
};

namespace {

// ---------------------------------------------------------------------------
// Generation: A (padded), the FP64 diagonal d and the right-hand sides.
// ---------------------------------------------------------------------------

// item = (system, first column): 32 columns of all P_s rows.  Real entries
// are the generator's values rounded to FP32 (fill_one_panel_with_rand,
// hpl_rand.hpp:59-106); the padding is the identity.  The real diagonal is
// written afterwards by bdiag_kernel.
__global__ void __launch_bounds__(256) bfill_kernel(const BSys *__restrict__ sys, const int2 *__restrict__ items,
	float *__restrict__ A, int64_t lda, JumpT tab)
{
	const int2 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const int c0 = it.y, c1 = min(c0 + 32, S.P);
	const Coeff jn = jump(tab, static_cast<uint64_t>(S.n));
	for (int i = threadIdx.x; i < S.P; i += 256) {
		float *col = A + i + (S.C + c0) * lda;
		if (i < S.n) {
			uint64_t s = coeff_apply(jump(tab, static_cast<uint64_t>(i) + static_cast<uint64_t>(S.n) * c0), S.state0);
			for (int c = c0; c < c1; ++c, col += lda) {
				*col = c < S.n ? __double2float_rn(state_value(s)) : 0.f;
				s = coeff_apply(jn, s);
			}
		} else {
			for (int c = c0; c < c1; ++c, col += lda) *col = (c == i) ? 1.f : 0.f;
		}
	}
}

// d_i = sum_{j != i} |a_ij| in sequential FP64 (hpl_rand.hpp:108-123); the
// FP32 rounding also becomes A's diagonal.  item = (system, first row).
__global__ void __launch_bounds__(128) bdiag_kernel(const BSys *__restrict__ sys, const int2 *__restrict__ items,
	float *__restrict__ A, int64_t lda, double *__restrict__ d, JumpT tab)
{
	const int2 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const int i = it.y + threadIdx.x;
	if (i >= S.n) return;
	const int n = S.n;
	const Coeff jn = jump(tab, static_cast<uint64_t>(n));
	const Coeff jn4 = coeff_mul(coeff_mul(jn, jn), coeff_mul(jn, jn));
	uint64_t s0 = coeff_apply(jump(tab, static_cast<uint64_t>(i)), S.state0);
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
	d[S.doff + i] = sum;
	A[i + (S.C + i) * lda] = __double2float_rn(sum);
}

// rhs column q = stream column n + q (item = (system, first row)).
__global__ void __launch_bounds__(128) brhs_kernel(const BSys *__restrict__ sys, const int2 *__restrict__ items,
	double *__restrict__ rhs, JumpT tab)
{
	const int2 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const int i = it.y + threadIdx.x;
	if (i >= S.n) return;
	const Coeff jn = jump(tab, static_cast<uint64_t>(S.n));
	uint64_t s = coeff_apply(jump(tab, static_cast<uint64_t>(i) + static_cast<uint64_t>(S.n) * S.n), S.state0);
	for (int q = 0; q < S.nrhs; ++q) {
		rhs[S.voff + static_cast<int64_t>(q) * S.n + i] = state_value(s);
		s = coeff_apply(jn, s);
	}
}

// ---------------------------------------------------------------------------
// Factorisation step k.
// ---------------------------------------------------------------------------
constexpr int kLdS = kBB + 1;   // shared-memory column pitch (bank-conflict free)
constexpr int kLdT = kBB + 4;   // pitch of the TRSM triangle: rows of 16-byte aligned float4

// The diagonal block (k, k) of system blockIdx.x (the active prefix).
__global__ void __launch_bounds__(512) bgetrf_kernel(const BSys *__restrict__ sys, float *__restrict__ A, int64_t lda,
	int k)
{
	extern __shared__ float sm[];
	const BSys S = sys[blockIdx.x];
	float *blk = A + static_cast<int64_t>(k) * kBB + (S.C + static_cast<int64_t>(k) * kBB) * lda;
	for (int e = threadIdx.x; e < kBB * kBB; e += 512) {
		const int r = e % kBB, c = e / kBB;
		sm[c * kLdS + r] = blk[r + static_cast<int64_t>(c) * lda];
	}
	__syncthreads();
	for (int p = 0; p < kBB; ++p) {
		// multipliers a_ip * (1 / u_pp), then the rank-1 update of the trailing block
		const float inv = 1.0f / sm[p * kLdS + p];
		for (int i = p + 1 + threadIdx.x; i < kBB; i += 512) sm[p * kLdS + i] *= inv;
		__syncthreads();
		const int w = kBB - 1 - p;
		for (int e = threadIdx.x; e < w * w; e += 512) {
			const int i = p + 1 + e % w, j = p + 1 + e / w;
			sm[j * kLdS + i] = fmaf(-sm[p * kLdS + i], sm[j * kLdS + p], sm[j * kLdS + i]);
		}
		__syncthreads();
	}
	for (int e = threadIdx.x; e < kBB * kBB; e += 512) {
		const int r = e % kBB, c = e / kBB;
		blk[r + static_cast<int64_t>(c) * lda] = sm[c * kLdS + r];
	}
}

// One 128-row chunk of a system's L panel below the diagonal block (side 0:
// L = A_col U^-1) or one 128-column chunk of its U panel (side 1:
// U = L^-1 A_row); item = (system, chunk, side).  The netlib strsm order
//   strsm("R","U","N","N"): for j: for i < j: b_j -= u_ij b_i; b_j *= 1/u_jj
//   strsm("L","L","N","U"): for i: if b_i != 0: for r > i: b_r -= l_ri b_i
// with each multiply-add one fmaf (getrf_nopiv.hpp:14-28 as the reference's
// -ffp-contract=fast build runs it), applied right-looking: at step i the
// final b_i is published and every later element takes its update, so each
// element sees the same updates in the same order as the netlib loops.
// 256 threads; thread (lane, warp) holds 4 panel rows (side 0; columns for
// side 1) 4 lane .. 4 lane + 3 times 16 elements 16 warp .. 16 warp + 15 in
// registers, so the owner of step i is one warp and every other thread
// updates 64 elements per step from two 16-byte shared-memory reads.
// The 128 steps of one panel chunk.  Warp oi owns steps 16 oi .. 16 oi + 15
// (its elements); within a warp's 16 steps the step index is a
// compile-time constant, so the owner reads and scales its element directly
// and a thread of a later warp updates all 16 of its elements unpredicated.
template <bool UPPER>
__device__ __forceinline__ void trsm_steps(float (&b)[4][16], const float *tri, float *pub, int p0, int e0, int wp)
{
	for (int oi = 0; oi < 8; ++oi) {
#pragma unroll
		for (int li = 0; li < 16; ++li) {
			const int i = 16 * oi + li;
			float *pb = pub + (li & 1) * kBB;
			if (wp == oi) {
				if (!UPPER) {
					const float inv = 1.0f / tri[i * kLdT + i];
#pragma unroll
					for (int r = 0; r < 4; ++r) b[r][li] = inv * b[r][li];
				}
				*reinterpret_cast<float4 *>(pb + p0) = make_float4(b[0][li], b[1][li], b[2][li], b[3][li]);
			}
			__syncthreads();
			if (wp < oi) continue;
			const float4 b4 = *reinterpret_cast<const float4 *>(pb + p0);
			const float bi[4] = {b4.x, b4.y, b4.z, b4.w};
			const float4 *row = reinterpret_cast<const float4 *>(tri + i * kLdT + e0);
			const int cfirst = (wp > oi) ? 0 : li + 1;   // a later warp: all 16; the owner: after li
#pragma unroll
			for (int g = 0; g < 4; ++g) {
				if (wp == oi && 4 * g + 3 <= li) continue;
				const float4 m4 = row[g];
				const float mg[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
				for (int h = 0; h < 4; ++h) {
					const int c = 4 * g + h;
					if (c < cfirst) continue;
					if (UPPER) {
#pragma unroll
						for (int r = 0; r < 4; ++r)
							if (bi[r] != 0.0f) b[r][c] = fmaf(-bi[r], mg[h], b[r][c]);
					} else if (mg[h] != 0.0f) {
#pragma unroll
						for (int r = 0; r < 4; ++r) b[r][c] = fmaf(-mg[h], bi[r], b[r][c]);
					}
				}
			}
		}
	}
}

constexpr int kTrsmThreads = 256;
__global__ void __launch_bounds__(kTrsmThreads, 2) btrsm_kernel(const BSys *__restrict__ sys,
	const int4 *__restrict__ items, float *__restrict__ A, int64_t lda, __half *__restrict__ L16,
	__half *__restrict__ U16, int k)
{
	extern __shared__ __align__(16) float sm[];
	// side 0: tri[i * kLdT + j] = U(i, j) (rows of U); side 1: tri[i * kLdT + r] = L(r, i) (columns of L)
	float *tri = sm;
	float *pub = sm + kBB * kLdT;    // pub[2][128]: step i's final element of each panel row (column)
	const int4 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const bool upper = it.z != 0;
	const int64_t kb = static_cast<int64_t>(k) * kBB;
	const int64_t off = kb + kBB + static_cast<int64_t>(it.y) * kBB;   // first panel row / column
	const float *diag = A + kb + (S.C + kb) * lda;
	for (int e = threadIdx.x; e < kBB * kBB; e += kTrsmThreads) {
		const int r = e % kBB, c = e / kBB;   // diag(r, c)
		tri[upper ? c * kLdT + r : r * kLdT + c] = diag[r + static_cast<int64_t>(c) * lda];
	}
	const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
	const int p0 = 4 * lane, e0 = 16 * wp;   // panel rows (columns) p0..p0+3, elements e0..e0+15
	float b[4][16];
	// element e of panel row p: side 0 A(off + p, kb + e); side 1 A(kb + e, off + p)
#pragma unroll
	for (int r = 0; r < 4; ++r)
#pragma unroll
		for (int c = 0; c < 16; ++c)
			b[r][c] = upper ? A[kb + e0 + c + (S.C + off + p0 + r) * lda] : A[off + p0 + r + (S.C + kb + e0 + c) * lda];
	__syncthreads();
	if (upper) trsm_steps<true>(b, tri, pub, p0, e0, wp);
	else trsm_steps<false>(b, tri, pub, p0, e0, wp);
#pragma unroll
	for (int r = 0; r < 4; ++r) {
#pragma unroll
		for (int c = 0; c < 16; ++c) {
			if (upper) A[kb + e0 + c + (S.C + off + p0 + r) * lda] = b[r][c];
			else A[off + p0 + r + (S.C + kb + e0 + c) * lda] = b[r][c];
		}
		__half *o = (upper ? U16 : L16) + (S.R + off + p0 + r) * kBB + e0;
#pragma unroll
		for (int q = 0; q < 2; ++q) {
			uint4 w;
			uint32_t *wq = reinterpret_cast<uint32_t *>(&w);
#pragma unroll
			for (int h = 0; h < 4; ++h) {
				const __half2 h2 = __floats2half2_rn(b[r][8 * q + 2 * h], b[r][8 * q + 2 * h + 1]);
				wq[h] = *reinterpret_cast<const uint32_t *>(&h2);
			}
			*reinterpret_cast<uint4 *>(o + 8 * q) = w;
		}
	}
}

// ---------------------------------------------------------------------------
// Refinement.
// ---------------------------------------------------------------------------

// x = rhs ./ d (iterative_refinement.hpp:31-34); item = (system, first row)
__global__ void __launch_bounds__(128) bdiv_kernel(const BSys *__restrict__ sys, const int2 *__restrict__ items,
	const double *__restrict__ rhs, const double *__restrict__ d, double *__restrict__ x)
{
	const int2 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const int i = it.y + threadIdx.x;
	if (i >= S.n) return;
	for (int q = 0; q < S.nrhs; ++q) {
		const int64_t e = S.voff + static_cast<int64_t>(q) * S.n + i;
		x[e] = rhs[e] / d[S.doff + i];
	}
}

// Partial sums of A x over one column chunk for every right-hand side, A
// regenerated in FP64: sum of int64(state) * x_j over the off-diagonal
// columns times the generator scale, plus d_i x_i on the diagonal (the
// on-the-fly GEMV of otf_gemv.cpp:5-131 / panel_gemv.hpp:16-180).  item =
// (system, row block, column chunk).
__global__ void __launch_bounds__(kGemvRows) bgemv_kernel(const BSys *__restrict__ sys, const int4 *__restrict__ items,
	const double *__restrict__ x, const double *__restrict__ d, double *__restrict__ part, JumpT tab)
{
	__shared__ double xs[kMaxRhs][kGemvCols];
	const int4 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const int i = it.y + threadIdx.x, c = it.z;
	const int j0 = c * kGemvCols, j1 = min(j0 + kGemvCols, S.n);
	for (int q = 0; q < S.nrhs; ++q)
		for (int j = threadIdx.x; j < j1 - j0; j += kGemvRows) xs[q][j] = x[S.voff + static_cast<int64_t>(q) * S.n + j0 + j];
	__syncthreads();
	if (i >= S.n) return;
	const Coeff jn = jump(tab, static_cast<uint64_t>(S.n));
	uint64_t s = coeff_apply(jump(tab, static_cast<uint64_t>(i) + static_cast<uint64_t>(S.n) * j0), S.state0);
	double acc[kMaxRhs];
#pragma unroll
	for (int q = 0; q < kMaxRhs; ++q) acc[q] = 0.0;
	for (int j = 0; j < j1 - j0; ++j) {
		const double v = (j0 + j == i) ? 0.0 : __ll2double_rn(static_cast<long long>(s));
#pragma unroll
		for (int q = 0; q < kMaxRhs; ++q)
			if (q < S.nrhs) acc[q] = fma(v, xs[q][j], acc[q]);
		s = coeff_apply(jn, s);
	}
	const bool dg = i >= j0 && i < j1;
	for (int q = 0; q < S.nrhs; ++q) {
		double r = acc[q] * kValueScale;
		if (dg) r = fma(d[S.doff + i], xs[q][i - j0], r);
		part[S.poff + (static_cast<int64_t>(c) * S.nrhs + q) * S.n + i] = r;
	}
}

// r = rhs - (A x), the chunks folded in order; item = (system, first row).
__global__ void __launch_bounds__(128) bfold_kernel(const BSys *__restrict__ sys, const int2 *__restrict__ items,
	const double *__restrict__ part, const double *__restrict__ rhs, double *__restrict__ r)
{
	const int2 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const int i = it.y + threadIdx.x;
	if (i >= S.n) return;
	const int nch = (S.n + kGemvCols - 1) / kGemvCols;
	for (int q = 0; q < S.nrhs; ++q) {
		double sum = 0.0;
		for (int c = 0; c < nch; ++c) sum += part[S.poff + (static_cast<int64_t>(c) * S.nrhs + q) * S.n + i];
		const int64_t e = S.voff + static_cast<int64_t>(q) * S.n + i;
		r[e] = rhs[e] - sum;
	}
}

// Per (system, right-hand side) pair: the hpl-harness of this step
// (iterative_refinement.hpp:36-48); a pair below 16 is done, a non-finite
// one failed; pairs still refining are counted.  state: 0 refining, 1
// converged, 2 failed.
__global__ void __launch_bounds__(256) bnorm_kernel(const BSys *__restrict__ sys, const int2 *__restrict__ pairs,
	const double *__restrict__ rhs, const double *__restrict__ x, const double *__restrict__ r,
	const double *__restrict__ d, int *__restrict__ state, double *__restrict__ res, int *__restrict__ iters,
	int *__restrict__ active, int step)
{
	const int2 pq = pairs[blockIdx.x];
	const int p = blockIdx.x;
	if (state[p] != 0) return;
	const BSys S = sys[pq.x];
	const int64_t base = S.voff + static_cast<int64_t>(pq.y) * S.n;
	double mr = 0.0, mx = 0.0, mb = 0.0, md = 0.0;
	for (int i = threadIdx.x; i < S.n; i += 256) {
		const double rv = r[base + i];
		mr = (rv != rv) ? rv : fmax(mr, fabs(rv));   // a NaN residual propagates
		mx = fmax(mx, fabs(x[base + i]));
		mb = fmax(mb, fabs(rhs[base + i]));
		md = fmax(md, d[S.doff + i]);
	}
	__shared__ double sh[4][8];
	for (int o = 16; o; o >>= 1) {
		const double t = __shfl_xor_sync(0xffffffffu, mr, o);
		mr = (mr != mr) ? mr : ((t != t) ? t : fmax(mr, t));
		mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
		mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
		md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
	}
	if ((threadIdx.x & 31) == 0) {
		sh[0][threadIdx.x >> 5] = mr;
		sh[1][threadIdx.x >> 5] = mx;
		sh[2][threadIdx.x >> 5] = mb;
		sh[3][threadIdx.x >> 5] = md;
	}
	__syncthreads();
	if (threadIdx.x != 0) return;
	for (int w = 1; w < 8; ++w) {
		mr = (mr != mr) ? mr : ((sh[0][w] != sh[0][w]) ? sh[0][w] : fmax(mr, sh[0][w]));
		mx = fmax(mx, sh[1][w]);
		mb = fmax(mb, sh[2][w]);
		md = fmax(md, sh[3][w]);
	}
	const double norma = 2.0 * md;   // hpl_infnorm: the diagonal is the off-diagonal row 1-norm
	const double hpl = mr / fma(norma, mx, mb) * 1. / (S.n * 2.220446049250313e-16 / 2);
	iters[p] = step + 1;
	res[2 * p] = mr;
	res[2 * p + 1] = hpl;
	if (hpl < 16.) {
		state[p] = 1;
	} else if (!isfinite(hpl)) {
		state[p] = 2;
	} else {
		atomicAdd(active, 1);
	}
}

// r <- U^-1 L^-1 r for the refining (system, right-hand side) pairs, the
// FP32 factors applied to FP64 vectors (panel_trsvL / panel_trsvU,
// panel_trsv.hpp:310-758), 128 rows at a time: at step t of the L pass each
// system solves its diagonal block t (btrsv_diag_kernel) and then every
// 128-row chunk below it is updated in parallel with that block column
// (btrsv_off_kernel); the U pass does the same from each system's last block
// up.  The steps of one correction are a CUDA graph.
constexpr int kTrsvThreads = 256;   // 8 warps: one per right-hand side

__device__ __forceinline__ bool any_live(const BSys &S, const int *__restrict__ state)
{
	for (int q = 0; q < S.nrhs; ++q)
		if (state[S.pair0 + q] == 0) return true;
	return false;
}

// One CTA per system: its diagonal block (L pass: block t; U pass: block
// nbk-1-t) staged in shared memory and solved by one warp per right-hand
// side, the solved entry broadcast by shuffle (no block barrier inside).
__global__ void __launch_bounds__(kTrsvThreads) btrsv_diag_kernel(const BSys *__restrict__ sys,
	const float *__restrict__ A, int64_t lda, const int *__restrict__ state, double *__restrict__ r, int t, int up)
{
	extern __shared__ __align__(16) float blk[];   // blk[j * kLdS + i] = T(j0 + i, j0 + j)
	const BSys S = sys[blockIdx.x];
	const int n = S.n, nbk = (n + kBB - 1) / kBB;
	if (t >= nbk || !any_live(S, state)) return;
	const int jb = up ? nbk - 1 - t : t;
	const int j0 = jb * kBB, w = min(kBB, n - j0);
	const float *a = A + S.C * lda;
	for (int e = threadIdx.x; e < kBB * kBB; e += kTrsvThreads) {
		const int i = e % kBB, j = e / kBB;
		blk[j * kLdS + i] = (i < w && j < w) ? a[j0 + i + static_cast<int64_t>(j0 + j) * lda] : 0.f;
	}
	__syncthreads();
	const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (q >= S.nrhs || state[S.pair0 + q] != 0) return;
	double *rv = r + S.voff + static_cast<int64_t>(q) * n + j0;
	double v[4];
#pragma unroll
	for (int m = 0; m < 4; ++m) {
		const int i = lane + 32 * m;
		v[m] = i < w ? rv[i] : 0.0;
	}
	if (!up) {
		// unit lower: y_j final in order, then y_i -= L(i, j) y_j for i > j
		for (int j = 0; j < w; ++j) {
			double vj = 0.0;
#pragma unroll
			for (int m = 0; m < 4; ++m)
				if (m == (j >> 5)) vj = __shfl_sync(0xffffffffu, v[m], j & 31);
#pragma unroll
			for (int m = 0; m < 4; ++m) {
				const int i = lane + 32 * m;
				if (i > j && i < w) v[m] = fma(-static_cast<double>(blk[j * kLdS + i]), vj, v[m]);
			}
		}
	} else {
		// upper: y_j = v_j / U(j, j) from the last row up, then y_i -= U(i, j) y_j for i < j
		for (int j = w - 1; j >= 0; --j) {
#pragma unroll
			for (int m = 0; m < 4; ++m)
				if (m == (j >> 5) && lane == (j & 31)) v[m] = v[m] / static_cast<double>(blk[j * kLdS + j]);
			double vj = 0.0;
#pragma unroll
			for (int m = 0; m < 4; ++m)
				if (m == (j >> 5)) vj = __shfl_sync(0xffffffffu, v[m], j & 31);
#pragma unroll
			for (int m = 0; m < 4; ++m) {
				const int i = lane + 32 * m;
				if (i < j) v[m] = fma(-static_cast<double>(blk[j * kLdS + i]), vj, v[m]);
			}
		}
	}
#pragma unroll
	for (int m = 0; m < 4; ++m) {
		const int i = lane + 32 * m;
		if (i < w) rv[i] = v[m];
	}
}

// item = (system, chunk): 128 rows below (L pass) or above (U pass) the
// block solved at step t take its update, r_i -= sum_j T(i, j0 + j) y_j,
// one thread per row, every refining right-hand side at once.
__global__ void __launch_bounds__(kBB) btrsv_off_kernel(const BSys *__restrict__ sys, const int2 *__restrict__ items,
	const float *__restrict__ A, int64_t lda, const int *__restrict__ state, double *__restrict__ r, int t, int up)
{
	__shared__ double y[kMaxRhs][kBB];
	const int2 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const int n = S.n, nq = S.nrhs, nbk = (n + kBB - 1) / kBB;
	if (!any_live(S, state)) return;
	const int jb = up ? nbk - 1 - t : t;
	const int j0 = jb * kBB, w = min(kBB, n - j0);
	const int rbase = up ? it.y * kBB : j0 + kBB + it.y * kBB;
	double *rv = r + S.voff;
	for (int e = threadIdx.x; e < kMaxRhs * kBB; e += kBB) {
		const int q = e / kBB, j = e % kBB;
		y[q][j] = (q < nq && j < w) ? rv[static_cast<int64_t>(q) * n + j0 + j] : 0.0;
	}
	__syncthreads();
	const int i = rbase + threadIdx.x;
	if (i >= (up ? j0 : n)) return;
	const float *arow = A + i + (S.C + j0) * lda;
	double acc[kMaxRhs];
#pragma unroll
	for (int q = 0; q < kMaxRhs; ++q) acc[q] = 0.0;
	for (int j = 0; j < w; ++j) {
		const double l = arow[static_cast<int64_t>(j) * lda];
#pragma unroll
		for (int q = 0; q < kMaxRhs; ++q)
			if (q < nq) acc[q] = fma(l, y[q][j], acc[q]);
	}
	for (int q = 0; q < nq; ++q)
		if (state[S.pair0 + q] == 0) rv[static_cast<int64_t>(q) * n + i] -= acc[q];
}

// x += r for the pairs still refining; item = (system, first row)
__global__ void __launch_bounds__(128) bxupd_kernel(const BSys *__restrict__ sys, const int2 *__restrict__ items,
	const int *__restrict__ state, const double *__restrict__ r, double *__restrict__ x)
{
	const int2 it = items[blockIdx.x];
	const BSys S = sys[it.x];
	const int i = it.y + threadIdx.x;
	if (i >= S.n) return;
	for (int q = 0; q < S.nrhs; ++q) {
		if (state[S.pair0 + q] != 0) continue;
		const int64_t e = S.voff + static_cast<int64_t>(q) * S.n + i;
		x[e] += r[e];
	}
}

} // namespace

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
struct BatchEngine {
	int count = 0, pmax = 0, nsteps = 0, npairs = 0;
	int64_t rows = 0, cols = 0, lda = 0;
	std::vector<BSys> sys;                 // factorisation order
	std::vector<int> active;               // systems still factoring at step k (a prefix)
	std::vector<int> tile_off, tile_cnt;   // each step's slice of the tile table
	std::vector<int> trsm_off, trsm_cnt;   // each step's slice of the panel-chunk list
	std::vector<int> off_off, off_cnt;     // each refinement step's slice of the row-chunk list
	int2 *off_items = nullptr;
	cudaGraph_t cgraph = nullptr;          // one correction (both triangular solves and x += r)
	cudaGraphExec_t cexec = nullptr;

	int n_fill = 0, n_rows = 0, n_gemv = 0, max_chunks = 0;
	float *A = nullptr;
	__half *L16 = nullptr, *U16 = nullptr;
	double *d = nullptr, *rhs = nullptr, *x = nullptr, *r = nullptr, *part = nullptr, *res = nullptr;
	int4 *trsm_items = nullptr;
	int *state = nullptr, *iters = nullptr, *counter = nullptr, *host_counter = nullptr;
	BSys *dsys = nullptr;
	int2 *fill_items = nullptr, *row_items = nullptr, *pairs = nullptr;
	int4 *gemv_items = nullptr, *tiles = nullptr;
	SchurMaps maps;
	unsigned *status = nullptr;
	cudaStream_t st = nullptr;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	std::vector<double> h_res;
	std::vector<int> h_state, h_iters;
	unsigned long long launches_per_solve = 0, correction_launches = 0;
};

namespace {

void engine_free(BatchEngine *e)
{
	if (!e) return;
	if (e->exec) cudaGraphExecDestroy(e->exec);
	if (e->graph) cudaGraphDestroy(e->graph);
	if (e->cexec) cudaGraphExecDestroy(e->cexec);
	if (e->cgraph) cudaGraphDestroy(e->cgraph);
	cudaFree(e->off_items);
	cudaFree(e->A);
	cudaFree(e->L16);
	cudaFree(e->U16);
	cudaFree(e->d);
	cudaFree(e->rhs);
	cudaFree(e->x);
	cudaFree(e->r);
	cudaFree(e->part);
	cudaFree(e->res);
	cudaFree(e->state);
	cudaFree(e->iters);
	cudaFree(e->counter);
	cudaFree(e->dsys);
	cudaFree(e->fill_items);
	cudaFree(e->row_items);
	cudaFree(e->pairs);
	cudaFree(e->gemv_items);
	cudaFree(e->tiles);
	cudaFree(e->trsm_items);
	cudaFree(e->status);
	if (e->host_counter) cudaFreeHost(e->host_counter);
	if (e->st) cudaStreamDestroy(e->st);
	delete e;
}

template <typename T>
int upload(T **dst, const std::vector<T> &v)
{
	if (v.empty()) return HPLAI_OK;
	HPLAI_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(dst), sizeof(T) * v.size()));
	HPLAI_CUDA_TRY(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
	return HPLAI_OK;
}

constexpr size_t kGetrfSmem = sizeof(float) * kBB * kLdS;
constexpr size_t kTrsmSmem = sizeof(float) * (kBB * kLdT + 2 * kBB);
constexpr size_t kTrsvSmem = sizeof(float) * kBB * kLdS;

// Generation and factorisation of every system, in stream order.
int enqueue_factor(BatchEngine *e)
{
	static const JumpT tab = make_jump();
	cudaStream_t st = e->st;
	bfill_kernel<<<e->n_fill, 256, 0, st>>>(e->dsys, e->fill_items, e->A, e->lda, tab);
	bdiag_kernel<<<e->n_rows, 128, 0, st>>>(e->dsys, e->row_items, e->A, e->lda, e->d, tab);
	brhs_kernel<<<e->n_rows, 128, 0, st>>>(e->dsys, e->row_items, e->rhs, tab);
	HPLAI_CUDA_TRY(cudaGetLastError());
	unsigned long long launches = 3;
	for (int k = 0; k < e->nsteps; ++k) {
		const int m = e->active[k];
		if (m <= 0) break;
		bgetrf_kernel<<<m, 512, kGetrfSmem, st>>>(e->dsys, e->A, e->lda, k);
		HPLAI_CUDA_TRY(cudaGetLastError());
		++launches;
		if (e->trsm_cnt[k] <= 0) continue;
		btrsm_kernel<<<e->trsm_cnt[k], kTrsmThreads, kTrsmSmem, st>>>(e->dsys, e->trsm_items + e->trsm_off[k], e->A, e->lda,
			e->L16, e->U16, k);
		HPLAI_CUDA_TRY(cudaGetLastError());
		++launches;
		if (e->tile_cnt[k] > 0) {
			HPLAI_TRY(launch_schur_tiles(e->maps, e->tiles + e->tile_off[k], e->tile_cnt[k], 0, st));
			++launches;
		}
	}
	e->launches_per_solve = launches;
	return HPLAI_OK;
}

// One correction of every refining pair: U^-1 L^-1 r, then x += r.
int enqueue_correction(BatchEngine *e, unsigned long long *launches)
{
	cudaStream_t st = e->st;
	unsigned long long nl = 0;
	for (int up = 0; up < 2; ++up)
		for (int t = 0; t < e->nsteps; ++t) {
			const int m = e->active[t];
			if (m <= 0) break;
			btrsv_diag_kernel<<<m, kTrsvThreads, kTrsvSmem, st>>>(e->dsys, e->A, e->lda, e->state, e->r, t, up);
			HPLAI_CUDA_TRY(cudaGetLastError());
			++nl;
			if (e->off_cnt[t] > 0) {
				btrsv_off_kernel<<<e->off_cnt[t], kBB, 0, st>>>(e->dsys, e->off_items + e->off_off[t], e->A, e->lda,
					e->state, e->r, t, up);
				HPLAI_CUDA_TRY(cudaGetLastError());
				++nl;
			}
		}
	bxupd_kernel<<<e->n_rows, 128, 0, st>>>(e->dsys, e->row_items, e->state, e->r, e->x);
	HPLAI_CUDA_TRY(cudaGetLastError());
	*launches = nl + 1;
	return HPLAI_OK;
}

// Captures the work enqueue() puts on e->st into a graph.
template <typename F>
int capture(BatchEngine *e, cudaGraph_t *graph, cudaGraphExec_t *exec, F enqueue)
{
	if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return HPLAI_ECUDA;
	const int er = enqueue();
	cudaGraph_t g = nullptr;
	const cudaError_t ce = cudaStreamEndCapture(e->st, &g);
	(void)cudaGetLastError();
	if (er != HPLAI_OK || ce != cudaSuccess) {
		if (g) cudaGraphDestroy(g);
		return er != HPLAI_OK ? er : HPLAI_ECUDA;
	}
	*graph = g;
	return cudaGraphInstantiate(exec, g, 0) == cudaSuccess ? HPLAI_OK : HPLAI_ECUDA;
}

} // namespace

int batched_create(BatchEngine **out, int count, const int *n, const int *nrhs, const uint64_t *seeds)
{
	*out = nullptr;
	if (count <= 0) return HPLAI_EINVAL;
	for (int s = 0; s < count; ++s)
		if (n[s] < 1 || nrhs[s] < 1 || nrhs[s] > kMaxRhs) return HPLAI_EINVAL;
	BatchEngine *e = new BatchEngine;
	e->count = count;
	std::vector<int> order(count);
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return n[p] > n[q]; });
	int64_t rows = 0, cols = 0, voff = 0, doff = 0, poff = 0;
	int pair = 0;
	std::vector<int2> pairs;
	for (int s : order) {
		BSys S{};
		S.n = n[s];
		S.P = (n[s] + kBB - 1) / kBB * kBB;
		S.nrhs = nrhs[s];
		S.orig = s;
		S.R = rows;
		S.C = cols;
		S.voff = voff;
		S.doff = doff;
		S.poff = poff;
		S.pair0 = pair;
		S.state0 = state_initial(seeds[s]);
		rows += S.P;
		cols += S.P + kBB;
		voff += static_cast<int64_t>(S.n) * S.nrhs;
		doff += S.n;
		poff += static_cast<int64_t>((S.n + kGemvCols - 1) / kGemvCols) * S.nrhs * S.n;
		for (int q = 0; q < S.nrhs; ++q) pairs.push_back(make_int2(static_cast<int>(e->sys.size()), q));
		pair += S.nrhs;
		e->sys.push_back(S);
		e->pmax = std::max(e->pmax, S.P);
	}
	e->npairs = pair;
	e->rows = rows;
	e->cols = cols;
	e->lda = e->pmax;   // a multiple of 128 floats: 16-byte TMA strides
	e->nsteps = e->pmax / kBB;
	for (int k = 0; k < e->nsteps; ++k) {
		int m = 0;
		while (m < count && e->sys[m].P > k * kBB) ++m;
		e->active.push_back(m);
	}
	// work lists
	std::vector<int2> fill, rowi;
	std::vector<int4> gemv, tiles, trsm;
	for (int i = 0; i < count; ++i) {
		const BSys &S = e->sys[i];
		for (int c = 0; c < S.P; c += 32) fill.push_back(make_int2(i, c));
		for (int r = 0; r < S.n; r += 128) rowi.push_back(make_int2(i, r));
		for (int r = 0; r < S.n; r += kGemvRows)
			for (int c = 0; c * kGemvCols < S.n; ++c) gemv.push_back(make_int4(i, r, c, 0));
	}
	// refinement step t: the 128-row chunks off the diagonal block (below it
	// in the L pass, above it in the U pass: nbk - 1 - t either way)
	std::vector<int2> offi;
	for (int t = 0; t < e->nsteps; ++t) {
		e->off_off.push_back(static_cast<int>(offi.size()));
		for (int i = 0; i < e->active[t]; ++i) {
			const int nbk = e->sys[i].P / kBB;
			for (int c = 0; c < nbk - 1 - t; ++c) offi.push_back(make_int2(i, c));
		}
		e->off_cnt.push_back(static_cast<int>(offi.size()) - e->off_off.back());
	}
	// panel chunks of step k: 128 rows of L and 128 columns of U at a time
	for (int k = 0; k < e->nsteps; ++k) {
		e->trsm_off.push_back(static_cast<int>(trsm.size()));
		for (int i = 0; i < e->active[k]; ++i) {
			const int nch = e->sys[i].P / kBB - k - 1;
			for (int c = 0; c < nch; ++c)
				for (int side = 0; side < 2; ++side) trsm.push_back(make_int4(i, c, side, 0));
		}
		e->trsm_cnt.push_back(static_cast<int>(trsm.size()) - e->trsm_off.back());
	}
	// tiles of step k: the trailing rows and columns from (k + 1) * 128 of every
	// system still factoring, 128-row x 256-column tiles
	for (int k = 0; k < e->nsteps; ++k) {
		e->tile_off.push_back(static_cast<int>(tiles.size()));
		for (int i = 0; i < e->active[k]; ++i) {
			const BSys &S = e->sys[i];
			const int t0 = (k + 1) * kBB;
			for (int c = t0; c < S.P; c += 256)
				for (int rr = t0; rr < S.P; rr += kBB)
					tiles.push_back(make_int4(static_cast<int>(S.R + rr), static_cast<int>(S.R + c), rr,
						static_cast<int>(S.C + c)));
		}
		e->tile_cnt.push_back(static_cast<int>(tiles.size()) - e->tile_off.back());
	}
	e->n_fill = static_cast<int>(fill.size());
	e->n_rows = static_cast<int>(rowi.size());
	e->n_gemv = static_cast<int>(gemv.size());

	int rc = HPLAI_OK;
	auto alloc = [&](void **p, size_t bytes) {
		if (rc == HPLAI_OK && cudaMalloc(p, bytes) != cudaSuccess) {
			(void)cudaGetLastError();
			rc = HPLAI_ENOMEM;
		}
	};
	if (rows > (int64_t(1) << 31) - 1 || cols > (int64_t(1) << 31) - 1) rc = HPLAI_EUNSUPPORTED;   // int tile coordinates
	alloc(reinterpret_cast<void **>(&e->A), sizeof(float) * static_cast<size_t>(e->lda) * e->cols);
	alloc(reinterpret_cast<void **>(&e->L16), sizeof(__half) * static_cast<size_t>(rows) * kBB);
	alloc(reinterpret_cast<void **>(&e->U16), sizeof(__half) * static_cast<size_t>(rows) * kBB);
	alloc(reinterpret_cast<void **>(&e->d), sizeof(double) * static_cast<size_t>(doff));
	alloc(reinterpret_cast<void **>(&e->rhs), sizeof(double) * static_cast<size_t>(voff));
	alloc(reinterpret_cast<void **>(&e->x), sizeof(double) * static_cast<size_t>(voff));
	alloc(reinterpret_cast<void **>(&e->r), sizeof(double) * static_cast<size_t>(voff));
	alloc(reinterpret_cast<void **>(&e->part), sizeof(double) * static_cast<size_t>(poff));

	alloc(reinterpret_cast<void **>(&e->res), sizeof(double) * 2 * pair);
	alloc(reinterpret_cast<void **>(&e->state), sizeof(int) * pair);
	alloc(reinterpret_cast<void **>(&e->iters), sizeof(int) * pair);
	alloc(reinterpret_cast<void **>(&e->counter), sizeof(int));
	alloc(reinterpret_cast<void **>(&e->status), sizeof(unsigned));
	if (rc == HPLAI_OK && (upload(&e->dsys, e->sys) != HPLAI_OK || upload(&e->fill_items, fill) != HPLAI_OK ||
		upload(&e->row_items, rowi) != HPLAI_OK || upload(&e->pairs, pairs) != HPLAI_OK ||
		upload(&e->gemv_items, gemv) != HPLAI_OK || upload(&e->tiles, tiles) != HPLAI_OK ||
		upload(&e->trsm_items, trsm) != HPLAI_OK || upload(&e->off_items, offi) != HPLAI_OK))
		rc = HPLAI_ECUDA;
	if (rc == HPLAI_OK && cudaHostAlloc(reinterpret_cast<void **>(&e->host_counter), sizeof(int), 0) != cudaSuccess)
		rc = HPLAI_ENOMEM;
	if (rc == HPLAI_OK && cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) rc = HPLAI_ECUDA;
	if (rc == HPLAI_OK && (cudaFuncSetAttribute(bgetrf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(kGetrfSmem)) != cudaSuccess || cudaFuncSetAttribute(btrsm_kernel,
		cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kTrsmSmem)) != cudaSuccess ||
		cudaFuncSetAttribute(btrsv_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(kTrsvSmem)) != cudaSuccess))
		rc = HPLAI_ECUDA;
	if (rc == HPLAI_OK && cudaMemset(e->status, 0, sizeof(unsigned)) != cudaSuccess) rc = HPLAI_ECUDA;
	if (rc == HPLAI_OK) rc = schur_make_maps(&e->maps, reinterpret_cast<const uint16_t *>(e->L16),
		static_cast<int>(rows), kBB, reinterpret_cast<const uint16_t *>(e->U16), static_cast<int>(rows), kBB, kBB);
	if (rc == HPLAI_OK) rc = schur_set_cmap(&e->maps, e->A, e->pmax, static_cast<int>(e->cols), e->lda);
	if (rc == HPLAI_OK && !e->maps.has_cmap) rc = HPLAI_EINVAL;
	e->maps.status = e->status;
	// the generation and the factorisation as one graph, replayed per solve,
	// and one correction as another, replayed per refinement step
	if (rc == HPLAI_OK) rc = capture(e, &e->graph, &e->exec, [&] { return enqueue_factor(e); });
	unsigned long long cl = 0;
	if (rc == HPLAI_OK) rc = capture(e, &e->cgraph, &e->cexec, [&] { return enqueue_correction(e, &cl); });
	e->correction_launches = cl;
	if (rc != HPLAI_OK) {
		engine_free(e);
		return rc;
	}
	e->h_res.assign(2 * pair, -1.0);
	e->h_state.assign(pair, 0);
	e->h_iters.assign(pair, 0);
	*out = e;
	return HPLAI_OK;
}

void batched_destroy(BatchEngine *e) { engine_free(e); }

int batched_solve(BatchEngine *e, int maxit, unsigned long long *launches)
{
	static const JumpT tab = make_jump();
	cudaStream_t st = e->st;
	HPLAI_CUDA_TRY(cudaGraphLaunch(e->exec, st));
	unsigned long long nl = e->launches_per_solve;
	HPLAI_CUDA_TRY(cudaMemsetAsync(e->state, 0, sizeof(int) * e->npairs, st));
	HPLAI_CUDA_TRY(cudaMemsetAsync(e->iters, 0, sizeof(int) * e->npairs, st));
	bdiv_kernel<<<e->n_rows, 128, 0, st>>>(e->dsys, e->row_items, e->rhs, e->d, e->x);
	HPLAI_CUDA_TRY(cudaGetLastError());
	++nl;
	for (int it = 0; it < maxit; ++it) {
		HPLAI_CUDA_TRY(cudaMemsetAsync(e->counter, 0, sizeof(int), st));
		bgemv_kernel<<<e->n_gemv, kGemvRows, 0, st>>>(e->dsys, e->gemv_items, e->x, e->d, e->part, tab);
		bfold_kernel<<<e->n_rows, 128, 0, st>>>(e->dsys, e->row_items, e->part, e->rhs, e->r);
		bnorm_kernel<<<e->npairs, 256, 0, st>>>(e->dsys, e->pairs, e->rhs, e->x, e->r, e->d, e->state, e->res,
			e->iters, e->counter, it);
		HPLAI_CUDA_TRY(cudaGetLastError());
		nl += 3;
		HPLAI_CUDA_TRY(cudaMemcpyAsync(e->host_counter, e->counter, sizeof(int), cudaMemcpyDeviceToHost, st));
		HPLAI_CUDA_TRY(cudaStreamSynchronize(st));
		if (*e->host_counter == 0) break;
		HPLAI_CUDA_TRY(cudaGraphLaunch(e->cexec, st));
		nl += e->correction_launches;
	}
	HPLAI_CUDA_TRY(cudaMemcpyAsync(e->h_res.data(), e->res, sizeof(double) * 2 * e->npairs, cudaMemcpyDeviceToHost,
		st));
	HPLAI_CUDA_TRY(cudaMemcpyAsync(e->h_state.data(), e->state, sizeof(int) * e->npairs, cudaMemcpyDeviceToHost, st));
	HPLAI_CUDA_TRY(cudaMemcpyAsync(e->h_iters.data(), e->iters, sizeof(int) * e->npairs, cudaMemcpyDeviceToHost, st));
	unsigned ks = 0;
	HPLAI_CUDA_TRY(cudaMemcpyAsync(&ks, e->status, sizeof ks, cudaMemcpyDeviceToHost, st));
	HPLAI_CUDA_TRY(cudaStreamSynchronize(st));
	count_launches(static_cast<int>(nl));
	if (launches) *launches = nl;
	if (ks) return HPLAI_ETIMEOUT;
	int rc = HPLAI_OK;
	for (int p = 0; p < e->npairs; ++p)
		if (e->h_state[p] != 1) rc = HPLAI_ENOTCONV;
	return rc;
}

// System `orig` (the caller's index): the worst pair's {residual, harness},
// the most refinement steps, its status.
int batched_result(BatchEngine *e, int orig, hplai_ir_errors *worst, int *iters, int *status)
{
	for (const BSys &S : e->sys) {
		if (S.orig != orig) continue;
		hplai_ir_errors w{0.0, 0.0};
		int itmax = 0, st = HPLAI_OK;
		for (int q = 0; q < S.nrhs; ++q) {
			const int p = S.pair0 + q;
			itmax = std::max(itmax, e->h_iters[p]);
			if (e->h_state[p] != 1) {
				st = HPLAI_ENOTCONV;
				w = hplai_ir_errors{-1.0, -1.0};
			} else if (st == HPLAI_OK && e->h_res[2 * p + 1] > w.hpl_harness) {
				w = hplai_ir_errors{e->h_res[2 * p], e->h_res[2 * p + 1]};
			}
		}
		if (worst) *worst = w;
		if (iters) *iters = itmax;
		if (status) *status = st;
		return HPLAI_OK;
	}
	return HPLAI_EINVAL;
}

int batched_get_x(BatchEngine *e, int orig, double *x, int64_t ldx)
{
	for (const BSys &S : e->sys) {
		if (S.orig != orig) continue;
		if (ldx < S.n) return HPLAI_EINVAL;
		HPLAI_CUDA_TRY(cudaMemcpy2D(x, sizeof(double) * ldx, e->x + S.voff, sizeof(double) * S.n,
			sizeof(double) * S.n, S.nrhs, cudaMemcpyDeviceToHost));
		return HPLAI_OK;
	}
	return HPLAI_EINVAL;
}

// The factors of system `orig` (n x n, FP32, column-major with lda >= n).
int batched_get_lu(BatchEngine *e, int orig, float *a, int64_t lda)
{
	for (const BSys &S : e->sys) {
		if (S.orig != orig) continue;
		if (lda < S.n) return HPLAI_EINVAL;
		HPLAI_CUDA_TRY(cudaMemcpy2D(a, sizeof(float) * lda, e->A + S.C * e->lda, sizeof(float) * e->lda, sizeof(float) * S.n,
			S.n, cudaMemcpyDeviceToHost));
		return HPLAI_OK;
	}
	return HPLAI_EINVAL;
}

int batched_pad(BatchEngine *e, int orig)
{
	for (const BSys &S : e->sys)
		if (S.orig == orig) return S.P;
	return -1;
}

unsigned long long batched_launches(const BatchEngine *e) { return e->launches_per_solve; }

} // namespace hplai
