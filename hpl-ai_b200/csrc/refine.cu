// refine.cu -- FP64 kernels of the iterative refinement.
//
//  otf_gemv        y <- beta*y + alpha*A x with A regenerated from the LCG in
//                  FP64 (panel_gemv.hpp:57-180, otf_gemv.cpp:5-131); the
//                  diagonal comes from the FP64 diagonal vector.
//  trsv            x <- L^{-1} x or U^{-1} x with the FP32 LU factors and an
//                  FP64 vector (panel_trsv.hpp:310-758), one persistent
//                  cooperative launch with block-row flags.
//  infnorm, div, axpy   the vector helpers of panel_norm.hpp / panel.hpp.
#include "common.cuh"
#include "internal.h"

#include <mutex>

namespace hplai {

namespace {

struct JumpTable64 {
	Coeff p[64];
};

JumpTable64 make_table()
{
	JumpTable64 t;
	Coeff p{kLcgA, kLcgC};
	for (int k = 0; k < 64; ++k) {
		t.p[k] = p;
		p = coeff_mul(p, p);
	}
	return t;
}

const JumpTable64 &table()
{
	static const JumpTable64 t = make_table();
	return t;
}

__device__ __forceinline__ Coeff jump_of(const JumpTable64 &t, uint64_t m)
{
	Coeff r{1ULL, 0ULL};
	for (int k = 0; m; ++k, m >>= 1)
		if (m & 1ULL) r = coeff_mul(r, t.p[k]);
	return r;
}

// ---------------------------------------------------------------------------
// On-the-fly GEMV.  CTA = 256 rows x GEMV_COLS columns; each thread walks
// its row across the column chunk with four interleaved LCG chains
// (state jumps by n per column) and two FP64 accumulators.  Partial sums
// go to the workspace and a second kernel folds them in a fixed order, so
// the result does not depend on scheduling.
// ---------------------------------------------------------------------------
constexpr int GEMV_ROWS = 256;
constexpr int GEMV_COLS = 2048;

// TRANS: y = A^T x, output i walks column i of A (element (j, i) is state
// j + n*i, so the chain steps by 1 instead of n).
template <bool TRANS>
__global__ void __launch_bounds__(GEMV_ROWS) otf_partial_kernel(int64_t n, int mb, int nb, double alpha,
	const double *__restrict__ x, uint64_t state00, int with_diag, const double *__restrict__ diag,
	double *__restrict__ part, JumpTable64 tab)
{
	__shared__ __align__(16) double xs[GEMV_COLS];
	const int j0 = blockIdx.y * GEMV_COLS;
	const int j1 = min(j0 + GEMV_COLS, nb);
	for (int j = threadIdx.x; j < j1 - j0; j += GEMV_ROWS) xs[j] = x[j0 + j];
	__syncthreads();
	const int i = blockIdx.x * GEMV_ROWS + threadIdx.x;
	if (i >= mb) return;
	const Coeff jn = jump_of(tab, TRANS ? 1ULL : static_cast<uint64_t>(n));
	const Coeff jn4 = coeff_mul(coeff_mul(jn, jn), coeff_mul(jn, jn));
	const uint64_t idx0 = TRANS ? static_cast<uint64_t>(j0) + static_cast<uint64_t>(n) * static_cast<uint64_t>(i)
	                            : static_cast<uint64_t>(i) + static_cast<uint64_t>(n) * j0;
	uint64_t s0 = coeff_apply(jump_of(tab, idx0), state00);
	uint64_t s1 = coeff_apply(jn, s0);
	uint64_t s2 = coeff_apply(jn, s1);
	uint64_t s3 = coeff_apply(jn, s2);
	double a0 = 0.0, a1 = 0.0;
	const int len = j1 - j0;
	const int dj = (with_diag && i >= j0 && i < j1) ? i - j0 : -1;   // diagonal column inside the chunk
	int j = 0;
	if (dj < 0) {
		// no diagonal in this chunk (every CTA but those on the diagonal):
		// the same sums without the per-group test, x read two at a time
		for (; j + 3 < len; j += 4) {
			const double2 x01 = *reinterpret_cast<const double2 *>(&xs[j]);
			const double2 x23 = *reinterpret_cast<const double2 *>(&xs[j + 2]);
			a0 = fma(__ll2double_rn(static_cast<long long>(s0)), x01.x, a0);
			a1 = fma(__ll2double_rn(static_cast<long long>(s1)), x01.y, a1);
			a0 = fma(__ll2double_rn(static_cast<long long>(s2)), x23.x, a0);
			a1 = fma(__ll2double_rn(static_cast<long long>(s3)), x23.y, a1);
			s0 = coeff_apply(jn4, s0);
			s1 = coeff_apply(jn4, s1);
			s2 = coeff_apply(jn4, s2);
			s3 = coeff_apply(jn4, s3);
		}
	} else {
		for (; j + 3 < len; j += 4) {
			double v0 = __ll2double_rn(static_cast<long long>(s0));
			double v1 = __ll2double_rn(static_cast<long long>(s1));
			double v2 = __ll2double_rn(static_cast<long long>(s2));
			double v3 = __ll2double_rn(static_cast<long long>(s3));
			if (dj >= j && dj < j + 4) {
				if (dj == j) v0 = 0.0;
				if (dj == j + 1) v1 = 0.0;
				if (dj == j + 2) v2 = 0.0;
				if (dj == j + 3) v3 = 0.0;
			}
			a0 = fma(v0, xs[j], a0);
			a1 = fma(v1, xs[j + 1], a1);
			a0 = fma(v2, xs[j + 2], a0);
			a1 = fma(v3, xs[j + 3], a1);
			s0 = coeff_apply(jn4, s0);
			s1 = coeff_apply(jn4, s1);
			s2 = coeff_apply(jn4, s2);
			s3 = coeff_apply(jn4, s3);
		}
	}
	for (; j < len; ++j) {
		const double v = (j == dj) ? 0.0 : __ll2double_rn(static_cast<long long>(s0));
		a0 = fma(v, xs[j], a0);
		s0 = coeff_apply(jn, s0);
	}
	double r = (a0 + a1) * (alpha * kValueScale);
	if (dj >= 0) r = fma(alpha * diag[i], xs[dj], r);
	part[static_cast<int64_t>(blockIdx.y) * mb + i] = r;
}

__global__ void otf_reduce_kernel(int mb, int nchunks, double beta, const double *__restrict__ part, double *y,
	int overwrite)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= mb) return;
	double s = 0.0;
	for (int c = 0; c < nchunks; ++c) s += part[static_cast<int64_t>(c) * mb + i];
	y[i] = overwrite ? s : fma(beta, y[i], s);
}

int otf_launch(int64_t n, int mb, int nb, double alpha, const double *x, double beta, double *y,
	uint64_t state00, int with_diag, const double *diag, void *work, size_t work_bytes, cudaStream_t st,
	bool trans = false)
{
	if (mb <= 0) return HPLAI_OK;
	const int nchunks = (nb + GEMV_COLS - 1) / GEMV_COLS;
	if (work_bytes < static_cast<size_t>(nchunks) * mb * sizeof(double)) return HPLAI_EINVAL;
	double *part = static_cast<double *>(work);
	if (nb > 0) {
		dim3 grid((mb + GEMV_ROWS - 1) / GEMV_ROWS, nchunks);
		if (trans)
			otf_partial_kernel<true><<<grid, GEMV_ROWS, 0, st>>>(n, mb, nb, alpha, x, state00, with_diag, diag, part,
				table());
		else
			otf_partial_kernel<false><<<grid, GEMV_ROWS, 0, st>>>(n, mb, nb, alpha, x, state00, with_diag, diag, part,
				table());
		count_launches();
		HPLAI_CUDA_TRY(cudaGetLastError());
	}
	otf_reduce_kernel<<<(mb + 255) / 256, 256, 0, st>>>(mb, nb > 0 ? nchunks : 0, beta, part, y,
		beta == 0.0 ? 1 : 0);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

// ---------------------------------------------------------------------------
// On-the-fly GEMV over Higham's HPL-AI matrix (hmg_gemv_up/low/diag,
// otf_gemv.cpp:133-314): the entries of row i are the lower constants
// fma(ab, j, cl) of the columns j < i, the diagonal d_i and the upper
// constant fma(ab, i, cu) of the row; A^T swaps the two constants.  Same
// CTA shape, accumulators and fixed-order fold as the LCG GEMV.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(GEMV_ROWS) higham_partial_kernel(int n, double alpha, const double *__restrict__ x,
	double ab, double cu, double cl, const double *__restrict__ diag, double *__restrict__ part)
{
	__shared__ double xs[GEMV_COLS];
	__shared__ double ls[GEMV_COLS];
	const int j0 = blockIdx.y * GEMV_COLS;
	const int j1 = min(j0 + GEMV_COLS, n);
	for (int j = threadIdx.x; j < j1 - j0; j += GEMV_ROWS) {
		xs[j] = x[j0 + j];
		ls[j] = fma(ab, static_cast<double>(j0 + j), cl);
	}
	__syncthreads();
	const int i = blockIdx.x * GEMV_ROWS + threadIdx.x;
	if (i >= n) return;
	const double up = fma(ab, static_cast<double>(i), cu);
	const int len = j1 - j0;
	double a0 = 0.0, a1 = 0.0;
	int j = 0;
	for (; j + 1 < len; j += 2) {
		const int g = j0 + j;
		const double v0 = g < i ? ls[j] : (g > i ? up : 0.0);
		const double v1 = g + 1 < i ? ls[j + 1] : (g + 1 > i ? up : 0.0);
		a0 = fma(v0, xs[j], a0);
		a1 = fma(v1, xs[j + 1], a1);
	}
	if (j < len) {
		const int g = j0 + j;
		a0 = fma(g < i ? ls[j] : (g > i ? up : 0.0), xs[j], a0);
	}
	double r = (a0 + a1) * alpha;
	if (i >= j0 && i < j1) r = fma(alpha * diag[i], xs[i - j0], r);
	part[static_cast<int64_t>(blockIdx.y) * n + i] = r;
}

// ---------------------------------------------------------------------------
// Triangular solves.  Block rows of TB; CTA c handles block rows c, c+G, ...
// in solve order, accumulating the off-diagonal products as the block
// columns it depends on are published (flag[cb] == epoch), then solving its
// diagonal block with warp shuffles and publishing x for that block.
// Progress is guaranteed because every CTA is resident (cooperative launch)
// and each works through its rows in dependency order.  Every spin is
// bounded; a timeout sets the status word and the kernel returns.
// ---------------------------------------------------------------------------
constexpr int TB = 128;
constexpr int TRSV_THREADS = 256;

struct TrsvWork {
	uint32_t epoch;
	uint32_t status;
	uint32_t pad[2];
	// followed by flags[nbt]
};

__global__ void trsv_epoch_kernel(TrsvWork *w)
{
	w->epoch += 1;
	w->status = 0;
}

// FP64 inverses of the TB x TB diagonal blocks of the stored factors:
// dinv[(2*r + 0) * TB*TB + c*TB + i] = (L_rr^{-1})[i][c] (unit lower) and
// dinv[(2*r + 1) * TB*TB + c*TB + i] = (U_rr^{-1})[i][c], rows/columns past
// n padded with the identity.  Thread c solves T x = e_c by substitution in
// FP64 (the FP32 factor entries convert exactly).  Computed once per
// factorisation; the triangular solves then apply a block as one product.
__global__ void __launch_bounds__(TB) trsv_dinv_kernel(int n, const float *__restrict__ a, int64_t lda,
	double *__restrict__ dinv, int blk0)
{
	extern __shared__ __align__(16) float dyn_smem[];
	float (*tb)[TB + 1] = reinterpret_cast<float (*)[TB + 1]>(dyn_smem);                 // tb[i][j] = A[r0+i][r0+j]
	double *xc = reinterpret_cast<double *>(dyn_smem + TB * (TB + 1) + 1);             // xc[i * TB + c], 8-aligned
	xc = reinterpret_cast<double *>((reinterpret_cast<uintptr_t>(xc) + 7) & ~static_cast<uintptr_t>(7));
	const int r = blk0 + blockIdx.x, upper = blockIdx.y;
	const int r0 = r * TB, rows = min(TB, n - r0);
	const int c = threadIdx.x;
	for (int e = c; e < TB * TB; e += TB) {
		const int i = e % TB, j = e / TB;
		tb[i][j] = (i < rows && j < rows) ? a[static_cast<int64_t>(r0 + j) * lda + r0 + i] : (i == j ? 1.f : 0.f);
	}
	__syncthreads();
	if (!upper) {
		for (int i = 0; i < TB; ++i) {
			double v = (i == c) ? 1.0 : 0.0;
			if (i > c)
				for (int j = c; j < i; ++j) v = fma(-static_cast<double>(tb[i][j]), xc[j * TB + c], v);
			xc[i * TB + c] = v;
		}
	} else {
		for (int i = TB - 1; i >= 0; --i) {
			double v = (i == c) ? 1.0 : 0.0;
			if (i < c)
				for (int j = i + 1; j <= c; ++j) v = fma(-static_cast<double>(tb[i][j]), xc[j * TB + c], v);
			xc[i * TB + c] = (i <= c) ? v / static_cast<double>(tb[i][i]) : 0.0;
		}
	}
	double *out = dinv + (static_cast<int64_t>(2 * r + upper) * TB) * TB;
	for (int i = 0; i < TB; ++i) out[static_cast<int64_t>(c) * TB + i] = xc[i * TB + c];
}

// Copy block (rows r0.., cols c0..) of M into shared memory with cp.async:
// TRANS (M[i][j] = a[i*lda + j]) as blk[i*TB + j], otherwise
// (M[i][j] = a[j*lda + i]) as blk[j*TB + i]; rows >= rows / cols >= cols
// are zero.  vec: 16-byte copies through L2 (a 16-byte aligned, lda % 4 == 0),
// else 4-byte copies.  The matrix is read-only for the whole solve.
template <bool TRANS>
__device__ __forceinline__ void stage_block(float *blk, const float *a, int64_t lda, int r0, int c0, int rows,
	int cols, bool vec, const double *xsrc = nullptr, double *xdst = nullptr)
{
	const int t = threadIdx.x;
	// x of the block column in the same copy group (its values are published)
	if (xsrc && t < TB / 2) {
		int bytes = (cols - 2 * t) * 8;
		bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
		asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(xdst + 2 * t)),
			"l"(xsrc + (bytes ? 2 * t : 0)), "r"(bytes) : "memory");
	}
	// contiguous index of the stored matrix: rows for M = stored, columns for M^T
	const int ncont = TRANS ? cols : rows, nline = TRANS ? rows : cols;
	if (vec) {
		for (int e = t; e < TB * TB / 4; e += TRSV_THREADS) {
			const int line = e / (TB / 4), g = (e % (TB / 4)) * 4;
			int bytes = (line < nline) ? (ncont - g) * 4 : 0;
			bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
			const float *src = TRANS ? a + static_cast<int64_t>(r0 + (bytes ? line : 0)) * lda + c0 + (bytes ? g : 0)
			                         : a + static_cast<int64_t>(c0 + (bytes ? line : 0)) * lda + r0 + (bytes ? g : 0);
			asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(blk + line * TB + g)),
				"l"(src), "r"(bytes) : "memory");
		}
	} else {
		for (int e = t; e < TB * TB; e += TRSV_THREADS) {
			const int line = e / TB, g = e % TB;
			const bool in = line < nline && g < ncont;
			const float *src = TRANS ? a + static_cast<int64_t>(r0 + (in ? line : 0)) * lda + c0 + (in ? g : 0)
			                         : a + static_cast<int64_t>(c0 + (in ? line : 0)) * lda + r0 + (in ? g : 0);
			asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(blk + line * TB + g)), "l"(src),
				"r"(in ? 4 : 0) : "memory");
		}
	}
	asm volatile("cp.async.commit_group;" ::: "memory");
}

// TRANS: the triangle solved is the transpose of the stored one, M[i][j] =
// a[i*lda + j]: lower = U^T (non-unit), upper = L^T (unit).  Otherwise
// M[i][j] = a[j*lda + i]: lower = L (unit), upper = U (non-unit).
// The off-diagonal blocks of a block row stream through two shared-memory
// buffers: block q+1 is being copied while block q waits for its x and is
// applied, so the latency of the factor reads leaves the dependency chain.
// With dinv (the FP64 inverses of the diagonal blocks, trsv_dinv_kernel) a
// diagonal block is applied as one product instead of 128 dependent
// substitution steps.
template <bool TRANS>
__global__ void __launch_bounds__(TRSV_THREADS, 1) trsv_kernel(int lower, int n, const float *__restrict__ a,
	int64_t lda, double *x, TrsvWork *w, const double *__restrict__ dinv)
{
	extern __shared__ __align__(16) float dyn_smem[];
	float (*dblk)[TB + 1] = reinterpret_cast<float (*)[TB + 1]>(dyn_smem);   // dblk[i][j] = M[r0+i][r0+j]
	float *bufs = dyn_smem + TB * (TB + 1) + 3;   // two TB x TB blocks, 16-byte aligned
	bufs = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(bufs) + 15) & ~static_cast<uintptr_t>(15));
	// With the diagonal inverses the staged diagonal block is not needed and
	// its space becomes a third block buffer: two blocks in flight while one
	// is applied.
	const int NB = dinv ? 3 : 2;
	float *const bufp[3] = {bufs, bufs + TB * TB, dyn_smem};
	const bool unit = TRANS ? !lower : lower;
	const bool vec = ((reinterpret_cast<uintptr_t>(a) & 15u) == 0) && ((lda & 3) == 0);
	const bool xvec = (reinterpret_cast<uintptr_t>(x) & 15u) == 0;   // x copies of 16 bytes
	__shared__ __align__(16) double xsb[3][TB];   // x of the staged block columns, one per block buffer
	__shared__ double part[2][TB];       // partial sums of the two column halves
	__shared__ double rhs[TB];
	__shared__ int ready_upto;
	__shared__ int abort_flag;

	uint32_t *flags = reinterpret_cast<uint32_t *>(w + 1);
	const uint32_t epoch = *reinterpret_cast<volatile uint32_t *>(&w->epoch);
	const int nbt = (n + TB - 1) / TB;
	const int t = threadIdx.x;
	const int lr = t % TB, grp = t / TB;   // row within the block, column half

	// the published prefix seen so far: flags only advance during a launch,
	// so it carries over from one block row of this CTA to its next
	if (t == 0) {
		abort_flag = 0;
		ready_upto = lower ? 0 : nbt - 1;
	}
	__syncthreads();
	for (int idx = blockIdx.x; idx < nbt; idx += gridDim.x) {
		const int r = lower ? idx : nbt - 1 - idx;
		const int r0 = r * TB;
		const int rows = min(TB, n - r0);
		const int nblk = lower ? r : nbt - 1 - r;
		// the first NB - 1 off-diagonal blocks in flight before anything waits;
		// one copy group per block (empty past the last) keeps the count fixed
		// With the block goes its x when the block column is already known to
		// be solved (the published prefix warp 0 has seen; the same for every
		// thread between two barriers), so that applying it waits on nothing
		// but its copy group.
		bool xpre[3] = {false, false, false};
		auto stage_q = [&](int q) {
			if (q < nblk) {
				const int cb = lower ? q : nbt - 1 - q;
				const bool known = xvec && (lower ? (cb < ready_upto) : (cb > ready_upto));
				xpre[q % NB] = known;
				stage_block<TRANS>(bufp[q % NB], a, lda, r0, cb * TB, rows, min(TB, n - cb * TB), vec,
					known ? x + static_cast<int64_t>(cb) * TB : nullptr, xsb[q % NB]);
			} else {
				asm volatile("cp.async.commit_group;" ::: "memory");
			}
		};
		// the diagonal block's inverse (M^{-1} = T^{-1} or its transpose) into L2
		const double *dblock = nullptr;
		if (dinv) {
			const int tri = (lower != 0) == !TRANS ? 0 : 1;   // L for lower / L^T, U for upper / U^T
			dblock = dinv + (static_cast<int64_t>(2 * r + tri) * TB) * TB;
			if (t < 8)
				asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(dblock + t * (TB * TB / 8)),
					"r"(static_cast<unsigned>(sizeof(double) * TB * TB / 8)) : "memory");
		}
		// Not transposed: this thread's 64 entries of the inverse go to registers
		// now, while the block row is summed, so that the diagonal step (the
		// chain's critical path) does not wait on L2.
		// this block's right-hand side (only this CTA writes it, at the end)
		const double xr = (t < rows) ? __ldcg(&x[r0 + t]) : 0.0;
		double dv[TB / 2];
		if (!TRANS && dinv) {
			const int jb = grp * (TB / 2);
#pragma unroll
			for (int q = 0; q < TB / 2; ++q) dv[q] = __ldcg(&dblock[static_cast<int64_t>(jb + q) * TB + lr]);
		}
		// Stage the diagonal block (independent of other CTAs).
		for (int e = t; !dinv && e < TB * TB; e += TRSV_THREADS) {
			// consecutive threads take the contiguous index of the stored matrix
			const int i = TRANS ? e / TB : e % TB, jj = TRANS ? e % TB : e / TB;
			const int64_t off = TRANS ? static_cast<int64_t>(r0 + i) * lda + r0 + jj : static_cast<int64_t>(r0 + jj) * lda + r0 + i;
			dblk[i][jj] = (i < rows && jj < rows) ? a[off] : 0.f;
		}
		double acc4[4] = {0.0, 0.0, 0.0, 0.0};
		// TRANS: warp `wv` takes rows wv, wv + 8, ...; lane takes 4 columns
		double tacc[TB / 8];
#pragma unroll
		for (int q = 0; q < TB / 8; ++q) tacc[q] = 0.0;
		__syncthreads();
		for (int q = 0; q < NB - 1; ++q) stage_q(q);
		// Off-diagonal block columns in dependency order: one barrier per
		// block.  Before it, warp 0 makes sure x of the block is published and
		// loads it, and every thread waits for its own copies of the block;
		// after it, the buffer of the previous block (every thread is done
		// with it) receives the block NB - 1 ahead, and the block is applied.
		for (int q = 0; q < nblk; ++q) {
			const int cb = lower ? q : nbt - 1 - q;
			const int cols = min(TB, n - cb * TB);
			const float *cur = bufp[q % NB];
			double *xs = xsb[q % NB];
			if (t < 32 && !xpre[q % NB]) {
				// Learn how far the published prefix reaches, 32 flags at a time.
				bool have = lower ? (cb < ready_upto) : (cb > ready_upto);
				if (!have) {
					const uint64_t t0 = global_ns();
					while (true) {
						const int probe = lower ? cb + t : cb - t;
						const bool inb = lower ? (probe < r) : (probe > r);
						const bool rdy = inb && ld_acquire_u32(&flags[probe]) == epoch;
						const unsigned m = __ballot_sync(0xffffffffu, rdy);
						const int cnt = __ffs(~m) - 1;   // leading ready flags
						const int c = (m == 0xffffffffu) ? 32 : cnt;
						if (c > 0) {
							if (t == 0) ready_upto = lower ? cb + c : cb - c;
							break;
						}
						// the decision to give up is taken by the whole warp at once
						if (__ballot_sync(0xffffffffu, global_ns() - t0 > kWaitLimitNs)) {
							if (t == 0) abort_flag = 1;
							break;
						}
						__nanosleep(100);
					}
				}
				// x of this block column, published by another CTA: bypass L1
#pragma unroll
				for (int k = 0; k < TB / 32; ++k) {
					const int j = cb * TB + t + 32 * k;
					xs[t + 32 * k] = (j < n) ? __ldcg(&x[j]) : 0.0;
				}
			}
			// block q has landed (the NB - 2 blocks after it may still be in flight)
			if (NB == 3)
				asm volatile("cp.async.wait_group 1;" ::: "memory");
			else
				asm volatile("cp.async.wait_group 0;" ::: "memory");
			__syncthreads();
			if (abort_flag) break;
			stage_q(q + NB - 1);
			if (TRANS) {
				const int wv = t >> 5, ln = t & 31;
				const int j = 4 * ln;
				if (j < cols) {
					const double x0 = xs[j], x1 = xs[j + 1], x2 = xs[j + 2], x3 = xs[j + 3];
#pragma unroll
					for (int qq = 0; qq < TB / 8; ++qq) {
						const int i = wv + 8 * qq;
						const float4 v = *reinterpret_cast<const float4 *>(cur + i * TB + j);
						double s4 = tacc[qq];
						s4 = fma(static_cast<double>(v.x), x0, s4);
						s4 = fma(static_cast<double>(v.y), x1, s4);
						s4 = fma(static_cast<double>(v.z), x2, s4);
						s4 = fma(static_cast<double>(v.w), x3, s4);
						tacc[qq] = s4;
					}
				}
			} else if (lr < rows) {
				// four independent FMA chains: one chain of 64 dependent FMAs per
				// block left the FP64 pipe waiting on its own latency
				const int jb = grp * (TB / 2), je = min(jb + TB / 2, cols);
				int j = jb;
				for (; j + 3 < je; j += 4) {
					acc4[0] = fma(static_cast<double>(cur[j * TB + lr]), xs[j], acc4[0]);
					acc4[1] = fma(static_cast<double>(cur[(j + 1) * TB + lr]), xs[j + 1], acc4[1]);
					acc4[2] = fma(static_cast<double>(cur[(j + 2) * TB + lr]), xs[j + 2], acc4[2]);
					acc4[3] = fma(static_cast<double>(cur[(j + 3) * TB + lr]), xs[j + 3], acc4[3]);
				}
				for (; j < je; ++j) acc4[0] = fma(static_cast<double>(cur[j * TB + lr]), xs[j], acc4[0]);
			}
		}
		if (abort_flag) break;
		if (TRANS) {
			// fold the lanes' partial sums of each row in a fixed order
			const int wv = t >> 5, ln = t & 31;
#pragma unroll
			for (int qq = 0; qq < TB / 8; ++qq) {
				double v = tacc[qq];
				for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
				if (ln == 0) {
					part[0][wv + 8 * qq] = v;
					part[1][wv + 8 * qq] = 0.0;
				}
			}
		} else {
			part[grp][lr] = (acc4[0] + acc4[1]) + (acc4[2] + acc4[3]);
		}
		__syncthreads();
		if (t < TB) rhs[t] = (t < rows) ? xr - (part[0][t] + part[1][t]) : 0.0;
		__syncthreads();
		if (dinv) {
			// x_r = M_rr^{-1} rhs: element (i, j) of M^{-1} is dblock[j*TB + i], or
			// dblock[i*TB + j] for the transpose
			if (TRANS) {
				const int wv = t >> 5, ln = t & 31;
#pragma unroll 4
				for (int qq = 0; qq < TB / 8; ++qq) {
					const int i = wv + 8 * qq;
					const double *row = dblock + static_cast<int64_t>(i) * TB + 4 * ln;
					double v = row[0] * rhs[4 * ln];
					v = fma(row[1], rhs[4 * ln + 1], v);
					v = fma(row[2], rhs[4 * ln + 2], v);
					v = fma(row[3], rhs[4 * ln + 3], v);
					for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
					if (ln == 0) {
						part[0][i] = v;
						part[1][i] = 0.0;
					}
				}
			} else {
				const int jb = grp * (TB / 2);
				double v = 0.0;
#pragma unroll
				for (int q = 0; q < TB / 2; ++q) v = fma(dv[q], rhs[jb + q], v);
				part[grp][lr] = v;
			}
			__syncthreads();
			if (t < rows) rhs[t] = part[0][t] + part[1][t];
			__syncthreads();
		}
		// Diagonal block: 32-row sub-blocks solved by warp 0 with shuffles,
		// the remaining rows updated by all threads.
		const int nsb = dinv ? 0 : (rows + 31) / 32;
		for (int sblk = 0; sblk < nsb; ++sblk) {
			const int sb = lower ? sblk : nsb - 1 - sblk;
			const int base = sb * 32;
			if (t < 32) {
				const int i = base + t;
				double v = (i < rows) ? rhs[i] : 0.0;
				if (lower) {
					for (int jj = 0; jj < 32; ++jj) {
						if (!unit && t == jj && i < rows) v = v / static_cast<double>(dblk[i][i]);
						const double xj = __shfl_sync(0xffffffffu, v, jj);
						if (t > jj && base + jj < rows) v = fma(-static_cast<double>(dblk[i][base + jj]), xj, v);
					}
				} else {
					for (int jj = 31; jj >= 0; --jj) {
						if (!unit && t == jj && i < rows) v = v / static_cast<double>(dblk[i][i]);
						const double xj = __shfl_sync(0xffffffffu, v, jj);
						if (t < jj && base + jj < rows) v = fma(-static_cast<double>(dblk[i][base + jj]), xj, v);
					}
				}
				if (i < rows) rhs[i] = v;
			}
			__syncthreads();
			// rows still to solve: below (lower) or above (upper) this sub-block
			const int lo = lower ? base + 32 : 0;
			const int hi = lower ? rows : base;
			for (int i = lo + t; i < hi; i += TRSV_THREADS) {
				double v = rhs[i];
				for (int jj = 0; jj < 32 && base + jj < rows; ++jj) v = fma(-static_cast<double>(dblk[i][base + jj]), rhs[base + jj], v);
				rhs[i] = v;
			}
			__syncthreads();
		}
		if (t < rows) x[r0 + t] = rhs[t];
		__threadfence();
		__syncthreads();
		if (t == 0) st_release_u32(&flags[r], epoch);
	}
	// copies still in flight after a timeout land before the CTA exits
	asm volatile("cp.async.wait_all;" ::: "memory");
	if (t == 0 && abort_flag) atomicOr(&w->status, 1u);
}

// ---------------------------------------------------------------------------
// Vector helpers.
// ---------------------------------------------------------------------------
__global__ void infnorm_kernel(int n, const double *__restrict__ x, unsigned long long *out)
{
	// max that propagates NaN, so a diverged vector cannot report a finite norm
	auto vmax = [](double p, double q) { return (q != q || q > p) ? q : p; };
	double m = 0.0;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = vmax(m, fabs(x[i]));
	for (int o = 16; o; o >>= 1) m = vmax(m, __shfl_xor_sync(0xffffffffu, m, o));
	__shared__ double wm[32];
	if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
	__syncthreads();
	if (threadIdx.x < 32) {
		m = (threadIdx.x < (blockDim.x + 31) / 32) ? wm[threadIdx.x] : 0.0;
		for (int o = 16; o; o >>= 1) m = vmax(m, __shfl_xor_sync(0xffffffffu, m, o));
		// non-negative doubles order like their bit patterns
		if (threadIdx.x == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(m)));
	}
}

// Checksum of the factored matrix (panel_check.hpp:9-65): FP64 sums of
// |a_ij| over the diagonal, the strict upper and the strict lower triangle.
// HBM-bound (4 n^2 bytes read once).  One warp per column, grid-stride over
// columns, two float4 loads in flight per lane where a and lda allow them;
// each CTA writes its three partial sums and one CTA folds them in a fixed
// order, so the result depends on n and the matrix only.
constexpr int kCheckWarps = 8;

int check_blocks(int n)
{
	const int need = (n + kCheckWarps - 1) / kCheckWarps;
	return need < 1184 ? (need > 0 ? need : 1) : 1184;   // 148 SMs x 8 CTAs
}

__device__ __forceinline__ void check_add(float v, int r, int j, double &sd, double &su, double &sl)
{
	const double t = fabs(static_cast<double>(v));
	if (r < j) su += t;
	else if (r == j) sd += t;
	else sl += t;
}

__global__ void __launch_bounds__(kCheckWarps * 32) check_partial_kernel(int n, const float *__restrict__ a,
	int64_t lda, int vec, double *__restrict__ part)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	double sd = 0.0, su = 0.0, sl = 0.0;
	const int n4 = vec ? (n & ~3) : 0;
	for (int j = blockIdx.x * kCheckWarps + warp; j < n; j += gridDim.x * kCheckWarps) {
		const float *col = a + static_cast<int64_t>(j) * lda;
		int i = lane * 4;
		for (; i + 128 < n4; i += 256) {
			const float4 v0 = __ldcs(reinterpret_cast<const float4 *>(col + i));
			const float4 v1 = __ldcs(reinterpret_cast<const float4 *>(col + i + 128));
			check_add(v0.x, i, j, sd, su, sl);
			check_add(v0.y, i + 1, j, sd, su, sl);
			check_add(v0.z, i + 2, j, sd, su, sl);
			check_add(v0.w, i + 3, j, sd, su, sl);
			check_add(v1.x, i + 128, j, sd, su, sl);
			check_add(v1.y, i + 129, j, sd, su, sl);
			check_add(v1.z, i + 130, j, sd, su, sl);
			check_add(v1.w, i + 131, j, sd, su, sl);
		}
		if (i < n4) {
			const float4 v0 = __ldcs(reinterpret_cast<const float4 *>(col + i));
			check_add(v0.x, i, j, sd, su, sl);
			check_add(v0.y, i + 1, j, sd, su, sl);
			check_add(v0.z, i + 2, j, sd, su, sl);
			check_add(v0.w, i + 3, j, sd, su, sl);
		}
		for (int r = n4 + lane; r < n; r += 32) check_add(__ldcs(col + r), r, j, sd, su, sl);
	}
	for (int o = 16; o; o >>= 1) {
		sd += __shfl_xor_sync(0xffffffffu, sd, o);
		su += __shfl_xor_sync(0xffffffffu, su, o);
		sl += __shfl_xor_sync(0xffffffffu, sl, o);
	}
	__shared__ double ws[3][kCheckWarps];
	if (lane == 0) {
		ws[0][warp] = sd;
		ws[1][warp] = su;
		ws[2][warp] = sl;
	}
	__syncthreads();
	if (threadIdx.x < 3) {
		double s = 0.0;
		for (int w = 0; w < kCheckWarps; ++w) s += ws[threadIdx.x][w];
		part[3 * blockIdx.x + threadIdx.x] = s;
	}
}

__global__ void __launch_bounds__(256) check_fold_kernel(int nparts, const double *__restrict__ part, double *sigs)
{
	__shared__ double s[3][256];
	const int t = threadIdx.x;
	double d = 0.0, u = 0.0, l = 0.0;
	for (int p = t; p < nparts; p += 256) {
		d += part[3 * p];
		u += part[3 * p + 1];
		l += part[3 * p + 2];
	}
	s[0][t] = d;
	s[1][t] = u;
	s[2][t] = l;
	for (int o = 128; o; o >>= 1) {
		__syncthreads();
		if (t < o) {
			s[0][t] += s[0][t + o];
			s[1][t] += s[1][t + o];
			s[2][t] += s[2][t + o];
		}
	}
	__syncthreads();
	if (t < 3) sigs[t] = s[t][0];
}

__global__ void div_kernel(int n, const double *__restrict__ num, const double *__restrict__ den, double *out)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = num[i] / den[i];
}

__global__ void axpy1_kernel(int n, const double *__restrict__ x, double *y)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) y[i] += x[i];
}

} // namespace

size_t otf_gemv_workspace(int n)
{
	if (n <= 0) return 0;
	const size_t nchunks = (static_cast<size_t>(n) + GEMV_COLS - 1) / GEMV_COLS;
	return nchunks * static_cast<size_t>(n) * sizeof(double);
}

int launch_otf_gemv(int n, double alpha, const double *x, double beta, double *y, uint64_t seed, const double *diag,
	void *work, size_t work_bytes, cudaStream_t st, bool trans)
{
	return otf_launch(n, n, n, alpha, x, beta, y, state_initial(seed), 1, diag, work, work_bytes, st, trans);
}

int launch_higham_gemv(int n, double alpha, const double *x, double beta, double *y, double halpha, double hbeta,
	const double *diag, void *work, size_t work_bytes, cudaStream_t st, bool trans)
{
	if (n <= 0) return HPLAI_OK;
	const int nchunks = (n + GEMV_COLS - 1) / GEMV_COLS;
	if (work_bytes < static_cast<size_t>(nchunks) * n * sizeof(double)) return HPLAI_EINVAL;
	double *part = static_cast<double *>(work);
	const double ab = halpha * hbeta;
	// A: upper constants -beta + ab i, lower -alpha + ab j; A^T the other way round
	const double cu = trans ? -halpha : -hbeta, cl = trans ? -hbeta : -halpha;
	higham_partial_kernel<<<dim3((n + GEMV_ROWS - 1) / GEMV_ROWS, nchunks), GEMV_ROWS, 0, st>>>(n, alpha, x, ab, cu, cl,
		diag, part);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	otf_reduce_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, nchunks, beta, part, y, beta == 0.0 ? 1 : 0);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_otf_gemv_block(int64_t n, int mb, int nb, double alpha, const double *x, double *y, uint64_t state00,
	void *work, size_t work_bytes, cudaStream_t st)
{
	return otf_launch(n, mb, nb, alpha, x, 1.0, y, state00, 0, nullptr, work, work_bytes, st);
}

size_t trsv_workspace(int n)
{
	const size_t nbt = (static_cast<size_t>(n) + TB - 1) / TB;
	return sizeof(TrsvWork) + nbt * sizeof(uint32_t);
}

int launch_trsv(bool lower, int n, const float *a, int64_t lda, double *x, void *work, size_t work_bytes,
	cudaStream_t st, bool trans, const double *dinv)
{
	if (n <= 0) return HPLAI_OK;
	if (!work || work_bytes < trsv_workspace(n)) return HPLAI_EINVAL;
	constexpr size_t dsmem = sizeof(float) * (TB * (TB + 1) + 3 + 4 + 2 * TB * TB);
	// co-resident CTAs of the cooperative launch on this device
	static DeviceOnce grid_once;
	int max_blocks = 0;
	HPLAI_TRY(grid_once.get([&](int dev, int *v) -> int {
		int per_sm = 0, per_sm_t = 0, sms = 0;
		HPLAI_CUDA_TRY(cudaFuncSetAttribute(trsv_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			static_cast<int>(dsmem)));
		HPLAI_CUDA_TRY(cudaFuncSetAttribute(trsv_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			static_cast<int>(dsmem)));
		HPLAI_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsv_kernel<false>, TRSV_THREADS, dsmem));
		HPLAI_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_t, trsv_kernel<true>, TRSV_THREADS, dsmem));
		HPLAI_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
		*v = (per_sm < per_sm_t ? per_sm : per_sm_t) * sms;
		return HPLAI_OK;
	}, &max_blocks));
	if (max_blocks <= 0) return HPLAI_EUNSUPPORTED;
	// the transposed solve reads rows of the stored matrix as float4
	if (trans && ((reinterpret_cast<uintptr_t>(a) & 15u) || (lda & 3))) return HPLAI_EINVAL;
	TrsvWork *w = static_cast<TrsvWork *>(work);
	trsv_epoch_kernel<<<1, 1, 0, st>>>(w);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	const int nbt = (n + TB - 1) / TB;
	const int grid = nbt < max_blocks ? nbt : max_blocks;
	int lw = lower ? 1 : 0;
	void *args[] = {(void *)&lw, (void *)&n, (void *)&a, (void *)&lda, (void *)&x, (void *)&w, (void *)&dinv};
	void *fn = trans ? reinterpret_cast<void *>(trsv_kernel<true>) : reinterpret_cast<void *>(trsv_kernel<false>);
	HPLAI_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(TRSV_THREADS), args, dsmem, st));
	count_launches();
	return HPLAI_OK;
}

size_t trsv_dinv_doubles(int n)
{
	const size_t nbt = (static_cast<size_t>(n) + TB - 1) / TB;
	return 2 * nbt * TB * TB;
}

int launch_trsv_dinv(int n, const float *a, int64_t lda, double *dinv, cudaStream_t st, int blk0, int nblk)
{
	if (n <= 0) return HPLAI_OK;
	const int nbt = (n + TB - 1) / TB;
	if (nblk < 0) nblk = nbt - blk0;
	if (blk0 < 0 || nblk <= 0 || blk0 + nblk > nbt) return nblk == 0 ? HPLAI_OK : HPLAI_EINVAL;
	constexpr size_t smem = sizeof(float) * (TB * (TB + 1) + 3) + sizeof(double) * TB * TB;
	static DeviceOnce attr;
	HPLAI_TRY(attr.get([&](int, int *) -> int {
		HPLAI_CUDA_TRY(cudaFuncSetAttribute(trsv_dinv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			static_cast<int>(smem)));
		return HPLAI_OK;
	}));
	trsv_dinv_kernel<<<dim3(nblk, 2), TB, smem, st>>>(n, a, lda, dinv, blk0);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int trsv_status(void *work, cudaStream_t st, int *status)
{
	uint32_t v = 0;
	TrsvWork *w = static_cast<TrsvWork *>(work);
	HPLAI_CUDA_TRY(cudaMemcpyAsync(&v, &w->status, sizeof(v), cudaMemcpyDeviceToHost, st));
	HPLAI_CUDA_TRY(cudaStreamSynchronize(st));
	*status = v ? HPLAI_ETIMEOUT : HPLAI_OK;
	return HPLAI_OK;
}

int launch_infnorm(int n, const double *x, double *out, cudaStream_t st)
{
	HPLAI_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double), st));
	if (n <= 0) return HPLAI_OK;
	int blocks = (n + 255) / 256;
	if (blocks > 1184) blocks = 1184;
	infnorm_kernel<<<blocks, 256, 0, st>>>(n, x, reinterpret_cast<unsigned long long *>(out));
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

size_t panel_check_workspace(int n)
{
	return 3 * sizeof(double) * static_cast<size_t>(check_blocks(n));
}

int launch_panel_check(int n, const float *a, int64_t lda, double *sigs, void *work, size_t work_bytes,
	cudaStream_t st)
{
	if (n <= 0) {
		HPLAI_CUDA_TRY(cudaMemsetAsync(sigs, 0, 3 * sizeof(double), st));
		return HPLAI_OK;
	}
	if (work_bytes < panel_check_workspace(n)) return HPLAI_EINVAL;
	const int blocks = check_blocks(n);
	const int vec = (reinterpret_cast<uintptr_t>(a) % 16 == 0 && lda % 4 == 0) ? 1 : 0;
	double *part = static_cast<double *>(work);
	check_partial_kernel<<<blocks, kCheckWarps * 32, 0, st>>>(n, a, lda, vec, part);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	check_fold_kernel<<<1, 256, 0, st>>>(blocks, part, sigs);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_div(int n, const double *num, const double *den, double *out, cudaStream_t st)
{
	if (n <= 0) return HPLAI_OK;
	div_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, num, den, out);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_axpy1(int n, const double *x, double *y, cudaStream_t st)
{
	if (n <= 0) return HPLAI_OK;
	axpy1_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, x, y);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free on-the-fly GEMV.
//
// Callers that cannot allocate device memory (code that is handed every
// device buffer by another runtime's allocator and has none of its own, or a
// solve loop that must not call cudaMalloc because it can synchronise the
// device) get the GEMV's partial-sum scratch from this fixed array instead
// of a caller workspace.  It is part of the library image: every GPU that
// loads libhplai holds its 4 MiB until the process exits.  It covers orders
// up to kNoAllocMaxN (ceil(n/2048) * n doubles).  All calls share it.
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxN = 32768;
constexpr size_t kNoAllocScratchDoubles =
	static_cast<size_t>((kNoAllocMaxN + GEMV_COLS - 1) / GEMV_COLS) * kNoAllocMaxN;
static __device__ __align__(256) double g_gemv_noalloc_scratch[kNoAllocScratchDoubles];

namespace {
std::mutex g_noalloc_mu;
constexpr int kMaxDevices = 64;
void *g_noalloc_addr[kMaxDevices] = {};
} // namespace

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side handle, so the address is looked up
// once per device (with that device current) and cached.
static int noalloc_scratch(void **out)
{
	int dev = 0;
	HPLAI_CUDA_TRY(cudaGetDevice(&dev));
	if (dev < 0 || dev >= kMaxDevices) return HPLAI_EUNSUPPORTED;
	std::lock_guard<std::mutex> lk(g_noalloc_mu);
	if (!g_noalloc_addr[dev]) {
		void *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_gemv_noalloc_scratch);
		if (e != cudaSuccess) {
			set_last_cuda_error(e, "cudaGetSymbolAddress(g_gemv_noalloc_scratch)", __FILE__, __LINE__);
			return HPLAI_ECUDA;
		}
		g_noalloc_addr[dev] = p;
	}
	*out = g_noalloc_addr[dev];
	return HPLAI_OK;
}

} // namespace hplai

extern "C" size_t hplai_otf_gemv_workspace(int n) { return hplai::otf_gemv_workspace(n); }

extern "C" int hplai_otf_gemv(int n, double alpha, const double *x, double beta, double *y, uint64_t seed,
	const double *diag, void *work, size_t work_bytes, void *stream)
{
	if (n <= 0 || !x || !y || !diag || !work) return HPLAI_EINVAL;
	return hplai::launch_otf_gemv(n, alpha, x, beta, y, seed, diag, work, work_bytes, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_otf_gemv_block(int64_t n, int mb, int nb, double alpha, const double *x, double *y,
	uint64_t state00, void *work, size_t work_bytes, void *stream)
{
	if (n <= 0 || mb < 0 || nb < 0 || !x || !y || !work) return HPLAI_EINVAL;
	return hplai::launch_otf_gemv_block(n, mb, nb, alpha, x, y, state00, work, work_bytes,
		static_cast<cudaStream_t>(stream));
}

extern "C" size_t hplai_trsv_workspace(int n) { return hplai::trsv_workspace(n); }

extern "C" int hplai_trsv_lower(int n, const float *a, int64_t lda, double *x, void *work, size_t work_bytes,
	void *stream)
{
	if (n <= 0 || !a || !x || lda < n) return HPLAI_EINVAL;
	return hplai::launch_trsv(true, n, a, lda, x, work, work_bytes, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_trsv_upper(int n, const float *a, int64_t lda, double *x, void *work, size_t work_bytes,
	void *stream)
{
	if (n <= 0 || !a || !x || lda < n) return HPLAI_EINVAL;
	return hplai::launch_trsv(false, n, a, lda, x, work, work_bytes, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_infnorm(int n, const double *x, double *out, void *stream)
{
	if (n < 0 || (!x && n) || !out) return HPLAI_EINVAL;
	return hplai::launch_infnorm(n, x, out, static_cast<cudaStream_t>(stream));
}

extern "C" size_t hplai_panel_check_workspace(int n)
{
	return hplai::panel_check_workspace(n);
}

extern "C" int hplai_panel_check(int n, const float *a, int64_t lda, double *sigs, void *work, size_t work_bytes,
	void *stream)
{
	if (n < 0 || !sigs || (n > 0 && (!a || lda < n || !work))) return HPLAI_EINVAL;
	if (n > 0 && work_bytes < hplai::panel_check_workspace(n)) {
		hplai::set_last_error_message("hplai_panel_check: work is smaller than hplai_panel_check_workspace(n)");
		return HPLAI_EINVAL;
	}
	return hplai::launch_panel_check(n, a, lda, sigs, work, work_bytes, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_otf_gemv_noalloc(int n, double alpha, const double *x, double beta, double *y, uint64_t seed,
	const double *diag, void *stream)
{
	if (n <= 0 || !x || !y || !diag) return HPLAI_EINVAL;
	if (n > hplai::kNoAllocMaxN) {
		hplai::set_last_error_message("hplai_otf_gemv_noalloc: n exceeds HPLAI_OTF_GEMV_NOALLOC_MAX_N (32768)");
		return HPLAI_EINVAL;
	}
	void *scratch = nullptr;
	HPLAI_TRY(hplai::noalloc_scratch(&scratch));
	// Every partial sum the fold reads is written by this call's first
	// kernel, so the shared array needs no clearing between calls.
	return hplai::launch_otf_gemv(n, alpha, x, beta, y, seed, diag, scratch,
		hplai::kNoAllocScratchDoubles * sizeof(double), static_cast<cudaStream_t>(stream));
}
