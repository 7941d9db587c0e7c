// getrf.cu -- b x b diagonal block LU without pivoting, spread over the GPU.
//
// getrf_nopiv (getrf_nopiv.hpp:30-141) on the diagonal block of each step.
// The block is cut into 32 x 32 tiles that go through the steps of a
// right-looking LU:
//   step r < min(ti, tj):  X -= L(ti, r) U(r, tj)              (trailing update)
//   step r = ti = tj:      X <- LU of X                        (tile factor)
//   step r = tj < ti:      X <- X U(r, r)^{-1}                 (L tile)
//   step r = ti < tj:      X <- L(r, r)^{-1} X  (unit lower)   (U tile)
// Each tile publishes a progress word, epoch * 64 + (steps applied), where a
// tile with min(ti, tj) = r is final at r + 1; consumers wait for the value
// they need.
//
// The diagonal is the critical chain, so one CTA (CTA 0) does nothing
// else: at step r it takes L(r+1, r) and U(r, r+1) once their owners have
// applied their first r updates, solves them with the factored tile (r, r)
// it still holds (four warps each, a step per named barrier), publishes
// them, applies the last update to tile (r+1, r+1) and factors it (all
// eight warps).  There is no flag hop between two diagonal tiles, and its
// code stays hot in its SM's instruction cache.  Worker warps (the other
// CTAs) own every other tile and walk them step by step, panel tiles before
// updates.  Every wait is on work the producer reaches
// without waiting on the waiter, so the dataflow always completes (all
// warps are resident: cooperative launch); every wait is bounded, and a
// timeout sets the status word and the warp stops.
//
// Each element receives a_ij <- fmaf(-l_ik, u_kj, a_ij) in increasing k,
// multipliers are a_ik * (1/u_kk) and the U tiles use the same unit-lower
// sequence as netlib strsm: the operation sequence of a sequential FP32
// factorisation, so the result is bit for bit that of the reference's
// unblocked kernel with any blocking (getrf_nopiv.hpp:33-44).
#include "common.cuh"
#include "internal.h"

#include <mutex>

namespace hplai {

namespace {

constexpr int T = 32;
constexpr int kWarps = 8;       // worker warps per CTA
constexpr int kMaxTiles = 32;   // b <= 1024

// One progress word per 128-byte line, so that polling warps and publishing
// warps do not queue on a few L2 lines.
constexpr int kFlagStride = 32;

struct GetrfWork {
	uint32_t status;
	uint32_t pad[31];
	uint32_t prog[kMaxTiles * kMaxTiles * kFlagStride];
};

// Wait until *f >= target (values of earlier launches are below every target
// of this one).  Lane 0 reads the word; the whole warp stays in the loop
// and learns the outcome through a shuffle, so the warp never diverges
// around a wait (a warp left split after a long divergent spin runs the
// following shuffles many times slower).
__device__ __forceinline__ bool wait_prog(const uint32_t *f, uint32_t target)
{
	const bool lead = (threadIdx.x & 31) == 0;
	uint64_t t0 = 0;
	for (int it = 0;; ++it) {
		int ready = lead ? (ld_acquire_u32(f) >= target) : 0;
		ready = __shfl_sync(0xffffffffu, ready, 0);
		if (ready) return true;
		if (it == 0) t0 = global_ns();
		else if (global_ns() - t0 > kWaitLimitNs) return false;
		__nanosleep(32);
	}
}

__device__ __forceinline__ void publish(uint32_t *f, uint32_t v)
{
	__syncwarp();
	if ((threadIdx.x & 31) == 0) {
		__threadfence();
		st_release_u32(f, v);
	}
}

// A staged tile: column-major, element (i, j) at t[j * kLd + i]; rows of 16
// bytes so that cp.async can fill it.  Lane i works on row i (conflict-free
// along a column); all lanes reading one element is a broadcast.
constexpr int kLd = 36;
constexpr int kTileFloats = T * kLd;

// Tile (rows r0.., cols c0..) -> t, rows >= rv and columns >= cv zero.
// vec: a, lda and r0 allow 16-byte copies (cp.async.cg, L2 only); otherwise
// 4-byte loads through L2.  The caller waits with stage_wait().
__device__ __forceinline__ void stage_tile(float *t, const float *a, int64_t lda, int r0, int c0, int rv, int cv,
	bool vec, int lane)
{
	if (vec) {
#pragma unroll 1
		for (int q = 0; q < 8; ++q) {
			const int e = lane + 32 * q, j = e >> 3, g = (e & 7) * 4;
			int bytes = (j < cv) ? (rv - g) * 4 : 0;
			bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
			const float *src = a + static_cast<int64_t>(c0 + (j < cv ? j : 0)) * lda + r0 + (bytes ? g : 0);
			asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(t + j * kLd + g)), "l"(src),
				"r"(bytes) : "memory");
		}
		asm volatile("cp.async.commit_group;" ::: "memory");
	} else {
#pragma unroll 4
		for (int j = 0; j < T; ++j)
			t[j * kLd + lane] = (lane < rv && j < cv) ? __ldcg(&a[static_cast<int64_t>(c0 + j) * lda + r0 + lane]) : 0.f;
	}
}

__device__ __forceinline__ void stage_wait()
{
	asm volatile("cp.async.wait_all;" ::: "memory");
	__syncwarp();
}

__device__ __forceinline__ void store_tile(const float *t, float *a, int64_t lda, int r0, int c0, int rv, int cv,
	int lane)
{
	if (lane < rv) {
#pragma unroll 4
		for (int j = 0; j < cv; ++j) a[static_cast<int64_t>(c0 + j) * lda + r0 + lane] = t[j * kLd + lane];
	}
}

// One-warp tile operations on staged tiles (the worker warps').  The solves
// keep a row (or column) of the tile in registers, fully unrolled so that
// every register index is static: 496 FMAs and their loads per lane, with no
// register moves between pivots.

// L tile x <- x U^{-1}, U = upper part of the factored tile d (kv x kv); row `lane`.
__device__ __noinline__ void op_solve_l(float *x, const float *d, int kv)
{
	const int lane = threadIdx.x & 31;
	float v[T];
#pragma unroll
	for (int j = 0; j < T; ++j) v[j] = x[j * kLd + lane];
	// 1/u_jj, lane j's (the staged tile is zero past kv: those lanes' values go unused)
	const float inv = 1.0f / d[lane * kLd + lane];
#pragma unroll
	for (int j = 0; j < T; ++j) {
		if (j < kv) {
			v[j] *= __shfl_sync(0xffffffffu, inv, j);
			// U(j, t) at d[t * kLd + j]
#pragma unroll
			for (int t = j + 1; t < T; ++t) v[t] = fmaf(-v[j], d[t * kLd + j], v[t]);
		}
	}
#pragma unroll
	for (int j = 0; j < T; ++j)
		if (j < kv) x[j * kLd + lane] = v[j];
	__syncwarp();
}

// U tile x <- L^{-1} x, L = unit lower part of d (kv x kv); column `lane`.
__device__ __noinline__ void op_solve_u(float *x, const float *d, int kv)
{
	const int lane = threadIdx.x & 31;
	float v[T];
	float *col = x + lane * kLd;
#pragma unroll
	for (int q = 0; q < T / 4; ++q) {
		const float4 c = reinterpret_cast<const float4 *>(col)[q];
		v[4 * q] = c.x;
		v[4 * q + 1] = c.y;
		v[4 * q + 2] = c.z;
		v[4 * q + 3] = c.w;
	}
#pragma unroll
	for (int k = 0; k < T; ++k) {
		if (k < kv) {
			// L(i, k) at d[k * kLd + i]
#pragma unroll
			for (int i = k + 1; i < T; ++i) v[i] = fmaf(-v[k], d[k * kLd + i], v[i]);
		}
	}
#pragma unroll
	for (int k = 0; k < T; ++k)
		if (k < kv) col[k] = v[k];
	__syncwarp();
}

// x -= l u (K = T); column `lane` of x in registers: per k, u_kj from the
// lane's own column of u and column k of l as eight 16-byte broadcasts
// (columns are 16-byte aligned: kLd * 4 = 144 bytes).
__device__ __noinline__ void op_update(float *x, const float *l, const float *u)
{
	const int lane = threadIdx.x & 31;
	float v[T];
	float4 *xc = reinterpret_cast<float4 *>(x + lane * kLd);
#pragma unroll
	for (int q = 0; q < T / 4; ++q) {
		const float4 c = xc[q];
		v[4 * q] = c.x;
		v[4 * q + 1] = c.y;
		v[4 * q + 2] = c.z;
		v[4 * q + 3] = c.w;
	}
	const float4 *uc = reinterpret_cast<const float4 *>(u + lane * kLd);
#pragma unroll 1
	for (int k4 = 0; k4 < T / 4; ++k4) {
		const float4 u4 = uc[k4];
		const float uk[4] = {u4.x, u4.y, u4.z, u4.w};
#pragma unroll
		for (int kk = 0; kk < 4; ++kk) {
			const float4 *lc = reinterpret_cast<const float4 *>(l + (4 * k4 + kk) * kLd);
#pragma unroll
			for (int q = 0; q < T / 4; ++q) {
				const float4 l4 = lc[q];
				v[4 * q] = fmaf(-l4.x, uk[kk], v[4 * q]);
				v[4 * q + 1] = fmaf(-l4.y, uk[kk], v[4 * q + 1]);
				v[4 * q + 2] = fmaf(-l4.z, uk[kk], v[4 * q + 2]);
				v[4 * q + 3] = fmaf(-l4.w, uk[kk], v[4 * q + 3]);
			}
		}
	}
#pragma unroll
	for (int q = 0; q < T / 4; ++q) xc[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
	__syncwarp();
}

constexpr int kDiagWarps = kWarps;

// Barrier and AND-vote of the diagonal CTA's warps (named barrier 1).
__device__ __forceinline__ void diag_sync()
{
	asm volatile("bar.sync 1, %0;" ::"n"(kDiagWarps * 32) : "memory");
}

__device__ __forceinline__ bool diag_all(bool p)
{
	int r;
	asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.and.pred q, 1, %2, p;\n\t"
	             "selp.s32 %0, 1, 0, q;\n\t}"
	             : "=r"(r) : "r"(p ? 1 : 0), "n"(kDiagWarps * 32) : "memory");
	return r != 0;
}

// Columns c0 .. c0 + T/kDiagWarps - 1 of x -= l u (K = T); row `lane`.
__device__ __noinline__ void op_update_cols(float *x, const float *l, const float *u, int c0)
{
	constexpr int C = T / kDiagWarps;
	const int lane = threadIdx.x & 31;
	float v[C];
#pragma unroll
	for (int j = 0; j < C; ++j) v[j] = x[(c0 + j) * kLd + lane];
#pragma unroll 4
	for (int k = 0; k < T; ++k) {
		const float lk = l[k * kLd + lane];
#pragma unroll
		for (int j = 0; j < C; ++j) v[j] = fmaf(-lk, u[(c0 + j) * kLd + k], v[j]);
	}
#pragma unroll
	for (int j = 0; j < C; ++j) x[(c0 + j) * kLd + lane] = v[j];
}

// The diagonal CTA's tile operations over several warps: warp w of a group
// owns C = T / (warps in the group) columns (rows for the U solve), lane =
// row (column); the value each step broadcasts (a multiplier column or a
// solved row) goes through shared memory, double-buffered, one named
// barrier per step.  Every element receives the same operations in the same
// order as in an unblocked one-warp factorisation and in the workers'
// op_solve_l / op_solve_u.
__device__ __forceinline__ void group_sync(int id, int threads)
{
	asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Unblocked LU of the kv x kv tile x, all kDiagWarps warps (barrier 1).
__device__ __noinline__ void coop_factor(float *x, int kv, float *mbuf, int warp)
{
	constexpr int C = T / kDiagWarps;
	const int lane = threadIdx.x & 31, c0 = warp * C;
	float v[C];
#pragma unroll
	for (int c = 0; c < C; ++c) v[c] = x[(c0 + c) * kLd + lane];
#pragma unroll 1
	for (int k = 0; k < kv; ++k) {
		float *m = mbuf + (k & 1) * T;
		const bool own = k >= c0 && k < c0 + C;
		float lreg = 0.f;
#pragma unroll
		for (int c = 0; c < C; ++c)
			if (k == c0 + c) {
				const float inv = 1.0f / __shfl_sync(0xffffffffu, v[c], k);
				const float lik = v[c] * inv;
				if (lane > k) v[c] = lik;
				m[lane] = lik;
				lreg = lik;
			}
		group_sync(1, kDiagWarps * 32);
		const float l = own ? lreg : m[lane];
#pragma unroll
		for (int c = 0; c < C; ++c) {
			const float ukj = __shfl_sync(0xffffffffu, v[c], k);
			if (lane > k && c0 + c > k) v[c] = fmaf(-l, ukj, v[c]);
		}
	}
#pragma unroll
	for (int c = 0; c < C; ++c) x[(c0 + c) * kLd + lane] = v[c];
}

// L tile x <- x U^{-1} (T columns), warps w = 0 .. kSolveWarps - 1 of the
// group on barrier `bar`; row `lane`.
constexpr int kSolveWarps = kDiagWarps / 2;
__device__ __noinline__ void coop_solve_l(float *x, const float *d, float *mbuf, int w, int bar)
{
	constexpr int C = T / kSolveWarps;
	const int lane = threadIdx.x & 31, c0 = w * C;
	float v[C];
#pragma unroll
	for (int c = 0; c < C; ++c) v[c] = x[(c0 + c) * kLd + lane];
	const float inv = 1.0f / d[lane * kLd + lane];   // lane j: 1/u_jj
#pragma unroll 1
	for (int j = 0; j < T; ++j) {
		float *m = mbuf + (j & 1) * T;
		const bool own = j >= c0 && j < c0 + C;
		const float invj = __shfl_sync(0xffffffffu, inv, j);
		float xreg = 0.f;
#pragma unroll
		for (int c = 0; c < C; ++c)
			if (j == c0 + c) {
				v[c] *= invj;
				m[lane] = v[c];
				xreg = v[c];
			}
		group_sync(bar, kSolveWarps * 32);
		const float xij = own ? xreg : m[lane];
#pragma unroll
		for (int c = 0; c < C; ++c)
			if (c0 + c > j) v[c] = fmaf(-xij, d[(c0 + c) * kLd + j], v[c]);
	}
#pragma unroll
	for (int c = 0; c < C; ++c) x[(c0 + c) * kLd + lane] = v[c];
}

// U tile x <- L^{-1} x (T rows, L unit lower), warp w of its group owning
// rows w * C ..; column `lane`.
__device__ __noinline__ void coop_solve_u(float *x, const float *d, float *mbuf, int w, int bar)
{
	constexpr int C = T / kSolveWarps;
	const int lane = threadIdx.x & 31, r0 = w * C;
	float v[C];
#pragma unroll
	for (int r = 0; r < C; ++r) v[r] = x[lane * kLd + r0 + r];
#pragma unroll 1
	for (int k = 0; k < T; ++k) {
		float *m = mbuf + (k & 1) * T;
		const bool own = k >= r0 && k < r0 + C;
		float xreg = 0.f;
#pragma unroll
		for (int r = 0; r < C; ++r)
			if (k == r0 + r) {
				m[lane] = v[r];
				xreg = v[r];
			}
		group_sync(bar, kSolveWarps * 32);
		const float xkj = own ? xreg : m[lane];
#pragma unroll
		for (int r = 0; r < C; ++r)
			if (r0 + r > k) v[r] = fmaf(-xkj, d[k * kLd + r0 + r], v[r]);
	}
#pragma unroll
	for (int r = 0; r < C; ++r) x[lane * kLd + r0 + r] = v[r];
}

__global__ void __launch_bounds__(kWarps * 32) getrf_tiles_kernel(int b, float *a, int64_t lda, GetrfWork *w,
	uint32_t epoch)
{
	extern __shared__ __align__(16) float dyn[];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	float *X = dyn + warp * 4 * kTileFloats;   // this warp's tile
	float *D = X + kTileFloats;                // the factored diagonal tile it reads
	float *Lt = X + 2 * kTileFloats;           // an L tile it reads
	float *Ut = X + 3 * kTileFloats;           // a U tile it reads
	const int nt = (b + T - 1) / T, ntiles = nt * nt;
	const uint32_t base = epoch * 64u;
	uint32_t *prog = w->prog;
	auto pidx = [nt](int ti, int tj) { return (ti + nt * tj) * kFlagStride; };
	const bool vec = ((reinterpret_cast<uintptr_t>(a) & 15u) == 0) && ((lda & 3) == 0);
	bool ok = true;

	if (blockIdx.x == 0) {
		// ---------------- the diagonal chain (all kDiagWarps warps) ----------------
		// warps 0 .. 3 solve L(r+1, r) while warps 4 .. 7 solve U(r, r+1);
		// all share the update of tile (r+1, r+1) and its factorisation.
		// Their tiles are warp 0's four staging buffers; the broadcast rows
		// sit in warp 1's.
		float *Dd = dyn, *Xd = dyn + kTileFloats, *Ld = dyn + 2 * kTileFloats, *Ud = dyn + 3 * kTileFloats;
		float *mF = dyn + 4 * kTileFloats, *mL = mF + 2 * T, *mU = mL + 2 * T;
		const bool lgroup = warp < kSolveWarps;
		{
			const int kv = min(T, b);
			if (warp == 0) stage_tile(Dd, a, lda, 0, 0, kv, kv, vec, lane);
			stage_wait();
			diag_sync();
			coop_factor(Dd, kv, mF, warp);
			diag_sync();
			if (warp == 0) {
				store_tile(Dd, a, lda, 0, 0, kv, kv, lane);
				publish(&prog[0], base + 1);
			}
		}
		diag_sync();
		for (int r = 0; r + 1 < nt && ok; ++r) {
			const int k0 = r * T, r1 = k0 + T, v1 = min(T, b - r1);
			bool mine = true;
			if (r > 0 && warp < 3) {
				const int f = warp == 0 ? pidx(r + 1, r) : (warp == 1 ? pidx(r, r + 1) : pidx(r + 1, r + 1));
				mine = wait_prog(&prog[f], base + r);
			}
			ok = diag_all(mine);
			if (!ok) break;
			if (warp == 0) stage_tile(Ld, a, lda, r1, k0, v1, T, vec, lane);   // L(r+1, r) before its solve
			if (warp == 1) stage_tile(Ud, a, lda, k0, r1, T, v1, vec, lane);   // U(r, r+1) before its solve
			if (warp == 2) stage_tile(Xd, a, lda, r1, r1, v1, v1, vec, lane);  // tile (r+1, r+1)
			stage_wait();
			diag_sync();
			if (lgroup)
				coop_solve_l(Ld, Dd, mL, warp, 2);
			else
				coop_solve_u(Ud, Dd, mU, warp - kSolveWarps, 3);
			diag_sync();
			if (warp == 0)
				store_tile(Ld, a, lda, r1, k0, v1, T, lane);
			else if (warp == 1)
				store_tile(Ud, a, lda, k0, r1, T, v1, lane);
			__threadfence();
			diag_sync();
			if (warp == 0 && lane == 0) {
				st_release_u32(&prog[pidx(r + 1, r)], base + r + 1);
				st_release_u32(&prog[pidx(r, r + 1)], base + r + 1);
			}
			op_update_cols(Xd, Ld, Ud, warp * (T / kDiagWarps));
			diag_sync();
			coop_factor(Xd, v1, mF, warp);
			diag_sync();
			if (warp == 0) {
				store_tile(Xd, a, lda, r1, r1, v1, v1, lane);
				publish(&prog[pidx(r + 1, r + 1)], base + r + 2);
			}
			// the new diagonal tile is the next step's factor
			for (int e = threadIdx.x; e < kTileFloats; e += kDiagWarps * 32) Dd[e] = Xd[e];
			diag_sync();
		}
		if (!ok && threadIdx.x == 0) atomicOr(&w->status, 1u);
		return;
	}

	// ---------------- worker warps ----------------
	// worker warp w owns tiles w, w + nwarps, ... (column-major tile index);
	// warp numbers run across the CTAs first, so that neighbouring tiles sit
	// on different SMs (b = 1024: 0.57 ms against 0.62 with them on one SM;
	// ordering each warp's tiles nearest-the-diagonal first was slower)
	const int wid = warp * (gridDim.x - 1) + (blockIdx.x - 1), nwarps = (gridDim.x - 1) * kWarps;
	for (int r = 0; r < nt && ok; ++r) {
		const int k0 = r * T, kv = min(T, b - k0);
		const uint32_t diag_final = base + r + 1;
		// pass 0: panel tiles of step r; pass 1: trailing updates
		for (int pass = 0; pass < 2 && ok; ++pass) {
			for (int t = wid; t < ntiles && ok; t += nwarps) {
				const int ti = t % nt, tj = t / nt;
				const int mn = min(ti, tj);
				if (mn < r || ti == tj && ti <= r + 1) continue;                     // done, or the diagonal CTA's
				if ((ti == r + 1 && tj == r) || (ti == r && tj == r + 1)) continue;  // the diagonal CTA's
				if ((mn == r ? 0 : 1) != pass) continue;
				const int r0 = ti * T, c0 = tj * T;
				const int rv = min(T, b - r0), cv = min(T, b - c0);
				if (pass == 0) {
					// L tile X <- X U(r,r)^{-1}, or U tile X <- L(r,r)^{-1} X
					stage_tile(X, a, lda, r0, c0, rv, cv, vec, lane);
					if (!wait_prog(&prog[pidx(r, r)], diag_final)) { ok = false; break; }
					stage_tile(D, a, lda, k0, k0, kv, kv, vec, lane);
					stage_wait();
					if (tj == r)
						op_solve_l(X, D, kv);
					else
						op_solve_u(X, D, kv);
					store_tile(X, a, lda, r0, c0, rv, cv, lane);
					publish(&prog[t * kFlagStride], base + r + 1);
				} else {
					// X -= L(ti, r) U(r, tj)
					if (!wait_prog(&prog[pidx(ti, r)], base + r + 1) || !wait_prog(&prog[pidx(r, tj)], base + r + 1)) {
						ok = false;
						break;
					}
					stage_tile(X, a, lda, r0, c0, rv, cv, vec, lane);
					stage_tile(Lt, a, lda, r0, k0, rv, T, vec, lane);
					stage_tile(Ut, a, lda, k0, c0, T, cv, vec, lane);
					stage_wait();
					op_update(X, Lt, Ut);
					store_tile(X, a, lda, r0, c0, rv, cv, lane);
					// the next step's panel tiles, and the diagonal tile after next, announce
					// that they hold r + 1 updates
					if (mn == r + 1 || (ti == tj && ti == r + 2)) publish(&prog[t * kFlagStride], base + r + 1);
				}
				__syncwarp();   // this warp's staging tiles are free again
			}
		}
	}
	if (!ok && lane == 0) atomicOr(&w->status, 1u);
}

constexpr size_t kSmemBytes = static_cast<size_t>(kWarps) * 4 * kTileFloats * sizeof(float);

std::mutex g_static_mu;
__device__ GetrfWork g_static_work;
uint32_t g_static_epoch = 0;

int max_coresident_ctas()
{
	static DeviceOnce once;
	int n = 0;
	if (once.get([](int dev, int *v) -> int {
		int per_sm = 0, sms = 0;
		HPLAI_CUDA_TRY(cudaFuncSetAttribute(getrf_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			static_cast<int>(kSmemBytes)));
		HPLAI_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, getrf_tiles_kernel, kWarps * 32,
			kSmemBytes));
		HPLAI_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
		*v = per_sm * sms;
		return HPLAI_OK;
	}, &n) != HPLAI_OK) return 0;
	return n;
}

} // namespace

size_t getrf_workspace() { return sizeof(GetrfWork); }

int launch_getrf_tiles(int b, float *a, int64_t lda, void *work, uint32_t *epoch, int max_ctas, cudaStream_t st)
{
	if (b <= 0) return HPLAI_OK;
	if (b > T * kMaxTiles || !a || lda < b || !work || !epoch) return HPLAI_EINVAL;
	const int nt = (b + T - 1) / T;
	// CTA 0: the diagonal chain; then enough worker CTAs for one tile per warp
	int grid = 1 + (nt > 1 ? (nt * nt + kWarps - 1) / kWarps : 0);
	const int cap = max_coresident_ctas();
	if (cap < 2) return HPLAI_EUNSUPPORTED;
	if (grid > cap) grid = cap;
	if (max_ctas > 0 && grid > max_ctas) grid = max_ctas < 2 ? 2 : max_ctas;
	if (nt > 1 && grid < 2) grid = 2;
	GetrfWork *w = static_cast<GetrfWork *>(work);
	// progress words are epoch * 64 + steps (< 64): epochs stay below 2^26
	uint32_t ep = ++*epoch;
	if (ep >= (1u << 26)) return HPLAI_EUNSUPPORTED;
	void *args[] = {(void *)&b, (void *)&a, (void *)&lda, (void *)&w, (void *)&ep};
	HPLAI_CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<void *>(getrf_tiles_kernel), dim3(grid),
		dim3(kWarps * 32), args, kSmemBytes, st));
	count_launches();
	return HPLAI_OK;
}

int getrf_status(void *work, cudaStream_t st, int *status)
{
	uint32_t v = 0;
	GetrfWork *w = static_cast<GetrfWork *>(work);
	HPLAI_CUDA_TRY(cudaMemcpyAsync(&v, &w->status, sizeof(v), cudaMemcpyDeviceToHost, st));
	HPLAI_CUDA_TRY(cudaStreamSynchronize(st));
	*status = v ? HPLAI_ETIMEOUT : HPLAI_OK;
	return HPLAI_OK;
}

// The leaf entry point's workspace: one per library, calls serialised by
// the host lock (stream order then keeps their flags apart).
int launch_getrf(int b, float *a, int64_t lda, cudaStream_t st)
{
	std::lock_guard<std::mutex> lk(g_static_mu);
	void *w = nullptr;
	HPLAI_CUDA_TRY(cudaGetSymbolAddress(&w, g_static_work));
	HPLAI_TRY(launch_getrf_tiles(b, a, lda, w, &g_static_epoch, 0, st));
	int s = HPLAI_OK;
	HPLAI_TRY(getrf_status(w, st, &s));
	return s;
}

} // namespace hplai
