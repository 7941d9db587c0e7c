// getrf.cu -- b x b diagonal block LU without pivoting, spread over the GPU.
//
// getrf_nopiv (getrf_nopiv.hpp:30-141) on the diagonal block of each step.
// The block is cut into 32 x 32 tiles; every tile is owned by one warp and
// goes through the steps of a right-looking LU:
//   step r < min(ti, tj):  X -= L(ti, r) U(r, tj)              (trailing update)
//   step r = ti = tj:      X <- LU of X                        (tile factor)
//   step r = tj < ti:      X <- X U(r, r)^{-1}                 (L tile)
//   step r = ti < tj:      X <- L(r, r)^{-1} X  (unit lower)   (U tile)
// A tile that is final publishes a per-tile flag; consumers wait on the
// flags of the tiles they read.  All warps are resident (cooperative
// launch) and each walks its tiles step by step, within a step first the
// diagonal tile, then panel tiles, then trailing updates, so no warp can
// wait on work it has not yet reached and the dataflow always completes; it
// also runs the next step's tile factor as soon as its inputs exist (a
// look-ahead for free).  Every wait is bounded; a timeout sets the status
// word and the warp stops.
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
constexpr int kWarps = 8;
constexpr int kMaxTiles = 32;   // b <= 1024

struct GetrfWork {
	uint32_t status;
	uint32_t pad[31];
	uint32_t flags[kMaxTiles * kMaxTiles];
};

// Wait until *f == epoch; every lane polls, the warp gives up together.
__device__ __forceinline__ bool wait_tile(const uint32_t *f, uint32_t epoch)
{
	if (ld_acquire_u32(f) == epoch) return true;
	const uint64_t t0 = global_ns();
	while (true) {
		if (__all_sync(0xffffffffu, ld_acquire_u32(f) == epoch)) return true;
		if (__any_sync(0xffffffffu, global_ns() - t0 > kWaitLimitNs)) return false;
	}
}

__device__ __forceinline__ void publish(uint32_t *f, uint32_t epoch)
{
	__syncwarp();
	if ((threadIdx.x & 31) == 0) {
		__threadfence();
		st_release_u32(f, epoch);
	}
}

// Tile (rows r0.., cols c0..) -> S[i][j] (rows >= rv or cols >= cv read as 0).
__device__ __forceinline__ void load_tile(float (*S)[T + 1], const float *a, int64_t lda, int r0, int c0, int rv,
	int cv, int lane)
{
#pragma unroll 8
	for (int j = 0; j < T; ++j)
		S[lane][j] = (lane < rv && j < cv) ? __ldcg(&a[static_cast<int64_t>(c0 + j) * lda + r0 + lane]) : 0.f;
}

__device__ __forceinline__ void store_tile(const float (*S)[T + 1], float *a, int64_t lda, int r0, int c0, int rv,
	int cv, int lane)
{
	if (lane < rv) {
#pragma unroll 8
		for (int j = 0; j < T; ++j)
			if (j < cv) a[static_cast<int64_t>(c0 + j) * lda + r0 + lane] = S[lane][j];
	}
}

__global__ void __launch_bounds__(kWarps * 32) getrf_tiles_kernel(int b, float *a, int64_t lda, GetrfWork *w,
	uint32_t epoch)
{
	__shared__ float stage[kWarps][T][T + 1];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	// this warp's staging tile: its own tile (factor, U tile transpose) or the
	// tile it reads (U(r, tj) of an update, the factored diagonal tile)
	float (*S)[T + 1] = stage[warp];
	float (*D)[T + 1] = stage[warp];
	const int wid = blockIdx.x * kWarps + warp, nwarps = gridDim.x * kWarps;
	const int nt = (b + T - 1) / T, ntiles = nt * nt;
	uint32_t *flags = w->flags;
	bool ok = true;

	for (int r = 0; r < nt && ok; ++r) {
		const int k0 = r * T, kv = min(T, b - k0);
		for (int pass = 0; pass < 3 && ok; ++pass) {
			for (int t = wid; t < ntiles && ok; t += nwarps) {
				const int ti = t % nt, tj = t / nt;
				const int mn = min(ti, tj);
				if (mn < r) continue;
				const int kind = (ti == r && tj == r) ? 0 : (mn == r ? 1 : 2);
				if (kind != pass) continue;
				const int r0 = ti * T, c0 = tj * T;
				const int rv = min(T, b - r0), cv = min(T, b - c0);
				if (kind == 2) {
					// X -= L(ti, r) U(r, tj): row `lane` of X and of L in registers, U staged
					if (!wait_tile(&flags[ti + nt * r], epoch) || !wait_tile(&flags[r + nt * tj], epoch)) {
						ok = false;
						break;
					}
					float x[T], l[T];
#pragma unroll
					for (int j = 0; j < T; ++j) {
						x[j] = (lane < rv && j < cv) ? __ldcg(&a[static_cast<int64_t>(c0 + j) * lda + r0 + lane]) : 0.f;
						l[j] = (lane < rv) ? __ldcg(&a[static_cast<int64_t>(k0 + j) * lda + r0 + lane]) : 0.f;
					}
					load_tile(D, a, lda, k0, c0, T, cv, lane);
					__syncwarp();
#pragma unroll
					for (int k = 0; k < T; ++k)
#pragma unroll
						for (int j = 0; j < T; ++j) x[j] = fmaf(-l[k], D[k][j], x[j]);
					if (lane < rv) {
#pragma unroll
						for (int j = 0; j < T; ++j)
							if (j < cv) a[static_cast<int64_t>(c0 + j) * lda + r0 + lane] = x[j];
					}
					__syncwarp();
				} else if (kind == 0) {
					// unblocked LU of the diagonal tile (getrf_nopiv_small order)
					load_tile(S, a, lda, r0, c0, rv, cv, lane);
					__syncwarp();
					for (int k = 0; k < kv; ++k) {
						const float inv = 1.0f / S[k][k];
						if (lane > k && lane < kv) {
							const float lik = S[lane][k] * inv;
							S[lane][k] = lik;
							for (int j = k + 1; j < kv; ++j) S[lane][j] = fmaf(-lik, S[k][j], S[lane][j]);
						}
						__syncwarp();
					}
					store_tile(S, a, lda, r0, c0, rv, cv, lane);
					publish(&flags[t], epoch);
				} else if (tj == r) {
					// L tile: X <- X U(r,r)^{-1}, row `lane` of X in registers
					float x[T];
#pragma unroll
					for (int j = 0; j < T; ++j)
						x[j] = (lane < rv && j < kv) ? __ldcg(&a[static_cast<int64_t>(c0 + j) * lda + r0 + lane]) : 0.f;
					if (!wait_tile(&flags[r + nt * r], epoch)) {
						ok = false;
						break;
					}
					load_tile(D, a, lda, k0, k0, kv, kv, lane);
					__syncwarp();
#pragma unroll
					for (int j = 0; j < T; ++j) {
						if (j < kv) {
							x[j] *= 1.0f / D[j][j];
#pragma unroll
							for (int q = j + 1; q < T; ++q) x[q] = fmaf(-x[j], D[j][q], x[q]);
						}
					}
					if (lane < rv) {
#pragma unroll
						for (int j = 0; j < T; ++j)
							if (j < kv) a[static_cast<int64_t>(c0 + j) * lda + r0 + lane] = x[j];
					}
					publish(&flags[t], epoch);
				} else {
					// U tile: X <- L(r,r)^{-1} X, column `lane` of X in registers
					load_tile(S, a, lda, r0, c0, kv, cv, lane);
					__syncwarp();
					float y[T];
#pragma unroll
					for (int i = 0; i < T; ++i) y[i] = S[i][lane];
					__syncwarp();
					if (!wait_tile(&flags[r + nt * r], epoch)) {
						ok = false;
						break;
					}
					load_tile(D, a, lda, k0, k0, kv, kv, lane);
					__syncwarp();
#pragma unroll
					for (int k = 0; k < T; ++k) {
						if (k < kv) {
#pragma unroll
							for (int i = k + 1; i < T; ++i) y[i] = fmaf(-y[k], D[i][k], y[i]);
						}
					}
					__syncwarp();
#pragma unroll
					for (int i = 0; i < T; ++i) S[i][lane] = y[i];
					__syncwarp();
					store_tile(S, a, lda, r0, c0, kv, cv, lane);
					publish(&flags[t], epoch);
				}
			}
		}
	}
	if (!ok && lane == 0) atomicOr(&w->status, 1u);
}

std::mutex g_static_mu;
__device__ GetrfWork g_static_work;
uint32_t g_static_epoch = 0;

int max_coresident_ctas()
{
	static int cached = 0;
	if (!cached) {
		int per_sm = 0, dev = 0, sms = 0;
		HPLAI_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, getrf_tiles_kernel, kWarps * 32, 0));
		HPLAI_CUDA_TRY(cudaGetDevice(&dev));
		HPLAI_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
		cached = per_sm * sms;
	}
	return cached;
}

} // namespace

size_t getrf_workspace() { return sizeof(GetrfWork); }

int launch_getrf_tiles(int b, float *a, int64_t lda, void *work, uint32_t *epoch, int max_ctas, cudaStream_t st)
{
	if (b <= 0) return HPLAI_OK;
	if (b > T * kMaxTiles || !a || lda < b || !work || !epoch) return HPLAI_EINVAL;
	const int nt = (b + T - 1) / T;
	int grid = (nt * nt + kWarps - 1) / kWarps;
	const int cap = max_coresident_ctas();
	if (cap <= 0) return HPLAI_EUNSUPPORTED;
	if (grid > cap) grid = cap;
	if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
	GetrfWork *w = static_cast<GetrfWork *>(work);
	uint32_t ep = ++*epoch;
	if (ep == 0) ep = ++*epoch;   // flags start zeroed: never wait for 0
	void *args[] = {(void *)&b, (void *)&a, (void *)&lda, (void *)&w, (void *)&ep};
	HPLAI_CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<void *>(getrf_tiles_kernel), dim3(grid),
		dim3(kWarps * 32), args, 0, st));
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
