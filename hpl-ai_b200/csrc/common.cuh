// common.cuh -- device helpers shared by the libhplai kernels (sm_100a).
//
// LCG arithmetic of the HPL-AI matrix generator (hpl_rand.hpp:8-57 of the
// reference), status plumbing, and thin inline-PTX wrappers for mbarrier,
// TMA (cp.async.bulk.tensor) and tcgen05 (TMEM allocation, UMMA, loads).
// Every spin-wait here is bounded by wall-clock (%globaltimer) and reports a
// timeout instead of hanging.
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <mutex>

#include "../../include/hplai.h"

#define HPLAI_CUDA_TRY(expr)                                   \
	do {                                                       \
		cudaError_t e__ = (expr);                              \
		if (e__ != cudaSuccess) {                              \
			hplai::set_last_cuda_error(e__, #expr, __FILE__, __LINE__); \
			return HPLAI_ECUDA;                                \
		}                                                      \
	} while (0)

#define HPLAI_TRY(expr)                                        \
	do {                                                       \
		int s__ = (expr);                                      \
		if (s__ != HPLAI_OK) return s__;                       \
	} while (0)

namespace hplai {

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);
void set_last_error_message(const char *msg);

// Kernel attributes and occupancy belong to one device: a call site's
// set-up runs the first time the site is reached with each device current
// (under a lock, so concurrent first calls do it once), and its int result
// is cached per device.
struct DeviceOnce {
	static constexpr int kMax = 64;
	std::mutex mu;
	int value[kMax] = {};
	bool done[kMax] = {};
	template <class F> int get(F &&init, int *out = nullptr)
	{
		int dev = 0;
		HPLAI_CUDA_TRY(cudaGetDevice(&dev));
		if (dev < 0 || dev >= kMax) return HPLAI_EUNSUPPORTED;
		std::lock_guard<std::mutex> lk(mu);
		if (!done[dev]) {
			int v = 0;
			HPLAI_TRY(init(dev, &v));
			value[dev] = v;
			done[dev] = true;
		}
		if (out) *out = value[dev];
		return HPLAI_OK;
	}
};

// ---------------------------------------------------------------------------
// LCG x <- a*x + c mod 2^64 (hpl_rand.hpp:8-57).
// ---------------------------------------------------------------------------
struct Coeff {
	uint64_t a, c;
};

constexpr uint64_t kLcgA = 6364136223846793005ULL;
constexpr uint64_t kLcgC = 1ULL;
// int64 -> double scale of the generator: (1 - 2^-53) * 2^-64 (hpl_rand.hpp:51).
constexpr double kValueScale = 0x1.fffffffffffffP-65;

__host__ __device__ __forceinline__ Coeff coeff_mul(Coeff l, Coeff r)
{
	// (l * r)(x) = l(r(x))   hpl_rand.hpp:16-18
	return Coeff{l.a * r.a, l.a * r.c + l.c};
}

__host__ __device__ __forceinline__ uint64_t coeff_apply(Coeff c, uint64_t x) { return c.a * x + c.c; }

// inc1^m by binary powering (the same map as RandCoeff::pow, hpl_rand.hpp:20-32).
__host__ __device__ inline Coeff coeff_pow(uint64_t m)
{
	Coeff r{1ULL, 0ULL};
	Coeff p{kLcgA, kLcgC};
	while (m) {
		if (m & 1ULL) r = coeff_mul(r, p);
		p = coeff_mul(p, p);
		m >>= 1;
	}
	return r;
}

__host__ __device__ __forceinline__ Coeff coeff_pow_of(Coeff base, uint64_t m)
{
	Coeff r{1ULL, 0ULL};
	Coeff p = base;
	while (m) {
		if (m & 1ULL) r = coeff_mul(r, p);
		p = coeff_mul(p, p);
		m >>= 1;
	}
	return r;
}

// state_0 = a*seed + c   (hpl_rand.hpp:38-43)
__host__ __device__ __forceinline__ uint64_t state_initial(uint64_t seed) { return kLcgA * seed + kLcgC; }

// Jump table in shared memory: tab[k] = inc1^(2^k), k < 64.  Filled by the
// first 64 threads; caller synchronises.
__device__ __forceinline__ void jump_table_fill(Coeff *tab)
{
	if (threadIdx.x < 64) {
		Coeff p{kLcgA, kLcgC};
		for (unsigned k = 0; k < threadIdx.x; ++k) p = coeff_mul(p, p);
		tab[threadIdx.x] = p;
	}
}

__device__ __forceinline__ Coeff jump_from_table(const Coeff *tab, uint64_t m)
{
	Coeff r{1ULL, 0ULL};
	for (int k = 0; m; ++k, m >>= 1)
		if (m & 1ULL) r = coeff_mul(r, tab[k]);
	return r;
}

// value = int64(x) * (1-2^-53) * 2^-64, rounded once each step exactly as
// the reference's `static_cast<int64_t>(x) * 0x1.fffffffffffffP-65`.
__device__ __forceinline__ double state_value(uint64_t x)
{
	return __dmul_rn(__ll2double_rn((long long)x), kValueScale);
}

// ---------------------------------------------------------------------------
// Bounded waits.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t global_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// A device wait gives up after this many nanoseconds (2 s) and reports
// HPLAI_ETIMEOUT through the kernel's status word.
constexpr uint64_t kWaitLimitNs = 2000000000ULL;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------------------
// mbarrier
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
		: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}\n"
		: "=r"(ok)
		: "r"(smem_u32(bar)), "r"(parity)
		: "memory");
	return ok != 0;
}

// Waits for the phase with the given parity to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
	if (mbar_try_wait(bar, parity)) return true;
	const uint64_t t0 = global_ns();
	while (true) {
		if (mbar_try_wait(bar, parity)) return true;
		if (global_ns() - t0 > kWaitLimitNs) return false;
	}
}

// ---------------------------------------------------------------------------
// TMA (tiled, no multicast)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tma_prefetch_desc(const void *map)
{
	asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *smem_dst, const void *map, uint64_t *bar, int x, int y)
{
	asm volatile(
		"cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
		::"r"(smem_u32(smem_dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
		: "memory");
}

// L2 prefetch of a tensor box (no shared-memory destination).
__device__ __forceinline__ void tma_prefetch_l2_2d(const void *map, int x, int y)
{
	asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global [%0, {%1, %2}];"
		::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y)
		: "memory");
}

// ---------------------------------------------------------------------------
// tcgen05: tensor memory and UMMA (cta_group::1)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		::"r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem desc] * B[smem desc], kind::f16 (FP16/BF16 in, FP32 acc).
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
	uint32_t accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
		::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
		: "memory");
}

// kind::f8f6f4 (E4M3/E5M2 in, FP32 acc).
__device__ __forceinline__ void umma_f8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
	uint32_t accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n"
		::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
		: "memory");
}

// Arrive on an mbarrier once every previously issued tcgen05.mma of this
// thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
		::"r"(smem_u32(bar)) : "memory");
}

// 32 lanes x 32 consecutive columns of 32-bit TMEM cells into 32 registers
// (lane = warp's lane quarter + laneid).
__device__ __forceinline__ void tmem_ld_32x32b_x32(uint32_t taddr, uint32_t (&r)[32])
{
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x32.b32 "
		"{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
		"%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
		  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
		  "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
		  "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
		: "r"(taddr)
		: "memory");
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// UMMA shared-memory descriptor for a K-major operand tile written by TMA
// with 128-byte swizzle: rows of 128 bytes, 8-row (1024-byte) swizzle atoms
// stacked along M/N.  Fields: start>>4 [0,14), LBO>>4 [16,30) (unused for
// swizzled K-major, 1 by convention), SBO>>4 [32,46) = 1024 B between 8-row
// groups, version 1 [46,48), layout SWIZZLE_128B = 2 [61,64).
__device__ __forceinline__ uint64_t umma_desc_k_sw128(uint32_t smem_addr)
{
	uint64_t d = 0;
	d |= static_cast<uint64_t>((smem_addr >> 4) & 0x3FFFu);
	d |= static_cast<uint64_t>(1u) << 16;
	d |= static_cast<uint64_t>(1024u >> 4) << 32;
	d |= static_cast<uint64_t>(1u) << 46;
	d |= static_cast<uint64_t>(2u) << 61;
	return d;
}

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1),
// A/B FP16 (bits 7-9 / 10-12 = 0), both K-major, N>>3 at [17,23), M>>4 at [24,29).
__host__ __device__ constexpr uint32_t umma_idesc_f16(int m, int n)
{
	return (1u << 4) | (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

// Instruction descriptor, kind::f8f6f4 with E4M3 A and B (formats 0), FP32 acc.
__host__ __device__ constexpr uint32_t umma_idesc_e4m3(int m, int n)
{
	return (1u << 4) | (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

// ---------------------------------------------------------------------------
// CTA pairs (cluster of two, tcgen05 cta_group::2): the leader (rank 0)
// issues MMAs of M = 256 whose operands and accumulator rows are split
// between the two CTAs' shared and tensor memories.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t cluster_rank()
{
	uint32_t r;
	asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
	return r;
}

// The shared::cluster address of the same shared-memory offset in CTA `rank`.
__device__ __forceinline__ uint32_t smem_peer_u32(const void *p, uint32_t rank)
{
	uint32_t r;
	asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
	return r;
}

__device__ __forceinline__ void cluster_sync()
{
	asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Arrive on an mbarrier given by its shared::cluster address (possibly the peer's).
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar)
{
	asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar) : "memory");
}

// TMA load into this CTA's shared memory whose completion is counted on an
// mbarrier of either CTA of the pair (bar: shared::cluster address).
__device__ __forceinline__ void tma_load_2d_pair(void *smem_dst, const void *map, uint32_t bar, int x, int y)
{
	asm volatile(
		"cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
		::"r"(smem_u32(smem_dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
		: "memory");
}

// Executed by one warp in each CTA of the pair: the same columns in both.
__device__ __forceinline__ void tmem_alloc_pair(uint32_t *dst_smem, uint32_t ncols)
{
	asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;"
		::"r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tmem_relinquish_pair()
{
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols)
{
	asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void umma_f16_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
	uint32_t accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
		::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
		: "memory");
}

__device__ __forceinline__ void umma_f8_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
	uint32_t accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n"
		::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
		: "memory");
}

// Arrive on an mbarrier (shared::cluster address: this CTA's or the peer's)
// once the pair's previously issued MMAs have completed.
__device__ __forceinline__ void umma_commit_pair_at(uint32_t bar)
{
	asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];"
		::"r"(bar) : "memory");
}

__device__ __forceinline__ void umma_commit_pair(uint64_t *bar) { umma_commit_pair_at(smem_u32(bar)); }

// The same on the mbarrier at this shared-memory offset in both CTAs of the
// pair (two commits, one per CTA).
__device__ __forceinline__ void umma_commit_pair_both(uint64_t *bar)
{
	umma_commit_pair_at(smem_peer_u32(bar, 0));
	umma_commit_pair_at(smem_peer_u32(bar, 1));
}

// Memory-model helpers for flags exchanged between CTAs of one launch.
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p)
{
	uint32_t v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v)
{
	asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

} // namespace hplai
