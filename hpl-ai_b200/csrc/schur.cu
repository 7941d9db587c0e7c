// schur.cu -- the Schur complement update C -= L * U on tcgen05 tensor cores.
//
// The reference's gemmschur -> shgemm (schur_updator.hpp:24-31,
// fp16sim.hpp:216-233, kernels/avx2.cpp:249-302) multiplies FP16 panels
// and accumulates in FP32 into the FP32 trailing matrix.  Here one
// persistent, warp-specialised kernel does the same on sm_100a:
//
//   warp 0      TMA producer: 128x64 (L) and 256x64 (U) FP16 tiles, 128B
//               swizzle, into a 4-stage shared-memory ring.  (An L2 prefetch
//               of the C tile ahead of its epilogue measured 34-42% slower.)
//   warp 1      allocates 512 TMEM columns (two 128x256 FP32 accumulators)
//               and one elected thread issues tcgen05.mma (M=128, N=256,
//               K=16, kind::f16); tcgen05.commit releases ring stages and
//               publishes finished accumulators.
//   warps 2-5   epilogue: tcgen05.ld of the accumulator (lane = row), -acc
//               to shared memory and a TMA reduce-add into C (FP32, in L2);
//               when C's rows are not 16-byte aligned, C = C - acc with
//               coalesced loads and stores instead.
//
// The accumulator is double buffered so the epilogue of tile i overlaps
// the MMAs of tile i+1.  Every wait is bounded; a timeout sets the status
// word and the kernel drains and frees TMEM before returning.
#include "common.cuh"
#include "internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <atomic>
#include <cstring>

namespace hplai {

namespace {

constexpr int BM = 128;
constexpr int BN = 256;
constexpr int BK = 64;                 // one 128-byte swizzle row of FP16 (128 FP8 values)
// Pipeline shape (build-time tunables): operand stages, epilogue warps (4,
// or 8 = two per TMEM lane quarter, each taking half of the tile's
// columns) and staging buffers per epilogue warp.
#ifndef HPLAI_SCHUR_STAGES
#define HPLAI_SCHUR_STAGES 4
#endif
#ifndef HPLAI_SCHUR_EPI_WARPS
#define HPLAI_SCHUR_EPI_WARPS 4
#endif
#ifndef HPLAI_SCHUR_EPI_BUFS
#define HPLAI_SCHUR_EPI_BUFS 2
#endif
// Reduce box: 32 rows (one warp's TMEM quarter) or the tile's full 128 rows
// (the four epilogue warps stage one chunk together; 512-byte column runs).
#ifndef HPLAI_SCHUR_TALL_BOX
#define HPLAI_SCHUR_TALL_BOX 1
#endif
#ifndef HPLAI_SCHUR_EPI_CHUNK
#define HPLAI_SCHUR_EPI_CHUNK 32
#endif
constexpr int STAGES = HPLAI_SCHUR_STAGES;
constexpr int A_BYTES = BM * BK * 2;   // 16 KB
constexpr int B_BYTES = BN * BK * 2;   // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int EPI_WARPS = HPLAI_SCHUR_EPI_WARPS;
constexpr int EPI_BUFS = HPLAI_SCHUR_EPI_BUFS;
constexpr int EPI_SPLIT = EPI_WARPS / 4;            // warps per TMEM lane quarter
constexpr int EPI_COLS = BN / EPI_SPLIT;            // accumulator columns per epilogue warp
static_assert(EPI_WARPS == 4 || EPI_WARPS == 8, "one or two epilogue warps per lane quarter");
constexpr uint32_t TMEM_COLS = 2 * BN;
constexpr bool TALL = HPLAI_SCHUR_TALL_BOX != 0;
constexpr int EPI_CHUNK = HPLAI_SCHUR_EPI_CHUNK;    // columns per epilogue chunk
constexpr int EPI_BUF_BYTES = 32 * EPI_CHUNK * 4;   // one warp's 32 rows x EPI_CHUNK columns FP32
static_assert(!TALL || EPI_WARPS == 4, "the tall box is staged by the four lane-quarter warps");
static_assert(TALL || EPI_CHUNK == 32, "per-warp boxes are 32 x 32");
constexpr size_t RED_BYTES = static_cast<size_t>(EPI_WARPS) * EPI_BUFS * EPI_BUF_BYTES;   // = BM x EPI_CHUNK x EPI_BUFS when tall
// DECK epilogue: FP16 trailing matrix, chunks of 128 rows x DECK_CH columns
// loaded by TMA into a ring of DECK_BUFS buffers, updated and stored back.
// 64-column chunks with five buffers and three operand stages measured
// fastest at n = 65536, b = 512 (trailing update 220 ms against 280 ms for
// 32-column chunks with ten buffers).
#ifndef HPLAI_DECK_CH
#define HPLAI_DECK_CH 64
#endif
#ifndef HPLAI_DECK_BUFS
#define HPLAI_DECK_BUFS 5
#endif
#ifndef HPLAI_DECK_STAGES
#define HPLAI_DECK_STAGES 3
#endif
// Epilogue warps of the deck kernel: 8 = two per TMEM lane quarter, each
// taking half of every chunk's columns (the update is a few instructions per
// element, so one warp per SM sub-partition cannot keep up with the MMAs:
// 8 warps took the e4m3 trailing update at n = 131072, b = 1024 from 1.39 s
// to 0.98 s).
#ifndef HPLAI_DECK_EPI_WARPS
#define HPLAI_DECK_EPI_WARPS 8
#endif
constexpr int DECK_CH = HPLAI_DECK_CH;
constexpr int DECK_BUFS = HPLAI_DECK_BUFS;      // DECK_BUFS - 1 chunk loads in flight per SM
constexpr int DECK_STAGES = HPLAI_DECK_STAGES;  // operand stages of the deck kernel (its chunk ring takes the rest)
constexpr int DECK_EPI_WARPS = HPLAI_DECK_EPI_WARPS;
constexpr int DECK_CW = DECK_CH / (DECK_EPI_WARPS / 4);   // chunk columns per deck epilogue warp
static_assert(DECK_EPI_WARPS == 4 || DECK_EPI_WARPS == 8, "one or two deck epilogue warps per lane quarter");
static_assert(DECK_CW % 32 == 0 && BN % DECK_CH == 0, "deck chunks are whole 32-column TMEM loads per warp");
constexpr uint32_t DECK_CHUNK_BYTES = BM * DECK_CH * 2;
constexpr size_t DECK_BYTES = static_cast<size_t>(DECK_BUFS) * DECK_CHUNK_BYTES;
// epilogue kinds: 0 direct (plain loads/stores of FP32 C), 1 TMA reduce-add
// into FP32 C, 2 FP16 deck (load, update, store)
__host__ __device__ constexpr size_t epi_bytes(int epi) { return epi == 1 ? RED_BYTES : (epi == 2 ? DECK_BYTES : 0); }
__host__ __device__ constexpr int stages_for(int epi) { return epi == 2 ? DECK_STAGES : STAGES; }
__host__ __device__ constexpr int epi_warps_for(int epi) { return epi == 2 ? DECK_EPI_WARPS : EPI_WARPS; }
__host__ __device__ constexpr int threads_for(int epi) { return (2 + epi_warps_for(epi)) * 32; }
constexpr size_t smem_bytes(int epi)
{
	return static_cast<size_t>(stages_for(epi)) * STAGE_BYTES + epi_bytes(epi) + 1024 + 256;
}
static_assert(smem_bytes(2) <= 232448 && smem_bytes(1) <= 232448, "shared memory per CTA");

static_assert(TMEM_COLS <= 512, "two accumulators must fit in TMEM");

struct Params {
	float *c;
	int64_t ldc;
	int m, n;
	int num_kc;       // K chunks of BK
	int lrow0, urow0; // first L row / first U row (= C column) in the panel buffers
	int tiles_m, tiles_n;
	int crow0, ccol0; // coordinates of C(0,0) in the C tensor map (reduce epilogue)
	// FP8 operands: power-of-two dequantisation factors per 128 rows of L
	// (sl, block 0 starting at L row sl0) and per 128 columns of U (su, su0).
	const float *sl, *su;
	int sl0, su0;
	unsigned *status;   // set to 1 on a wait timeout
	float dscale;       // DECK: the deck holds dscale x (accumulated update)
	// Store form of the reduce epilogue (FP16 operands only): C = acc * *oscale
	// written by TMA store instead of C -= acc (null: the update)
	const float *oscale;
	// Batched form (FP16 operands, reduce epilogue): `ntiles` tiles whose L
	// row, U row, C row and C column come from this table instead of the
	// region's tile grid -- the tiles of many systems' updates in one launch.
	const int4 *tiles;
	int ntiles;
	int group_m;        // tile rows per group of the tile order (tile_coords)
	// Store form: block maxima of the written values (AmaxTargets)
	unsigned *amax_bits[2];
	int amax_base[2];
	int amax_dim;
};

__device__ unsigned int g_status;

// Tile order: groups of group_m tile rows (kGroupM unless the context's
// tuner chose another), each group swept column by column (tile rows
// fastest).  The CTAs in flight then share a few U blocks and the group's L
// blocks stay in L2 while the group crosses all tile columns, so each panel
// is read from HBM about once per group instead of once per tile column (the
// L panel alone is 256 MB at n = 131072, b = 1024).
constexpr int kGroupM = 32;

__device__ __forceinline__ void tile_coords(int tile, int tiles_m, int tiles_n, int group_m, int &tm, int &tn)
{
	const int per_group = group_m * tiles_n;
	const int g = tile / per_group;
	const int first = g * group_m;
	const int gm = min(group_m, tiles_m - first);
	const int in = tile - g * per_group;
	tm = first + in % gm;
	tn = in / gm;
}

__device__ __forceinline__ void tma_store_2d(const void *map, const void *smem_src, int x, int y)
{
	asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];"
		::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(smem_src)), "r"(x), "r"(y)
		: "memory");
}

// AND over the NW epilogue warps (named barrier 1), so that they take the same branch.
template <int NW = EPI_WARPS>
__device__ __forceinline__ bool epi_all(bool mine)
{
	int all_ok;
	asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\t"
	             "bar.red.and.pred q, 1, %2, p;\n\tselp.s32 %0, 1, 0, q;\n\t}"
	             : "=r"(all_ok) : "r"(mine ? 1 : 0), "n"(NW * 32) : "memory");
	return all_ok != 0;
}

// FP8: dequantisation factors of the 32 C columns c0 .. c0 + 31 of this
// launch (U rows urow0 + c0 ..).  When they share one 128-row block of U
// (always, for panels whose blocks start on a multiple of 32) the factor is
// returned in `uni` with true; otherwise lane j's `mine` is column c0 + j's
// factor.  Columns past n take the last column's block: the clipped C maps
// never store them.
__device__ __forceinline__ bool col_factors(const Params &p, int c0, int lane, float &uni, float &mine)
{
	const int a = (p.urow0 + min(c0, p.n - 1) - p.su0) >> 7;
	const int b = (p.urow0 + min(c0 + 31, p.n - 1) - p.su0) >> 7;
	if (a == b) {
		uni = __ldg(&p.su[a]);
		return true;
	}
	mine = __ldg(&p.su[(p.urow0 + min(c0 + lane, p.n - 1) - p.su0) >> 7]);
	return false;
}

__device__ __forceinline__ void tma_reduce_add_2d(const void *map, const void *smem_src, int x, int y)
{
	asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.bulk_group [%0, {%2, %3}], [%1];"
		::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(smem_src)), "r"(x), "r"(y)
		: "memory");
}

// RED: the epilogue writes -acc to shared memory and a TMA reduce-add folds
// it into C in L2 (C never passes through the SM); otherwise the epilogue
// loads C, subtracts and stores with plain coalesced accesses.
// FP8: e4m3 operands (kind::f8f6f4, K = 32 per MMA, 128 per 128-byte row)
// with the accumulator multiplied by the two blocks' power-of-two factors
// in the epilogue (exact); otherwise FP16 operands (kind::f16).
// DECK: C is an FP16 deck holding dscale x (the accumulated update); each
// chunk is loaded by TMA, deck - dscale * acc is rounded to FP16 once and
// stored back by TMA (the precision form's trailing matrix, half the bytes).
template <int EPI, bool FP8>
__global__ void __launch_bounds__(threads_for(EPI), 1) schur_kernel(const __grid_constant__ CUtensorMap lmap,
	const __grid_constant__ CUtensorMap umap, const __grid_constant__ CUtensorMap cmap, const Params p)
{
	constexpr bool RED = EPI == 1, DECK = EPI == 2;
	constexpr int NST = stages_for(EPI);   // operand ring stages
	constexpr int NW = epi_warps_for(EPI); // epilogue warps
	extern __shared__ uint8_t smem_raw[];
	const uint32_t raw_addr = smem_u32(smem_raw);
	uint8_t *smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
	uint8_t *sA = smem;
	uint8_t *sB = smem + NST * A_BYTES;
	float *sEpi = reinterpret_cast<float *>(smem + NST * STAGE_BYTES);   // RED staging / DECK chunks
	uint64_t *bars = reinterpret_cast<uint64_t *>(smem + NST * STAGE_BYTES + epi_bytes(EPI));
	uint64_t *full = bars;
	uint64_t *empty = bars + NST;
	uint64_t *accf = bars + 2 * NST;
	uint64_t *acce = accf + 2;
	uint64_t *drain = acce + 2;
	uint64_t *dbar = drain + 1;   // DECK chunk loads
	uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(dbar + DECK_BUFS);
	int *consumed = reinterpret_cast<int *>(tmem_holder + 1);   // stages the MMA warp consumed

	const int warp = threadIdx.x >> 5;
	const int lane = threadIdx.x & 31;

	if (threadIdx.x == 0) {
		for (int s = 0; s < NST; ++s) {
			mbar_init(&full[s], 1);
			mbar_init(&empty[s], 1);
		}
		for (int a = 0; a < 2; ++a) {
			mbar_init(&accf[a], 1);
			mbar_init(&acce[a], NW * 32);
		}
		mbar_init(drain, 1);
		for (int b = 0; b < DECK_BUFS; ++b) mbar_init(&dbar[b], 1);
		*consumed = 0;
		fence_mbar_init();
	}
	if (warp == 1) {
		tmem_alloc(tmem_holder, TMEM_COLS);
		tmem_relinquish();
	}
	if (warp == 0 && lane == 0) {
		tma_prefetch_desc(&lmap);
		tma_prefetch_desc(&umap);
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem_base = *tmem_holder;

	const int total = p.tiles ? p.ntiles : p.tiles_m * p.tiles_n;
	int issued = 0;   // producer: stages issued

	if (warp == 0) {
		// ---------------- TMA producer ----------------
		bool ok = true;
		int stage = 0;
		uint32_t phase = 0;
		for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
			int lrow, urow;
			if (p.tiles) {
				const int4 t = p.tiles[tile];
				lrow = t.x;
				urow = t.y;
			} else {
				int tm, tn;
				tile_coords(tile, p.tiles_m, p.tiles_n, p.group_m, tm, tn);
				lrow = p.lrow0 + tm * BM;
				urow = p.urow0 + tn * BN;
			}
			if (lane == 0) {
				for (int kc = 0; kc < p.num_kc; ++kc) {
					if (!mbar_wait(&empty[stage], phase ^ 1u)) { ok = false; break; }
					mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
					// K offset of this stage in elements: 64 FP16 or 128 FP8 per 128-byte row
					const int kx = kc * (FP8 ? 2 * BK : BK);
					tma_load_2d(sA + stage * A_BYTES, &lmap, &full[stage], kx, lrow);
					tma_load_2d(sB + stage * B_BYTES, &umap, &full[stage], kx, urow);
					++issued;
					if (++stage == NST) { stage = 0; phase ^= 1u; }
				}
			}
			ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
		}
		if (lane == 0 && !ok) atomicOr(p.status, 1u);
	} else if (warp == 1) {
		// ---------------- MMA issuer ----------------
		if (lane == 0) {
			bool ok = true;
			int stage = 0;
			uint32_t phase = 0;
			int acc = 0;
			uint32_t acc_phase = 0;
			int used = 0;
			const uint32_t idesc = umma_idesc_f16(BM, BN);
			for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
				if (!mbar_wait(&acce[acc], acc_phase ^ 1u)) { ok = false; break; }
				tc_fence_after();
				const uint32_t d_tmem = tmem_base + static_cast<uint32_t>(acc * BN);
				for (int kc = 0; kc < p.num_kc; ++kc) {
					if (!mbar_wait(&full[stage], phase)) { ok = false; break; }
					tc_fence_after();
					const uint64_t adesc = umma_desc_k_sw128(smem_u32(sA + stage * A_BYTES));
					const uint64_t bdesc = umma_desc_k_sw128(smem_u32(sB + stage * B_BYTES));
#pragma unroll
					for (int kk = 0; kk < 4; ++kk) {
						// advance 32 bytes (2 units of 16 B) along K inside the 128-byte swizzle row:
						// 16 FP16 or 32 FP8 values per MMA
						if (FP8)
							umma_f8(d_tmem, adesc + 2u * kk, bdesc + 2u * kk, idesc, (kc | kk) != 0 ? 1u : 0u);
						else
							umma_f16(d_tmem, adesc + 2u * kk, bdesc + 2u * kk, idesc, (kc | kk) != 0 ? 1u : 0u);
					}
					umma_commit(&empty[stage]);
					++used;
					if (++stage == NST) { stage = 0; phase ^= 1u; }
				}
				if (!ok) break;
				umma_commit(&accf[acc]);
				if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
			}
			// Every MMA of this thread completes before TMEM is released.
			umma_commit(drain);
			if (!mbar_wait(drain, 0)) ok = false;
			*consumed = used;
			if (!ok) atomicOr(p.status, 1u);
		}
	} else if (DECK) {
		// ---------------- FP16 deck epilogue ----------------
		// A rolling pipeline over this CTA's chunk sequence (its tiles in order,
		// BN / DECK_CH chunks each): warp 2's lane 0 keeps DECK_BUFS loads ahead.
		// Warp w updates TMEM lane quarter w & 3 (rows) and, with 8 warps, one
		// half of each chunk's columns.
		constexpr int CPT = BN / DECK_CH;
		const int q = warp & 3;
		const int cw0 = ((warp - 2) >> 2) * DECK_CW;   // first chunk column of this warp
		__half *dbuf = reinterpret_cast<__half *>(sEpi);
		const bool lead = (warp == 2 && lane == 0);
		const int my_tiles = (blockIdx.x < total) ? (total - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
		const int nseq = my_tiles * CPT;
		auto chunk_xy = [&](int sidx, int &x, int &y) {
			int tm, tn;
			tile_coords(blockIdx.x + (sidx / CPT) * gridDim.x, p.tiles_m, p.tiles_n, p.group_m, tm, tn);
			x = p.crow0 + tm * BM;
			y = p.ccol0 + tn * BN + (sidx % CPT) * DECK_CH;
		};
		int issued = 0;
		if (lead) {
			for (; issued < DECK_BUFS - 1 && issued < nseq; ++issued) {
				int x, y;
				chunk_xy(issued, x, y);
				mbar_arrive_expect_tx(&dbar[issued % DECK_BUFS], DECK_CHUNK_BYTES);
				tma_load_2d(dbuf + (issued % DECK_BUFS) * (BM * DECK_CH), &cmap, &dbar[issued % DECK_BUFS], x, y);
			}
		}
		bool ok = true;
		int acc = 0;
		uint32_t acc_phase = 0;
		int sidx = 0;
		for (int it = 0; it < my_tiles && ok; ++it) {
			int tm, tn;
			tile_coords(blockIdx.x + it * gridDim.x, p.tiles_m, p.tiles_n, p.group_m, tm, tn);
			ok = epi_all<NW>(mbar_wait(&accf[acc], acc_phase));
			if (!ok) break;
			tc_fence_after();
			const uint32_t tbase = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * BN);
			// this lane's row factor: dscale, times the row block's factor for FP8
			// (rows past m read the last row's block; never stored)
			float rf = p.dscale;
			if (FP8) rf *= p.sl[(p.lrow0 + min(tm * BM + q * 32 + lane, p.m - 1) - p.sl0) >> 7];
#pragma unroll 1
			for (int ch = 0; ch < CPT; ++ch, ++sidx) {
				const int bi = sidx % DECK_BUFS;
				ok = epi_all<NW>(mbar_wait(&dbar[bi], static_cast<uint32_t>((sidx / DECK_BUFS) & 1)));
				if (!ok) break;
#pragma unroll
				for (int g = 0; g < DECK_CW / 32; ++g) {
					const int cc = ch * DECK_CH + cw0 + 32 * g;   // tile column of this group
					uint32_t r[32];
					tmem_ld_32x32b_x32(tbase + static_cast<uint32_t>(cc), r);
					// element (row, j) of the chunk at j * BM + row; the deck values are
					// read while the accumulator load is in flight
					__half *sb = dbuf + bi * (BM * DECK_CH) + (cw0 + 32 * g) * BM + q * 32 + lane;
					float d[32];
#pragma unroll
					for (int j = 0; j < 32; ++j) d[j] = __half2float(sb[j * BM]);
					float fu = rf, fl = 0.f;
					const bool uni = FP8 ? col_factors(p, tn * BN + cc, lane, fu, fl) : true;
					if (FP8 && uni) fu *= rf;
					tmem_ld_wait();
					if (uni) {
#pragma unroll
						for (int j = 0; j < 32; ++j) sb[j * BM] = __float2half_rn(d[j] - __uint_as_float(r[j]) * fu);
					} else {
#pragma unroll
						for (int j = 0; j < 32; ++j) {
							const float f = rf * __shfl_sync(0xffffffffu, fl, j);
							sb[j * BM] = __float2half_rn(d[j] - __uint_as_float(r[j]) * f);
						}
					}
				}
				asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
				asm volatile("bar.sync 1, %0;" ::"n"(NW * 32) : "memory");
				if (lead) {
					int x, y;
					chunk_xy(sidx, x, y);
					tma_store_2d(&cmap, dbuf + bi * (BM * DECK_CH), x, y);
					asm volatile("cp.async.bulk.commit_group;" ::: "memory");
					if (issued < nseq) {
						// chunk sidx + DECK_BUFS - 1 goes into the buffer of chunk sidx - 1,
						// whose store (one group back) has read it
						const int nb2 = issued % DECK_BUFS;
						asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
						chunk_xy(issued, x, y);
						mbar_arrive_expect_tx(&dbar[nb2], DECK_CHUNK_BYTES);
						tma_load_2d(dbuf + nb2 * (BM * DECK_CH), &cmap, &dbar[nb2], x, y);
						++issued;
					}
				}
			}
			if (!ok) break;
			tc_fence_before();
			mbar_arrive(&acce[acc]);
			if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
		}
		if (lead) {
			asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
			// loads issued but never consumed (only after a timeout) land before exit
			for (int s2 = sidx; s2 < issued; ++s2)
				(void)mbar_wait(&dbar[s2 % DECK_BUFS], static_cast<uint32_t>((s2 / DECK_BUFS) & 1));
		}
		if (lane == 0 && !ok) atomicOr(p.status, 1u);
	} else {
		// ---------------- epilogue ----------------
		const int q = warp & 3;   // TMEM lane quarter this warp may access
		const int cbase = ((warp - 2) / 4) * EPI_COLS;   // first accumulator column of this warp
		bool ok = true;
		int acc = 0;
		uint32_t acc_phase = 0;
		int epi_buf = 0;
		for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
			int tm = 0, tn = 0, crow, ccol;
			if (p.tiles) {
				const int4 t = p.tiles[tile];
				crow = t.z;
				ccol = t.w;
			} else {
				tile_coords(tile, p.tiles_m, p.tiles_n, p.group_m, tm, tn);
				crow = p.crow0 + tm * BM;
				ccol = p.ccol0 + tn * BN;
			}
			// the epilogue warps decide together (their named barriers must not split)
			ok = epi_all(mbar_wait(&accf[acc], acc_phase));
			if (!ok) break;
			tc_fence_after();
			const uint32_t tbase = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * BN);
			// FP8: this lane's row factor (rows past the panel end read block 0; never stored)
			float rs = 1.f;
			if (FP8) {
				const int lr = p.lrow0 + tm * BM + q * 32 + lane - p.sl0;
				rs = (tm * BM + q * 32 + lane < p.m) ? p.sl[lr >> 7] : 0.f;
			}
			if (RED && TALL) {
				const bool issuer = (warp == 2 && lane == 0);
				// store form: |value| maxima of this lane's row over the tile's
				// two 128-column halves (values past the region are exact zeros)
				float vmax[2] = {0.f, 0.f};
#pragma unroll 1
				for (int ch = 0; ch < BN / EPI_CHUNK; ++ch) {
					const int cc = ch * EPI_CHUNK;
					float *sb = sEpi + (epi_buf % EPI_BUFS) * (BM * EPI_CHUNK);
					// the reduce issued EPI_BUFS chunks ago read this buffer; let it finish
					if (issuer) asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(EPI_BUFS - 1) : "memory");
					asm volatile("bar.sync 1, %0;" ::"n"(EPI_WARPS * 32) : "memory");
#pragma unroll
					for (int half = 0; half < EPI_CHUNK / 32; ++half) {
						uint32_t r[32];
						tmem_ld_32x32b_x32(tbase + static_cast<uint32_t>(cc + 32 * half), r);
						tmem_ld_wait();
						if (FP8) {
							float fu = 0.f, fl = 0.f;
							if (col_factors(p, tn * BN + cc + 32 * half, lane, fu, fl)) {
								fu *= rs;
#pragma unroll
								for (int j = 0; j < 32; ++j) sb[(32 * half + j) * BM + q * 32 + lane] = -(__uint_as_float(r[j]) * fu);
							} else {
#pragma unroll
								for (int j = 0; j < 32; ++j)
									sb[(32 * half + j) * BM + q * 32 + lane] =
										-(__uint_as_float(r[j]) * (rs * __shfl_sync(0xffffffffu, fl, j)));
							}
						} else if (p.oscale) {
							const float os = *p.oscale;
							float m = 0.f;
#pragma unroll
							for (int j = 0; j < 32; ++j) {
								const float v = __uint_as_float(r[j]) * os;
								sb[(32 * half + j) * BM + q * 32 + lane] = v;
								m = fmaxf(m, fabsf(v));
							}
							vmax[(cc + 32 * half) >> 7] = fmaxf(vmax[(cc + 32 * half) >> 7], m);
						} else {
#pragma unroll
							for (int j = 0; j < 32; ++j) sb[(32 * half + j) * BM + q * 32 + lane] = -__uint_as_float(r[j]);
						}
					}
					asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
					asm volatile("bar.sync 1, %0;" ::"n"(EPI_WARPS * 32) : "memory");
					if (issuer) {
						if (!FP8 && p.oscale)
							tma_store_2d(&cmap, sb, crow, ccol + cc);
						else
							tma_reduce_add_2d(&cmap, sb, crow, ccol + cc);
						asm volatile("cp.async.bulk.commit_group;" ::: "memory");
					}
					++epi_buf;
				}
				if (!FP8 && p.oscale && (p.amax_bits[0] || p.amax_bits[1])) {
					// dim 0: the tile's 128 rows are one block, every lane's row
					// max over both halves; dim 1: one block per 128-column half,
					// the max over this warp's 32 rows
					if (p.amax_dim == 0) vmax[0] = fmaxf(vmax[0], vmax[1]);
#pragma unroll
					for (int o = 16; o; o >>= 1) {
						vmax[0] = fmaxf(vmax[0], __shfl_xor_sync(0xffffffffu, vmax[0], o));
						vmax[1] = fmaxf(vmax[1], __shfl_xor_sync(0xffffffffu, vmax[1], o));
					}
					if (lane == 0) {
#pragma unroll
						for (int t2 = 0; t2 < 2; ++t2) {
							if (!p.amax_bits[t2]) continue;
							if (p.amax_dim == 0) {
								const int r0 = tm * BM - p.amax_base[t2];
								if (r0 >= 0) atomicMax(&p.amax_bits[t2][r0 >> 7], __float_as_uint(vmax[0]));
							} else {
#pragma unroll
								for (int h = 0; h < 2; ++h) {
									const int c0 = tn * BN + 128 * h - p.amax_base[t2];
									if (c0 >= 0 && tn * BN + 128 * h < p.n)
										atomicMax(&p.amax_bits[t2][c0 >> 7], __float_as_uint(vmax[h]));
								}
							}
						}
					}
				}
			} else if (RED) {
				float *mybuf = sEpi + (warp - 2) * EPI_BUFS * (EPI_BUF_BYTES / 4);
				const int gx = p.crow0 + tm * BM + q * 32;   // tensor-map row of this warp's lane 0
#pragma unroll 1
				for (int ch = 0; ch < EPI_COLS / EPI_CHUNK; ++ch) {
					const int cc = cbase + ch * EPI_CHUNK;   // accumulator column of the chunk
					uint32_t r[32];
					tmem_ld_32x32b_x32(tbase + static_cast<uint32_t>(cc), r);
					tmem_ld_wait();
					float *sb = mybuf + (epi_buf % EPI_BUFS) * (EPI_BUF_BYTES / 4);
					// the reduce issued EPI_BUFS chunks ago read this buffer; let it finish
					if (lane == 0) asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(EPI_BUFS - 1) : "memory");
					__syncwarp();
					if (FP8) {
						float fu = 0.f, fl = 0.f;
						if (col_factors(p, tn * BN + cc, lane, fu, fl)) {
							fu *= rs;
#pragma unroll
							for (int j = 0; j < 32; ++j) sb[j * 32 + lane] = -(__uint_as_float(r[j]) * fu);
						} else {
#pragma unroll
							for (int j = 0; j < 32; ++j)
								sb[j * 32 + lane] = -(__uint_as_float(r[j]) * (rs * __shfl_sync(0xffffffffu, fl, j)));
						}
					} else {
#pragma unroll
						for (int j = 0; j < 32; ++j) sb[j * 32 + lane] = -__uint_as_float(r[j]);
					}
					asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
					__syncwarp();
					if (lane == 0) {
						tma_reduce_add_2d(&cmap, sb, gx, p.ccol0 + tn * BN + cc);
						asm volatile("cp.async.bulk.commit_group;" ::: "memory");
					}
					++epi_buf;
				}
			} else {
				const int row = tm * BM + q * 32 + lane;
				const bool rok = row < p.m;
				float *crow = p.c + row;
#pragma unroll 1
				for (int ch = 0; ch < EPI_COLS / 32; ++ch) {
					uint32_t r[32];
					tmem_ld_32x32b_x32(tbase + static_cast<uint32_t>(cbase + ch * 32), r);
					tmem_ld_wait();
					const int col0 = tn * BN + cbase + ch * 32;
					if (rok) {
						float cv[32];
#pragma unroll
						for (int j = 0; j < 32; ++j)
							if (col0 + j < p.n) cv[j] = crow[static_cast<int64_t>(col0 + j) * p.ldc];
#pragma unroll
						for (int j = 0; j < 32; ++j) {
							if (col0 + j < p.n) {
								float v = __uint_as_float(r[j]);
								if (FP8) v *= rs * __ldg(&p.su[(p.urow0 + col0 + j - p.su0) >> 7]);
								crow[static_cast<int64_t>(col0 + j) * p.ldc] = cv[j] - v;
							}
						}
					}
				}
			}
			tc_fence_before();
			mbar_arrive(&acce[acc]);
			if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
		}
		// all reduces of this warp complete before the CTA exits
		if (RED && lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
		if (lane == 0 && !ok) atomicOr(p.status, 1u);
	}

	tc_fence_before();
	__syncthreads();
	if (warp == 0 && lane == 0) {
		// Loads issued but never consumed (only after a timeout) land before exit.
		int left = issued - *consumed;
		for (int s = 0; left > 0 && s < NST; ++s, --left) {
			(void)mbar_wait(&full[(*consumed + s) % NST], static_cast<uint32_t>(((*consumed + s) / NST) & 1));
		}
	}
	if (warp == 1) {
		tc_fence_after();
		tmem_dealloc(tmem_base, TMEM_COLS);
	}
}

// ---------------------------------------------------------------------------
// The deck update on CTA pairs (tcgen05 cta_group::2).  A cluster of two CTAs
// owns a 256 x 256 tile: CTA r loads rows 128 r .. 128 r + 127 of the tile's
// L block and of its U block (16 KB each per stage), the leader (r = 0)
// issues M = 256, N = 256 MMAs that read both CTAs' shared memory, and each
// CTA's tensor memory receives its 128 rows of the accumulator.  Per stage an
// SM then loads 32 KB for the MMA work that costs 48 KB in the single-CTA
// kernel (128 x 256 tile), which is what bounds that kernel's e4m3 rate: the
// operand stream from L2, not the tensor pipe.  Both CTAs' loads count on the
// leader's `full` barrier; the leader's commits arrive on both CTAs' `empty`
// and `accf` barriers; the epilogue warps of both CTAs arrive on the leader's
// `acce` barrier.  Every wait is bounded as in schur_kernel.
// ---------------------------------------------------------------------------
#ifndef HPLAI_PAIR_STAGES
#define HPLAI_PAIR_STAGES 4
#endif
constexpr int PAIR_STAGES = HPLAI_PAIR_STAGES;
constexpr int PAIR_BM = 2 * BM;                       // tile rows of a pair
constexpr int PAIR_HALF = BM * 128;                   // 16 KB: 128 rows x 128 bytes of one operand
constexpr int PAIR_STAGE_BYTES = 2 * PAIR_HALF;       // per CTA: its L rows and its U rows
constexpr size_t pair_smem_bytes()
{
	return static_cast<size_t>(PAIR_STAGES) * PAIR_STAGE_BYTES + DECK_BYTES + 1024 + 256;
}
static_assert(pair_smem_bytes() <= 232448, "shared memory per CTA of a pair");

template <bool FP8>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(threads_for(2), 1) schur_pair_kernel(
	const __grid_constant__ CUtensorMap lmap, const __grid_constant__ CUtensorMap umap,
	const __grid_constant__ CUtensorMap cmap, const Params p)
{
	constexpr int NST = PAIR_STAGES;
	constexpr int NW = DECK_EPI_WARPS;
	extern __shared__ uint8_t smem_raw[];
	const uint32_t raw_addr = smem_u32(smem_raw);
	uint8_t *smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
	uint8_t *sA = smem;
	uint8_t *sB = smem + NST * PAIR_HALF;
	__half *dbuf = reinterpret_cast<__half *>(smem + NST * PAIR_STAGE_BYTES);
	uint64_t *bars = reinterpret_cast<uint64_t *>(smem + NST * PAIR_STAGE_BYTES + DECK_BYTES);
	uint64_t *full = bars;          // leader: both CTAs' loads of a stage
	uint64_t *empty = bars + NST;   // both: the stage's MMAs completed
	uint64_t *accf = bars + 2 * NST;
	uint64_t *acce = accf + 2;      // leader: both CTAs' epilogues drained the accumulator
	uint64_t *drain = acce + 2;
	uint64_t *dbar = drain + 1;
	uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(dbar + DECK_BUFS);

	const int warp = threadIdx.x >> 5;
	const int lane = threadIdx.x & 31;
	const uint32_t rank = cluster_rank();
	const bool leader = rank == 0;
	const int cl = static_cast<int>(blockIdx.x >> 1), ncl = static_cast<int>(gridDim.x >> 1);

	if (threadIdx.x == 0) {
		for (int s = 0; s < NST; ++s) {
			mbar_init(&full[s], 1);
			mbar_init(&empty[s], 1);
		}
		for (int a = 0; a < 2; ++a) {
			mbar_init(&accf[a], 1);
			mbar_init(&acce[a], 2 * NW);
		}
		mbar_init(drain, 1);
		for (int b = 0; b < DECK_BUFS; ++b) mbar_init(&dbar[b], 1);
		fence_mbar_init();
	}
	if (warp == 1) {
		tmem_alloc_pair(tmem_holder, TMEM_COLS);
		tmem_relinquish_pair();
	}
	if (warp == 0 && lane == 0) {
		tma_prefetch_desc(&lmap);
		tma_prefetch_desc(&umap);
		tma_prefetch_desc(&cmap);
	}
	__syncwarp();
	tc_fence_before();
	cluster_sync();
	tc_fence_after();
	const uint32_t tmem_base = *tmem_holder;
	const int total = p.tiles_m * p.tiles_n;   // pair tiles (tiles_m counts 256-row tiles)
	bool ok = true;

	if (warp == 0) {
		// ---------------- TMA producer (both CTAs) ----------------
		if (lane == 0) {
			int stage = 0;
			uint32_t phase = 0;
			for (int tile = cl; tile < total && ok; tile += ncl) {
				int tm, tn;
				tile_coords(tile, p.tiles_m, p.tiles_n, p.group_m, tm, tn);
				const int lrow = p.lrow0 + tm * PAIR_BM + static_cast<int>(rank) * BM;
				const int urow = p.urow0 + tn * BN + static_cast<int>(rank) * BM;
				for (int kc = 0; kc < p.num_kc; ++kc) {
					if (!mbar_wait(&empty[stage], phase ^ 1u)) { ok = false; break; }
					if (leader) mbar_arrive_expect_tx(&full[stage], 2 * PAIR_STAGE_BYTES);
					const uint32_t fb = smem_peer_u32(&full[stage], 0);
					const int kx = kc * (FP8 ? 2 * BK : BK);
					tma_load_2d_pair(sA + stage * PAIR_HALF, &lmap, fb, kx, lrow);
					tma_load_2d_pair(sB + stage * PAIR_HALF, &umap, fb, kx, urow);
					if (++stage == NST) { stage = 0; phase ^= 1u; }
				}
			}
			if (!ok) atomicOr(p.status, 1u);
		}
	} else if (warp == 1) {
		// ---------------- MMA issuer (leader) ----------------
		if (leader && lane == 0) {
			int stage = 0;
			uint32_t phase = 0;
			int acc = 0;
			uint32_t acc_phase = 0;
			const uint32_t idesc = FP8 ? umma_idesc_e4m3(PAIR_BM, BN) : umma_idesc_f16(PAIR_BM, BN);
			for (int tile = cl; tile < total && ok; tile += ncl) {
				if (!mbar_wait(&acce[acc], acc_phase ^ 1u)) { ok = false; break; }
				tc_fence_after();
				const uint32_t d_tmem = tmem_base + static_cast<uint32_t>(acc * BN);
				for (int kc = 0; kc < p.num_kc; ++kc) {
					if (!mbar_wait(&full[stage], phase)) { ok = false; break; }
					tc_fence_after();
					const uint64_t adesc = umma_desc_k_sw128(smem_u32(sA + stage * PAIR_HALF));
					const uint64_t bdesc = umma_desc_k_sw128(smem_u32(sB + stage * PAIR_HALF));
#pragma unroll
					for (int kk = 0; kk < 4; ++kk) {
						if (FP8)
							umma_f8_pair(d_tmem, adesc + 2u * kk, bdesc + 2u * kk, idesc, (kc | kk) != 0 ? 1u : 0u);
						else
							umma_f16_pair(d_tmem, adesc + 2u * kk, bdesc + 2u * kk, idesc, (kc | kk) != 0 ? 1u : 0u);
					}
					umma_commit_pair_both(&empty[stage]);
					if (++stage == NST) { stage = 0; phase ^= 1u; }
				}
				if (!ok) break;
				umma_commit_pair_both(&accf[acc]);
				if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
			}
			// every MMA completes before the pair releases its shared and tensor memory
			umma_commit_pair(drain);
			if (!mbar_wait(drain, 0)) ok = false;
			if (!ok) atomicOr(p.status, 1u);
		}
	} else {
		// ---------------- FP16 deck epilogue (both CTAs, their own 128 rows) ----------------
		constexpr int CPT = BN / DECK_CH;
		const int q = warp & 3;
		const int cw0 = ((warp - 2) >> 2) * DECK_CW;
		const bool lead = (warp == 2 && lane == 0);
		const int my_tiles = (cl < total) ? (total - cl + ncl - 1) / ncl : 0;
		const int nseq = my_tiles * CPT;
		const int r0 = static_cast<int>(rank) * BM;   // first tile row of this CTA
		const uint32_t acce_leader[2] = {smem_peer_u32(&acce[0], 0), smem_peer_u32(&acce[1], 0)};
		auto chunk_xy = [&](int sidx, int &x, int &y, bool &rows_in) {
			int tm, tn;
			tile_coords(cl + (sidx / CPT) * ncl, p.tiles_m, p.tiles_n, p.group_m, tm, tn);
			x = p.crow0 + tm * PAIR_BM + r0;
			y = p.ccol0 + tn * BN + (sidx % CPT) * DECK_CH;
			rows_in = tm * PAIR_BM + r0 < p.m;
		};
		int issued = 0;
		if (lead) {
			for (; issued < DECK_BUFS - 1 && issued < nseq; ++issued) {
				int x, y;
				bool in;
				chunk_xy(issued, x, y, in);
				mbar_arrive_expect_tx(&dbar[issued % DECK_BUFS], DECK_CHUNK_BYTES);
				tma_load_2d(dbuf + (issued % DECK_BUFS) * (BM * DECK_CH), &cmap, &dbar[issued % DECK_BUFS], x, y);
			}
		}
		int acc = 0;
		uint32_t acc_phase = 0;
		int sidx = 0;
		for (int it = 0; it < my_tiles && ok; ++it) {
			int tm, tn;
			tile_coords(cl + it * ncl, p.tiles_m, p.tiles_n, p.group_m, tm, tn);
			ok = epi_all<NW>(mbar_wait(&accf[acc], acc_phase));
			if (!ok) break;
			tc_fence_after();
			const uint32_t tbase = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * BN);
			float rf = p.dscale;
			if (FP8) rf *= p.sl[(p.lrow0 + min(tm * PAIR_BM + r0 + q * 32 + lane, p.m - 1) - p.sl0) >> 7];
#pragma unroll 1
			for (int ch = 0; ch < CPT; ++ch, ++sidx) {
				const int bi = sidx % DECK_BUFS;
				ok = epi_all<NW>(mbar_wait(&dbar[bi], static_cast<uint32_t>((sidx / DECK_BUFS) & 1)));
				if (!ok) break;
#pragma unroll
				for (int g = 0; g < DECK_CW / 32; ++g) {
					const int cc = ch * DECK_CH + cw0 + 32 * g;
					uint32_t r[32];
					tmem_ld_32x32b_x32(tbase + static_cast<uint32_t>(cc), r);
					__half *sb = dbuf + bi * (BM * DECK_CH) + (cw0 + 32 * g) * BM + q * 32 + lane;
					float d[32];
#pragma unroll
					for (int j = 0; j < 32; ++j) d[j] = __half2float(sb[j * BM]);
					float fu = rf, fl = 0.f;
					const bool uni = FP8 ? col_factors(p, tn * BN + cc, lane, fu, fl) : true;
					if (FP8 && uni) fu *= rf;
					tmem_ld_wait();
					if (uni) {
#pragma unroll
						for (int j = 0; j < 32; ++j) sb[j * BM] = __float2half_rn(d[j] - __uint_as_float(r[j]) * fu);
					} else {
#pragma unroll
						for (int j = 0; j < 32; ++j) {
							const float f = rf * __shfl_sync(0xffffffffu, fl, j);
							sb[j * BM] = __float2half_rn(d[j] - __uint_as_float(r[j]) * f);
						}
					}
				}
				asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
				asm volatile("bar.sync 1, %0;" ::"n"(NW * 32) : "memory");
				if (lead) {
					int x, y;
					bool in;
					chunk_xy(sidx, x, y, in);
					// a half tile wholly below the region's last row stores nothing
					if (in) tma_store_2d(&cmap, dbuf + bi * (BM * DECK_CH), x, y);
					asm volatile("cp.async.bulk.commit_group;" ::: "memory");
					if (issued < nseq) {
						const int nb2 = issued % DECK_BUFS;
						asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
						chunk_xy(issued, x, y, in);
						mbar_arrive_expect_tx(&dbar[nb2], DECK_CHUNK_BYTES);
						tma_load_2d(dbuf + nb2 * (BM * DECK_CH), &cmap, &dbar[nb2], x, y);
						++issued;
					}
				}
			}
			if (!ok) break;
			tc_fence_before();
			__syncwarp();
			if (lane == 0) mbar_arrive_cluster(acce_leader[acc]);
			if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
		}
		if (lead) {
			asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
			for (int s2 = sidx; s2 < issued; ++s2)
				(void)mbar_wait(&dbar[s2 % DECK_BUFS], static_cast<uint32_t>((s2 / DECK_BUFS) & 1));
		}
		if (lane == 0 && !ok) atomicOr(p.status, 1u);
	}

	__syncwarp();
	tc_fence_before();
	cluster_sync();
	if (warp == 0 && lane == 0 && *static_cast<volatile unsigned *>(p.status)) {
		// After a timeout, operand loads of either CTA may still be in flight
		// (their completion is counted on the leader's barriers): give them
		// 100 us to land before the pair's shared memory is released.
		const uint64_t t0 = global_ns();
		while (global_ns() - t0 < 100000ULL) {
		}
	}
	cluster_sync();
	if (warp == 1) {
		tc_fence_after();
		tmem_dealloc_pair(tmem_base, TMEM_COLS);
	}
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
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

int make_map_2d(void *out, CUtensorMapDataType dt, int esize, const void *base, uint64_t inner, uint64_t outer,
	uint64_t ld_elems, uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle swz)
{
	auto fn = encode_fn();
	if (!fn) return HPLAI_ECUDA;
	if ((reinterpret_cast<uintptr_t>(base) & 15u) || ((ld_elems * esize) & 15u)) return HPLAI_EINVAL;
	CUtensorMap m;
	cuuint64_t dims[2] = {inner, outer};
	cuuint64_t strides[1] = {ld_elems * esize};
	cuuint32_t box[2] = {box_inner, box_outer};
	cuuint32_t estr[2] = {1, 1};
	CUresult r = fn(&m, dt, 2, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
		CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS) return HPLAI_EINVAL;
	std::memcpy(out, &m, sizeof(m));
	return HPLAI_OK;
}

int make_map_f16(void *out, const void *base, uint64_t inner, uint64_t outer, uint64_t ld_elems, uint32_t box_inner,
	uint32_t box_outer)
{
	return make_map_2d(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, base, inner, outer, ld_elems, box_inner, box_outer,
		CU_TENSOR_MAP_SWIZZLE_128B);
}

int num_sms()
{
	int dev = 0, sms = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return 148;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return 148;
	return sms;
}

} // namespace

static_assert(sizeof(CUtensorMap) <= sizeof(SchurMaps::lmap), "tensor map storage");

int schur_make_maps(SchurMaps *m, const uint16_t *lh, int lrows, int64_t ldl, const uint16_t *uh, int urows,
	int64_t ldu, int k)
{
	if (!m || !lh || !uh || lrows <= 0 || urows <= 0 || k <= 0 || ldl < k || ldu < k || (ldl % 8) || (ldu % 8))
		return HPLAI_EINVAL;
	HPLAI_TRY(make_map_f16(m->lmap, lh, static_cast<uint64_t>(k), static_cast<uint64_t>(lrows),
		static_cast<uint64_t>(ldl), BK, BM));
	HPLAI_TRY(make_map_f16(m->umap, uh, static_cast<uint64_t>(k), static_cast<uint64_t>(urows),
		static_cast<uint64_t>(ldu), BK, BN));
	HPLAI_TRY(make_map_f16(m->umap2, uh, static_cast<uint64_t>(k), static_cast<uint64_t>(urows),
		static_cast<uint64_t>(ldu), BK, BM));
	m->k = k;
	m->has_cmap = false;
	return HPLAI_OK;
}

int schur_set_cmap(SchurMaps *m, const float *c, int rows, int cols, int64_t ldc)
{
	m->has_cmap = false;
	if (!c || rows <= 0 || cols <= 0 || (reinterpret_cast<uintptr_t>(c) & 15u) || (ldc % 4)) return HPLAI_OK;
	m->cbase = const_cast<float *>(c);
	m->cld = ldc;
	m->crows = rows;
	m->ccols = cols;
	m->has_cmap = true;
	return HPLAI_OK;
}

template <int EPI, bool FP8>
int set_smem_attr()
{
	HPLAI_CUDA_TRY(cudaFuncSetAttribute(schur_kernel<EPI, FP8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		static_cast<int>(smem_bytes(EPI))));
	return HPLAI_OK;
}

// Off by default: in the solves the trailing update runs under the 1000 W
// cap, where the pairs' lighter operand stream gave 2 % more throughput on
// long leaf runs (32768^2 e4m3 deck, K = 2048: 2112 against 2064 TFLOP/s at
// 1.27 against 1.24 GHz) but nothing measurable in a serial C3 solve, and
// under look-ahead the pairs, which need two free SMs of one TPC, lost
// 1 % to the side stream's scattered CTAs.
std::atomic<int> g_pairs_default{0};

// Shared memory of the pair kernel, and the most clusters of two that the
// device keeps resident at once (the persistent pair kernel launches no more:
// its clusters stride over the tiles and none waits for another).
int pair_cluster_limit(int *limit)
{
	static DeviceOnce once;
	return once.get([](int, int *v) -> int {
		HPLAI_CUDA_TRY(cudaFuncSetAttribute(schur_pair_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			static_cast<int>(pair_smem_bytes())));
		HPLAI_CUDA_TRY(cudaFuncSetAttribute(schur_pair_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			static_cast<int>(pair_smem_bytes())));
		cudaLaunchConfig_t cfg;
		std::memset(&cfg, 0, sizeof cfg);
		cfg.gridDim = dim3(2 * (num_sms() / 2), 1, 1);
		cfg.blockDim = dim3(threads_for(2), 1, 1);
		cfg.dynamicSmemBytes = pair_smem_bytes();
		int n = 0;
		if (cudaOccupancyMaxActiveClusters(&n, schur_pair_kernel<true>, &cfg) != cudaSuccess || n <= 0) {
			(void)cudaGetLastError();
			n = num_sms() / 2;
		}
		*v = n;
		return HPLAI_OK;
	}, limit);
}

// deck: C is the FP16 deck (c = its base, ldc its leading dimension in
// halves) updated as deck - dscale * acc; otherwise FP32 C.
static int launch_schur_any(const SchurMaps &maps, bool fp8, const float *sl, int sl0, const float *su, int su0,
	int lrow0, int urow0, int m, int n, void *c, int64_t ldc, int crow0, int ccol0, bool deck, float dscale,
	int max_ctas, cudaStream_t st, const float *oscale = nullptr, const AmaxTargets *amax = nullptr)
{
	if (m <= 0 || n <= 0) return HPLAI_OK;
	Params p;
	for (int t = 0; t < 2; ++t) {
		p.amax_bits[t] = amax ? amax->bits[t] : nullptr;
		p.amax_base[t] = amax ? amax->base[t] : 0;
	}
	p.amax_dim = amax ? amax->dim : 0;
	if (amax && (!oscale || amax->base[0] % 128 || amax->base[1] % 128)) return HPLAI_EINVAL;
	p.c = static_cast<float *>(c);
	p.ldc = ldc;
	p.m = m;
	p.n = n;
	p.num_kc = fp8 ? (maps.k + 127) / 128 : (maps.k + BK - 1) / BK;
	p.lrow0 = lrow0;
	p.urow0 = urow0;
	p.tiles_m = (m + BM - 1) / BM;
	p.tiles_n = (n + BN - 1) / BN;
	p.crow0 = crow0;
	p.ccol0 = ccol0;
	p.sl = sl;
	p.su = su;
	p.sl0 = sl0;
	p.su0 = su0;
	p.dscale = dscale;
	p.oscale = oscale;
	p.tiles = nullptr;
	p.ntiles = 0;
	p.group_m = maps.group_m > 0 ? maps.group_m : kGroupM;
	p.status = maps.status;
	if (!p.status) {
		void *g = nullptr;
		HPLAI_CUDA_TRY(cudaGetSymbolAddress(&g, g_status));
		p.status = static_cast<unsigned *>(g);
	}
	const int total = p.tiles_m * p.tiles_n;
	int grid = (max_ctas > 0 && max_ctas < num_sms()) ? max_ctas : num_sms();
	if (grid > total) grid = total;
	// The reduce epilogue needs each warp's first row 16-byte aligned in the map.
	// Its map ends at the region's last row and column: a TMA reduce clips
	// only at the tensor's extent, and a tile reaching past a region that
	// does not end at the matrix edge must not touch the neighbouring blocks.
	// The deck's loads and stores use a map clipped the same way; its rows
	// start and end on multiples of 8 (a TMA store clips a column in whole
	// 16-byte units, so a region ending inside one would overwrite the rows
	// after it with the out-of-range fill).
	int epi = 0;
	alignas(64) unsigned char cmap[128];
	if (deck) {
		if (crow0 % 8 || m % 8 || !maps.deck_base) return HPLAI_EINVAL;
		HPLAI_TRY(make_map_2d(cmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, maps.deck_base,
			static_cast<uint64_t>(crow0 + m), static_cast<uint64_t>(ccol0 + n), static_cast<uint64_t>(maps.deck_ld), BM,
			DECK_CH, CU_TENSOR_MAP_SWIZZLE_NONE));
		epi = 2;
	} else if (maps.has_cmap && (crow0 % 4 == 0) &&
		make_map_2d(cmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, maps.cbase, static_cast<uint64_t>(crow0 + m),
			static_cast<uint64_t>(ccol0 + n), static_cast<uint64_t>(maps.cld), TALL ? BM : 32, EPI_CHUNK,
			CU_TENSOR_MAP_SWIZZLE_NONE) == HPLAI_OK) {
		epi = 1;
	}
	// The store form writes whole 16-byte units of a column, so its region
	// starts and ends on multiples of 4 rows; it needs the tall-box reduce path.
	if (oscale && (fp8 || deck || epi != 1 || !TALL || (m % 4))) return HPLAI_EINVAL;
	// 256-row tiles on CTA pairs for the updates of K >= 2048 (two-panel groups
	// at b = 1024), where the single-CTA kernel's operand stream from L2 limits
	// it (16384^2 e4m3 deck, short runs: 2518 against 2375 TFLOP/s); at
	// K = 1024 the deck epilogue bounds both and the pairs' coupled tile steps
	// measured 17 % slower (1506 against 1817 TFLOP/s)
	if (epi == 2 && m > BM && maps.k >= 2048 && (maps.pairs > 0 || (maps.pairs < 0 && g_pairs_default.load() != 0))) {
		p.tiles_m = (m + PAIR_BM - 1) / PAIR_BM;
		const int ptotal = p.tiles_m * p.tiles_n;
		int limit = 0;
		HPLAI_TRY(pair_cluster_limit(&limit));
		int ncl = ((max_ctas > 0 && max_ctas < num_sms()) ? max_ctas : num_sms()) / 2;
		if (ncl > limit) ncl = limit;
		if (ncl > ptotal) ncl = ptotal;
		if (ncl >= 1) {
			CUtensorMap lm, um, cm;
			std::memcpy(&lm, maps.lmap, sizeof(lm));
			std::memcpy(&um, maps.umap2, sizeof(um));
			std::memcpy(&cm, cmap, sizeof(cm));
			if (fp8)
				schur_pair_kernel<true><<<2 * ncl, threads_for(2), pair_smem_bytes(), st>>>(lm, um, cm, p);
			else
				schur_pair_kernel<false><<<2 * ncl, threads_for(2), pair_smem_bytes(), st>>>(lm, um, cm, p);
			count_launches();
			HPLAI_CUDA_TRY(cudaGetLastError());
			return HPLAI_OK;
		}
		p.tiles_m = (m + BM - 1) / BM;
	}
	static DeviceOnce attr;
	HPLAI_TRY(attr.get([](int, int *) -> int {
		HPLAI_TRY((set_smem_attr<0, false>()));
		HPLAI_TRY((set_smem_attr<1, false>()));
		HPLAI_TRY((set_smem_attr<2, false>()));
		HPLAI_TRY((set_smem_attr<0, true>()));
		HPLAI_TRY((set_smem_attr<1, true>()));
		HPLAI_TRY((set_smem_attr<2, true>()));
		return HPLAI_OK;
	}));
	CUtensorMap lm, um, cm;
	std::memcpy(&lm, maps.lmap, sizeof(lm));
	std::memcpy(&um, maps.umap, sizeof(um));
	std::memcpy(&cm, epi ? cmap : maps.lmap, sizeof(cm));
	const size_t sm = smem_bytes(epi);
	if (fp8) {
		if (epi == 2) schur_kernel<2, true><<<grid, threads_for(2), sm, st>>>(lm, um, cm, p);
		else if (epi == 1) schur_kernel<1, true><<<grid, threads_for(1), sm, st>>>(lm, um, cm, p);
		else schur_kernel<0, true><<<grid, threads_for(0), sm, st>>>(lm, um, cm, p);
	} else {
		if (epi == 2) schur_kernel<2, false><<<grid, threads_for(2), sm, st>>>(lm, um, cm, p);
		else if (epi == 1) schur_kernel<1, false><<<grid, threads_for(1), sm, st>>>(lm, um, cm, p);
		else schur_kernel<0, false><<<grid, threads_for(0), sm, st>>>(lm, um, cm, p);
	}
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int launch_schur(const SchurMaps &maps, int lrow0, int urow0, int m, int n, float *c, int64_t ldc, int crow0,
	int ccol0, int max_ctas, cudaStream_t st)
{
	return launch_schur_any(maps, false, nullptr, 0, nullptr, 0, lrow0, urow0, m, n, c, ldc, crow0, ccol0, false, 0.f,
		max_ctas, st);
}

int launch_schur_fp8(const SchurMaps &maps8, const float *sl, int sl0, const float *su, int su0, int lrow0, int urow0,
	int m, int n, float *c, int64_t ldc, int crow0, int ccol0, int max_ctas, cudaStream_t st)
{
	return launch_schur_any(maps8, true, sl, sl0, su, su0, lrow0, urow0, m, n, c, ldc, crow0, ccol0, false, 0.f,
		max_ctas, st);
}

int launch_schur_store(const SchurMaps &maps, int lrow0, int urow0, int m, int n, float *c, int64_t ldc, int crow0,
	int ccol0, const float *oscale, int max_ctas, cudaStream_t st, const AmaxTargets *amax)
{
	if (!oscale) return HPLAI_EINVAL;
	return launch_schur_any(maps, false, nullptr, 0, nullptr, 0, lrow0, urow0, m, n, c, ldc, crow0, ccol0, false, 0.f,
		max_ctas, st, oscale, amax);
}

int launch_schur_deck(const SchurMaps &maps, bool fp8, const float *sl, int sl0, const float *su, int su0, int lrow0,
	int urow0, int m, int n, int crow0, int ccol0, float dscale, int max_ctas, cudaStream_t st)
{
	return launch_schur_any(maps, fp8, sl, sl0, su, su0, lrow0, urow0, m, n, maps.deck_base, maps.deck_ld, crow0, ccol0,
		true, dscale, max_ctas, st);
}

int launch_schur_tiles(const SchurMaps &maps, const int4 *tiles, int ntiles, int max_ctas, cudaStream_t st)
{
	if (ntiles <= 0) return HPLAI_OK;
	if (!maps.has_cmap || !TALL || !tiles) return HPLAI_EINVAL;
	Params p;
	std::memset(&p, 0, sizeof p);
	p.c = maps.cbase;
	p.ldc = maps.cld;
	p.num_kc = (maps.k + BK - 1) / BK;
	p.tiles = tiles;
	p.ntiles = ntiles;
	p.group_m = kGroupM;
	p.dscale = 0.f;
	p.status = maps.status;
	if (!p.status) {
		void *g = nullptr;
		HPLAI_CUDA_TRY(cudaGetSymbolAddress(&g, g_status));
		p.status = static_cast<unsigned *>(g);
	}
	// one C map over the whole matrix holding every system's C: a tile past a
	// system's last column lands in columns no system reads (the batched
	// layout leaves them), past the matrix end it is clipped
	alignas(64) unsigned char cmap[128];
	HPLAI_TRY(make_map_2d(cmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, maps.cbase, static_cast<uint64_t>(maps.crows),
		static_cast<uint64_t>(maps.ccols), static_cast<uint64_t>(maps.cld), BM, EPI_CHUNK, CU_TENSOR_MAP_SWIZZLE_NONE));
	static DeviceOnce attr;
	HPLAI_TRY(attr.get([](int, int *) -> int {
		HPLAI_TRY((set_smem_attr<1, false>()));
		return HPLAI_OK;
	}));
	CUtensorMap lm, um, cm;
	std::memcpy(&lm, maps.lmap, sizeof(lm));
	std::memcpy(&um, maps.umap, sizeof(um));
	std::memcpy(&cm, cmap, sizeof(cm));
	int grid = (max_ctas > 0 && max_ctas < num_sms()) ? max_ctas : num_sms();
	if (grid > ntiles) grid = ntiles;
	schur_kernel<1, false><<<grid, threads_for(1), smem_bytes(1), st>>>(lm, um, cm, p);
	count_launches();
	HPLAI_CUDA_TRY(cudaGetLastError());
	return HPLAI_OK;
}

int schur_make_maps_fp8(SchurMaps *m, const uint8_t *l8, int lrows, int64_t ldl, const uint8_t *u8, int urows,
	int64_t ldu, int k)
{
	if (!m || !l8 || !u8 || lrows <= 0 || urows <= 0 || k <= 0 || ldl < k || ldu < k || (ldl % 16) || (ldu % 16))
		return HPLAI_EINVAL;
	HPLAI_TRY(make_map_2d(m->lmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, l8, static_cast<uint64_t>(k),
		static_cast<uint64_t>(lrows), static_cast<uint64_t>(ldl), 128, BM, CU_TENSOR_MAP_SWIZZLE_128B));
	HPLAI_TRY(make_map_2d(m->umap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, u8, static_cast<uint64_t>(k),
		static_cast<uint64_t>(urows), static_cast<uint64_t>(ldu), 128, BN, CU_TENSOR_MAP_SWIZZLE_128B));
	HPLAI_TRY(make_map_2d(m->umap2, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, u8, static_cast<uint64_t>(k),
		static_cast<uint64_t>(urows), static_cast<uint64_t>(ldu), 128, BM, CU_TENSOR_MAP_SWIZZLE_128B));
	m->k = k;
	m->has_cmap = false;
	return HPLAI_OK;
}

void schur_set_pairs_default(bool on) { g_pairs_default.store(on ? 1 : 0); }

int schur_status()
{
	unsigned int v = 0;
	if (cudaMemcpyFromSymbol(&v, g_status, sizeof(v)) != cudaSuccess) return HPLAI_ECUDA;
	return v ? HPLAI_ETIMEOUT : HPLAI_OK;
}

void schur_status_reset()
{
	unsigned int z = 0;
	(void)cudaMemcpyToSymbol(g_status, &z, sizeof(z));
}

} // namespace hplai

extern "C" int hplai_shgemm_minus(int m, int n, int k, const uint16_t *lh, int64_t ldlh, const uint16_t *uh,
	int64_t lduh, float *c, int64_t ldc, void *stream)
{
	if (m < 0 || n < 0 || k <= 0 || !lh || !uh || !c || ldc < m || ldlh < k || lduh < k) return HPLAI_EINVAL;
	if (m == 0 || n == 0) return HPLAI_OK;
	hplai::SchurMaps maps;
	HPLAI_TRY(hplai::schur_make_maps(&maps, lh, m, ldlh, uh, n, lduh, k));
	HPLAI_TRY(hplai::schur_set_cmap(&maps, c, m, n, ldc));
	return hplai::launch_schur(maps, 0, 0, m, n, c, ldc, 0, 0, 0, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_f8gemm_minus(int m, int n, int k, const uint8_t *l8, int64_t ldl, const float *sl,
	const uint8_t *u8, int64_t ldu, const float *su, float *c, int64_t ldc, void *stream)
{
	if (m < 0 || n < 0 || k <= 0 || !l8 || !u8 || !sl || !su || !c || ldc < m || ldl < k || ldu < k) return HPLAI_EINVAL;
	if (m == 0 || n == 0) return HPLAI_OK;
	hplai::SchurMaps maps;
	HPLAI_TRY(hplai::schur_make_maps_fp8(&maps, l8, m, ldl, u8, n, ldu, k));
	HPLAI_TRY(hplai::schur_set_cmap(&maps, c, m, n, ldc));
	return hplai::launch_schur_fp8(maps, sl, 0, su, 0, 0, 0, m, n, c, ldc, 0, 0, 0, static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_shgemm_deck_minus(int m, int n, int k, const uint16_t *lh, int64_t ldlh, const uint16_t *uh,
	int64_t lduh, uint16_t *deck, int64_t ldd, float dscale, void *stream)
{
	if (m < 0 || n < 0 || k <= 0 || !lh || !uh || !deck || ldd < m || (ldd % 8) || (m % 8) || ldlh < k || lduh < k ||
		(reinterpret_cast<uintptr_t>(deck) & 15))
		return HPLAI_EINVAL;
	if (m == 0 || n == 0) return HPLAI_OK;
	hplai::SchurMaps maps;
	HPLAI_TRY(hplai::schur_make_maps(&maps, lh, m, ldlh, uh, n, lduh, k));
	maps.deck_base = deck;
	maps.deck_ld = ldd;
	return hplai::launch_schur_deck(maps, false, nullptr, 0, nullptr, 0, 0, 0, m, n, 0, 0, dscale, 0,
		static_cast<cudaStream_t>(stream));
}

extern "C" int hplai_f8gemm_deck_minus(int m, int n, int k, const uint8_t *l8, int64_t ldl, const float *sl,
	const uint8_t *u8, int64_t ldu, const float *su, uint16_t *deck, int64_t ldd, float dscale, void *stream)
{
	if (m < 0 || n < 0 || k <= 0 || !l8 || !u8 || !sl || !su || !deck || ldd < m || (ldd % 8) || (m % 8) || ldl < k ||
		ldu < k ||
		(reinterpret_cast<uintptr_t>(deck) & 15))
		return HPLAI_EINVAL;
	if (m == 0 || n == 0) return HPLAI_OK;
	hplai::SchurMaps maps;
	HPLAI_TRY(hplai::schur_make_maps_fp8(&maps, l8, m, ldl, u8, n, ldu, k));
	maps.deck_base = deck;
	maps.deck_ld = ldd;
	return hplai::launch_schur_deck(maps, true, sl, 0, su, 0, 0, 0, m, n, 0, 0, dscale, 0,
		static_cast<cudaStream_t>(stream));
}
