// batch.cu -- the batched C API: many independent HPL-AI systems on one GPU.
//
// The reference solves one system per run (main.cpp:144-492).  A batch holds
// `count` systems; system s is the HPL-AI matrix of order n[s] generated from
// seed[s] (state_0 = a*seed + 1, hpl_rand.hpp:35-57) with nrhs[s]
// right-hand sides: columns n, n+1, ... of the same stream (pcolvgen,
// matgen.hpp:193-207, extended past column n).
//
// The plain form (F32_F16, IR; up to 8 right-hand sides per system) runs on
// the batched engine of batched.cu: every kernel covers all systems, and
// generation plus factorisation are one CUDA graph.  Other forms (the e4m3
// precision form with GMRES-IR, the FP16 deck, more right-hand sides) give
// each system its own context, fed by a pool of host worker threads that
// take systems largest first (by n^3) from a shared counter.
#include "common.cuh"
#include "internal.h"

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

struct hplai_batch {
	int count = 0, precision = 0;
	int device = 0;
	int workers = 1;
	std::vector<int> n, nrhs, b;
	std::vector<uint64_t> seed;
	std::vector<hplai_ctx *> ctx;
	std::vector<std::vector<double>> x;      // n[s] x nrhs[s], column-major
	std::vector<hplai_ir_errors> worst;      // largest harness over the system's right-hand sides
	std::vector<int> iters, status;
	std::vector<int> order;                  // systems by decreasing n
	hplai::BatchEngine *eng = nullptr;       // the batched engine (plain form), else per-system contexts
};

namespace {

// The largest block size <= 512 that is a multiple of 16 and divides n:
// fewer, larger steps (each step costs a fixed number of launches).
int pick_block(int n)
{
	for (int b = 512; b >= 16; b -= 16)
		if (n % b == 0 && n >= b) return b;
	return 0;
}

void destroy(hplai_batch *bt)
{
	if (!bt) return;
	if (bt->eng) hplai::batched_destroy(bt->eng);
	for (hplai_ctx *c : bt->ctx)
		if (c) hplai_destroy(c);
	delete bt;
}

void solve_one(hplai_batch *bt, int s, int maxit)
{
	hplai_ctx *c = bt->ctx[s];
	int rc = hplai_generate(c, bt->seed[s]);
	if (rc == HPLAI_OK) rc = hplai_factor(c);
	hplai_ir_errors worst{0.0, 0.0};
	int itmax = 0;
	for (int r = 0; rc == HPLAI_OK && r < bt->nrhs[s]; ++r) {
		hplai_ir_errors e{-1.0, -1.0};
		int it = 0;
		const int rr = hplai_ctx_solve_stream_rhs(c, r, bt->x[s].data() + static_cast<size_t>(r) * bt->n[s], maxit, &e,
			&it);
		itmax = std::max(itmax, it);
		if (rr != HPLAI_OK) {
			rc = rr;
			worst = e;
			break;
		}
		if (e.hpl_harness > worst.hpl_harness) worst = e;
	}
	bt->worst[s] = rc == HPLAI_OK ? worst : hplai_ir_errors{-1.0, -1.0};
	bt->iters[s] = itmax;
	bt->status[s] = rc;
}

} // namespace

extern "C" int hplai_batch_create(hplai_batch **out, int count, const int *n, const int *nrhs, const uint64_t *seeds,
	int precision, unsigned flags, int workers)
{
	if (!out || count <= 0 || !n || !nrhs || !seeds) return HPLAI_EINVAL;
	*out = nullptr;
	hplai_batch *bt = new hplai_batch;
	bt->count = count;
	bt->precision = precision;
	bt->workers = workers > 0 ? workers : 8;
	HPLAI_CUDA_TRY(cudaGetDevice(&bt->device));
	bt->n.assign(n, n + count);
	bt->nrhs.assign(nrhs, nrhs + count);
	bt->seed.assign(seeds, seeds + count);
	bt->b.resize(count);
	bt->ctx.assign(count, nullptr);
	bt->x.resize(count);
	bt->worst.assign(count, hplai_ir_errors{-1.0, -1.0});
	bt->iters.assign(count, 0);
	bt->status.assign(count, HPLAI_ESTATE);
	bool engine = precision == HPLAI_F32_F16 && flags == 0;
	for (int s = 0; s < count; ++s) {
		if (n[s] < 1 || nrhs[s] < 1) {
			destroy(bt);
			return HPLAI_EINVAL;
		}
		if (nrhs[s] > 8) engine = false;
	}
	if (engine) {
		std::vector<uint64_t> sd(seeds, seeds + count);
		const int rc = hplai::batched_create(&bt->eng, count, n, nrhs, sd.data());
		if (rc != HPLAI_OK) {
			destroy(bt);
			return rc;
		}
		for (int s = 0; s < count; ++s) bt->b[s] = 128;
		*out = bt;
		return HPLAI_OK;
	}
	for (int s = 0; s < count; ++s) {
		const int bs = pick_block(n[s]);
		if (bs == 0 || nrhs[s] < 1) {
			destroy(bt);
			return HPLAI_EINVAL;
		}
		bt->b[s] = bs;
		const int rc = hplai_create(&bt->ctx[s], n[s], bs, precision, flags);
		if (rc != HPLAI_OK) {
			destroy(bt);
			return rc;
		}
		bt->x[s].assign(static_cast<size_t>(n[s]) * nrhs[s], 0.0);
	}
	bt->order.resize(count);
	for (int s = 0; s < count; ++s) bt->order[s] = s;
	std::stable_sort(bt->order.begin(), bt->order.end(), [bt](int p, int q) { return bt->n[p] > bt->n[q]; });
	*out = bt;
	return HPLAI_OK;
}

extern "C" int hplai_batch_destroy(hplai_batch *bt)
{
	destroy(bt);
	return HPLAI_OK;
}

extern "C" int hplai_batch_solve(hplai_batch *bt, int maxit)
{
	if (!bt || maxit < 0) return HPLAI_EINVAL;
	if (bt->eng) {
		if (cudaSetDevice(bt->device) != cudaSuccess) return HPLAI_ECUDA;
		return hplai::batched_solve(bt->eng, maxit, nullptr);
	}
	// the first (largest) system on this thread: every lazily initialised
	// library setting is in place before the pool starts
	solve_one(bt, bt->order[0], maxit);
	std::atomic<int> next{1};
	auto work = [bt, maxit, &next]() {
		cudaSetDevice(bt->device);
		for (int k = next.fetch_add(1); k < bt->count; k = next.fetch_add(1)) solve_one(bt, bt->order[k], maxit);
	};
	const int nw = std::min(bt->workers, bt->count - 1);
	std::vector<std::thread> pool;
	pool.reserve(nw);
	for (int w = 0; w < nw; ++w) pool.emplace_back(work);
	for (auto &t : pool) t.join();
	int rc = HPLAI_OK;
	for (int s = 0; s < bt->count; ++s) {
		const int st = bt->status[s];
		if (st != HPLAI_OK && st != HPLAI_ENOTCONV) return st;
		if (st == HPLAI_ENOTCONV) rc = HPLAI_ENOTCONV;
	}
	return rc;
}

extern "C" int hplai_batch_result(hplai_batch *bt, int s, hplai_ir_errors *worst, int *iters, int *status)
{
	if (!bt || s < 0 || s >= bt->count) return HPLAI_EINVAL;
	if (bt->eng) return hplai::batched_result(bt->eng, s, worst, iters, status);
	if (worst) *worst = bt->worst[s];
	if (iters) *iters = bt->iters[s];
	if (status) *status = bt->status[s];
	return HPLAI_OK;
}

extern "C" int hplai_batch_get_x(hplai_batch *bt, int s, double *x, int64_t ldx)
{
	if (!bt || s < 0 || s >= bt->count || !x || ldx < bt->n[s]) return HPLAI_EINVAL;
	if (bt->eng) return hplai::batched_get_x(bt->eng, s, x, ldx);
	for (int r = 0; r < bt->nrhs[s]; ++r)
		std::copy_n(bt->x[s].data() + static_cast<size_t>(r) * bt->n[s], bt->n[s], x + static_cast<size_t>(r) * ldx);
	return HPLAI_OK;
}

extern "C" int hplai_batch_block(hplai_batch *bt, int s)
{
	if (!bt || s < 0 || s >= bt->count) return -1;
	return bt->b[s];
}

extern "C" int hplai_batch_get_lu(hplai_batch *bt, int s, float *a, int64_t lda)
{
	if (!bt || s < 0 || s >= bt->count || !a || lda < bt->n[s]) return HPLAI_EINVAL;
	if (bt->eng) return hplai::batched_get_lu(bt->eng, s, a, lda);
	return hplai_get_lu(bt->ctx[s], a, lda);
}

extern "C" unsigned long long hplai_batch_launches(hplai_batch *bt)
{
	if (!bt) return 0;
	return bt->eng ? hplai::batched_launches(bt->eng) : 0;
}
