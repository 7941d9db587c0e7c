// api.cu -- the solve context of libhplai: allocation, generation, the
// blocked LU driver and the iterative-refinement driver.
//
// This is the single-GPU collapse of the reference's driver
// (main.cpp:185-488): one n x n FP32 matrix in HBM instead of 2D
// block-cyclic panels, FP16 copies of the current L and U panels instead of
// the broadcast buffers, CUDA streams instead of MPI requests.
#include "common.cuh"
#include "internal.h"

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

namespace hplai {

namespace {
std::mutex g_err_mu;
std::string g_err;
std::atomic<unsigned long long> g_launches{0};
} // namespace

void count_launches(int k) { g_launches.fetch_add(static_cast<unsigned long long>(k), std::memory_order_relaxed); }

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line)
{
	std::lock_guard<std::mutex> lk(g_err_mu);
	char buf[512];
	std::snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
	g_err = buf;
}

void set_last_error_message(const char *msg)
{
	std::lock_guard<std::mutex> lk(g_err_mu);
	g_err = msg;
}

static int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

} // namespace hplai

using namespace hplai;

struct hplai_ctx {
	int n = 0, b = 0, nb = 0, precision = 0;
	unsigned flags = 0;
	int64_t lda = 0, ldh = 0;
	float *A = nullptr;
	uint16_t *Lh = nullptr, *Uh = nullptr;
	SchurMaps maps;
	TcPanels tc;
	float *tcbuf = nullptr;   // phi, plo (n x ldp) and the four b x ldp inverse buffers
	double *rhs = nullptr, *d = nullptr, *x = nullptr, *r = nullptr, *scal = nullptr;
	void *gemv_work = nullptr;
	size_t gemv_bytes = 0;
	void *trsv_work = nullptr;
	size_t trsv_bytes = 0;
	cudaStream_t st = nullptr;
	uint64_t seed = 0;
	bool have_inputs = false, factored = false;
	double norma = 0.0, normb = 0.0;
	std::vector<double> log_resid, log_harness;
	double phase_ms[HPLAI_PH_COUNT] = {};
};

namespace {

int ctx_free(hplai_ctx *c)
{
	if (!c) return HPLAI_OK;
	cudaFree(c->A);
	cudaFree(c->Lh);
	cudaFree(c->Uh);
	cudaFree(c->tcbuf);
	cudaFree(c->rhs);
	cudaFree(c->d);
	cudaFree(c->x);
	cudaFree(c->r);
	cudaFree(c->scal);
	cudaFree(c->gemv_work);
	cudaFree(c->trsv_work);
	if (c->st) cudaStreamDestroy(c->st);
	delete c;
	return HPLAI_OK;
}

#define CTX_ALLOC(ptr, bytes)                                                         \
	do {                                                                              \
		cudaError_t e__ = cudaMalloc(reinterpret_cast<void **>(&(ptr)), (bytes));     \
		if (e__ != cudaSuccess) {                                                     \
			set_last_cuda_error(e__, "cudaMalloc(" #ptr ")", __FILE__, __LINE__);     \
			(void)cudaGetLastError();                                                 \
			ctx_free(c);                                                              \
			return HPLAI_ENOMEM;                                                      \
		}                                                                             \
	} while (0)

// Elapsed milliseconds between event pairs recorded around each phase.
struct PhaseEvents {
	std::vector<cudaEvent_t> ev;
	std::vector<int> phase;
	int record(cudaStream_t st, int ph)
	{
		cudaEvent_t a, b;
		HPLAI_CUDA_TRY(cudaEventCreate(&a));
		HPLAI_CUDA_TRY(cudaEventCreate(&b));
		HPLAI_CUDA_TRY(cudaEventRecord(a, st));
		ev.push_back(a);
		ev.push_back(b);
		phase.push_back(ph);
		return HPLAI_OK;
	}
	int end(cudaStream_t st) { return cudaEventRecord(ev.back(), st) == cudaSuccess ? HPLAI_OK : HPLAI_ECUDA; }
	void collect(double *ms)
	{
		for (size_t i = 0; i < phase.size(); ++i) {
			float t = 0.f;
			if (cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) ms[phase[i]] += t;
		}
	}
	~PhaseEvents()
	{
		for (auto e : ev) cudaEventDestroy(e);
	}
};

int compute_norms(hplai_ctx *c)
{
	HPLAI_TRY(launch_infnorm(c->n, c->rhs, c->scal + 0, c->st));
	HPLAI_TRY(launch_infnorm(c->n, c->d, c->scal + 1, c->st));
	double h[2];
	HPLAI_CUDA_TRY(cudaMemcpyAsync(h, c->scal, sizeof h, cudaMemcpyDeviceToHost, c->st));
	HPLAI_CUDA_TRY(cudaStreamSynchronize(c->st));
	c->normb = h[0];
	c->norma = 2.0 * h[1];   // hpl_infnorm: the diagonal is the off-diagonal row 1-norm
	return HPLAI_OK;
}

} // namespace

extern "C" const char *hplai_status_string(int status)
{
	switch (status) {
	case HPLAI_OK: return "ok";
	case HPLAI_EINVAL: return "invalid argument";
	case HPLAI_ENOMEM: return "out of memory";
	case HPLAI_ECUDA: return "CUDA error";
	case HPLAI_ENOTCONV: return "refinement did not converge";
	case HPLAI_ETIMEOUT: return "device wait timed out";
	case HPLAI_ESTATE: return "call out of order";
	case HPLAI_EUNSUPPORTED: return "unsupported configuration";
	default: return "unknown status";
	}
}

extern "C" int hplai_version(void) { return HPLAI_VERSION; }

extern "C" unsigned long long hplai_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" int hplai_last_error(char *buf, size_t len)
{
	std::lock_guard<std::mutex> lk(g_err_mu);
	if (buf && len) {
		std::strncpy(buf, g_err.c_str(), len - 1);
		buf[len - 1] = 0;
	}
	return HPLAI_OK;
}

extern "C" int hplai_create(hplai_ctx **out, int n, int b, int precision, unsigned flags)
{
	if (!out) return HPLAI_EINVAL;
	*out = nullptr;
	if (n <= 0 || b < 16 || b > 1024 || n % b) return HPLAI_EINVAL;
	if (precision != HPLAI_F32_F16) return HPLAI_EUNSUPPORTED;
	hplai_ctx *c = new hplai_ctx;
	c->n = n;
	c->b = b;
	c->nb = n / b;
	c->precision = precision;
	c->flags = flags;
	// lda padded to 64 floats plus 64 more so that columns do not share a
	// power-of-two stride (the reference's calc_lda_c, panel.hpp:10-18, for HBM).
	c->lda = round_up(n, 64) + 64;
	c->ldh = round_up(b, 64);
	HPLAI_CUDA_TRY(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
	CTX_ALLOC(c->A, sizeof(float) * static_cast<size_t>(c->lda) * n);
	CTX_ALLOC(c->Lh, sizeof(uint16_t) * static_cast<size_t>(c->ldh) * n);
	CTX_ALLOC(c->Uh, sizeof(uint16_t) * static_cast<size_t>(c->ldh) * n);
	const int64_t ldp = round_up(b, 32);
	const size_t tc_elems = static_cast<size_t>(ldp) * (2 * static_cast<size_t>(n) + 4 * static_cast<size_t>(b));
	CTX_ALLOC(c->tcbuf, sizeof(float) * tc_elems);
	CTX_ALLOC(c->rhs, sizeof(double) * n);
	CTX_ALLOC(c->d, sizeof(double) * n);
	CTX_ALLOC(c->x, sizeof(double) * n);
	CTX_ALLOC(c->r, sizeof(double) * n);
	CTX_ALLOC(c->scal, sizeof(double) * 8);
	c->gemv_bytes = otf_gemv_workspace(n);
	CTX_ALLOC(c->gemv_work, c->gemv_bytes);
	c->trsv_bytes = trsv_workspace(n);
	CTX_ALLOC(c->trsv_work, c->trsv_bytes);
	if (cudaMemset(c->trsv_work, 0, c->trsv_bytes) != cudaSuccess) {
		ctx_free(c);
		return HPLAI_ECUDA;
	}
	int s = schur_make_maps(&c->maps, c->Lh, n, c->ldh, c->Uh, n, c->ldh, b);
	if (s == HPLAI_OK) s = schur_set_cmap(&c->maps, c->A, n, n, c->lda);
	if (s == HPLAI_OK) {
		float *base = c->tcbuf;
		const size_t pn = static_cast<size_t>(ldp) * n, pb = static_cast<size_t>(ldp) * b;
		s = tc_panels_make(&c->tc, n, b, base, base + pn, ldp, base + 2 * pn, base + 2 * pn + pb,
			base + 2 * pn + 2 * pb, base + 2 * pn + 3 * pb);
	}
	if (s != HPLAI_OK) {
		ctx_free(c);
		return s;
	}
	*out = c;
	return HPLAI_OK;
}

extern "C" int hplai_destroy(hplai_ctx *c) { return ctx_free(c); }

extern "C" int hplai_generate(hplai_ctx *c, uint64_t seed)
{
	if (!c) return HPLAI_EINVAL;
	const int n = c->n;
	// pmatgen (matgen.hpp:7-22): the whole matrix, then the diagonal as the
	// FP32 rounding of the sequential FP64 row sums (which are also d).
	HPLAI_TRY(launch_fill(n, 0, 0, n, n, c->A, c->lda, seed, 0, c->st));
	HPLAI_TRY(launch_diag(n, 0, n, c->d, c->A, c->lda, seed, c->st));
	HPLAI_TRY(launch_rhs(n, c->rhs, seed, c->st));
	c->seed = seed;
	HPLAI_TRY(compute_norms(c));
	c->have_inputs = true;
	c->factored = false;
	return HPLAI_OK;
}

extern "C" int hplai_upload(hplai_ctx *c, const float *a, int64_t lda, const double *rhs, const double *diag,
	uint64_t seed)
{
	if (!c || !a || !rhs || !diag || lda < c->n) return HPLAI_EINVAL;
	const int n = c->n;
	HPLAI_CUDA_TRY(cudaMemcpy2DAsync(c->A, sizeof(float) * c->lda, a, sizeof(float) * lda, sizeof(float) * n, n,
		cudaMemcpyHostToDevice, c->st));
	HPLAI_CUDA_TRY(cudaMemcpyAsync(c->rhs, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
	HPLAI_CUDA_TRY(cudaMemcpyAsync(c->d, diag, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
	c->seed = seed;
	HPLAI_TRY(compute_norms(c));
	c->have_inputs = true;
	c->factored = false;
	return HPLAI_OK;
}

extern "C" int hplai_factor(hplai_ctx *c)
{
	if (!c) return HPLAI_EINVAL;
	if (!c->have_inputs) return HPLAI_ESTATE;
	const int n = c->n, b = c->b, nb = c->nb;
	const int64_t lda = c->lda, ldh = c->ldh;
	cudaStream_t st = c->st;
	schur_status_reset();
	tc_status_reset();
	const bool simt = (c->flags & HPLAI_FLAG_SIMT_PANELS) != 0;
	for (double &v : c->phase_ms) v = 0.0;
	PhaseEvents pe;
	// Right-looking blocked LU without pivoting, one panel per step
	// (panel_lu, panel_trf.hpp:329-432, with GemmControl's pieces fused
	// into one trailing update per step).
	for (int k = 0; k < nb; ++k) {
		const int64_t kb = static_cast<int64_t>(k) * b;
		float *diag = c->A + kb + kb * lda;
		HPLAI_TRY(pe.record(st, HPLAI_PH_DIAG_LU));
		HPLAI_TRY(launch_getrf(b, diag, lda, st));
		HPLAI_TRY(pe.end(st));
		if (k == nb - 1) break;
		const int rem = n - static_cast<int>(kb) - b;
		HPLAI_TRY(pe.record(st, HPLAI_PH_TRSM_L));
		if (simt) {
			HPLAI_TRY(launch_trsm_right_upper(rem, b, diag, lda, diag + b, lda, c->Lh + (kb + b) * ldh, ldh, 1.0f, st));
		} else {
			HPLAI_TRY(launch_tri_inverses(c->tc, diag, lda, st));
			HPLAI_TRY(launch_lpanel_tc(c->tc, rem, diag + b, lda, c->Lh + (kb + b) * ldh, ldh, 1.0f, 0, st));
		}
		HPLAI_TRY(pe.end(st));
		HPLAI_TRY(pe.record(st, HPLAI_PH_TRSM_R));
		if (simt) {
			HPLAI_TRY(launch_trsm_left_lower(b, rem, diag, lda, diag + static_cast<int64_t>(b) * lda, lda,
				c->Uh + (kb + b) * ldh, ldh, 1.0f, st));
		} else {
			HPLAI_TRY(launch_upanel_tc(c->tc, rem, diag + static_cast<int64_t>(b) * lda, lda, c->Uh + (kb + b) * ldh,
				ldh, 1.0f, 0, st));
		}
		HPLAI_TRY(pe.end(st));
		HPLAI_TRY(pe.record(st, HPLAI_PH_GEMM_UPDATE));
		HPLAI_TRY(launch_schur(c->maps, static_cast<int>(kb) + b, static_cast<int>(kb) + b, rem, rem,
			diag + b + static_cast<int64_t>(b) * lda, lda, static_cast<int>(kb) + b, static_cast<int>(kb) + b, st));
		HPLAI_TRY(pe.end(st));
	}
	HPLAI_CUDA_TRY(cudaStreamSynchronize(st));
	pe.collect(c->phase_ms);
	HPLAI_TRY(schur_status());
	HPLAI_TRY(tc_status());
	c->factored = true;
	return HPLAI_OK;
}

extern "C" int hplai_refine(hplai_ctx *c, int mode, int maxit, hplai_ir_errors *err, int *iters)
{
	if (!c || maxit < 0) return HPLAI_EINVAL;
	if (!c->factored) return HPLAI_ESTATE;
	if (mode != HPLAI_IR) return HPLAI_EUNSUPPORTED;
	const int n = c->n;
	cudaStream_t st = c->st;
	c->log_resid.clear();
	c->log_harness.clear();
	if (err) *err = hplai_ir_errors{-1.0, -1.0};
	if (iters) *iters = 0;
	PhaseEvents pe;
	// x_0 = b ./ diag(A)   (iterative_refinement.hpp:31-34)
	HPLAI_TRY(launch_div(n, c->rhs, c->d, c->x, st));
	int rc = HPLAI_ENOTCONV;
	for (int it = 0; it < maxit; ++it) {
		HPLAI_CUDA_TRY(cudaMemcpyAsync(c->r, c->rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
		HPLAI_TRY(launch_infnorm(n, c->x, c->scal + 2, st));
		// r = b - A x with A regenerated in FP64 (panel_gemv(-1, ..., 1, r))
		HPLAI_TRY(pe.record(st, HPLAI_PH_IR_GEMV));
		HPLAI_TRY(launch_otf_gemv(n, -1.0, c->x, 1.0, c->r, c->seed, c->d, c->gemv_work, c->gemv_bytes, st));
		HPLAI_TRY(pe.end(st));
		HPLAI_TRY(launch_infnorm(n, c->r, c->scal + 3, st));
		double h[2];
		HPLAI_CUDA_TRY(cudaMemcpyAsync(h, c->scal + 2, sizeof h, cudaMemcpyDeviceToHost, st));
		HPLAI_CUDA_TRY(cudaStreamSynchronize(st));
		const double normx = h[0], normr = h[1];
		// iterative_refinement.hpp:43
		const double hpl = normr / std::fma(c->norma, normx, c->normb) * 1. / (n * DBL_EPSILON / 2);
		c->log_resid.push_back(normr);
		c->log_harness.push_back(hpl);
		if (iters) *iters = it + 1;
		if (hpl < 16.) {
			if (err) *err = hplai_ir_errors{normr, hpl};
			rc = HPLAI_OK;
			break;
		}
		// x += U^{-1} L^{-1} r   (iterative_refinement.hpp:50-53)
		HPLAI_TRY(pe.record(st, HPLAI_PH_IR_TRSV));
		HPLAI_TRY(launch_trsv(true, n, c->A, c->lda, c->r, c->trsv_work, c->trsv_bytes, st));
		HPLAI_TRY(launch_trsv(false, n, c->A, c->lda, c->r, c->trsv_work, c->trsv_bytes, st));
		HPLAI_TRY(pe.end(st));
		HPLAI_TRY(launch_axpy1(n, c->r, c->x, st));
		int ts = HPLAI_OK;
		HPLAI_TRY(trsv_status(c->trsv_work, st, &ts));
		if (ts != HPLAI_OK) return ts;
	}
	HPLAI_CUDA_TRY(cudaStreamSynchronize(st));
	double tmp[HPLAI_PH_COUNT] = {};
	pe.collect(tmp);
	c->phase_ms[HPLAI_PH_IR_GEMV] = tmp[HPLAI_PH_IR_GEMV];
	c->phase_ms[HPLAI_PH_IR_TRSV] = tmp[HPLAI_PH_IR_TRSV];
	return rc;
}

extern "C" int hplai_get_x(hplai_ctx *c, double *x)
{
	if (!c || !x) return HPLAI_EINVAL;
	HPLAI_CUDA_TRY(cudaMemcpyAsync(x, c->x, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->st));
	HPLAI_CUDA_TRY(cudaStreamSynchronize(c->st));
	return HPLAI_OK;
}

extern "C" int hplai_get_lu(hplai_ctx *c, float *a, int64_t lda)
{
	if (!c || !a || lda < c->n) return HPLAI_EINVAL;
	HPLAI_CUDA_TRY(cudaMemcpy2DAsync(a, sizeof(float) * lda, c->A, sizeof(float) * c->lda, sizeof(float) * c->n, c->n,
		cudaMemcpyDeviceToHost, c->st));
	HPLAI_CUDA_TRY(cudaStreamSynchronize(c->st));
	return HPLAI_OK;
}

extern "C" int hplai_get_rhs(hplai_ctx *c, double *rhs)
{
	if (!c || !rhs) return HPLAI_EINVAL;
	HPLAI_CUDA_TRY(cudaMemcpyAsync(rhs, c->rhs, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->st));
	HPLAI_CUDA_TRY(cudaStreamSynchronize(c->st));
	return HPLAI_OK;
}

extern "C" int hplai_get_diag(hplai_ctx *c, double *diag)
{
	if (!c || !diag) return HPLAI_EINVAL;
	HPLAI_CUDA_TRY(cudaMemcpyAsync(diag, c->d, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->st));
	HPLAI_CUDA_TRY(cudaStreamSynchronize(c->st));
	return HPLAI_OK;
}

extern "C" int hplai_get_ir_log(hplai_ctx *c, double *residual, double *harness, int cap, int *count)
{
	if (!c) return HPLAI_EINVAL;
	const int m = static_cast<int>(c->log_resid.size());
	for (int i = 0; i < m && i < cap; ++i) {
		if (residual) residual[i] = c->log_resid[i];
		if (harness) harness[i] = c->log_harness[i];
	}
	if (count) *count = m;
	return HPLAI_OK;
}

extern "C" int hplai_get_phase_ms(hplai_ctx *c, double *ms, int count)
{
	if (!c || !ms) return HPLAI_EINVAL;
	double total = 0.0;
	for (int i = 0; i < HPLAI_PH_TOTAL; ++i) total += c->phase_ms[i];
	for (int i = 0; i < count && i < HPLAI_PH_COUNT; ++i) ms[i] = (i == HPLAI_PH_TOTAL) ? total : c->phase_ms[i];
	return HPLAI_OK;
}

extern "C" void *hplai_get_stream(hplai_ctx *c) { return c ? static_cast<void *>(c->st) : nullptr; }

extern "C" int hplai_get_norms(hplai_ctx *c, double *norma, double *normb)
{
	if (!c) return HPLAI_EINVAL;
	if (norma) *norma = c->norma;
	if (normb) *normb = c->normb;
	return HPLAI_OK;
}

extern "C" int hplai_solve_host(hplai_ctx *c, const float *a, int64_t lda, const double *rhs, const double *diag,
	uint64_t seed, int maxit, double *x, hplai_ir_errors *err, int *iters)
{
	HPLAI_TRY(hplai_upload(c, a, lda, rhs, diag, seed));
	HPLAI_TRY(hplai_factor(c));
	const int rc = hplai_refine(c, HPLAI_IR, maxit, err, iters);
	if (rc != HPLAI_OK && rc != HPLAI_ENOTCONV) return rc;
	HPLAI_TRY(hplai_get_x(c, x));
	return rc;
}

extern "C" int hplai_format_report(int n, double seconds, hplai_ir_errors err, char *buf, size_t len)
{
	if (!buf || !len || seconds <= 0.0) return HPLAI_EINVAL;
	// main.cpp:440-452
	const double hplflops = 2. / 3 * n * static_cast<double>(n) * n + 3. / 2 * n * static_cast<double>(n);
	std::snprintf(buf, len, "%.9f sec. %.9f GFlop/s resid = %20.15e hpl-harness = %.9f", seconds,
		hplflops / seconds * 1e-9, err.residual, err.hpl_harness);
	return HPLAI_OK;
}
