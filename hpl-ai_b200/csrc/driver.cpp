// driver.cpp -- command-line driver with the reference's interface.
//
//   driver.out <n> <b> <P> [flags]
//
// Same positional arguments and report as the reference's driver
// (main.cpp:144-181, 437-453): n % b == 0, seed 42, LU + iterative
// refinement timed as one region, then
//   "%.9f sec. %.9f GFlop/s resid = %20.15e hpl-harness = %.9f".
// P (the process-grid rows) does not lay out anything -- the whole matrix
// lives on one GPU -- but sets the length of the `-w` warm-up as in the
// reference (the first P + 2 panels, main.cpp:57, panel_trf.hpp:726).  `-d`/`-l` (the double-decker layout with lazy
// initialisation, main.cpp:52-53) select the FP16 trailing-update deck; `--fp8` the
// precision form (e4m3 Schur update, GMRES-IR); `--gmres` GMRES-IR.  The
// reference's layout/transport flags (-not, -r, -m, --pack, --numa, --nbuf,
// ...) are accepted and reported as not applicable.
#include "../../include/hplai.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>
#include <unistd.h>

// Timer::show / Timer::dump_mp (timer.hpp:174-218) as main.cpp:470-478 calls
// them on one process: the file Timerdump.<job>.<n>.<b>.<size>.<rank> in the
// working directory, one line per timer item (seconds, share of TOTAL,
// accumulated operation count, Gop/s) and the GEMM rate.  Items of the
// distributed reference that have no work on one GPU (broadcasts, tests,
// waits, separate down-casts, write-back, communication) read 0; MISC is
// TOTAL minus the other items, as in the reference.  With look-ahead the
// side stream's items (DIAG_LU, TRSM_L, TRSM_R) run while GEMM_UPDATE does,
// so the items can add up to more than TOTAL: MISC is then clamped at 0 and
// a comment line says that the items overlap.
static void write_timerdump(int jobid, int n, int b, double total_s, const double *ms, long long matvecs,
	bool overlapped, bool warmup)
{
	enum { DIAG_LU = 5, TRSM_L = 6, TRSM_R = 7, GEMM_UPDATE = 10, GEMM_PROGRESS = 11, LAZY_INIT = 12, WRITE_BACK = 13, IR_GEMV = 14,
		IR_TRSV = 16, TOTAL = 19, MISC = 20, NUM_ITEMS = 21 };
	static const char *names[NUM_ITEMS] = {"DIAG_BCAST", "LCOL_BCAST", "RROW_BCAST", "TEST", "WAIT", "DIAG_LU",
		"TRSM_L", "TRSM_R", "CONV_L", "CONV_R", "GEMM_UPDATE", "GEMM_PROGRESS", "LAZY_INIT", "WRITE_BACK", "IR_GEMV",
		"IR_GEMV_COMM", "IR_TRSV", "IR_TRSV_MV", "IR_TRSV_COMM", "TOTAL", "MISC"};
	double t[NUM_ITEMS] = {};
	long long acc[NUM_ITEMS] = {};
	const long long nb = n / b, bb = b;
	t[DIAG_LU] = 1e-3 * ms[HPLAI_PH_DIAG_LU];
	t[TRSM_L] = 1e-3 * ms[HPLAI_PH_TRSM_L];
	t[TRSM_R] = 1e-3 * ms[HPLAI_PH_TRSM_R];
	t[GEMM_UPDATE] = 1e-3 * ms[HPLAI_PH_GEMM_UPDATE];
	t[LAZY_INIT] = 1e-3 * ms[HPLAI_PH_LAZY_INIT];
	t[WRITE_BACK] = 1e-3 * ms[HPLAI_PH_WRITE_BACK];
	t[IR_GEMV] = 1e-3 * ms[HPLAI_PH_IR_GEMV];
	t[IR_TRSV] = 1e-3 * ms[HPLAI_PH_IR_TRSV];
	t[TOTAL] = total_s;
	// operation counts the reference accumulates per item, summed over the
	// n/b steps (panel_trf.hpp:156,170,457; schur_updator.hpp:394; panel_gemv.hpp:156)
	acc[DIAG_LU] = nb * (bb * (bb * (4 * bb - 3) + 5) / 6);
	acc[TRSM_L] = bb * bb * bb * (nb * (nb - 1) / 2);
	acc[TRSM_R] = acc[TRSM_L];
	acc[GEMM_UPDATE] = 2 * bb * bb * bb * ((nb - 1) * nb * (2 * nb - 1) / 6);
	acc[IR_GEMV] = 2LL * n * n * matvecs;
	t[MISC] = t[TOTAL];
	for (int i = 0; i < NUM_ITEMS - 2; ++i) t[MISC] -= t[i];
	if (t[MISC] < 0.0) t[MISC] = 0.0;
	char fname[128];
	std::snprintf(fname, sizeof fname, warmup ? "Warmup.%06d.%09d.%04d.%05d.%05d" : "Timerdump.%06d.%09d.%04d.%05d.%05d",
		jobid, n, b, 1, 0);
	FILE *fp = std::fopen(fname, "w");
	if (!fp) return;
	char host[256] = "";
	gethostname(host, sizeof host - 1);
	std::fprintf(fp, "# row=%d, col=%d, host=%s\n", 0, 0, host);
	if (overlapped)
		std::fprintf(fp, "# look-ahead: DIAG_LU, TRSM_L and TRSM_R ran on a side stream during GEMM_UPDATE; "
		                 "items overlap, MISC clamped at 0\n");
	for (int i = 0; i < NUM_ITEMS; ++i)
		std::fprintf(fp, " %-12s : %e sec : %6.2f %% : %20lld : %e Gop/s\n", names[i], t[i], 100.0 * t[i] / t[TOTAL],
			acc[i], 1e-9 * static_cast<double>(acc[i]) / t[i]);
	const double flops = static_cast<double>(acc[GEMM_UPDATE] + acc[GEMM_PROGRESS]) / (t[GEMM_UPDATE] + t[GEMM_PROGRESS]);
	std::fprintf(fp, "GEMM_TOTAL: %f Tflops\n", 1.e-12 * flops);
	std::fclose(fp);
}

static void print_ctime(const char *msg)
{
	std::time_t t;
	std::time(&t);
	std::printf("%s%s", msg, std::ctime(&t));
}

static int usage()
{
	std::printf(
		"HPL-AI on one B200\n\n"
		"usage: driver.out <n> <b> <P> [arguments]\n\n"
		"Arguments:\n"
		"   n                       The matrix size.\n"
		"   b                       The block size. Requires mod(n,b) = 0 and 16 <= b <= 1024.\n"
		"   P                       Process-grid rows of the distributed reference; ignored.\n"
		"   --maxit <k>             Refinement steps before giving up (default 50).\n"
		"   --seed <s>              LCG seed (default 42, as the reference).\n"
		"   -d, -l, --delayed, --lazy-init\n"
		"                           Keep the trailing updates in an FP16 deck (double-decker form).\n"
		"   --ref-deck              The reference's -d arithmetic bit for bit: A regenerated at panel\n"
		"                           time, FP16-accumulating Schur update on CUDA cores (parity mode).\n"
		"   --back_buffer           With --ref-deck (implied): the reference's back-buffer form bit for bit.\n"
		"   --lazy-a                With --fp8 (implies -d): store no A; each block is regenerated from the\n"
		"                           LCG when it joins a panel and the deck shares the factors' storage.\n"
		"   --highammat             Higham's HPL-AI matrix (cond 1000) instead of the LCG matrix.\n"
		"   --fp8                   e4m3 Schur update with GMRES refinement.\n"
		"   --gmres                 GMRES refinement instead of the classical correction.\n"
		"   --lookahead             Factor the next panel while the trailing update runs.\n"
		"   --group <g>             Panels per trailing update: 1 (default), 2 or 4 (K = g b; b %% 128 == 0).\n"
		"   --autotune              Choose the schedule (groups, look-ahead) by timing it first.\n"
		"   --checksum              Print sums of |diag|, |upper|, |lower| of the factors after the LU.\n"
		"   -w, --warmup            Factor the first P+2 panels only, one refinement step (benchmark warm-up).\n"
		"   --l1est                 Approximate the LU factors from the matrix instead of factoring it.\n"
		"   --job-id <id>           Job number in the name of the Timerdump file (default 0).\n"
		"   --help or -h            Print this message.\n"
		"Layout and transport flags of the distributed reference (-not, -r, -m, --pack,\n"
		"--numa, --numa-map, --nbuf, --pwrtune) are accepted, echoed in the settings lines\n"
		"and have no effect on one GPU.\n");
	return 0;
}

int main(int argc, char **argv)
{
	int n = 120, b = 30, maxit = 50;
	unsigned long long seed = 42;
	int precision = HPLAI_F32_F16, mode = HPLAI_IR;
	unsigned flags = 0;
	bool checksum = false, autotune = false, warmup = false, l1est = false, higham = false;
	int nrow = 2;
	int jobid = 0;
	// layout and transport settings of the distributed reference: accepted,
	// echoed in its settings lines, without effect on one GPU
	bool tile = true, rdma = false, pack = false;
	int numasize = 0, nbuf = 2;
	const char *numamap = "ROWDIST";
	if (argc > 1) n = std::atoi(argv[1]);
	if (argc > 2) b = std::atoi(argv[2]);
	if (argc > 3) nrow = std::atoi(argv[3]);
	for (int i = 4; i < argc; ++i) {
		if (!std::strcmp(argv[i], "--help") || !std::strcmp(argv[i], "-h")) return usage();
		else if (!std::strcmp(argv[i], "--maxit") && i + 1 < argc) maxit = std::atoi(argv[++i]);
		else if (!std::strcmp(argv[i], "--seed") && i + 1 < argc) seed = std::strtoull(argv[++i], nullptr, 10);
		else if (!std::strcmp(argv[i], "-d") || !std::strcmp(argv[i], "--delayed") || !std::strcmp(argv[i], "-l") ||
			!std::strcmp(argv[i], "--lazy-init"))
			flags |= HPLAI_FLAG_FP16_DECK;
		else if (!std::strcmp(argv[i], "--ref-deck")) flags |= HPLAI_FLAG_REF_DECK;
		else if (!std::strcmp(argv[i], "--lazy-a")) flags |= HPLAI_FLAG_FP16_DECK | HPLAI_FLAG_LAZY_A;
		else if (!std::strcmp(argv[i], "--back_buffer")) flags |= HPLAI_FLAG_REF_DECK | HPLAI_FLAG_REF_BACKBUF;
		else if (!std::strcmp(argv[i], "--highammat")) higham = true;
		else if (!std::strcmp(argv[i], "--fp8")) { precision = HPLAI_F32_F8; mode = HPLAI_GMRES; }
		else if (!std::strcmp(argv[i], "--gmres")) mode = HPLAI_GMRES;
		else if (!std::strcmp(argv[i], "--lookahead")) flags |= HPLAI_FLAG_LOOKAHEAD;
		else if (!std::strcmp(argv[i], "--group") && i + 1 < argc) {
			const int g = std::atoi(argv[++i]);
			if (g == 2) flags |= HPLAI_FLAG_GROUP2;
			else if (g == 4) flags |= HPLAI_FLAG_GROUP4;
		}
		else if (!std::strcmp(argv[i], "--autotune")) autotune = true;
		else if (!std::strcmp(argv[i], "--checksum")) checksum = true;
		else if (!std::strcmp(argv[i], "-w") || !std::strcmp(argv[i], "--warmup")) warmup = true;
		else if (!std::strcmp(argv[i], "--l1est")) l1est = true;
		else if (!std::strcmp(argv[i], "-not") || !std::strcmp(argv[i], "-nt") || !std::strcmp(argv[i], "--notile"))
			tile = false;
		else if (!std::strcmp(argv[i], "-r") || !std::strcmp(argv[i], "--rdma")) rdma = true;
		else if (!std::strcmp(argv[i], "--pack")) pack = true;
		else if (!std::strcmp(argv[i], "-m") || !std::strcmp(argv[i], "--manual-progress") ||
			!std::strcmp(argv[i], "--pwrtune")) continue;
		else if (!std::strcmp(argv[i], "--numa")) {
			if (i + 1 < argc) numasize = std::atoi(argv[++i]);
		} else if (!std::strcmp(argv[i], "--numa-map")) {
			if (i + 1 < argc) {
				++i;
				for (const char *m : {"ROWCONT", "COLCONT", "ROWDIST", "COLDIST"})
					if (!std::strcmp(argv[i], m)) numamap = m;
			}
		} else if (!std::strcmp(argv[i], "--nbuf")) {
			if (i + 1 < argc) nbuf = std::atoi(argv[++i]);
		}
		else if (!std::strcmp(argv[i], "--job-id") && i + 1 < argc) jobid = std::atoi(argv[++i]);
		else if (argv[i][0] == '-') std::printf("Ignoring option not applicable on one GPU: %s\n", argv[i]);
		else std::printf("Ignoring unknown option: %s\n", argv[i]);
	}
	if (argc > 1 && (!std::strcmp(argv[1], "-h") || !std::strcmp(argv[1], "--help"))) return usage();
	if (flags & HPLAI_FLAG_REF_DECK) {
		// one fixed schedule: nothing to tune
		flags &= ~(HPLAI_FLAG_FP16_DECK | HPLAI_FLAG_GROUP2 | HPLAI_FLAG_GROUP4 | HPLAI_FLAG_LOOKAHEAD | HPLAI_FLAG_LAZY_A);
		autotune = false;
	}

	// the reference's settings lines (main.cpp:214-232), then this build's
	const bool lazy = (flags & (HPLAI_FLAG_FP16_DECK | HPLAI_FLAG_REF_DECK)) != 0;
	std::printf("jobid=%d\n", jobid);
	std::printf("n=%d b=%d r=1 c=1\n", n, b);
	std::printf("%s %s %s %s %s %s %s %s\n", tile ? "tile" : "2dbc",
		(flags & HPLAI_FLAG_REF_BACKBUF) ? "back_buffer" : lazy ? "lazy" : "precomp", rdma ? "rdma" : "mpi",
		warmup ? "warmup" : "full", pack ? "pack" : "nopack", checksum ? "checksum" : "nocheck",
		l1est ? "skiplu" : "noskiplu", higham ? "hmat" : "ddmat");
	std::printf("numasize=%d numamap=%s nbuf=%d\n", numasize, numamap, nbuf);
	std::printf("1gpu %s full fp32/%s%s%s\n", (flags & (HPLAI_FLAG_FP16_DECK | HPLAI_FLAG_REF_DECK)) ? "lazy" : "precomp",
		precision == HPLAI_F32_F8 ? "e4m3" : "fp16",
		(flags & HPLAI_FLAG_REF_BACKBUF) ? " fp16-deck-ref back_buffer"
		: (flags & HPLAI_FLAG_REF_DECK) ? " fp16-deck-ref"
		: (flags & HPLAI_FLAG_LAZY_A) ? " fp16-deck no-stored-A" : (flags & HPLAI_FLAG_FP16_DECK) ? " fp16-deck" : "",
		higham ? " hmat" : " ddmat");

	// Warm-up on a small system with the same block size so that every kernel
	// is loaded before the timed region (the reference warms BLAS up the same
	// way, getrf_nopiv.hpp:161-167 / main.cpp:281).
	{
		hplai_ctx *w = nullptr;
		int rc = hplai_create(&w, 2 * b, b, precision, flags);
		if (rc == HPLAI_OK) {
			hplai_ir_errors e;
			int it;
			if (higham) hplai_set_matrix(w, HPLAI_MATRIX_HIGHAM, 1000., 0.5);
			hplai_generate(w, seed);
			hplai_factor(w);
			hplai_refine(w, mode, maxit, &e, &it);
			hplai_destroy(w);
		}
	}

	hplai_ctx *ctx = nullptr;
	int rc = HPLAI_OK;
	if (autotune && b % 128 == 0 && !(flags & (HPLAI_FLAG_GROUP2 | HPLAI_FLAG_GROUP4 | HPLAI_FLAG_REF_DECK))) {
		// buffers for four-panel groups, so that the tuner can choose them (skipped when they do not fit)
		rc = hplai_create(&ctx, n, b, precision, flags | HPLAI_FLAG_GROUP4);
		if (rc == HPLAI_OK) rc = hplai_set_schedule(ctx, flags & HPLAI_FLAG_LOOKAHEAD, 32);
		if (rc != HPLAI_OK && ctx) {
			hplai_destroy(ctx);
			ctx = nullptr;
		}
	}
	if (!ctx) rc = hplai_create(&ctx, n, b, precision, flags);
	if (rc != HPLAI_OK) {
		std::fprintf(stderr, "hplai_create(n=%d, b=%d): %s\n", n, b, hplai_status_string(rc));
		return 1;
	}
	if (higham) {
		// HMGen(n, 1000., 0.5, ...) (main.cpp:258-259)
		rc = hplai_set_matrix(ctx, HPLAI_MATRIX_HIGHAM, 1000., 0.5);
		if (rc != HPLAI_OK) {
			std::fprintf(stderr, "hplai_set_matrix(higham): %s\n", hplai_status_string(rc));
			return 1;
		}
	}
	if (autotune) {
		unsigned tf = 0;
		int side = 0;
		double tms = 0.0;
		rc = hplai_autotune(ctx, seed, &tf, &side, &tms);
		if (rc != HPLAI_OK) {
			std::fprintf(stderr, "hplai_autotune: %s\n", hplai_status_string(rc));
			return 1;
		}
		flags = tf;
		std::printf("autotune: %d panel(s) per update, %s, factorisation %.3f ms\n",
			(tf & HPLAI_FLAG_GROUP4) ? 4 : (tf & HPLAI_FLAG_GROUP2) ? 2 : 1,
			(tf & HPLAI_FLAG_LOOKAHEAD) ? "look-ahead" : "serial", tms);
		if (tf & HPLAI_FLAG_LOOKAHEAD) std::printf("autotune: %d side-stream SMs\n", side);
	}
	auto tg0 = std::chrono::steady_clock::now();
	rc = hplai_generate(ctx, seed);
	auto tg1 = std::chrono::steady_clock::now();
	if (rc != HPLAI_OK) {
		std::fprintf(stderr, "hplai_generate: %s\n", hplai_status_string(rc));
		return 1;
	}
	std::printf("generation: %.6f sec. (outside the timed region, as in the reference)\n",
		std::chrono::duration<double>(tg1 - tg0).count());
	print_ctime("#BEGIN: ");
	std::fflush(stdout);

	hplai_ir_errors er{-1.0, -1.0};
	int iters = 0;
	// with -w the refinement gets one step (main.cpp:322: maxit = warmup ? 1 : 50)
	if (warmup) maxit = 1;
	auto t0 = std::chrono::steady_clock::now();
	if (l1est) rc = hplai_l1est(ctx);
	else if (warmup) rc = hplai_factor_steps(ctx, nrow + 2);
	else rc = hplai_factor(ctx);
	if (rc == HPLAI_OK && checksum) {
		// inside the timed region, between the LU and the refinement (main.cpp:298-302)
		double sigs[3];
		const int rs = hplai_checksum(ctx, sigs);
		if (rs != HPLAI_OK) {
			std::fprintf(stderr, "hplai_checksum: %s\n", hplai_status_string(rs));
			return 1;
		}
		std::printf("check %22.17e %22.17e, %22.17e\n", sigs[0], sigs[1], sigs[2]);
		std::fflush(stdout);
	}
	int rr = HPLAI_OK;
	if (rc == HPLAI_OK) rr = hplai_refine(ctx, mode, maxit, &er, &iters);
	auto t1 = std::chrono::steady_clock::now();
	if (rc != HPLAI_OK) {
		std::fprintf(stderr, "hplai_factor: %s\n", hplai_status_string(rc));
		return 1;
	}
	std::vector<double> res(maxit > 0 ? maxit : 1), har(maxit > 0 ? maxit : 1);
	int cnt = 0;
	hplai_get_ir_log(ctx, res.data(), har.data(), maxit, &cnt);
	for (int i = 0; i < cnt; ++i)
		std::printf("# iterative refinement: step=%3d, residual=%20.16e hpl-harness=%f\n", i, res[i], har[i]);
	print_ctime("#END__: ");
	char line[256];
	const double secs = std::chrono::duration<double>(t1 - t0).count();
	if (warmup) {
		// the skipped trailing part leaves the flop count (main.cpp:441-446)
		const double nn = static_cast<double>(n) - static_cast<double>(nrow + 2) * b;
		const double flops = 2. / 3 * n * static_cast<double>(n) * n + 3. / 2 * n * static_cast<double>(n) -
			(2. / 3 * nn * nn * nn + 3. / 2 * nn * nn);
		std::snprintf(line, sizeof line, "%.9f sec. %.9f GFlop/s resid = %20.15e hpl-harness = %.9f", secs,
			flops / secs * 1e-9, er.residual, er.hpl_harness);
	} else {
		hplai_format_report(n, secs, er, line, sizeof line);
	}
	std::printf("%s\n", line);
	double ms[HPLAI_PH_COUNT];
	hplai_get_phase_ms(ctx, ms, HPLAI_PH_COUNT);
	std::printf("phases [ms]: DIAG_LU %.3f TRSM_L %.3f TRSM_R %.3f GEMM_UPDATE %.3f LAZY_INIT %.3f IR_GEMV %.3f "
	            "IR_TRSV %.3f\n",
		ms[HPLAI_PH_DIAG_LU], ms[HPLAI_PH_TRSM_L], ms[HPLAI_PH_TRSM_R], ms[HPLAI_PH_GEMM_UPDATE], ms[HPLAI_PH_LAZY_INIT],
		ms[HPLAI_PH_IR_GEMV], ms[HPLAI_PH_IR_TRSV]);
	std::fflush(stdout);
	int outer = 0, inner = 0;
	hplai_get_refine_counts(ctx, &outer, &inner);
	write_timerdump(jobid, n, b, secs, ms, static_cast<long long>(outer) + inner, (flags & HPLAI_FLAG_LOOKAHEAD) != 0,
		warmup);
	hplai_destroy(ctx);
	if (rr != HPLAI_OK && rr != HPLAI_ENOTCONV) {
		std::fprintf(stderr, "hplai_refine: %s\n", hplai_status_string(rr));
		return 1;
	}
	if (warmup) return 0;   // one refinement step of a partial factorisation: {-1, -1} by design
	return rr == HPLAI_OK ? 0 : 2;
}
