// ref_xdump.cpp -- compiles the reference's main.cpp unchanged (it is
// #included from the reference tree by oracle/build_ref.sh, with main
// renamed to hplai_rank_main) and hands the solution vector of its
// iterative refinement to the thread-rank runtime, which writes it to the
// file named by TMPI_XDUMP; with TMPI_LUDUMP=<file> the factored matrix
// (FP32, n x n column-major: unit L below the diagonal, U on and above) as
// the LU left it, before the refinement.  The reference prints the residual and the
// harness but never x (iterative_refinement.hpp:18-57, main.cpp:319-441).
//
// TEST INFRASTRUCTURE ONLY (see mpi.h).
#include "iterative_refinement.hpp"

extern "C" void tmpi_xdump_put(long long first, const double *x, int count, long long n);
extern "C" void tmpi_xdump_rank_done(void);
extern "C" void tmpi_ludump_put(long long row0, long long col0, const float *blk, long long ld, int b, long long n);
extern "C" void tmpi_ludump_rank_done(void);

// The reference's refinement, then every block of x this rank owns: a
// column-vector block i is held by the rank whose process column owns the
// diagonal block of the same index (panel.hpp:277-291).
template <typename P, typename M, typename G>
IRErrors tmpi_refine_and_dump(P const &p, M &mg, double *x, double *w, size_t ldv, double *rhs, double norma,
	double normb, int maxit, G &grid)
{
	const long long n = static_cast<long long>(p.nblocks) * p.b;
	// local block (i, j) is global block (i1 + i istride, j1 + j jstride);
	// its element (ii, jj) lies at panel_address(i, j)[jj lda + ii] (panel.hpp:20-60, 135-230)
	if (sizeof(*p(0, 0)) == sizeof(float)) {
		for (int j = 0; j < p.npcol; ++j)
			for (int i = 0; i < p.nprow; ++i)
				tmpi_ludump_put(static_cast<long long>(p.i1 + i * p.istride) * p.b,
					static_cast<long long>(p.j1 + j * p.jstride) * p.b, reinterpret_cast<const float *>(p(i, j)),
					static_cast<long long>(p.lda), p.b, n);
	}
	tmpi_ludump_rank_done();
	IRErrors e = iterative_refinement(p, mg, x, w, ldv, rhs, norma, normb, maxit, grid);
	for (int i = 0; i < p.nprow; ++i) {
		const int ipos = p.i1 + i * p.istride;
		if (ipos % p.jstride == p.j1) tmpi_xdump_put(static_cast<long long>(ipos) * p.b, x + p.b * i, p.b, n);
	}
	tmpi_xdump_rank_done();
	return e;
}

// Only the calls in main.cpp see this: the template above was defined first.
#define iterative_refinement(...) tmpi_refine_and_dump(__VA_ARGS__)
#include "main.cpp"
