"""Parity at the full benchmark sizes: n = 65536 (b = 512, plain form) and
n = 131072 (b = 1024, plain and precision forms).

The CPU oracle cannot factor these systems in test time, so the checks are
the size-independent ones:
  * the solution's FP64 residual r = b - A x (A regenerated in FP64 by the
    GPU's on-the-fly GEMV, as the refinement does) agrees on 64 sampled rows
    with the oracle's long-double row sums of the same generated matrix, to
    1e-13 ||A||_inf ||x||_inf;
  * the diagonal (the sequential FP64 row sums) equals the oracle's on the
    sampled rows bit for bit;
  * the hpl-harness recomputed from that residual
    (iterative_refinement.hpp:43) is below 16 and equals the harness the
    solver reported for its last step.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


def _check_solution(hplai, oracle, torch, s, n, rep, seed=42, nsample=64):
    x = s.x()
    rhs = s.rhs()
    d = s.diag()
    norma, normb = s.norms()
    # the diagonal on the sampled rows, bit for bit
    rng = np.random.default_rng(n + 7)
    rows = np.sort(rng.choice(n, size=nsample, replace=False)).astype(np.int64)
    rows[0], rows[-1] = 0, n - 1
    want_d = np.array([oracle.calc_diag(int(i), n, seed) for i in rows[:8]])
    assert np.array_equal(d[rows[:8]], want_d)
    assert norma == 2.0 * d.max() and normb == np.abs(rhs).max()
    # the GPU's full residual through the on-the-fly GEMV leaf
    xd = torch.from_numpy(x).cuda()
    rd = torch.from_numpy(rhs).cuda()
    dd = torch.from_numpy(d).cuda()
    ws = hplai.otf_gemv_workspace(n)
    w = torch.empty(ws // 8 + 1, dtype=torch.float64, device="cuda")
    hplai.check(hplai.otf_gemv(n, -1.0, xd.data_ptr(), 1.0, rd.data_ptr(), seed, dd.data_ptr(), w.data_ptr(), ws,
                               None))
    torch.cuda.synchronize()
    r_gpu = rd.cpu().numpy()
    normx = np.abs(x).max()
    # the oracle's rows of the same residual
    r_orc = oracle.residual_rows(n, x, rows, seed=seed)
    tol = 1e-13 * norma * normx
    err = np.abs(r_gpu[rows] - r_orc).max()
    assert err <= tol, (err, tol)
    # the harness from the verified residual
    normr = np.abs(r_gpu).max()
    harness = normr / (norma * normx + normb) * 2.0 / (n * EPS)
    assert 0 <= harness < 16, harness
    assert abs(harness - rep.hpl_harness) <= 1e-9 * max(harness, 1e-300), (harness, rep.hpl_harness)
    assert abs(normr - rep.residual) <= 1e-9 * max(normr, 1e-300)
    # the sampled oracle rows cannot exceed the full norm beyond the tolerance
    assert np.abs(r_orc).max() <= normr + tol


def test_c2_plain_residual_vs_oracle_rows(hplai, oracle, torch_cuda):
    n, b = 65536, 512
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.factor()
        rep = s.iterative_refinement(50)
        assert rep.status == hplai.HPLAI_OK, rep
        _check_solution(hplai, oracle, torch_cuda, s, n, rep)


def test_c2_lookahead_deck_residual_vs_oracle_rows(hplai, oracle, torch_cuda):
    """The C2 size with look-ahead and the FP16 deck (the schedule and the
    trailing-matrix form the autotuned bench may pick)."""
    n, b = 65536, 512
    with hplai.Solver(n, b, flags=hplai.FLAG_LOOKAHEAD | hplai.FLAG_FP16_DECK) as s:
        s.generate(42)
        s.factor()
        rep = s.iterative_refinement(50)
        assert rep.status == hplai.HPLAI_OK, rep
        _check_solution(hplai, oracle, torch_cuda, s, n, rep)


def test_c2_group2_residual_vs_oracle_rows(hplai, oracle, torch_cuda):
    """The C2 size with two-panel groups (K = 1024 trailing updates)."""
    n, b = 65536, 512
    with hplai.Solver(n, b, flags=hplai.FLAG_GROUP2) as s:
        s.generate(42)
        s.factor()
        rep = s.iterative_refinement(50)
        assert rep.status == hplai.HPLAI_OK, rep
        _check_solution(hplai, oracle, torch_cuda, s, n, rep)


@pytest.mark.parametrize("form", ["precision", "plain", "precision-group2", "plain-group2"])
def test_c3_residual_vs_oracle_rows(hplai, oracle, torch_cuda, form):
    """n = 131072, b = 1024: the precision form (e4m3 Schur into the FP16
    deck, GMRES-IR) and the plain form (FP16 Schur into the FP32 trailing
    matrix, IR), with one- and two-panel trailing updates, one after the
    other."""
    n, b = 131072, 1024
    if form.startswith("precision"):
        prec, flags, mode = hplai.F32_F8, hplai.FLAG_FP16_DECK, hplai.GMRES
    else:
        prec, flags, mode = hplai.F32_F16, 0, hplai.IR
    if form.endswith("group2"):
        flags |= hplai.FLAG_GROUP2
    with hplai.Solver(n, b, precision=prec, flags=flags) as s:
        s.generate(42)
        s.factor()
        rep = s.iterative_refinement(50, mode=mode)
        assert rep.status == hplai.HPLAI_OK, rep
        outer, inner = s.refine_counts()
        assert outer <= 5 and (mode == hplai.IR or inner <= 30)
        _check_solution(hplai, oracle, torch_cuda, s, n, rep)


def test_l1est_beyond_the_grid_y_limit(hplai, torch_cuda):
    """--l1est at an order above 65535 (one CTA row per column no longer
    fits a launch's y dimension): the scaling covers every column, and the
    refinement from those approximate factors converges."""
    n, b = 65664, 128
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.l1est()
        res = s.iterative_refinement(50)
        assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, res
