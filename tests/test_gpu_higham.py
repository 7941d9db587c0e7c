"""Higham's HPL-AI matrix (hplai_set_matrix(HPLAI_MATRIX_HIGHAM), the
reference's --highammat) on the B200.

* Generation: the FP32 matrix and the FP64 diagonal bit for bit against the
  oracle (the reference's float formula, one fused multiply-add per entry).
* The refinement's GEMV regenerates the FP64 entries: the step-0 residual
  equals the oracle's long-double residual.
* Every form converges to hpl-harness < 16 -- plain IR, plain GMRES, the
  e4m3 precision form with the FP16 deck and two-panel groups -- and the
  solution matches the dense FP64 solve to the forward-error bound of a
  converged solve, cond(A, inf) x 16 n eps (cond = 1000), or, at n = 65536,
  the oracle's residual rows bound the harness below 16.
* The LU of A = L U recovers Higham's factors (constant -alpha, -beta): the
  first block row and column (no Schur update yet) to b FP32 roundings, the
  rest within the drift of the FP16-operand updates (5 % of beta after 4096
  rows); hplai_l1est writes them exactly.
* The adjoint solve (A^T, the two constants swapped) and the driver flag.
"""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
EPS = np.finfo(np.float64).eps


def _solver(hplai, n, b, precision=0, flags=0):
    s = hplai.Solver(n, b, precision=precision, flags=flags)
    s.set_matrix(hplai.MATRIX_HIGHAM)
    s.generate(42)
    return s


def test_generation_bit_exact(hplai, oracle, torch_cuda):
    n, b = 1200, 60
    a, be = oracle.higham_params(n)
    with _solver(hplai, n, b) as s:
        assert np.array_equal(s.lu().view(np.uint32), oracle.higham_matrix(n, a, be).view(np.uint32))
        assert np.array_equal(s.diag(), oracle.higham_diag(n, a, be))
        assert np.array_equal(s.rhs(), oracle.rhs(n))
        norma, _ = s.norms()
        assert abs(norma - oracle.higham_norm(n, a, be)) <= 1e-14 * norma


def test_step0_residual_is_the_fp64_residual(hplai, oracle, torch_cuda):
    n, b = 1200, 60
    a, be = oracle.higham_params(n)
    with _solver(hplai, n, b) as s:
        s.factor()
        s.iterative_refinement(1)
        r0 = s.ir_log()[0][0]
    x0 = oracle.rhs(n) / oracle.higham_diag(n, a, be)
    want = np.abs(oracle.higham_residual_rows(n, a, be, x0, np.arange(n), oracle.rhs(n))).max()
    assert abs(r0 - want) <= 1e-13 * want


@pytest.mark.parametrize("n,b,precision,flags,mode", [
    (1200, 60, 0, 0, 0), (1200, 60, 0, 0, 1), (1200, 60, 1, 0, 1),
    (4096, 256, 0, 0, 0), (4096, 256, 0, 8, 1), (4096, 256, 1, 4, 1), (4096, 512, 1, 4 | 8 | 2, 1)])
def test_solves_match_dense(hplai, oracle, torch_cuda, n, b, precision, flags, mode):
    a, be = oracle.higham_params(n)
    with _solver(hplai, n, b, precision, flags) as s:
        s.factor()
        res = s.iterative_refinement(50, mode=mode)
        x = s.x()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, res
    xs = np.linalg.solve(oracle.higham_dense_f64(n, a, be), oracle.rhs(n))
    assert np.abs(x - xs).max() / np.abs(xs).max() < 1000.0 * 16 * n * EPS


@pytest.mark.parametrize("precision,flags,mode", [(0, 8, 0), (1, 4 | 8, 1)])
def test_large_solves_vs_oracle_rows(hplai, oracle, torch_cuda, precision, flags, mode):
    n, b = 65536, 1024
    a, be = oracle.higham_params(n)
    with _solver(hplai, n, b, precision, flags) as s:
        s.factor()
        res = s.iterative_refinement(50, mode=mode)
        x = s.x()
        norma, normb = s.norms()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, res
    rows = np.sort(np.random.default_rng(5).choice(n, 48, replace=False))
    r = oracle.higham_residual_rows(n, a, be, x, rows, oracle.rhs(n))
    bound = np.abs(r).max() / (norma * np.abs(x).max() + normb) * 2.0 / (n * EPS)
    assert bound < 16.0
    assert abs(norma - oracle.higham_norm(n, a, be)) <= 1e-13 * norma


def test_lu_recovers_highams_factors_and_l1est_writes_them(hplai, oracle, torch_cuda):
    n, b = 4096, 256
    a, be = oracle.higham_params(n)
    exact = np.where(np.tri(n, k=-1, dtype=bool), -a, np.where(np.eye(n, dtype=bool), 1.0, -be))
    with _solver(hplai, n, b) as s:
        s.factor()
        lu = s.lu().astype(np.float64)
        err = np.abs(lu - exact)
        # FP32 LU of the first diagonal block: b roundings of entries near 1
        tol = 2 * b * 2.0 ** -24
        assert err[:, :b].max() <= tol and err[:b, :].max() <= tol
        assert err.max() <= 0.05 * be
        s.l1est()
        assert np.array_equal(s.lu(), exact.astype(np.float32))
        res = s.iterative_refinement(50)
        assert res.status == hplai.HPLAI_OK and len(s.ir_log()) <= 3


def test_transpose_solve(hplai, oracle, torch_cuda):
    n, b = 2048, 128
    a, be = oracle.higham_params(n)
    g = np.random.default_rng(3).standard_normal(n)
    with _solver(hplai, n, b) as s:
        s.factor()
        lam, res = s.solve_transpose(g)
    assert res.status == hplai.HPLAI_OK
    want = np.linalg.solve(oracle.higham_dense_f64(n, a, be).T, g)
    assert np.abs(lam - want).max() / np.abs(want).max() < 1000.0 * 16 * n * EPS


def test_driver_highammat(hplai, torch_cuda, tmp_path):
    exe = os.path.abspath(os.path.join(HERE, "..", "hpl-ai_b200", "driver.out"))
    for extra in ([], ["--fp8"]):
        out = subprocess.run([exe, "4096", "256", "2", "-not", "-r", "--highammat"] + extra, capture_output=True,
                             text=True, timeout=300, cwd=tmp_path)
        assert out.returncode == 0, out.stderr
        assert " hmat" in out.stdout
        m = re.search(r"resid = (\S+) hpl-harness = (\S+)$", out.stdout, re.M)
        assert m and 0 <= float(m.group(2)) < 16, out.stdout
