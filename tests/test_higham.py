"""Higham's HPL-AI matrix (`--highammat`) on the CPU: parameters, definition
and the pin against the reference's own numbers (tests/golden/ref_c1.json,
written by tests/golden/make_ref_fixtures.py from the reference built here).

* alpha and beta: the reference's higham_mat_comp_beta (its source compiled
  alone) against the oracle's restatement and the library's host code, bit for
  bit, for 42 (n, cond, rho) triples -- including n >= 46341, where the
  reference's 32-bit integer terms wrap (at n = 65536 that moves beta by 1 %).
* The matrix is Higham's definition: A = L U with constant strictly
  triangular parts -alpha (L) and -beta (U), cond(A, inf) = 1000.
* The reference's `--highammat` refinement diverges.  Its printed step-0
  residual and harness are reproduced here from its own evaluation
  conventions -- the entries of its pmatgen (matgen.hpp:25-77: +alpha, +beta)
  with alpha and beta swapped in the diagonal blocks (hmg_gemv_diag,
  otf_gemv.cpp:296-314), its ||A|| (higham_infnorm, panel_norm.hpp:86-141),
  x_0 = b ./ diag, b the LCG's column n -- which pins alpha, beta, the
  diagonal and the right-hand side to the reference's numbers, and shows that
  the matrix it refines against is neither the one its precomputed path
  factors nor Higham's.
"""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_c1.json")))
H = FIX["higham"]


def test_beta_matches_the_reference_bit_for_bit(oracle, hplai):
    for rec in H["betas"]:
        want = float.fromhex(rec["beta"])
        a, b = oracle.higham_params(rec["n"], rec["cond"], rec["rho"])
        assert b == want, rec
        la, lb = hplai.higham_params(rec["n"], rec["cond"], rec["rho"])
        assert lb == want and la == rec["rho"] * want, rec


def test_matrix_is_highams_with_condition_1000(oracle):
    n = 1200
    a, b = oracle.higham_params(n)
    A = oracle.higham_dense_f64(n, a, b)
    L = np.eye(n) + np.tril(np.full((n, n), -a), -1)
    U = np.eye(n) + np.triu(np.full((n, n), -b), 1)
    assert np.abs(L @ U - A).max() <= 4 * np.finfo(np.float64).eps
    assert abs(np.linalg.cond(A, np.inf) - 1000.0) <= 1e-6
    assert abs(oracle.higham_norm(n, a, b) - np.abs(A).sum(1).max()) <= 1e-14 * np.abs(A).sum(1).max()
    f32 = oracle.higham_matrix(n, a, b)
    assert np.abs(f32.astype(np.float64) - A).max() <= 2 ** -24 * np.abs(A).max()


@pytest.mark.parametrize("run", ["not_r", "not_d_r"])
def test_reference_step0_from_its_own_conventions(oracle, run):
    n, bs = FIX["n"], FIX["b"]
    a, b = oracle.higham_params(n)
    ab = a * b
    i = np.arange(n, dtype=np.float64)
    I, J = np.meshgrid(i, i, indexing="ij")
    # pmatgen's entries (+alpha, +beta) ...
    gen = np.where(I < J, b + ab * I, np.where(I > J, a + ab * J, 1 + ab * I))
    # ... and the GEMV's, whose diagonal blocks swap alpha and beta
    same = (I // bs) == (J // bs)
    gemv = gen.copy()
    gemv[same & (I > J)] = (b + ab * J)[same & (I > J)]
    gemv[same & (I < J)] = (a + ab * I)[same & (I < J)]
    rhs = oracle.rhs(n)
    d = 1 + ab * i
    x0 = rhs / d
    normr = np.abs(rhs - gemv @ x0).max()
    norma = gen.sum(1).max()
    harness = normr / (norma * np.abs(x0).max() + np.abs(rhs).max()) / (n * np.finfo(np.float64).eps / 2)
    want = H["runs"][run]["first_steps"][0]
    assert abs(normr - want["residual"]) <= 1e-13 * want["residual"]
    assert abs(harness - want["hpl_harness"]) <= 1e-12 * want["hpl_harness"]
    # neither the matrix its precomputed path factors nor Higham's gives that residual
    for other in (gen, oracle.higham_dense_f64(n, a, b)):
        assert abs(np.abs(rhs - other @ x0).max() - want["residual"]) > 1e-4
    # and the refinement diverges: IRErrors {-1, -1} after 50 steps
    assert H["runs"][run]["steps"] == 50 and H["runs"][run]["hpl_harness"] == -1.0


def test_params_arguments(hplai):
    for n, cond, rho in [(1200, 0.5, 0.5), (1200, 1000.0, 0.0), (1, 1000.0, 0.5)]:
        with pytest.raises(hplai.HplaiError):
            hplai.higham_params(n, cond, rho)
