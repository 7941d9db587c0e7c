"""End-to-end solves through the context API against the oracle (B200)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_c1_solve_matches_reference_and_oracle(hplai, oracle, torch_cuda):
    """n=1200, b=60, seed 42: hpl-harness < 16, the step-0 residual equals the
    reference's published value to 1e-13 (summation order differs), and x
    matches the oracle's x and a dense FP64 solve to 1e-12 relative."""
    g = json.load(open(os.path.join(HERE, "golden", "readme_step0.json")))
    n, b = g["n"], g["b"]
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.factor()
        r = s.iterative_refinement(50)
        x = s.x()
        log = s.ir_log()
        assert np.array_equal(s.rhs(), oracle.rhs(n))
        assert np.array_equal(s.diag(), oracle.diag(n))
        norma, normb = s.norms()
    assert r.status == hplai.HPLAI_OK and 0 <= r.hpl_harness < 16
    assert abs(log[0][0] - g["step0_residual"]) <= 1e-13 * g["step0_residual"]
    assert abs(log[0][1] - g["step0_harness"]) <= 1e-12 * g["step0_harness"]
    rc, xo, res, har, steps = oracle.solve(n, b, q=1)
    assert rc == 0
    assert np.abs(x - xo).max() <= 1e-12 * np.abs(xo).max()
    a = oracle.dense_matrix_f64(n)
    xr = np.linalg.solve(a, oracle.rhs(n))
    assert np.abs(x - xr).max() <= 1e-12 * np.abs(xr).max()
    assert norma == 2 * oracle.diag(n).max() and normb == np.abs(oracle.rhs(n)).max()


def test_c1_factors_close_to_oracle(hplai, oracle, torch_cuda):
    """LU factors: the first panel step is bit-exact, the rest differs only by
    the Schur update's FP32 summation order."""
    n, b = 1200, 60
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.factor()
        lu = s.lu()
    ref = oracle.lu(oracle.matrix(n), b)
    assert np.array_equal(lu[:, :b].view(np.uint32), ref[:, :b].view(np.uint32))
    assert np.array_equal(lu[:b, :].view(np.uint32), ref[:b, :].view(np.uint32))
    rel = np.abs(lu.astype(np.float64) - ref) / (np.abs(ref) + 1e-3 * np.abs(ref).max())
    assert rel.max() < 1e-3


@pytest.mark.parametrize("n,b", [(2048, 64), (3000, 100), (8192, 256), (16384, 512)])
def test_larger_solves_converge(hplai, oracle, torch_cuda, n, b):
    """Size-independent checks: hpl-harness < 16 (the FP64 backward-error
    criterion on the regenerated matrix) and the step-0 residual, which only
    involves the generator and the FP64 GEMV, against the oracle."""
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.factor()
        r = s.iterative_refinement(50)
        log = s.ir_log()
    assert r.status == hplai.HPLAI_OK and 0 <= r.hpl_harness < 16 and r.iters <= 6
    zero = np.zeros((n, n), dtype=np.float32, order="F") if n <= 4096 else None
    if zero is not None:
        _, _, _, _, steps = oracle.refine(zero, b, 42, oracle.rhs(n), oracle.diag(n), maxit=1)
        assert abs(log[0][0] - steps[0][0]) <= 1e-12 * steps[0][0]


def test_solve_host_matches_device_path(hplai, oracle, torch_cuda):
    n, b = 1200, 60
    a = oracle.matrix(n)
    with hplai.Solver(n, b) as s:
        x, r = s.solve_host(a, oracle.rhs(n), oracle.diag(n), 42, 50)
        assert r.status == hplai.HPLAI_OK and r.hpl_harness < 16
        s.generate(42)
        s.factor()
        s.iterative_refinement(50)
        assert np.array_equal(s.x(), x)


def test_call_order_and_nonconvergence(hplai, torch_cuda):
    with hplai.Solver(480, 60) as s:
        with pytest.raises(hplai.HplaiError) as e:
            s.factor()
        assert e.value.status == hplai.HPLAI_ESTATE
        s.generate(42)
        with pytest.raises(hplai.HplaiError):
            s.iterative_refinement(5)          # before factor
        s.factor()
        r = s.iterative_refinement(1)          # one step cannot reach < 16: IRErrors {-1,-1}
        assert r.status == hplai.HPLAI_ENOTCONV and r.residual == -1 and r.hpl_harness == -1
        r = s.iterative_refinement(50)
        assert r.status == hplai.HPLAI_OK
