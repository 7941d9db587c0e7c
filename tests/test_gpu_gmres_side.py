"""GMRES-IR with right (flexible) and left preconditioning by the e4m3 LU.

Right preconditioning keeps z_j = M^{-1} v_j and corrects by Z y: one
application of (L U)^{-1} per inner step, none before or after, where the
left form needs one more per cycle.  Both must converge to hpl-harness < 16
in about as many residual evaluations, and agree with the dense FP64
solution."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,b,flags", [(4096, 512, 4), (8192, 1024, 4 | 128 | 2), (3072, 256, 0)])
def test_gmres_sides_agree(hplai, oracle, torch_cuda, n, b, flags):
    out = {}
    with hplai.Solver(n, b, precision=hplai.F32_F8, flags=flags) as s:
        s.generate(42)
        s.factor()
        for right in (True, False):
            s.set_gmres_side(right)
            res = s.iterative_refinement(50, mode=hplai.GMRES)
            assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, (right, res)
            out[right] = (s.x(), s.refine_counts())
    assert out[True][1][0] <= out[False][1][0] + 1    # residual evaluations (equal in practice)
    if n <= 4096:
        xs = np.linalg.solve(oracle.dense_matrix_f64(n, 42), oracle.rhs(n, 42))
        for right in (True, False):
            assert np.abs(out[right][0] - xs).max() / np.abs(xs).max() < 1e-11, right


def test_gmres_side_arguments(hplai):
    with hplai.Solver(1024, 128, precision=hplai.F32_F8) as s:
        s.set_gmres_side(True)
        s.set_gmres_side(False)
    assert hplai._set_gmres_side(None, 1) == hplai.HPLAI_EINVAL
