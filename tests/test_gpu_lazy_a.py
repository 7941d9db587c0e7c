"""HPLAI_FLAG_LAZY_A: the precision form's FP16 deck without a stored A.

The matrix is regenerated from the LCG when a block joins a panel and the
deck lives in the upper half of each FP32 column of the factors' storage.
The arithmetic is the stored-A deck form's (the same FP32 values of A, the
same fold a + deck / s), so the factors must be bit-identical to it under
every schedule; the solves converge as the stored-A form's do.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
DECK = 4   # HPLAI_FLAG_FP16_DECK


def _lu(hplai, n, b, flags, steps=None):
    with hplai.Solver(n, b, precision=hplai.F32_F8, flags=flags) as s:
        s.generate(42)
        if steps is None:
            s.factor()
        else:
            s.factor_steps(steps)
        return s.lu()


@pytest.mark.parametrize("n,b,extra", [(2048, 256, 0), (4096, 512, 8), (4096, 1024, 8 | 2), (3072, 128, 2),
                                       (8192, 1024, 8 | 2)])
def test_lazy_a_factors_bit_identical(hplai, torch_cuda, n, b, extra):
    want = _lu(hplai, n, b, DECK | extra)
    got = _lu(hplai, n, b, DECK | extra | hplai.FLAG_LAZY_A)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_lazy_a_solves_and_refuses_host_matrices(hplai, oracle, torch_cuda):
    n, b = 4096, 512
    with hplai.Solver(n, b, precision=hplai.F32_F8, flags=DECK | 8 | hplai.FLAG_LAZY_A) as s:
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=hplai.GMRES)
        x = s.x()
        assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0
        with pytest.raises(hplai.HplaiError):
            s.upload(oracle.matrix(n), oracle.rhs(n), oracle.diag(n), 42)
    xs = np.linalg.solve(oracle.dense_matrix_f64(n, 42), oracle.rhs(n))
    assert np.abs(x - xs).max() / np.abs(xs).max() < 1e-12


def test_lazy_a_flag_combinations(hplai):
    for prec, flags in [(1, 64), (0, 4 | 64), (1, 4 | 1 | 64)]:
        with pytest.raises(hplai.HplaiError):
            hplai.Solver(1024, 128, precision=prec, flags=flags)
    # the lazy form regenerates the LCG matrix: Higham's matrix is refused
    with hplai.Solver(1024, 128, precision=hplai.F32_F8, flags=DECK | hplai.FLAG_LAZY_A) as s:
        with pytest.raises(hplai.HplaiError):
            s.set_matrix(hplai.MATRIX_HIGHAM, 1000.0, 0.5)


def test_lazy_a_l1est_and_checksum(hplai, torch_cuda):
    """--l1est regenerates the whole matrix into the factors' storage (the
    deck is cleared again by the next factorisation) and gives the stored-A
    form's approximation; the checksum of the lazy factors equals the
    stored-A form's."""
    n, b = 2048, 256
    sig = []
    for flags in (DECK, DECK | hplai.FLAG_LAZY_A):
        with hplai.Solver(n, b, precision=hplai.F32_F8, flags=flags) as s:
            s.generate(42)
            s.l1est()
            e0 = s.lu()
            s.generate(42)
            s.factor()
            sig.append((e0, s.checksum()))
    assert np.array_equal(sig[0][0].view(np.uint32), sig[1][0].view(np.uint32))
    assert np.array_equal(sig[0][1], sig[1][1])
