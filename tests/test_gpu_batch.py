"""The batched solver (many independent systems on one GPU) on the B200.

System s is the HPL-AI matrix of order n[s] from seed[s], with nrhs[s]
right-hand sides taken from columns n, n+1, ... of its LCG stream.  The
extra columns are integer/generator work and must match the oracle bit for
bit; solutions are compared with a dense FP64 solve of the same system
(1e-12 relative, converged solutions of a matrix with cond_inf of a few
units), and every right-hand side must reach hpl-harness < 16.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def stream_columns(oracle, n, seed, first, count):
    return np.array([[oracle.elem(n, i, n + first + r, seed) for i in range(n)] for r in range(count)]).T


def test_rhs_columns_bit_exact(hplai, oracle, torch_cuda):
    torch = torch_cuda
    n, seed = 640, 7
    out = torch.empty(n * 3, dtype=torch.float64, device="cuda")
    hplai.check(hplai.gen_rhs_cols(n, seed, 0, 3, out.data_ptr(), None))
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(3, n).T
    assert np.array_equal(got[:, 0], oracle.rhs(n, seed))
    assert np.array_equal(got, stream_columns(oracle, n, seed, 0, 3))


def test_small_batch_vs_dense(hplai, oracle, torch_cuda):
    n = [256, 192, 512, 320, 128, 1024, 448, 64]
    nrhs = [1, 3, 2, 1, 4, 2, 1, 3]
    seeds = [11, 12, 13, 14, 15, 16, 17, 18]
    with hplai.Batch(n, nrhs, seeds, workers=4) as bt:
        assert bt.solve() == hplai.HPLAI_OK
        for s in range(len(n)):
            res = bt.result(s)
            assert res.status == hplai.HPLAI_OK and 0.0 <= res.hpl_harness < 16.0, (s, res)
            assert n[s] % bt.block(s) == 0
            x = bt.x(s)
            a = oracle.dense_matrix_f64(n[s], seeds[s])
            rhs = stream_columns(oracle, n[s], seeds[s], 0, nrhs[s])
            ref = np.linalg.solve(a, rhs)
            err = np.max(np.abs(x - ref)) / np.max(np.abs(ref))
            assert err < 1e-12, (s, err)


def test_batch_rejects_bad_sizes(hplai):
    with pytest.raises(hplai.HplaiError):
        hplai.Batch([100], [1], [1])          # no multiple of 16 divides 100
    with pytest.raises(hplai.HplaiError):
        hplai.Batch([256], [0], [1])


def test_batch_workload_512_systems(hplai, torch_cuda):
    """The 512-system workload: log-uniform orders 256..4096, 1..8
    right-hand sides each, system s seeded with s."""
    n, nrhs = hplai.batch_sizes(512)
    assert n.min() >= 256 and n.max() <= 4096 and np.all(n % 64 == 0)
    with hplai.Batch(n, nrhs, np.arange(512), workers=8) as bt:
        assert bt.solve() == hplai.HPLAI_OK
        worst = max(bt.result(s).hpl_harness for s in range(512))
        assert worst < 16.0
