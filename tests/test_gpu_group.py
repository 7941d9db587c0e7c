"""Two-panel groups (HPLAI_FLAG_GROUP2): the trailing matrix is updated once
per two panels with K = 2b (C -= [L_k L_k+1][U_k; U_k+1]), the group's
second block first receiving its first panel's update alone.

* The schedule is exact arithmetic reordered: with look-ahead (both panels of
  the next group formed on the side stream) the factors are bit-identical to
  the one-stream schedule.
* Against one-panel groups the factors differ only by where the FP32
  accumulator is rounded into C (once per two panels instead of once per
  panel): elementwise within the FP16 operand level.
* Every form's solve converges to hpl-harness < 16 and matches the dense FP64
  solution to 1e-11 (the same bar as the one-panel forms).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lu(hplai, n, b, flags, precision=0):
    with hplai.Solver(n, b, precision=precision, flags=flags) as s:
        s.generate(42)
        s.factor()
        return s.lu()


def _dense_x(oracle, n):
    a = oracle.dense_matrix_f64(n, 42)
    return np.linalg.solve(a, oracle.rhs(n, 42))


@pytest.mark.parametrize("n,b,extra,precision", [(4096, 512, 0, 0), (3840, 256, 0, 0), (6144, 1024, 0, 0),
                                                 (4096, 256, 1, 0), (4096, 512, 4, 1), (3584, 256, 4, 0)])
def test_group2_lookahead_matches_serial(hplai, torch_cuda, n, b, extra, precision):
    """Both schedules issue the same kernels on the same data in the same
    order per element; odd and even panel counts, SIMT panels, the deck."""
    g = hplai.FLAG_GROUP2 | extra
    a = _lu(hplai, n, b, g | hplai.FLAG_LOOKAHEAD, precision)
    z = _lu(hplai, n, b, g, precision)
    assert np.array_equal(a.view(np.uint32), z.view(np.uint32))


@pytest.mark.parametrize("n,b", [(4096, 512), (3840, 256)])
def test_group2_factors_close_to_one_panel_groups(hplai, torch_cuda, n, b):
    """Only the accumulator's rounding into C moves: far below the FP16
    operands' own error (relative to the entry scale)."""
    one = _lu(hplai, n, b, 0).astype(np.float64)
    two = _lu(hplai, n, b, hplai.FLAG_GROUP2).astype(np.float64)
    scale = np.abs(one) + 1e-3 * np.abs(one).max()
    assert (np.abs(one - two) / scale).max() < 1e-3


@pytest.mark.parametrize("precision,flags,mode,n,b", [
    (0, 0, 0, 4096, 512), (0, 0, 0, 3840, 256), (0, 4, 0, 4096, 256),
    (1, 4, 1, 4096, 512), (1, 0, 1, 3072, 1024), (1, 4 | 2, 1, 8192, 1024)])
def test_group2_solves_match_dense(hplai, oracle, torch_cuda, precision, flags, mode, n, b):
    with hplai.Solver(n, b, precision=precision, flags=flags | hplai.FLAG_GROUP2) as s:
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=mode)
        x = s.x()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, res
    if n <= 4096:
        xs = _dense_x(oracle, n)
        assert np.max(np.abs(x - xs)) / np.max(np.abs(xs)) < 1e-11


def test_group2_needs_block_multiple_of_128(hplai):
    with pytest.raises(hplai.HplaiError):
        hplai.Solver(1200, 60, flags=hplai.FLAG_GROUP2)


def test_autotune_considers_groups(hplai, oracle, torch_cuda):
    """The tuner times one- and two-panel groups (b = 512 allows both) after a
    warm-up, records every trial, and the chosen schedule solves."""
    n, b = 4096, 512
    with hplai.Solver(n, b) as s:
        flags, side, ms = s.autotune(42)
        log = s.autotune_log()
        groups = {bool(f & hplai.FLAG_GROUP2) for f, _, _ in log}
        assert groups == {False, True} and len(log) >= 11 and ms > 0
        assert flags & ~(hplai.FLAG_LOOKAHEAD | hplai.FLAG_GROUP2) == 0
        s.factor()
        res = s.iterative_refinement(50)
        x = s.x()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0
    xs = _dense_x(oracle, n)
    assert np.max(np.abs(x - xs)) / np.max(np.abs(xs)) < 1e-12


@pytest.mark.parametrize("precision,flags", [(0, 0), (0, 8), (1, 4 | 8)])
def test_tile_group_does_not_change_results(hplai, torch_cuda, precision, flags):
    """The tile order only decides which CTA computes which tile when: every
    C element still receives each update once, so the factors are
    bit-identical under any tile group."""
    n, b = 4096, 512
    out = []
    for gm in (0, 1, 16, 64, 1024):
        with hplai.Solver(n, b, precision=precision, flags=flags) as s:
            s.set_tile_group(gm)
            assert s.tile_group() == (gm if gm else 32)
            s.generate(42)
            s.factor()
            out.append(s.lu().view(np.uint32))
    for o in out[1:]:
        assert np.array_equal(out[0], o)


def test_autotune_trials_cover_tile_groups(hplai, torch_cuda):
    with hplai.Solver(4096, 512) as s:
        s.autotune(42)
        trials = s.autotune_trials()
        assert {tg for _, _, tg, _ in trials} >= {16, 32, 64}
        assert len(trials) == len(s.autotune_log())
        assert s.tile_group() in (16, 32, 64)
        with pytest.raises(hplai.HplaiError):
            s.set_tile_group(-1)
