"""Four-panel groups (HPLAI_FLAG_GROUP4): the trailing matrix is updated once
per four panels with K = 4b, the group's block e + j first receiving the
updates of panels e .. e + j - 1 each alone.

* Look-ahead (the next group's four panels formed on the side stream) is
  bit-identical to the one-stream schedule, for panel counts that are and are
  not multiples of four, with FP32 C, the FP16 deck, e4m3 operands and the
  matrix regenerated (HPLAI_FLAG_LAZY_A).
* Against two-panel groups the factors move only by the accumulator's
  rounding into C (FP32 C; e4m3: also the group's shared factors).
* Every form's solve converges to hpl-harness < 16 and matches the dense FP64
  solution to 1e-11.
* A context created with HPLAI_FLAG_GROUP4 can be set to one-, two- or
  four-panel groups; one created without it refuses four.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G2, G4, LA, DECK, LAZY = 8, 128, 2, 4, 64


def _lu(hplai, n, b, flags, precision=0):
    with hplai.Solver(n, b, precision=precision, flags=flags) as s:
        s.generate(42)
        s.factor()
        return s.lu()


def _dense_x(oracle, n):
    a = oracle.dense_matrix_f64(n, 42)
    return np.linalg.solve(a, oracle.rhs(n, 42))


@pytest.mark.parametrize("n,b,extra,precision", [(4096, 512, 0, 0), (5120, 512, 0, 0), (6144, 1024, 0, 0),
                                                 (3584, 256, 1, 0), (4608, 512, DECK, 1), (8192, 1024, DECK, 1),
                                                 (7168, 1024, DECK | LAZY, 1), (3840, 256, DECK, 0)])
def test_group4_lookahead_matches_serial(hplai, torch_cuda, n, b, extra, precision):
    a = _lu(hplai, n, b, G4 | extra | LA, precision)
    z = _lu(hplai, n, b, G4 | extra, precision)
    assert np.array_equal(a.view(np.uint32), z.view(np.uint32))


@pytest.mark.parametrize("n,b", [(4096, 512), (5120, 256)])
def test_group4_factors_close_to_two_panel_groups(hplai, torch_cuda, n, b):
    two = _lu(hplai, n, b, G2).astype(np.float64)
    four = _lu(hplai, n, b, G4).astype(np.float64)
    scale = np.abs(two) + 1e-3 * np.abs(two).max()
    assert (np.abs(two - four) / scale).max() < 1e-3


@pytest.mark.parametrize("precision,flags,mode,n,b", [
    (0, 0, 0, 4096, 512), (0, 0, 0, 5120, 256), (0, DECK, 0, 4096, 256),
    (1, DECK, 1, 4096, 512), (1, 0, 1, 5120, 1024), (1, DECK | LA, 1, 8192, 1024),
    (1, DECK | LA | LAZY, 1, 9216, 1024)])
def test_group4_solves_match_dense(hplai, oracle, torch_cuda, precision, flags, mode, n, b):
    with hplai.Solver(n, b, precision=precision, flags=flags | G4) as s:
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=mode)
        x = s.x()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, res
    if n <= 5120:
        xs = _dense_x(oracle, n)
        assert np.max(np.abs(x - xs)) / np.max(np.abs(xs)) < 1e-11


def test_group4_schedule_switching(hplai, torch_cuda):
    """A four-panel context runs every group size; each schedule's factors
    equal those of a context created for it."""
    n, b = 4096, 512
    with hplai.Solver(n, b, precision=1, flags=G4 | DECK) as s:
        for g, want_flags in ((0, DECK), (G2, DECK | G2), (G4, DECK | G4)):
            s.set_schedule(g | LA, -16)
            s.generate(42)
            s.factor()
            got = s.lu()
            want = _lu(hplai, n, b, want_flags, 1)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), g
        with pytest.raises(hplai.HplaiError):
            s.set_schedule(G2 | G4, 16)
    with hplai.Solver(n, b, precision=1, flags=DECK) as s:
        with pytest.raises(hplai.HplaiError):
            s.set_schedule(G4, 16)


def test_group4_flag_checks(hplai):
    with pytest.raises(hplai.HplaiError):
        hplai.Solver(1200, 60, flags=G4)
    with pytest.raises(hplai.HplaiError):
        hplai.Solver(1024, 128, flags=G4 | G2)
    with pytest.raises(hplai.HplaiError):
        hplai.Solver(1024, 128, flags=G4 | 16)   # HPLAI_FLAG_REF_DECK


def test_autotune_considers_four_panel_groups(hplai, torch_cuda):
    n, b = 4096, 512
    with hplai.Solver(n, b, precision=1, flags=G4 | DECK) as s:
        flags, side, ms = s.autotune(42)
        groups = {4 if f & G4 else 2 if f & G2 else 1 for f, _, _ in s.autotune_log()}
        assert groups == {1, 2, 4}
        s.factor()
        res = s.iterative_refinement(50, mode=1)
        assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0


@pytest.mark.parametrize("args", [["--fp8", "-d", "--group", "4", "--lookahead"], ["--group", "4"],
                                  ["--fp8", "--lazy-a", "--autotune"]])
def test_driver_four_panel_groups(hplai, torch_cuda, tmp_path, args):
    """driver.out with --group 4 (and the tuner, which may pick it) converges
    and prints the reference's report line."""
    import os
    import re
    import subprocess
    exe = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", "hpl-ai_b200", "driver.out"))
    out = subprocess.run([exe, "8192", "1024", "2"] + args, capture_output=True, text=True, timeout=300,
                         cwd=tmp_path)
    assert out.returncode == 0, out.stderr
    m = re.search(r"^(\S+) sec\. (\S+) GFlop/s resid = (\S+) hpl-harness = (\S+)$", out.stdout, re.M)
    assert m and 0 <= float(m.group(4)) < 16, out.stdout
