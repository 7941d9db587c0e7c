"""The oracle and the GPU path against the reference's own outputs at C1
(n = 1200, b = 60, seed 42, 2 x 2 grid), from tests/golden/ref_c1.json
(written by tests/golden/make_ref_fixtures.py from the reference's CPU driver
built by oracle/build_ref.sh).

* The oracle's LU is the reference's LU bit for bit when the reference is
  linked with a netlib-order BLAS (its own BLAS is unpinned): the SHA-256 of
  the FP32 factors match.
* The refinement's step-0 residual and harness equal the reference's in every
  run; step 1 depends on the grid's TRSV summation order (the oracle follows a
  single process column), so it is compared to 1e-8.
* The driver's two other factor paths pin the same way: `--l1est`
  (approximate factors without a decomposition) bit for bit, and the `-w`
  warm-up (the first P + 2 = 4 block steps) bit for bit against the oracle's
  truncated LU; on the GPU, hplai_l1est is bit-exact and the refinement from
  it reaches the reference's x.
* The `-d` path (lazy initialisation, FP16 deck, FP16-accumulating Schur
  update in k-chunks of 100): the oracle's factors are the reference's bit
  for bit at C1 and at n = 2400, b = 120 (two chunks per panel); on the GPU,
  HPLAI_FLAG_REF_DECK reproduces them bit for bit and refines to the
  reference's x.
* Every solution -- the oracle's, the GPU's plain form, the GPU's precision
  form (e4m3 Schur, GMRES-IR; the FP16 deck needs b % 8 == 0, which b = 60 is
  not) -- equals the reference's x from each of its four runs (`-not -r`,
  `-not -d -r`, netlib and OpenBLAS builds) to FP64 relative error 1e-12.
"""
import hashlib
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_c1.json")))
N, B = FIX["n"], FIX["b"]


def ref_x(run):
    return np.array([float.fromhex(v) for v in FIX["runs"][run]["x"]])


SOLVED = sorted(r for r in FIX["runs"] if "x" in FIX["runs"][r] and "l1est" not in r)


def digest(a):
    return hashlib.sha256(np.asfortranarray(a, dtype=np.float32).tobytes(order="F")).hexdigest()


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_oracle_lu_is_the_references_bit_for_bit(oracle):
    lu = oracle.lu(oracle.matrix(N), B)
    assert digest(lu) == FIX["runs"]["netlib_not_r"]["lu_sha256"]


def test_oracle_warmup_lu_is_the_references_bit_for_bit(oracle):
    """-w: the first P + 2 = 4 block steps (panel_trf.hpp:726)."""
    lu = oracle.lu_steps(oracle.matrix(N), B, 4)
    assert digest(lu) == FIX["runs"]["netlib_warmup"]["lu_sha256"]


DECK_RUNS = {"netlib_not_d_r": (N, B, False), "netlib_not_d_r_2400": (2400, 120, False),
             "netlib_not_r_bb_2400": (2400, 60, True), "netlib_not_r_bb_4800": (4800, 60, True)}


def _deck_command(n, b, bb):
    return f"driver.out {n} {b} 2 " + ("-not -r --back_buffer" if bb else "-not -d -r")


@pytest.mark.parametrize("run", ["netlib_not_d_r", "netlib_not_d_r_2400", "netlib_not_r_bb_2400"])
def test_oracle_deck_lu_is_the_references_bit_for_bit(oracle, run):
    """-d: lazy init + FP16 deck + hgemm_opt numerics (lazy_init.hpp:92-227,
    kernels/avx2.cpp:82-189); --back_buffer: the deck written back every 32
    steps (back_buffer.hpp:81-170) -- one write-back at n = 2400, b = 60."""
    n, b, bb = DECK_RUNS[run]
    assert FIX["runs"][run]["command"] == _deck_command(n, b, bb)
    assert digest(oracle.lu_deck(n, b, back_buffer=bb)) == FIX["runs"][run]["lu_sha256"]


def test_oracle_deck_refinement_vs_reference(oracle):
    lu = oracle.lu_deck(N, B)
    rc, x, res, har, steps = oracle.refine(lu, B, 42, oracle.rhs(N), oracle.diag(N), q=2)
    ref = FIX["runs"]["netlib_not_d_r"]
    assert rc == 0 and len(steps) == len(ref["steps"])
    assert steps[0][0] == ref["steps"][0]["residual"]
    assert abs(steps[1][0] - ref["steps"][1]["residual"]) <= 1e-8 * ref["steps"][1]["residual"]
    assert rel(x, ref_x("netlib_not_d_r")) <= 1e-12


def test_oracle_l1est_is_the_references_bit_for_bit(oracle):
    a = oracle.l1est(oracle.matrix(N), oracle.diag(N))
    assert digest(a) == FIX["runs"]["netlib_l1est"]["lu_sha256"]


def test_oracle_l1est_refinement_vs_reference(oracle):
    a = oracle.l1est(oracle.matrix(N), oracle.diag(N))
    rc, x, res, har, steps = oracle.refine(a, B, 42, oracle.rhs(N), oracle.diag(N), q=2)
    ref = FIX["runs"]["netlib_l1est"]
    assert rc == 0 and len(steps) == len(ref["steps"])
    assert steps[0][0] == ref["steps"][0]["residual"]
    # the grid's TRSV sums in another order: while the residual is far above
    # rounding level the steps agree to 1e-8; the last ones are rounding-level
    for i, (got, want) in enumerate(zip(steps[1:], ref["steps"][1:]), 1):
        tol = 1e-8 if i <= 2 else 1e-3
        assert abs(got[0] - want["residual"]) <= tol * want["residual"], i
    assert rel(x, ref_x("netlib_l1est")) <= 1e-12


def test_oracle_refinement_vs_reference_steps(oracle):
    rc, x, res, har, steps = oracle.solve(N, B, q=2)
    assert rc == 0
    for run in FIX["runs"].values():
        if not run["command"].startswith(f"driver.out {N} {B} "):
            continue
        assert steps[0][0] == run["steps"][0]["residual"]
        assert abs(steps[0][1] - run["steps"][0]["hpl_harness"]) <= 1e-12 * steps[0][1]
    ref = FIX["runs"]["netlib_not_r"]["steps"]
    assert len(steps) == len(ref)
    assert abs(steps[1][0] - ref[1]["residual"]) <= 1e-8 * ref[1]["residual"]
    assert 0 <= har < 16 and 0 <= FIX["runs"]["netlib_not_r"]["hpl_harness"] < 16


@pytest.mark.parametrize("run", SOLVED)
def test_oracle_x_matches_reference_x(oracle, run):
    rc, x, _, _, _ = oracle.solve(N, B, q=2)
    assert rc == 0
    assert rel(x, ref_x(run)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["plain", "precision"])
def test_gpu_x_matches_reference_x(hplai, torch_cuda, form):
    """C1's parity bar: x equals the reference's x to FP64 relative 1e-12,
    against all four of the reference's runs."""
    prec, flags, mode = hplai.F32_F16, 0, hplai.IR
    if form == "precision":
        prec, mode = hplai.F32_F8, hplai.GMRES
    with hplai.Solver(N, B, precision=prec, flags=flags) as s:
        s.generate(42)
        s.factor()
        r = s.iterative_refinement(50, mode=mode)
        x = s.x()
    assert r.status == hplai.HPLAI_OK and 0 <= r.hpl_harness < 16
    for run in SOLVED:
        assert rel(x, ref_x(run)) <= 1e-12, run


@pytest.mark.gpu
def test_gpu_l1est_bit_exact_and_refines_to_reference_x(hplai, oracle, torch_cuda):
    with hplai.Solver(N, B) as s:
        s.generate(42)
        s.l1est()
        a = s.lu()
        r = s.iterative_refinement(50)
        x = s.x()
        log = s.ir_log()
    want = oracle.l1est(oracle.matrix(N), oracle.diag(N))
    assert np.array_equal(a.view(np.uint32), want.view(np.uint32))
    assert digest(a) == FIX["runs"]["netlib_l1est"]["lu_sha256"]
    assert r.status == hplai.HPLAI_OK and 0 <= r.hpl_harness < 16
    assert len(log) == len(FIX["runs"]["netlib_l1est"]["steps"])
    assert rel(x, ref_x("netlib_l1est")) <= 1e-12


@pytest.mark.gpu
def test_gpu_warmup_factor_steps(hplai, oracle, torch_cuda):
    """hplai_factor_steps(4): panels 0..3 factored and applied; with the SIMT
    panels the diagonal blocks and panels of step 0 are the reference's bit
    for bit, and the whole truncated matrix is within the FP16 Schur
    update's reordering of the oracle's (the reference's) truncated LU."""
    with hplai.Solver(N, B, flags=hplai.FLAG_SIMT_PANELS) as s:
        s.generate(42)
        s.factor_steps(4)
        lu = s.lu().astype(np.float64)
        r = s.iterative_refinement(1)
    ref = oracle.lu_steps(oracle.matrix(N), B, 4).astype(np.float64)
    assert np.array_equal(lu[:, :B].astype(np.float32).view(np.uint32), ref[:, :B].astype(np.float32).view(np.uint32))
    relerr = np.abs(lu - ref) / (np.abs(ref) + 1e-3 * np.abs(ref).max())
    assert relerr.max() < 1e-3
    assert r.status == hplai.HPLAI_ENOTCONV and r.hpl_harness == -1.0



@pytest.mark.gpu
@pytest.mark.parametrize("run", sorted(DECK_RUNS))
def test_gpu_ref_deck_lu_is_the_references_bit_for_bit(hplai, torch_cuda, run):
    """HPLAI_FLAG_REF_DECK: A regenerated at panel time, the FP16-accumulating
    deck update on CUDA cores -- the reference's `-d` factors bit for bit
    (C1 and n = 2400, b = 120: two k-chunks of 100 per panel); with
    HPLAI_FLAG_REF_BACKBUF its `--back_buffer` factors (one and two
    write-backs at n = 2400 and 4800, b = 60)."""
    n, b, bb = DECK_RUNS[run]
    assert FIX["runs"][run]["command"] == _deck_command(n, b, bb)
    flags = hplai.FLAG_REF_DECK | (hplai.FLAG_REF_BACKBUF if bb else 0)
    with hplai.Solver(n, b, flags=flags) as s:
        s.generate(42)
        s.factor()
        assert digest(s.lu()) == FIX["runs"][run]["lu_sha256"]
        s.factor()   # A is regenerated from the seed: a second factorisation is the same
        assert digest(s.lu()) == FIX["runs"][run]["lu_sha256"]
        if run == "netlib_not_d_r":
            res = s.iterative_refinement(50)
            assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0
            assert rel(s.x(), ref_x(run)) <= 1e-12
            log = s.ir_log()   # the device GEMV sums in another order: step 0 to 1e-13
            want = FIX["runs"][run]["steps"][0]["residual"]
            assert abs(log[0][0] - want) <= 1e-13 * want


@pytest.mark.gpu
def test_gpu_ref_deck_matches_oracle_beyond_c1(hplai, oracle, torch_cuda):
    """b = 256 (chunks of 100, 100, 56), the uploaded-matrix form (the lazy
    initialisation reads A instead of regenerating it) and a truncated LU."""
    n, b = 2048, 256
    want = oracle.lu_deck(n, b)
    with hplai.Solver(n, b, flags=hplai.FLAG_REF_DECK) as s:
        s.generate(42)
        s.factor()
        assert np.array_equal(s.lu().view(np.uint32), want.view(np.uint32))
        s.upload(oracle.matrix(n), oracle.rhs(n), oracle.diag(n), 42)
        s.factor()
        assert np.array_equal(s.lu().view(np.uint32), want.view(np.uint32))
        s.generate(42)
        s.factor_steps(3)
        part = oracle.lu_deck(n, b, kend=3)
        assert np.array_equal(s.lu()[:, :3 * b].view(np.uint32), part[:, :3 * b].view(np.uint32))
        assert np.array_equal(s.lu()[:3 * b, :].view(np.uint32), part[:3 * b, :].view(np.uint32))


def test_ref_deck_flag_combinations(hplai):
    for flags, prec in [(hplai.FLAG_REF_DECK | hplai.FLAG_FP16_DECK, 0), (hplai.FLAG_REF_DECK | hplai.FLAG_LOOKAHEAD, 0),
                        (hplai.FLAG_REF_DECK, 1), (hplai.FLAG_REF_BACKBUF, 0)]:
        with pytest.raises(hplai.HplaiError):
            hplai.Solver(1200, 60, precision=prec, flags=flags)
