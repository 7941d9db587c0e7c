"""The CPU oracle against the reference's published golden values and an
independent restatement of the generator (CPU only)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
MASK = (1 << 64) - 1
A_LCG, C_LCG = 6364136223846793005, 1
SCALE = float.fromhex("0x1.fffffffffffffp-65")


def py_state(n, i, j, seed):
    """hpl_rand.hpp:35-57 in Python integers: state_0 = a*seed + c, then
    i + n*j single steps (done by binary powering of the affine map)."""
    x = (A_LCG * seed + C_LCG) & MASK
    m = i + n * j
    a, c = A_LCG, C_LCG
    while m:
        if m & 1:
            x = (a * x + c) & MASK
        a, c = (a * a) & MASK, (a * c + c) & MASK
        m >>= 1
    return x


def py_value(x):
    s = x - (1 << 64) if x >= (1 << 63) else x
    return float(s) * SCALE


def test_readme_step0_pin(oracle):
    """The oracle reproduces the reference's published step-0 residual and
    hpl-harness (README:50) bit for bit on the 2x2 grid's summation order."""
    g = json.load(open(os.path.join(HERE, "golden", "readme_step0.json")))
    n, b, seed = g["n"], g["b"], g["seed"]
    rhs, d = oracle.rhs(n, seed), oracle.diag(n, seed)
    lu = np.zeros((n, n), dtype=np.float32, order="F")   # step 0 does not touch the factors
    rc, x, res, har, steps = oracle.refine(lu, b, seed, rhs, d, maxit=1, q=g["grid_cols"])
    r0, h0 = steps[0]
    assert r0 == g["step0_residual"]
    assert f"{h0:.6f}" == f"{g['step0_harness']:.6f}"
    assert rc == 1 and res == -1.0 and har == -1.0   # maxit=1 without convergence -> IRErrors {-1,-1}


def test_step0_sequential_order_close(oracle):
    """The one-process summation order differs only in rounding."""
    g = json.load(open(os.path.join(HERE, "golden", "readme_step0.json")))
    n, b = g["n"], g["b"]
    rhs, d = oracle.rhs(n), oracle.diag(n)
    lu = np.zeros((n, n), dtype=np.float32, order="F")
    _, _, _, _, steps = oracle.refine(lu, b, 42, rhs, d, maxit=1, q=1)
    assert abs(steps[0][0] - g["step0_residual"]) <= 1e-13 * g["step0_residual"]


@pytest.mark.parametrize("n,i,j", [(1200, 0, 0), (1200, 7, 1199), (65536, 65535, 123), (131072, 5, 131071),
                                   (1200, 3, 1200)])
def test_generator_matches_python_restatement(oracle, n, i, j):
    assert oracle.state_at(n, i, j, 42) == py_state(n, i, j, 42)
    assert oracle.elem(n, i, j, 42) == py_value(py_state(n, i, j, 42))


def test_generator_range_and_diag(oracle):
    n = 300
    a = oracle.matrix(n)
    off = a.astype(np.float64)
    np.fill_diagonal(off, 0.0)
    assert np.all(np.abs(off) <= 0.5)
    d = oracle.diag(n)
    a64 = oracle.dense_matrix_f64(n)
    off64 = a64.copy()
    np.fill_diagonal(off64, 0.0)
    # diagonal = FP64 sum of |a_ij|, j != i, summed in j order (checked loosely here, exactly below)
    assert np.allclose(d, np.abs(off64).sum(axis=1), rtol=1e-14, atol=0)
    for i in (0, 17, n - 1):
        s = 0.0
        for jj in range(n):
            if jj != i:
                s += abs(py_value(py_state(n, i, jj, 42)))
        assert d[i] == s
    assert np.array_equal(np.diag(a), d.astype(np.float32))
    # rhs = column n of the stream, FP64
    rhs = oracle.rhs(n)
    assert rhs[5] == py_value(py_state(n, 5, n, 42))


def test_panels_equal_whole_matrix(oracle):
    """pmatgen fills block by block; any blocking gives the same matrix."""
    n, b = 240, 60
    a = oracle.matrix(n)
    for (bi, bj) in [(0, 0), (1, 2), (3, 3), (2, 0)]:
        p = oracle.fill_panel(n, bi * b, bj * b, b, b)
        assert np.array_equal(p, a[bi * b:(bi + 1) * b, bj * b:(bj + 1) * b])


def test_coeff_pow_composes(oracle):
    a1, c1 = oracle.coeff_pow(1000)
    a2, c2 = oracle.coeff_pow(2345)
    a3, c3 = oracle.coeff_pow(3345)
    assert (a1 * a2) & MASK == a3 and (a1 * c2 + c1) & MASK == c3


def test_getrf_nopiv_reconstructs(oracle):
    rng = np.random.default_rng(1)
    for b in (16, 60, 100):
        m = rng.uniform(-0.5, 0.5, (b, b)).astype(np.float32)
        m[np.arange(b), np.arange(b)] = np.abs(m).sum(1)
        f = oracle.getrf_nopiv(m)
        l = np.tril(f.astype(np.float64), -1) + np.eye(b)
        u = np.triu(f.astype(np.float64))
        assert np.abs(l @ u - m).max() <= 1e-5 * np.abs(m).max()


def test_trsv_against_dense_solve(oracle):
    rng = np.random.default_rng(2)
    n, b = 480, 60
    m = rng.uniform(-0.5, 0.5, (n, n)).astype(np.float32)
    m[np.arange(n), np.arange(n)] = np.abs(m).sum(1)
    x = rng.uniform(-1, 1, n)
    l = np.tril(m.astype(np.float64), -1) + np.eye(n)
    u = np.triu(m.astype(np.float64))
    y = oracle.trsv_lower(m, x, b)
    assert np.abs(y - np.linalg.solve(l, x)).max() <= 1e-12 * np.abs(y).max()
    z = oracle.trsv_upper(m, x, b)
    assert np.abs(z - np.linalg.solve(u, x)).max() <= 1e-12 * np.abs(z).max()


def test_otf_gemv_matches_dense(oracle):
    n, b = 600, 60
    a = oracle.dense_matrix_f64(n)
    d = oracle.diag(n)
    x = np.random.default_rng(3).uniform(-1, 1, n)
    y0 = np.random.default_rng(4).uniform(-1, 1, n)
    y = oracle.otf_gemv(n, b, -1.0, x, y0, 42, d)
    ref = y0 - a @ x
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(a).sum(1).max()


def test_full_solve_c1(oracle):
    """n=1200, b=60: converges, and x matches a dense FP64 solve to 1e-12."""
    n, b = 1200, 60
    rc, x, res, har, steps = oracle.solve(n, b, q=1)
    assert rc == 0 and 0 <= har < 16
    a = oracle.dense_matrix_f64(n)
    xr = np.linalg.solve(a, oracle.rhs(n))
    assert np.abs(x - xr).max() <= 1e-12 * np.abs(xr).max()
    assert len(steps) <= 5


def test_bad_block_rejected(oracle):
    with pytest.raises(ValueError):
        oracle.lu(np.eye(100, dtype=np.float32), 30)


def test_nonconvergence_reports_minus_one(oracle):
    """Planted fault on the CPU: factors of the wrong matrix never converge
    within maxit, and refinement returns IRErrors {-1,-1}."""
    n, b = 240, 60
    bad = np.eye(n, dtype=np.float32, order="F") * 1e-3
    rc, x, res, har, steps = oracle.refine(bad, b, 42, oracle.rhs(n), oracle.diag(n), maxit=3)
    assert rc == 1 and res == -1.0 and har == -1.0 and len(steps) == 3


def test_e4m3_restatement_matches_torch_conversion(oracle):
    """The oracle's e4m3 rounding (restated from the format definition) agrees
    with torch's independent float -> float8_e4m3fn conversion on a dense sweep
    of the finite range and on random values across 20 binades."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.linspace(-448, 448, 100001, dtype=np.float32),
                         (rng.standard_normal(100000) * np.float32(2.0) ** rng.integers(-14, 8, 100000))
                         .astype(np.float32)])
    xs = np.clip(xs, -448, 448)
    mine = np.fromiter((oracle.e4m3_rn(float(v)) for v in xs), dtype=np.uint8, count=len(xs))
    ref = torch.from_numpy(xs.copy()).to(torch.float8_e4m3fn).view(torch.uint8).numpy()
    assert np.array_equal(mine, ref)
    for b in range(256):
        if (b & 0x7F) != 0x7F:
            assert oracle.e4m3_rn(oracle.e4m3_to_f32(b)) == b


def test_quantize_e4m3_block_factors(oracle):
    """One power-of-two factor per 128 rows; the scaled block maximum lies in
    [224, 448]; an all-zero block gets factor 1 and zero bytes."""
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (300, 60)).astype(np.float32)
    x[:128] *= 1e-3
    x[128:256] = 0
    q, s = oracle.quantize_e4m3(x, col_major=True)
    assert q.shape == (300, 128) and s.shape == (3,)
    assert s[1] == 1.0 and not q[128:256].any() and not q[:, 60:].any()
    for blk in (0, 2):
        amax = np.abs(x[blk * 128:(blk + 1) * 128]).max() / s[blk]
        assert 224.0 <= amax < 448.0
        assert np.log2(s[blk]) == int(np.log2(s[blk]))


def test_panel_check_restatement_matches_triangle_sums(oracle):
    """panel_check (panel_check.hpp:9-65) in the reference's block order agrees
    with order-free FP64 sums of the diagonal and the strict triangles of the
    factored matrix (to 1e-13: only the summation order differs), and the
    block size changes only the order."""
    n, b = 360, 60
    lu = oracle.lu(oracle.matrix(n), b)
    s = oracle.panel_check(lu, b)
    a = np.abs(lu.astype(np.float64))
    want = np.array([np.trace(a), np.triu(a, 1).sum(), np.tril(a, -1).sum()])
    assert np.all(np.abs(s - want) <= 1e-13 * want)
    assert np.all(np.abs(oracle.panel_check(lu, 120) - s) <= 1e-13 * s)
