"""The precision form (e4m3 Schur update) and GMRES refinement on the B200.

The e4m3 down-cast is integer-exact work (a power-of-two factor per 128
rows, then round-to-nearest-even), so the device bytes and factors must
equal the oracle's restatement bit for bit.  The e4m3 GEMM forms exact
products and sums them in FP32 on the tensor cores, so it is checked
against FP64 sums of the same products with a stated tolerance.  Whole
solves have no reference counterpart: they must reach hpl-harness < 16 and
agree with a dense FP64 solve of the same matrix.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def panel_values(rng, rows, k):
    """Panel-like values whose magnitude changes from one 128-row block to the
    next (one block all zero, one tiny enough to reach e4m3 subnormals)."""
    x = rng.uniform(-1.0, 1.0, (rows, k)).astype(np.float32)
    for blk in range((rows + 127) // 128):
        x[blk * 128:(blk + 1) * 128] *= np.float32(2.0) ** int(rng.integers(-20, 6))
    if rows > 256:
        x[128:256] = 0.0
    x[::37, ::5] *= np.float32(1e-4)   # values far below the block maximum
    return x


@pytest.mark.parametrize("rows,k", [(1000, 60), (777, 512), (300, 1024), (128, 128)])
@pytest.mark.parametrize("col_major", [True, False])
def test_quantize_e4m3_bit_exact(hplai, oracle, torch_cuda, rows, k, col_major):
    torch = torch_cuda
    rng = np.random.default_rng(rows * 7 + k)
    x = panel_values(rng, rows, k)
    ld8 = (k + 127) // 128 * 128
    if col_major:
        src = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()     # column p of x contiguous, ld = rows
        lds = rows
    else:
        src = torch.from_numpy(np.ascontiguousarray(x)).cuda()       # row r contiguous, ld = k
        lds = k
    dst = torch.full((rows, ld8), 0xAB, dtype=torch.uint8, device="cuda")
    scale = torch.zeros((rows + 127) // 128, dtype=torch.float32, device="cuda")
    bits = torch.zeros((rows + 127) // 128 + 1, dtype=torch.int32, device="cuda")
    hplai.check(hplai.quantize_e4m3(rows, k, src.data_ptr(), lds, 1 if col_major else 0, dst.data_ptr(), ld8,
                                    scale.data_ptr(), bits.data_ptr(), None))
    torch.cuda.synchronize()
    ref8, refs = oracle.quantize_e4m3(x, col_major=True, ld8=ld8)
    assert np.array_equal(scale.cpu().numpy(), refs)
    got = dst.cpu().numpy()
    assert np.array_equal(got, ref8), f"{np.count_nonzero(got != ref8)} bytes differ"


def test_quantize_e4m3_rejects_bad_ld(hplai):
    assert hplai.quantize_e4m3(10, 60, 0, 10, 1, 0, 100, 0, 0, None) == hplai.HPLAI_EINVAL


@pytest.mark.parametrize("m,n,k", [(700, 500, 256), (1000, 1000, 60), (256, 384, 1024), (129, 131, 512)])
def test_f8gemm_minus_vs_fp64_products(hplai, oracle, torch_cuda, m, n, k):
    torch = torch_cuda
    rng = np.random.default_rng(m + n + k)
    l8, sl = oracle.quantize_e4m3(panel_values(rng, m, k), col_major=True)
    u8, su = oracle.quantize_e4m3(panel_values(rng, n, k), col_major=False)
    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(np.float32))
    cd = torch.from_numpy(np.ascontiguousarray(c.T)).cuda()
    l8d, u8d = torch.from_numpy(l8).cuda(), torch.from_numpy(u8).cuda()
    sld, sud = torch.from_numpy(sl).cuda(), torch.from_numpy(su).cuda()
    hplai.check(hplai.f8gemm_minus(m, n, k, l8d.data_ptr(), l8.shape[1], sld.data_ptr(), u8d.data_ptr(), u8.shape[1],
                                   sud.data_ptr(), cd.data_ptr(), m, None))
    torch.cuda.synchronize()
    got = np.asfortranarray(cd.cpu().numpy().T)
    ref = oracle.f8gemm_minus(c, l8, sl, u8, su, k)
    # bound: FP32 summation of k exact products, then one rounding of the update
    lv = np.vectorize(oracle.e4m3_to_f32)(l8[:, :k]).astype(np.float64) * np.repeat(sl, 128)[:m, None]
    uv = np.vectorize(oracle.e4m3_to_f32)(u8[:, :k]).astype(np.float64) * np.repeat(su, 128)[:n, None]
    mag = np.abs(lv) @ np.abs(uv).T
    tol = 2.0 ** -19 * mag + 2.0 ** -22 * np.abs(ref)
    err = np.abs(got.astype(np.float64) - ref)
    assert np.all(err <= tol), f"max err/tol {np.max(err / np.maximum(tol, 1e-300)):.3g}"


def dense_solution(oracle, n, seed=42):
    a = oracle.dense_matrix_f64(n, seed)
    return np.linalg.solve(a, oracle.rhs(n, seed))


@pytest.mark.parametrize("precision,mode", [(1, 1), (0, 1)])
def test_c1_solve_precision_and_mode(hplai, oracle, torch_cuda, precision, mode):
    n, b = 1200, 60
    with hplai.Solver(n, b, precision=precision) as s:
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=mode)
        outer, inner = s.refine_counts()
        x = s.x()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, (res, outer, inner)
    assert inner >= 1 and outer <= 4
    xs = dense_solution(oracle, n)
    rel = np.max(np.abs(x - xs)) / np.max(np.abs(xs))
    assert rel < 1e-11, rel


@pytest.mark.parametrize("n,b", [(8192, 512), (4096, 1024), (6144, 256)])
def test_fp8_gmres_converges(hplai, torch_cuda, n, b):
    with hplai.Solver(n, b, precision=hplai.F32_F8) as s:
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=hplai.GMRES)
        outer, inner = s.refine_counts()
        log = s.ir_log()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, (res, log)
    # one GMRES cycle per residual evaluation; a few residual evaluations in all
    assert outer <= 4 and inner <= 30 * (outer - 1), (outer, inner)


def test_fp8_classical_ir_still_terminates(hplai, torch_cuda):
    """The e4m3 factor with the reference's classical correction: either it
    converges or it stops with {-1,-1} (never a hang or an error)."""
    with hplai.Solver(4096, 512, precision=hplai.F32_F8) as s:
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=hplai.IR)
    assert res.status in (hplai.HPLAI_OK, hplai.HPLAI_ENOTCONV)
    if res.status == hplai.HPLAI_OK:
        assert res.hpl_harness < 16.0
    else:
        assert (res.residual, res.hpl_harness) == (-1.0, -1.0)


def test_fp8_factor_close_to_fp16_factor(hplai, torch_cuda):
    """Each e4m3 rounding moves a panel value by at most 2^-4 relative, so the
    two factors of the same matrix differ by a few percent of the Schur
    contribution, far below the diagonal."""
    n, b = 2048, 256
    lus = []
    for prec in (hplai.F32_F16, hplai.F32_F8):
        with hplai.Solver(n, b, precision=prec) as s:
            s.generate(42)
            s.factor()
            lus.append(s.lu().astype(np.float64))
    d = np.abs(lus[0] - lus[1])
    assert np.max(d) < 0.05, np.max(d)
    assert np.all(np.isfinite(lus[1]))


def test_gmres_parameters_validated(hplai, torch_cuda):
    with hplai.Solver(512, 128) as s:
        with pytest.raises(hplai.HplaiError):
            s.set_gmres(0, 1e-12)
        with pytest.raises(hplai.HplaiError):
            s.set_gmres(32, 1e-12)
        with pytest.raises(hplai.HplaiError):
            s.set_gmres(10, 0.0)
        s.set_gmres(5, 1e-10)
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=hplai.GMRES)
        assert res.status == hplai.HPLAI_OK


# ---------------------------------------------------------------------------
# FP16 deck (HPLAI_FLAG_FP16_DECK): the trailing updates accumulate in FP16
# and are applied to a block column/row just before it is factored.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision,mode,n,b", [(0, 0, 2048, 256), (0, 0, 1536, 128), (1, 1, 4096, 512),
                                               (1, 1, 8192, 1024)])
def test_deck_solves_converge(hplai, oracle, torch_cuda, precision, mode, n, b):
    with hplai.Solver(n, b, precision=precision, flags=hplai.FLAG_FP16_DECK) as s:
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=mode)
        x = s.x()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, res
    if n <= 4096:
        xs = dense_solution(oracle, n)
        assert np.max(np.abs(x - xs)) / np.max(np.abs(xs)) < 1e-11


def test_deck_factor_close_to_fp32_trailing(hplai, torch_cuda):
    """FP16 accumulation of the updates moves each factor entry by far less
    than the FP16 operands already do."""
    n, b = 2048, 256
    lus = []
    for flags in (0, hplai.FLAG_FP16_DECK):
        with hplai.Solver(n, b, flags=flags) as s:
            s.generate(42)
            s.factor()
            lus.append(s.lu().astype(np.float64))
    assert np.max(np.abs(lus[0] - lus[1])) < 1e-2


def test_deck_needs_block_multiple_of_8(hplai):
    with pytest.raises(hplai.HplaiError):
        hplai.Solver(1200, 60, flags=hplai.FLAG_FP16_DECK)


def _deck_check(got, ref, mag, dscale):
    """FP32 accumulation of the products (2^-19 of the magnitude sum, as for
    the FP32 updates), then one FP16 rounding of the deck element."""
    acc_err = dscale * 2.0 ** -19 * mag
    tol = acc_err + 2.0 ** -11 * (np.abs(ref) + acc_err) + 2.0 ** -25
    err = np.abs(got.astype(np.float64) - ref)
    assert np.all(err <= tol), f"max err/tol {np.max(err / tol):.3g}"


@pytest.mark.parametrize("m,n,k", [(704, 500, 256), (136, 131, 512), (1000, 1000, 64), (256, 768, 1024)])
def test_shgemm_deck_minus_vs_fp64_products(hplai, torch_cuda, m, n, k):
    """deck <- half(deck - dscale L U) on an FP16 column-major deck (m a
    multiple of 8, n ragged); the rows between m and ldd and the column
    after n are not touched."""
    torch = torch_cuda
    rng = np.random.default_rng(m * 3 + n + k)
    ld = (k + 7) // 8 * 8
    l16 = rng.uniform(-0.5, 0.5, (m, ld)).astype(np.float16)
    u16 = rng.uniform(-0.5, 0.5, (n, ld)).astype(np.float16)
    ldd = (m + 7) // 8 * 8 + 8
    deck0 = rng.uniform(-100, 100, (n + 1, ldd)).astype(np.float16)     # column j at deck0[j]
    dscale = 64.0
    dd = torch.from_numpy(deck0.copy()).cuda()
    ld_, ud = torch.from_numpy(l16).cuda(), torch.from_numpy(u16).cuda()
    hplai.check(hplai.shgemm_deck_minus(m, n, k, ld_.data_ptr(), ld, ud.data_ptr(), ld, dd.data_ptr(), ldd,
                                        dscale, None))
    torch.cuda.synchronize()
    got = dd.cpu().numpy()
    lv, uv = l16[:, :k].astype(np.float64), u16[:, :k].astype(np.float64)
    ref = deck0[:n, :m].astype(np.float64).T - dscale * (lv @ uv.T)
    _deck_check(got[:n, :m].T, ref, np.abs(lv) @ np.abs(uv).T, dscale)
    assert np.array_equal(got[:, m:], deck0[:, m:]) and np.array_equal(got[n], deck0[n])


@pytest.mark.parametrize("m,n,k", [(704, 500, 256), (136, 131, 512), (256, 384, 1024)])
def test_f8gemm_deck_minus_vs_fp64_products(hplai, oracle, torch_cuda, m, n, k):
    torch = torch_cuda
    rng = np.random.default_rng(m + 5 * n + k)
    l8, sl = oracle.quantize_e4m3(panel_values(rng, m, k), col_major=True)
    u8, su = oracle.quantize_e4m3(panel_values(rng, n, k), col_major=False)
    ldd = (m + 7) // 8 * 8 + 8
    deck0 = rng.uniform(-100, 100, (n + 1, ldd)).astype(np.float16)
    dscale = 2.0 ** -8
    dd = torch.from_numpy(deck0.copy()).cuda()
    l8d, u8d = torch.from_numpy(l8).cuda(), torch.from_numpy(u8).cuda()
    sld, sud = torch.from_numpy(sl).cuda(), torch.from_numpy(su).cuda()
    hplai.check(hplai.f8gemm_deck_minus(m, n, k, l8d.data_ptr(), l8.shape[1], sld.data_ptr(), u8d.data_ptr(),
                                        u8.shape[1], sud.data_ptr(), dd.data_ptr(), ldd, dscale, None))
    torch.cuda.synchronize()
    got = dd.cpu().numpy()
    lv = np.vectorize(oracle.e4m3_to_f32)(l8[:, :k]).astype(np.float64) * np.repeat(sl, 128)[:m, None]
    uv = np.vectorize(oracle.e4m3_to_f32)(u8[:, :k]).astype(np.float64) * np.repeat(su, 128)[:n, None]
    ref = deck0[:n, :m].astype(np.float64).T - dscale * (lv @ uv.T)
    _deck_check(got[:n, :m].T, ref, np.abs(lv) @ np.abs(uv).T, dscale)
    assert np.array_equal(got[:, m:], deck0[:, m:]) and np.array_equal(got[n], deck0[n])


def test_deck_minus_rejects_bad_layouts(hplai):
    assert hplai.shgemm_deck_minus(64, 64, 64, 16, 64, 16, 64, 16, 60, 1.0, None) == hplai.HPLAI_EINVAL  # ldd < m
    assert hplai.shgemm_deck_minus(64, 64, 64, 16, 64, 16, 64, 16, 68, 1.0, None) == hplai.HPLAI_EINVAL  # ldd % 8
    assert hplai.shgemm_deck_minus(60, 64, 64, 16, 64, 16, 64, 16, 64, 1.0, None) == hplai.HPLAI_EINVAL  # m % 8
    assert hplai.f8gemm_deck_minus(64, 64, 128, 16, 128, 16, 16, 128, 16, 24, 64, 1.0, None) == hplai.HPLAI_EINVAL


@pytest.mark.parametrize("precision,flags,n,b", [(0, 4, 2048, 256), (1, 0, 4096, 512), (1, 4, 4096, 512)])
def test_checksum_over_factors_of_every_form(hplai, oracle, torch_cuda, precision, flags, n, b):
    """hplai_checksum (panel_check.hpp:9-65) reads the FP32 factors the
    refinement uses in the FP16-deck and e4m3 forms too: it equals the
    oracle's sums in the reference's block order over hplai_get_lu's copy,
    to 1e-13 relative."""
    assert flags in (0, hplai.FLAG_FP16_DECK)
    with hplai.Solver(n, b, precision=precision, flags=flags) as s:
        s.generate(42)
        s.factor()
        got = s.checksum()
        lu = s.lu()
    want = oracle.panel_check(lu, b)
    assert np.all(np.abs(got - want) <= 1e-13 * want)
