"""ctypes binding of the CPU oracle (liboracle.so, built from hplai_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py (cpu_baseline and the reference arm).  The product never imports
this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build() -> str:
    """Compile liboracle.so with the Makefile next to this file (gcc, seconds)."""
    srcs = [os.path.join(HERE, f) for f in ("hplai_oracle.c", "hplai_oracle_f8.c", "Makefile")]
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(os.path.getmtime(s) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


build()
_lib = ctypes.CDLL(LIB_PATH)

_dp = ctypes.POINTER(ctypes.c_double)
_i64, _u64, _int, _dbl, _vp = ctypes.c_int64, ctypes.c_uint64, ctypes.c_int, ctypes.c_double, ctypes.c_void_p


def _proto(name, restype, *argtypes):
    f = getattr(_lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


state_at = _proto("orc_state_at", _u64, _int, _i64, _i64, _u64)
elem = _proto("orc_elem", _dbl, _int, _i64, _i64, _u64)
_coeff_pow = _proto("orc_coeff_pow", None, _u64, ctypes.POINTER(_u64), ctypes.POINTER(_u64))
calc_diag = _proto("orc_calc_diag", _dbl, _int, _int, _u64)
_fill_panel = _proto("orc_fill_panel", None, _int, _int, _int, _int, _int, _vp, _i64, _u64, _int)
_gen_rhs = _proto("orc_gen_rhs", None, _int, _u64, _vp)
_gen_diag = _proto("orc_gen_diag", None, _int, _u64, _vp)
_gen_rhs_cols = _proto("orc_gen_rhs_cols", None, _int, _u64, _int, _int, _vp)
_getrf = _proto("orc_getrf_nopiv", None, _int, _vp, _i64)
_trsm_ru = _proto("orc_trsm_right_upper", None, _int, _int, _vp, _i64, _vp, _i64)
_trsm_ll = _proto("orc_trsm_left_lower_unit", None, _int, _int, _vp, _i64, _vp, _i64)
_shgemm = _proto("orc_shgemm_minus", None, _int, _int, _int, _vp, _i64, _vp, _i64, _vp, _i64)
_lu = _proto("orc_lu", _int, _int, _int, _vp, _i64)
_lu_steps = _proto("orc_lu_steps", _int, _int, _int, _vp, _i64, _int)
_l1est = _proto("orc_l1est", None, _int, _vp, _i64, _vp)
_lu_deck_steps = _proto("orc_lu_deck_steps", _int, _int, _int, _u64, _vp, _vp, _i64, _int, _vp, _int)
_higham_beta = _proto("orc_higham_beta", _dbl, _int, _dbl, _dbl)
_higham_fill = _proto("orc_higham_fill", None, _int, _int, _int, _int, _dbl, _dbl, _vp, _i64)
_higham_elem = _proto("orc_higham_elem", _dbl, _i64, _i64, _dbl, _dbl)
_higham_diag = _proto("orc_higham_diag", None, _int, _dbl, _dbl, _vp)
_higham_norm = _proto("orc_higham_norm", _dbl, _int, _dbl, _dbl)
_higham_resid = _proto("orc_higham_residual_rows", None, _int, _dbl, _dbl, _vp, _vp, _int, _vp, _vp)
_deck_scales = _proto("orc_deck_scales", None, _int, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float))
_otf_gemv = _proto("orc_otf_gemv", None, _int, _int, _int, _dbl, _vp, _vp, _u64, _vp)
_trsv_l = _proto("orc_trsv_lower", None, _int, _int, _vp, _i64, _vp)
_trsv_u = _proto("orc_trsv_upper", None, _int, _int, _vp, _i64, _vp)
_refine = _proto("orc_refine", _int, _int, _int, _int, _vp, _i64, _u64, _vp, _vp, _int, _vp, _vp, _vp,
                 ctypes.POINTER(_int), _dp, _dp)
_solve = _proto("orc_solve", _int, _int, _int, _int, _u64, _int, _vp, _vp, _vp, ctypes.POINTER(_int), _dp, _dp)
_e4m3_rn = _proto("orc_e4m3_rn", ctypes.c_uint8, ctypes.c_float)
_e4m3_to_f32 = _proto("orc_e4m3_to_f32", ctypes.c_float, ctypes.c_uint8)
_quantize_e4m3 = _proto("orc_quantize_e4m3", None, _int, _int, _vp, _i64, _int, _vp, _i64, _vp)
_panel_check = _proto("orc_panel_check", None, _int, _int, _vp, _i64, _vp)
_residual_rows = _proto("orc_residual_rows", None, _int, _u64, _vp, _int, _vp, _int, _int, _vp, _vp)
_f8gemm = _proto("orc_f8gemm_minus", None, _int, _int, _int, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _i64)


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def coeff_pow(m: int):
    a, c = _u64(), _u64()
    _coeff_pow(m, ctypes.byref(a), ctypes.byref(c))
    return a.value, c.value


def fill_panel(n, i0, j0, nrow, ncol, seed=42, calc_diag=True) -> np.ndarray:
    a = np.zeros((nrow, ncol), dtype=np.float32, order="F")
    _fill_panel(n, i0, j0, nrow, ncol, _p(a), max(nrow, 1), seed, 1 if calc_diag else 0)
    return a


def matrix(n, seed=42) -> np.ndarray:
    return fill_panel(n, 0, 0, n, n, seed, True)


def rhs(n, seed=42) -> np.ndarray:
    out = np.zeros(n)
    _gen_rhs(n, seed, _p(out))
    return out


def rhs_cols(n, seed, first, count) -> np.ndarray:
    """Columns n + first .. of the generator stream (n x count)."""
    out = np.zeros((count, n))
    _gen_rhs_cols(n, seed, first, count, _p(out))
    return out.T


def diag(n, seed=42) -> np.ndarray:
    out = np.zeros(n)
    _gen_diag(n, seed, _p(out))
    return out


def getrf_nopiv(a: np.ndarray) -> np.ndarray:
    a = np.array(a, dtype=np.float32, order="F", copy=True)
    _getrf(a.shape[0], _p(a), a.shape[0])
    return a


def trsm_right_upper(u: np.ndarray, b: np.ndarray) -> np.ndarray:
    """B <- B * U^{-1}, U upper non-unit (netlib strsm R,U,N,N order)."""
    u = np.asfortranarray(u, dtype=np.float32)
    b = np.array(b, dtype=np.float32, order="F", copy=True)
    _trsm_ru(b.shape[0], b.shape[1], _p(u), u.shape[0], _p(b), b.shape[0])
    return b


def trsm_left_lower_unit(l: np.ndarray, b: np.ndarray) -> np.ndarray:
    """B <- L^{-1} B, L unit lower (netlib strsm L,L,N,U order)."""
    l = np.asfortranarray(l, dtype=np.float32)
    b = np.array(b, dtype=np.float32, order="F", copy=True)
    _trsm_ll(b.shape[0], b.shape[1], _p(l), l.shape[0], _p(b), b.shape[0])
    return b


def shgemm_minus(c: np.ndarray, l16: np.ndarray, u16: np.ndarray) -> np.ndarray:
    """C - L*U with FP16 inputs, FP32 accumulation in k-blocks of 100."""
    c = np.array(c, dtype=np.float32, order="F", copy=True)
    l16 = np.asfortranarray(l16, dtype=np.float16).view(np.uint16)
    u16 = np.asfortranarray(u16, dtype=np.float16).view(np.uint16)
    m, k = l16.shape
    n = u16.shape[1]
    _shgemm(m, n, k, _p(l16), m, _p(u16), k, _p(c), m)
    return c


def lu(a: np.ndarray, b: int) -> np.ndarray:
    a = np.array(a, dtype=np.float32, order="F", copy=True)
    rc = _lu(a.shape[0], b, _p(a), a.shape[0])
    if rc:
        raise ValueError(f"orc_lu: {rc}")
    return a


def lu_steps(a: np.ndarray, b: int, kend: int) -> np.ndarray:
    """The first kend block steps of the LU (the reference's -w warm-up):
    panels 0..kend-1 factored, the updates of panels 0..kend-2 applied."""
    a = np.array(a, dtype=np.float32, order="F", copy=True)
    rc = _lu_steps(a.shape[0], b, _p(a), a.shape[0], kend)
    if rc:
        raise ValueError(f"orc_lu_steps: {rc}")
    return a


def lu_deck(n: int, b: int, seed: int = 42, kend: int = None, with_deck: bool = False, back_buffer: bool = False):
    """The reference's lazy-initialised double-decker LU (`-d`): A never
    stored, trailing updates into an FP16 deck by the FP16-accumulating
    hgemm_opt, blocks formed as fma(downscale, deck, a_ij) when they join a
    panel; back_buffer: the `--back_buffer` form.  Returns the FP32 factors
    (and the final deck, n x n FP16 bits)."""
    a = np.zeros((n, n), dtype=np.float32, order="F")
    dk = np.zeros((n, n), dtype=np.uint16, order="F") if with_deck else None
    df = np.ascontiguousarray(diag(n, seed).astype(np.float32))
    rc = _lu_deck_steps(n, b, seed, _p(df), _p(a), n, n // b if kend is None else kend,
                        _p(dk) if with_deck else None, 1 if back_buffer else 0)
    if rc:
        raise ValueError(f"orc_lu_deck_steps: {rc}")
    return (a, dk) if with_deck else a


def deck_scales(n: int):
    """(scalea, downscale) of the `-d` LU as FP32: n^0.75 and 1 / n^0.75."""
    sa, ds = ctypes.c_float(), ctypes.c_float()
    _deck_scales(n, ctypes.byref(sa), ctypes.byref(ds))
    return sa.value, ds.value


def l1est(a: np.ndarray, d: np.ndarray) -> np.ndarray:
    """pmatl1est: approximate factors without a decomposition."""
    a = np.array(a, dtype=np.float32, order="F", copy=True)
    _l1est(a.shape[0], _p(a), a.shape[0], _p(np.ascontiguousarray(d, dtype=np.float64)))
    return a


def panel_check(lu_f32: np.ndarray, b: int) -> np.ndarray:
    """panel_check (panel_check.hpp:9-65): [sum |diag|, sum |strict upper|,
    sum |strict lower|] of the factored matrix, in the reference's order."""
    a = np.asfortranarray(lu_f32, dtype=np.float32)
    n = a.shape[0]
    if n % b:
        raise ValueError("panel_check: n % b != 0")
    sigs = np.zeros(3, dtype=np.float64)
    _panel_check(n, b, _p(a), n, _p(sigs))
    return sigs


def otf_gemv(n, b, alpha, x, y, seed, d, q=1) -> np.ndarray:
    y = np.array(y, dtype=np.float64, copy=True)
    x = np.ascontiguousarray(x, dtype=np.float64)
    d = np.ascontiguousarray(d, dtype=np.float64)
    _otf_gemv(n, b, q, alpha, _p(x), _p(y), seed, _p(d))
    return y


def trsv_lower(lu_f32: np.ndarray, x: np.ndarray, b: int) -> np.ndarray:
    x = np.array(x, dtype=np.float64, copy=True)
    a = np.asfortranarray(lu_f32, dtype=np.float32)
    _trsv_l(a.shape[0], b, _p(a), a.shape[0], _p(x))
    return x


def trsv_upper(lu_f32: np.ndarray, x: np.ndarray, b: int) -> np.ndarray:
    x = np.array(x, dtype=np.float64, copy=True)
    a = np.asfortranarray(lu_f32, dtype=np.float32)
    _trsv_u(a.shape[0], b, _p(a), a.shape[0], _p(x))
    return x


def refine(lu_f32, b, seed, rhs_v, d, maxit=50, q=1):
    n = lu_f32.shape[0]
    a = np.asfortranarray(lu_f32, dtype=np.float32)
    x = np.zeros(n)
    sr, sh = np.zeros(max(maxit, 1)), np.zeros(max(maxit, 1))
    ns = _int()
    res, har = _dbl(), _dbl()
    rc = _refine(n, b, q, _p(a), n, seed, _p(np.ascontiguousarray(rhs_v)), _p(np.ascontiguousarray(d)), maxit, _p(x),
                 _p(sr), _p(sh), ctypes.byref(ns), ctypes.byref(res), ctypes.byref(har))
    steps = list(zip(sr[:ns.value].tolist(), sh[:ns.value].tolist()))
    return rc, x, res.value, har.value, steps


def solve(n, b, seed=42, maxit=50, q=1):
    """Generate, factor and refine on the CPU; returns (rc, x, resid, harness, steps)."""
    x = np.zeros(n)
    sr, sh = np.zeros(max(maxit, 1)), np.zeros(max(maxit, 1))
    ns = _int()
    res, har = _dbl(), _dbl()
    rc = _solve(n, b, q, seed, maxit, _p(x), _p(sr), _p(sh), ctypes.byref(ns), ctypes.byref(res), ctypes.byref(har))
    steps = list(zip(sr[:ns.value].tolist(), sh[:ns.value].tolist()))
    return rc, x, res.value, har.value, steps


def dense_matrix_f64(n, seed=42) -> np.ndarray:
    """The FP64 HPL-AI matrix (off-diagonal generator values, FP64 row-sum
    diagonal), as Matgen<double> defines it for the residual.  Vectorised
    over rows: column j+1's states are column j's advanced by inc1^n."""
    scale = float.fromhex("0x1.fffffffffffffp-65")
    col = np.empty(n, dtype=np.uint64)
    s = state_at(n, 0, 0, seed)
    for i in range(n):
        col[i] = s
        s = (s * 6364136223846793005 + 1) & ((1 << 64) - 1)
    an, cn = coeff_pow(n)
    an, cn = np.uint64(an), np.uint64(cn)
    a = np.empty((n, n), order="F")
    with np.errstate(over="ignore"):
        for j in range(n):
            a[:, j] = col.view(np.int64).astype(np.float64) * scale
            col = col * an + cn
    a[np.arange(n), np.arange(n)] = diag(n, seed)
    return a


def e4m3_rn(x: float) -> int:
    return int(_e4m3_rn(x))


def e4m3_to_f32(b: int) -> float:
    return float(_e4m3_to_f32(b))


def quantize_e4m3(x: np.ndarray, col_major: bool, ld8: int = None):
    """e4m3 copy of the rows x k panel X with one power-of-two factor per 128
    rows.  col_major: X given as an (rows, k) array read down columns (an L
    panel); else X given as (rows, k) with k contiguous in memory.  Returns
    (bytes (rows, ld8) uint8, scale (ceil(rows/128),) float32)."""
    x = np.asarray(x, dtype=np.float32)
    rows, k = x.shape
    ld8 = ld8 or (k + 127) // 128 * 128
    if col_major:
        src = np.asfortranarray(x)
        lds = max(rows, 1)
    else:
        src = np.ascontiguousarray(x)
        lds = k
    dst = np.zeros((rows, ld8), dtype=np.uint8)
    scale = np.zeros((rows + 127) // 128, dtype=np.float32)
    _quantize_e4m3(rows, k, _p(src), lds, 1 if col_major else 0, _p(dst), ld8, _p(scale))
    return dst, scale


def f8gemm_minus(c: np.ndarray, l8: np.ndarray, sl: np.ndarray, u8: np.ndarray, su: np.ndarray, k: int) -> np.ndarray:
    """C - diag(sl) L8 U8^T diag(su), FP64 sums of the exact e4m3 products."""
    c = np.array(c, dtype=np.float32, order="F", copy=True)
    l8 = np.ascontiguousarray(l8, dtype=np.uint8)
    u8 = np.ascontiguousarray(u8, dtype=np.uint8)
    m, n = c.shape
    _f8gemm(m, n, k, _p(l8), l8.shape[1], _p(np.ascontiguousarray(sl, dtype=np.float32)), _p(u8), u8.shape[1],
            _p(np.ascontiguousarray(su, dtype=np.float32)), _p(c), m)
    return c


def residual_rows(n, x, rows, seed=42, trans=False, rhs_col=0, rhs_v=None) -> np.ndarray:
    """r_i = rhs_i - (A x)_i for the listed rows of the FP64 matrix the
    refinement regenerates (long-double sums; n generator steps per row).
    rhs_v: the right-hand side (host vector), else column n + rhs_col of the
    generator stream."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.zeros(len(rows))
    rv = None if rhs_v is None else np.ascontiguousarray(rhs_v, dtype=np.float64)
    _residual_rows(n, seed, _p(x), len(rows), _p(rows), 1 if trans else 0, rhs_col,
                   None if rv is None else _p(rv), _p(out))
    return out


# ---- Higham's HPL-AI matrix (--highammat) --------------------------------

def higham_params(n, cond=1000.0, rho=0.5):
    """(alpha, beta): higham_mat_comp_beta restated (32-bit int terms)."""
    b = _higham_beta(n, cond, rho)
    return rho * b, b


def higham_matrix(n, alpha, beta, i0=0, j0=0, nrow=None, ncol=None) -> np.ndarray:
    """The FP32 matrix (or a sub-matrix) as the reference forms it in float."""
    nrow = n if nrow is None else nrow
    ncol = n if ncol is None else ncol
    a = np.zeros((nrow, ncol), dtype=np.float32, order="F")
    _higham_fill(i0, j0, nrow, ncol, alpha, beta, _p(a), nrow)
    return a


def higham_dense_f64(n, alpha, beta) -> np.ndarray:
    """The FP64 matrix: row constants above the diagonal, column constants
    below it, each one fused multiply-add as orc_higham_elem."""
    up = np.array([_higham_elem(k, k + 1, alpha, beta) for k in range(n)])
    lo = np.array([_higham_elem(k + 1, k, alpha, beta) for k in range(n)])
    i = np.arange(n)
    a = np.where(i[:, None] < i[None, :], up[:, None], lo[None, :])
    np.fill_diagonal(a, higham_diag(n, alpha, beta))
    return a


def higham_diag(n, alpha, beta) -> np.ndarray:
    d = np.zeros(n)
    _higham_diag(n, alpha, beta, _p(d))
    return d


def higham_norm(n, alpha, beta) -> float:
    return _higham_norm(n, alpha, beta)


def higham_residual_rows(n, alpha, beta, x, rows, rhs_v) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    rhs_v = np.ascontiguousarray(rhs_v, dtype=np.float64)
    r = np.zeros(rows.size)
    _higham_resid(n, alpha, beta, _p(x), _p(rows), rows.size, _p(rhs_v), _p(r))
    return r
