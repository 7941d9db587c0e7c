"""ctypes binding of libhplai (include/hplai.h) for tests and benchmarks.

The product is the C ABI in libhplai.so plus the C++ driver (driver.out);
this module only marshals arguments.  It loads the in-tree shared library
and raises ImportError when it is missing: there is no fallback path.

Names follow the reference (RIKEN-RCCS/hpl-ai): `iterative_refinement`
returns IRErrors {residual, hpl_harness} = {-1, -1} on failure
(iterative_refinement.hpp:13-57) instead of raising.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhplai.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"libhplai.so not built at {LIB_PATH}; run `make -C {_HERE}`")

_lib = ctypes.CDLL(LIB_PATH)

HPLAI_OK, HPLAI_EINVAL, HPLAI_ENOMEM, HPLAI_ECUDA, HPLAI_ENOTCONV, HPLAI_ETIMEOUT, HPLAI_ESTATE, \
    HPLAI_EUNSUPPORTED = range(8)
F32_F16, F32_F8 = 0, 1
FLAG_SIMT_PANELS = 1
FLAG_LOOKAHEAD = 2
FLAG_FP16_DECK = 4
FLAG_GROUP2 = 8
FLAG_GROUP4 = 128
TRIAL_CTA_PAIRS = 0x80000000
FLAG_REF_DECK = 16
FLAG_REF_BACKBUF = 32
FLAG_LAZY_A = 64
MATRIX_LCG = 0
MATRIX_HIGHAM = 1
IR, GMRES = 0, 1
PHASES = ("DIAG_LU", "TRSM_L", "TRSM_R", "GEMM_UPDATE", "IR_GEMV", "IR_TRSV", "TOTAL", "LAZY_INIT", "WRITE_BACK")

_c_int, _c_i64, _c_u64, _c_dbl, _c_flt, _c_sz, _vp = (
    ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double, ctypes.c_float, ctypes.c_size_t,
    ctypes.c_void_p)


class IRErrors(ctypes.Structure):
    _fields_ = [("residual", ctypes.c_double), ("hpl_harness", ctypes.c_double)]


def _proto(name, restype, *argtypes):
    f = getattr(_lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


_status_string = _proto("hplai_status_string", ctypes.c_char_p, _c_int)
_last_error = _proto("hplai_last_error", _c_int, ctypes.c_char_p, _c_sz)
version = _proto("hplai_version", _c_int)
_create = _proto("hplai_create", _c_int, ctypes.POINTER(_vp), _c_int, _c_int, _c_int, ctypes.c_uint)
_destroy = _proto("hplai_destroy", _c_int, _vp)
_generate = _proto("hplai_generate", _c_int, _vp, _c_u64)
_upload = _proto("hplai_upload", _c_int, _vp, _vp, _c_i64, _vp, _vp, _c_u64)
_factor = _proto("hplai_factor", _c_int, _vp)
_set_matrix = _proto("hplai_set_matrix", _c_int, _vp, _c_int, ctypes.c_double, ctypes.c_double)
_higham_params = _proto("hplai_higham_params", _c_int, _c_int, ctypes.c_double, ctypes.c_double,
                        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double))
_factor_steps = _proto("hplai_factor_steps", _c_int, _vp, _c_int)
_l1est = _proto("hplai_l1est", _c_int, _vp)
_autotune = _proto("hplai_autotune", _c_int, _vp, _c_u64, _vp, _vp, _vp)
_set_schedule = _proto("hplai_set_schedule", _c_int, _vp, ctypes.c_uint, _c_int)
_autotune_log = _proto("hplai_get_autotune_log", _c_int, _vp, _vp, _vp, _vp, _c_int, ctypes.POINTER(_c_int))
_autotune_trials = _proto("hplai_get_autotune_trials", _c_int, _vp, _vp, _vp, _vp, _vp, _c_int,
                          ctypes.POINTER(_c_int))
_set_tile_group = _proto("hplai_set_tile_group", _c_int, _vp, _c_int)
_get_tile_group = _proto("hplai_get_tile_group", _c_int, _vp, ctypes.POINTER(_c_int))
_set_cta_pairs = _proto("hplai_set_cta_pairs", _c_int, _vp, _c_int)
_get_cta_pairs = _proto("hplai_get_cta_pairs", _c_int, _vp, ctypes.POINTER(_c_int))
_refine = _proto("hplai_refine", _c_int, _vp, _c_int, _c_int, ctypes.POINTER(IRErrors), ctypes.POINTER(_c_int))
_get_x = _proto("hplai_get_x", _c_int, _vp, _vp)
_get_lu = _proto("hplai_get_lu", _c_int, _vp, _vp, _c_i64)
_checksum = _proto("hplai_checksum", _c_int, _vp, _vp)
_get_rhs = _proto("hplai_get_rhs", _c_int, _vp, _vp)
_get_diag = _proto("hplai_get_diag", _c_int, _vp, _vp)
_get_ir_log = _proto("hplai_get_ir_log", _c_int, _vp, _vp, _vp, _c_int, ctypes.POINTER(_c_int))
_get_phase_ms = _proto("hplai_get_phase_ms", _c_int, _vp, _vp, _c_int)
_get_stream = _proto("hplai_get_stream", _vp, _vp)
launch_count = _proto("hplai_launch_count", ctypes.c_ulonglong)
_solve_rhs = _proto("hplai_solve_rhs", _c_int, _vp, _vp, _vp, _c_int, ctypes.POINTER(IRErrors), ctypes.POINTER(_c_int))
_solve_transpose = _proto("hplai_solve_transpose", _c_int, _vp, _vp, _vp, _c_int, ctypes.POINTER(IRErrors),
                          ctypes.POINTER(_c_int))
_set_gmres = _proto("hplai_set_gmres", _c_int, _vp, _c_int, _c_dbl)
_set_gmres_side = _proto("hplai_set_gmres_side", _c_int, _vp, _c_int)
_get_refine_counts = _proto("hplai_get_refine_counts", _c_int, _vp, ctypes.POINTER(_c_int), ctypes.POINTER(_c_int))
_get_norms = _proto("hplai_get_norms", _c_int, _vp, ctypes.POINTER(_c_dbl), ctypes.POINTER(_c_dbl))
_solve_host = _proto("hplai_solve_host", _c_int, _vp, _vp, _c_i64, _vp, _vp, _c_u64, _c_int, _vp,
                     ctypes.POINTER(IRErrors), ctypes.POINTER(_c_int))
_format_report = _proto("hplai_format_report", _c_int, _c_int, _c_dbl, IRErrors, ctypes.c_char_p, _c_sz)

fill_panel = _proto("hplai_fill_panel", _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _c_i64, _c_u64,
                    _c_int, _vp)
gen_rhs = _proto("hplai_gen_rhs", _c_int, _c_int, _c_u64, _vp, _vp)
gen_diag = _proto("hplai_gen_diag", _c_int, _c_int, _c_u64, _c_int, _c_int, _vp, _vp)
getrf_nopiv = _proto("hplai_getrf_nopiv", _c_int, _c_int, _vp, _c_i64, _vp)
trsm_right_upper = _proto("hplai_trsm_right_upper", _c_int, _c_int, _c_int, _vp, _c_i64, _vp, _c_i64, _vp, _c_i64,
                          _c_flt, _vp)
trsm_left_lower = _proto("hplai_trsm_left_lower", _c_int, _c_int, _c_int, _vp, _c_i64, _vp, _c_i64, _vp, _c_i64,
                         _c_flt, _vp)
shgemm_minus = _proto("hplai_shgemm_minus", _c_int, _c_int, _c_int, _c_int, _vp, _c_i64, _vp, _c_i64, _vp, _c_i64,
                      _vp)
quantize_e4m3 = _proto("hplai_quantize_e4m3", _c_int, _c_int, _c_int, _vp, _c_i64, _c_int, _vp, _c_i64, _vp, _vp,
                       _vp)
f8gemm_minus = _proto("hplai_f8gemm_minus", _c_int, _c_int, _c_int, _c_int, _vp, _c_i64, _vp, _vp, _c_i64, _vp, _vp,
                      _c_i64, _vp)
shgemm_deck_minus = _proto("hplai_shgemm_deck_minus", _c_int, _c_int, _c_int, _c_int, _vp, _c_i64, _vp, _c_i64, _vp,
                           _c_i64, _c_flt, _vp)
f8gemm_deck_minus = _proto("hplai_f8gemm_deck_minus", _c_int, _c_int, _c_int, _c_int, _vp, _c_i64, _vp, _vp, _c_i64,
                           _vp, _vp, _c_i64, _c_flt, _vp)
otf_gemv_workspace = _proto("hplai_otf_gemv_workspace", _c_sz, _c_int)
otf_gemv = _proto("hplai_otf_gemv", _c_int, _c_int, _c_dbl, _vp, _c_dbl, _vp, _c_u64, _vp, _vp, _c_sz, _vp)
otf_gemv_noalloc = _proto("hplai_otf_gemv_noalloc", _c_int, _c_int, _c_dbl, _vp, _c_dbl, _vp, _c_u64, _vp, _vp)
OTF_GEMV_NOALLOC_MAX_N = 32768
otf_gemv_block = _proto("hplai_otf_gemv_block", _c_int, _c_i64, _c_int, _c_int, _c_dbl, _vp, _vp, _c_u64, _vp,
                        _c_sz, _vp)
trsv_workspace = _proto("hplai_trsv_workspace", _c_sz, _c_int)
trsv_lower = _proto("hplai_trsv_lower", _c_int, _c_int, _vp, _c_i64, _vp, _vp, _c_sz, _vp)
trsv_upper = _proto("hplai_trsv_upper", _c_int, _c_int, _vp, _c_i64, _vp, _vp, _c_sz, _vp)
infnorm = _proto("hplai_infnorm", _c_int, _c_int, _vp, _vp, _vp)
panel_check_workspace = _proto("hplai_panel_check_workspace", _c_sz, _c_int)
panel_check = _proto("hplai_panel_check", _c_int, _c_int, _vp, _c_i64, _vp, _vp, _c_sz, _vp)


gen_rhs_cols = _proto("hplai_gen_rhs_cols", _c_int, _c_int, _c_u64, _c_int, _c_int, _vp, _vp)
_batch_create = _proto("hplai_batch_create", _c_int, ctypes.POINTER(_vp), _c_int, _vp, _vp, _vp, _c_int, ctypes.c_uint,
                       _c_int)
_batch_destroy = _proto("hplai_batch_destroy", _c_int, _vp)
_batch_solve = _proto("hplai_batch_solve", _c_int, _vp, _c_int)
_batch_get_lu = _proto("hplai_batch_get_lu", _c_int, _vp, _c_int, _vp, _c_i64)
_batch_launches = _proto("hplai_batch_launches", ctypes.c_ulonglong, _vp)
_batch_result = _proto("hplai_batch_result", _c_int, _vp, _c_int, ctypes.POINTER(IRErrors), ctypes.POINTER(_c_int),
                       ctypes.POINTER(_c_int))
_batch_get_x = _proto("hplai_batch_get_x", _c_int, _vp, _c_int, _vp, _c_i64)
_batch_block = _proto("hplai_batch_block", _c_int, _vp, _c_int)


class HplaiError(RuntimeError):
    def __init__(self, status: int, what: str):
        buf = ctypes.create_string_buffer(512)
        _last_error(buf, 512)
        detail = buf.value.decode(errors="replace")
        super().__init__(f"{what}: {status_string(status)}" + (f" [{detail}]" if detail else ""))
        self.status = status


def status_string(status: int) -> str:
    return _status_string(status).decode()


def check(status: int, what: str = "hplai") -> int:
    if status != HPLAI_OK:
        raise HplaiError(status, what)
    return status


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def format_report(n: int, seconds: float, residual: float, harness: float) -> str:
    buf = ctypes.create_string_buffer(256)
    check(_format_report(n, seconds, IRErrors(residual, harness), buf, 256), "hplai_format_report")
    return buf.value.decode()


@dataclass
class RefineResult:
    residual: float
    hpl_harness: float
    iters: int
    status: int


def set_cta_pairs_default(on: bool):
    """The library default for deck updates on CTA pairs (contexts at -1 and the leaf calls)."""
    check(_set_cta_pairs(None, 1 if on else 0), "hplai_set_cta_pairs")


def higham_params(n: int, cond: float = 1000.0, rho: float = 0.5):
    """(alpha, beta) of Higham's HPL-AI matrix of order n."""
    a, b = ctypes.c_double(), ctypes.c_double()
    check(_higham_params(n, cond, rho, ctypes.byref(a), ctypes.byref(b)), "hplai_higham_params")
    return a.value, b.value


class Solver:
    """One solve context: the single-GPU collapse of the reference driver."""

    def __init__(self, n: int, b: int, precision: int = F32_F16, flags: int = 0):
        h = _vp()
        check(_create(ctypes.byref(h), n, b, precision, flags), f"hplai_create(n={n}, b={b})")
        self._h = h
        self.n, self.b = n, b

    def close(self):
        if getattr(self, "_h", None):
            _destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def generate(self, seed: int = 42):
        check(_generate(self._h, seed), "hplai_generate")

    def set_matrix(self, kind: int, cond: float = 1000.0, rho: float = 0.5):
        """MATRIX_LCG (the benchmark matrix) or MATRIX_HIGHAM (--highammat)."""
        check(_set_matrix(self._h, kind, cond, rho), "hplai_set_matrix")

    def upload(self, a: np.ndarray, rhs: np.ndarray, diag: np.ndarray, seed: int = 42):
        a = np.asfortranarray(a, dtype=np.float32)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        check(_upload(self._h, _ptr(a), a.shape[0], _ptr(rhs), _ptr(diag), seed), "hplai_upload")

    def factor(self):
        check(_factor(self._h), "hplai_factor")

    def factor_steps(self, steps: int):
        """Panels 0 .. steps-1 only (the reference's -w warm-up)."""
        check(_factor_steps(self._h, steps), "hplai_factor_steps")

    def l1est(self):
        """Approximate factors without a decomposition (the reference's --l1est)."""
        check(_l1est(self._h), "hplai_l1est")

    def autotune(self, seed: int = 42):
        """Time the factorisation serially and with look-ahead at several
        side-stream SM counts, keep the fastest schedule; returns
        (flags, side_sms, best_ms).  The context is left generated from seed."""
        fl, side, ms = ctypes.c_uint(), _c_int(), ctypes.c_double()
        check(_autotune(self._h, seed, ctypes.byref(fl), ctypes.byref(side), ctypes.byref(ms)), "hplai_autotune")
        return fl.value, side.value, ms.value

    def set_schedule(self, flags: int, side_sms: int = 32):
        """Look-ahead / two-panel groups and the side stream's SMs, by hand."""
        check(_set_schedule(self._h, flags, side_sms), "hplai_set_schedule")

    def autotune_log(self):
        """The last autotune's trials: [(flags, side_sms, ms)], warm-up first."""
        cap = 64
        fl = (ctypes.c_uint * cap)()
        sd = (_c_int * cap)()
        ms = (ctypes.c_double * cap)()
        cnt = _c_int()
        check(_autotune_log(self._h, fl, sd, ms, cap, ctypes.byref(cnt)), "hplai_get_autotune_log")
        return [(fl[i], sd[i], ms[i]) for i in range(min(cnt.value, cap))]

    def autotune_trials(self):
        """The last autotune's trials: [(flags, side_sms, tile_group, ms)], warm-up first."""
        cap = 64
        fl = (ctypes.c_uint * cap)()
        sd = (_c_int * cap)()
        tg = (_c_int * cap)()
        ms = (ctypes.c_double * cap)()
        cnt = _c_int()
        check(_autotune_trials(self._h, fl, sd, tg, ms, cap, ctypes.byref(cnt)), "hplai_get_autotune_trials")
        return [(fl[i], sd[i], tg[i], ms[i]) for i in range(min(cnt.value, cap))]

    def set_cta_pairs(self, on: int):
        """Deck updates on CTA pairs (1), single CTAs (0) or the library default (-1)."""
        check(_set_cta_pairs(self._h, on), "hplai_set_cta_pairs")

    def cta_pairs(self) -> int:
        v = _c_int()
        check(_get_cta_pairs(self._h, ctypes.byref(v)), "hplai_get_cta_pairs")
        return v.value

    def set_tile_group(self, group_m: int):
        check(_set_tile_group(self._h, group_m), "hplai_set_tile_group")

    def tile_group(self) -> int:
        g = _c_int()
        check(_get_tile_group(self._h, ctypes.byref(g)), "hplai_get_tile_group")
        return g.value

    def iterative_refinement(self, maxit: int = 50, mode: int = IR) -> RefineResult:
        e = IRErrors()
        it = _c_int()
        s = _refine(self._h, mode, maxit, ctypes.byref(e), ctypes.byref(it))
        if s not in (HPLAI_OK, HPLAI_ENOTCONV):
            check(s, "hplai_refine")
        return RefineResult(e.residual, e.hpl_harness, it.value, s)

    def _solve_vec(self, fn, name, v, maxit):
        v = np.ascontiguousarray(v, dtype=np.float64)
        if v.shape != (self.n,):
            raise ValueError(f"{name}: expected a vector of {self.n} doubles")
        out = np.empty(self.n, dtype=np.float64)
        e = IRErrors()
        it = _c_int()
        s = fn(self._h, _ptr(v), _ptr(out), maxit, ctypes.byref(e), ctypes.byref(it))
        if s not in (HPLAI_OK, HPLAI_ENOTCONV):
            check(s, name)
        return out, RefineResult(e.residual, e.hpl_harness, it.value, s)

    def solve_rhs(self, b, maxit: int = 50):
        """x = A^{-1} b for a caller's right-hand side (the factors of the last factor())."""
        return self._solve_vec(_solve_rhs, "hplai_solve_rhs", b, maxit)

    def solve_transpose(self, g, maxit: int = 50):
        """lambda = A^{-T} g: the adjoint solve."""
        return self._solve_vec(_solve_transpose, "hplai_solve_transpose", g, maxit)

    def set_gmres(self, restart: int = 30, tol: float = 1e-12):
        check(_set_gmres(self._h, restart, tol), "hplai_set_gmres")

    def set_gmres_side(self, right: bool):
        """GMRES preconditioning: right (flexible, the default) or left."""
        check(_set_gmres_side(self._h, 1 if right else 0), "hplai_set_gmres_side")

    def refine_counts(self):
        """(residual evaluations, GMRES inner steps) of the last refinement."""
        o, i = _c_int(), _c_int()
        check(_get_refine_counts(self._h, ctypes.byref(o), ctypes.byref(i)), "hplai_get_refine_counts")
        return o.value, i.value

    def solve_host(self, a, rhs, diag, seed=42, maxit=50):
        a = np.asfortranarray(a, dtype=np.float32)
        x = np.empty(self.n, dtype=np.float64)
        e = IRErrors()
        it = _c_int()
        s = _solve_host(self._h, _ptr(a), a.shape[0], _ptr(rhs), _ptr(diag), seed, maxit, _ptr(x), ctypes.byref(e),
                        ctypes.byref(it))
        if s not in (HPLAI_OK, HPLAI_ENOTCONV):
            check(s, "hplai_solve_host")
        return x, RefineResult(e.residual, e.hpl_harness, it.value, s)

    def x(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(_get_x(self._h, _ptr(out)), "hplai_get_x")
        return out

    def lu(self) -> np.ndarray:
        out = np.empty((self.n, self.n), dtype=np.float32, order="F")
        check(_get_lu(self._h, _ptr(out), self.n), "hplai_get_lu")
        return out

    def checksum(self) -> np.ndarray:
        """panel_check (panel_check.hpp:9-65): [sum |diag|, sum |strict upper|,
        sum |strict lower|] of the context's matrix (the factors after factor())."""
        out = np.empty(3, dtype=np.float64)
        check(_checksum(self._h, _ptr(out)), "hplai_checksum")
        return out

    def rhs(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(_get_rhs(self._h, _ptr(out)), "hplai_get_rhs")
        return out

    def diag(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(_get_diag(self._h, _ptr(out)), "hplai_get_diag")
        return out

    def ir_log(self):
        cap = 64
        r = np.zeros(cap)
        h = np.zeros(cap)
        cnt = _c_int()
        check(_get_ir_log(self._h, _ptr(r), _ptr(h), cap, ctypes.byref(cnt)), "hplai_get_ir_log")
        m = min(cnt.value, cap)
        return list(zip(r[:m].tolist(), h[:m].tolist()))

    def phase_ms(self) -> dict:
        out = np.zeros(len(PHASES))
        check(_get_phase_ms(self._h, _ptr(out), len(PHASES)), "hplai_get_phase_ms")
        return dict(zip(PHASES, out.tolist()))

    def stream(self) -> int:
        """cudaStream_t of this context as an integer handle."""
        return _get_stream(self._h) or 0

    def solve_host_ptrs(self, a_ptr: int, lda: int, rhs_ptr: int, diag_ptr: int, seed: int, maxit: int,
                        x_ptr: int) -> RefineResult:
        """hplai_solve_host on raw host pointers (e.g. pinned torch tensors)."""
        e = IRErrors()
        it = _c_int()
        s = _solve_host(self._h, a_ptr, lda, rhs_ptr, diag_ptr, seed, maxit, x_ptr, ctypes.byref(e), ctypes.byref(it))
        if s not in (HPLAI_OK, HPLAI_ENOTCONV):
            check(s, "hplai_solve_host")
        return RefineResult(e.residual, e.hpl_harness, it.value, s)

    def norms(self):
        a, b = _c_dbl(), _c_dbl()
        check(_get_norms(self._h, ctypes.byref(a), ctypes.byref(b)), "hplai_get_norms")
        return a.value, b.value


class Batch:
    """Many independent systems (sizes n[s], nrhs[s] right-hand sides, seeds[s])."""

    def __init__(self, n, nrhs, seeds, precision: int = F32_F16, flags: int = 0, workers: int = 0):
        self.n = np.ascontiguousarray(n, dtype=np.int32)
        self.nrhs = np.ascontiguousarray(nrhs, dtype=np.int32)
        self.seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        if not (len(self.n) == len(self.nrhs) == len(self.seeds)):
            raise ValueError("n, nrhs and seeds must have the same length")
        h = _vp()
        check(_batch_create(ctypes.byref(h), len(self.n), _ptr(self.n), _ptr(self.nrhs), _ptr(self.seeds), precision,
                            flags, workers), "hplai_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve(self, maxit: int = 50) -> int:
        s = _batch_solve(self._h, maxit)
        if s not in (HPLAI_OK, HPLAI_ENOTCONV):
            check(s, "hplai_batch_solve")
        return s

    def result(self, s: int) -> RefineResult:
        e = IRErrors()
        it, st = _c_int(), _c_int()
        check(_batch_result(self._h, s, ctypes.byref(e), ctypes.byref(it), ctypes.byref(st)), "hplai_batch_result")
        return RefineResult(e.residual, e.hpl_harness, it.value, st.value)

    def x(self, s: int) -> np.ndarray:
        out = np.empty((int(self.nrhs[s]), int(self.n[s])), dtype=np.float64)   # rows = columns of x
        check(_batch_get_x(self._h, s, _ptr(out), int(self.n[s])), "hplai_batch_get_x")
        return out.T

    def block(self, s: int) -> int:
        return _batch_block(self._h, s)

    def lu(self, s: int) -> np.ndarray:
        """System s's FP32 factors (unit L below the diagonal, U on and above)."""
        m = int(self.n[s])
        out = np.empty((m, m), dtype=np.float32, order="F")
        check(_batch_get_lu(self._h, s, _ptr(out), m), "hplai_batch_get_lu")
        return out

    def launches(self) -> int:
        """Kernel launches of the batched engine's generation + factorisation graph."""
        return int(_batch_launches(self._h))


def batch_sizes(count: int = 512, rng_seed: int = 20240611, lo: int = 256, hi: int = 4096):
    """System orders n_s = round64(exp(U(ln lo, ln hi))) and right-hand-side
    counts U{1..8} from a fixed host generator (numpy PCG64, rng_seed)."""
    rng = np.random.default_rng(rng_seed)
    n = np.exp(rng.uniform(np.log(lo), np.log(hi), count))
    n = np.clip(np.rint(n / 64).astype(np.int64) * 64, lo, hi).astype(np.int32)
    nrhs = rng.integers(1, 9, count).astype(np.int32)
    return n, nrhs
