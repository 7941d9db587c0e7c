"""The C ABI library loads and exports every function include/hplai.h
declares (no GPU needed: nothing here launches a kernel)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "hplai.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(hplai_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "hplai_create" in names and "hplai_shgemm_minus" in names and len(names) >= 25


def test_library_exports_every_declared_symbol(hplai):
    lib = ctypes.CDLL(hplai.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_calls(hplai):
    assert hplai.version() == 100
    assert hplai.status_string(hplai.HPLAI_ENOTCONV) == "refinement did not converge"
    line = hplai.format_report(1200, 1.546135562, 3.899311429300667e-14, 0.181652325)
    # the reference's report format (main.cpp:451-452) on its published numbers
    # (README:56); the reference divided by the unrounded time, so the last
    # GFlop/s digit may differ
    m = re.fullmatch(r"(\d+\.\d{9}) sec\. (\d+\.\d{9}) GFlop/s resid = +(\S+) hpl-harness = (\d+\.\d{9})", line)
    assert m, line
    assert m.group(1) == "1.546135562" and m.group(3) == "3.899311429300667e-14" and m.group(4) == "0.181652325"
    assert abs(float(m.group(2)) - 0.746480470) < 2e-9
    assert hplai.otf_gemv_workspace(4096) == 2 * 4096 * 8
    assert hplai.trsv_workspace(256) > 0


def test_invalid_arguments_rejected_without_gpu(hplai):
    import pytest
    with pytest.raises(hplai.HplaiError) as e:
        hplai.Solver(1000, 60)           # n % b != 0
    assert e.value.status == hplai.HPLAI_EINVAL
    assert hplai.fill_panel(0, 0, 0, 1, 1, None, 1, 42, 0, None) == hplai.HPLAI_EINVAL
    assert hplai.getrf_nopiv(2048, None, 2048, None) == hplai.HPLAI_EINVAL
    # panel_check: lda < n, missing output, and work smaller than its workspace
    assert hplai.panel_check_workspace(1 << 20) == 3 * 8 * 1184
    assert hplai.panel_check(100, 16, 99, 16, 16, 1 << 20, None) == hplai.HPLAI_EINVAL
    assert hplai.panel_check(100, 16, 100, None, 16, 1 << 20, None) == hplai.HPLAI_EINVAL
    assert hplai.panel_check(100, 16, 100, 16, 16, hplai.panel_check_workspace(100) - 1, None) == hplai.HPLAI_EINVAL


def test_create_rejects_invalid_schedules_without_gpu(hplai):
    """hplai_create checks sizes, precision and flag combinations before any
    CUDA call, so each refusal is visible on a machine without a GPU."""
    import pytest
    F = hplai
    cases = [
        (1024, 8, F.F32_F16, 0, F.HPLAI_EINVAL),                                        # b < 16
        (4096, 2048, F.F32_F16, 0, F.HPLAI_EINVAL),                                     # b > 1024
        (4096, 256, 7, 0, F.HPLAI_EUNSUPPORTED),                                        # precision
        (4080, 60, F.F32_F16, F.FLAG_FP16_DECK, F.HPLAI_EINVAL),                        # deck: b % 8
        (4096, 64, F.F32_F16, F.FLAG_GROUP2, F.HPLAI_EINVAL),                           # groups: b % 128
        (4096, 64, F.F32_F8, F.FLAG_GROUP4, F.HPLAI_EINVAL),
        (4096, 256, F.F32_F16, F.FLAG_GROUP2 | F.FLAG_GROUP4, F.HPLAI_EINVAL),          # both group sizes
        (4096, 256, F.F32_F8, F.FLAG_REF_DECK, F.HPLAI_EINVAL),                         # -d arithmetic: FP16 form only
        (4096, 256, F.F32_F16, F.FLAG_REF_DECK | F.FLAG_LOOKAHEAD, F.HPLAI_EINVAL),
        (4096, 256, F.F32_F16, F.FLAG_REF_DECK | F.FLAG_GROUP2, F.HPLAI_EINVAL),
        (4096, 256, F.F32_F16, F.FLAG_REF_BACKBUF, F.HPLAI_EINVAL),                     # back buffer needs -d
        (4096, 256, F.F32_F8, F.FLAG_LAZY_A, F.HPLAI_EINVAL),                           # no stored A: deck form
        (4096, 256, F.F32_F16, F.FLAG_LAZY_A | F.FLAG_FP16_DECK, F.HPLAI_EINVAL),       # ... and e4m3
        (4096, 256, F.F32_F8, F.FLAG_LAZY_A | F.FLAG_FP16_DECK | F.FLAG_SIMT_PANELS, F.HPLAI_EINVAL),
    ]
    for n, b, prec, flags, status in cases:
        with pytest.raises(F.HplaiError) as e:
            F.Solver(n, b, precision=prec, flags=flags)
        assert e.value.status == status, (n, b, prec, flags)
