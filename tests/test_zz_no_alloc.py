"""hplai_otf_gemv_noalloc: the on-the-fly GEMV for callers that cannot
allocate device memory (they only receive device buffers from another
runtime's allocator, or must not call cudaMalloc inside a solve because it
can synchronise the device).  It takes its scratch from an array compiled
into the library, so it is checked here through the C ABI against the
workspace entry point, hplai_otf_gemv, on two calls in a row -- the array
keeps the previous call's contents, and the second call must not see them.

This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemv_pair(hplai, torch, n, seed, alpha, beta, rng):
    x = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
    y0 = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
    d = torch.from_numpy(rng.uniform(n / 5, n / 3, n)).cuda()
    y_ws, y_na = y0.clone(), y0.clone()
    ws = hplai.otf_gemv_workspace(n)
    w = torch.empty(ws // 8 + 1, dtype=torch.float64, device="cuda")
    hplai.check(hplai.otf_gemv(n, alpha, x.data_ptr(), beta, y_ws.data_ptr(), seed, d.data_ptr(), w.data_ptr(), ws,
                               None), "hplai_otf_gemv")
    hplai.check(hplai.otf_gemv_noalloc(n, alpha, x.data_ptr(), beta, y_na.data_ptr(), seed, d.data_ptr(), None),
                "hplai_otf_gemv_noalloc")
    torch.cuda.synchronize()
    scale = float(d.abs().max().item() + n / 2) * float(x.abs().max().item()) * abs(alpha) + abs(beta)
    return y_ws.cpu().numpy(), y_na.cpu().numpy(), scale


@pytest.mark.parametrize("n", [5000, 32768])
def test_noalloc_matches_workspace_entry_twice(hplai, torch_cuda, n):
    """Two calls in a row with different inputs (the second one smaller, so a
    stale partial sum of the first would show); same tolerance as the other
    GEMV tests: 1e-14 of ||A||_inf ||x||_inf."""
    torch = torch_cuda
    rng = np.random.default_rng(n)
    a, b, scale = _gemv_pair(hplai, torch, n, 42, -1.0, 1.0, rng)
    assert np.abs(a - b).max() <= 1e-14 * scale
    m = n // 2 + 7
    a2, b2, scale2 = _gemv_pair(hplai, torch, m, 7, 0.5, 0.0, rng)
    assert np.abs(a2 - b2).max() <= 1e-14 * scale2


def test_noalloc_rejects_orders_beyond_its_scratch(hplai, torch_cuda):
    n = hplai.OTF_GEMV_NOALLOC_MAX_N + 1
    # pointers are never touched: the size check comes first
    rc = hplai.otf_gemv_noalloc(n, 1.0, 16, 0.0, 16, 42, 16, None)
    assert rc == hplai.HPLAI_EINVAL
    with pytest.raises(hplai.HplaiError, match="HPLAI_OTF_GEMV_NOALLOC_MAX_N"):
        hplai.check(rc, "hplai_otf_gemv_noalloc")
