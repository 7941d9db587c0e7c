"""CPU checks of bench.py's roofline model of the Schur updates.

The model lists the updates one factorisation issues (hplai_factor's order:
per group of panels the next group's block columns, its block rows, the
thin updates of the group's later blocks by its earlier panels, then the
rest).  Grouping panels changes how the work is cut into launches, never the
work itself, so the flops must equal those of the one-panel right-looking LU
(sum over steps k of 2 b (n - (k+1) b)^2, panel_trf.hpp:434-633), and the
launch count at n = 131072, b = 1024 with four-panel groups must match the
472 trailing-update launches of the committed ncu launch list of that solve.
"""
import importlib.util
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_model", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def lu_update_flops(n, b):
    nb = n // b
    return sum(2.0 * b * (n - (k + 1) * b) ** 2 for k in range(nb - 1))


@pytest.mark.parametrize("n,b", [(4096, 256), (5120, 512), (65536, 512), (131072, 1024), (204800, 1024)])
@pytest.mark.parametrize("group", [1, 2, 4])
def test_grouping_keeps_the_flops(bench, n, b, group):
    flops, _, launches = bench.schur_algorithmic(n, b, 1, 4, group)
    assert flops == lu_update_flops(n, b)
    assert launches > 0


def test_c_elements_match_flops(bench):
    # bytes with c_bytes = 1 and no panel bytes count C elements: flops / (2 K) per launch,
    # so with one-panel updates the C elements are the flops over 2 b
    n, b = 65536, 512
    flops, c_elems, _ = bench.schur_algorithmic(n, b, 0, 1, 1)
    assert c_elems == flops / (2.0 * b)


def test_launch_count_matches_the_c3_launch_list(bench):
    # profiles/launches_bench_c3_precision_n131072_b1024.md: 472 schur_kernel<2, 1> launches
    # per solve with four-panel groups
    _, _, launches = bench.schur_algorithmic(131072, 1024, 1, 4, 4)
    assert launches == 472
    text = open(os.path.join(ROOT, "profiles", "launches_bench_c3_precision_n131072_b1024.md")).read()
    assert "| 472 |" in text


def test_traffic_model_uses_the_capture_at_the_schedule_k(bench):
    d = json.load(open(os.path.join(ROOT, "profiles", "schur_kernel_traffic.json")))["kernels"]
    n, b = 131072, 1024
    _, c_elems, launches = bench.schur_algorithmic(n, b, 0, 1, 4)
    got = bench.schur_traffic_per_launch(n, b, 4, "e4m3_deck")
    assert got == pytest.approx(d["e4m3_deck_k4096"]["dram_bytes_per_c_element"] * c_elems / launches)
    _, c_elems2, launches2 = bench.schur_algorithmic(n, b, 0, 1, 2)
    got2 = bench.schur_traffic_per_launch(n, b, 2, "e4m3_deck")
    assert got2 == pytest.approx(d["e4m3_deck"]["dram_bytes_per_c_element"] * c_elems2 / launches2)
