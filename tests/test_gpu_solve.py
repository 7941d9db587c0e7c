"""End-to-end solves through the context API against the oracle (B200)."""
import json
import re
import subprocess
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_c1_solve_matches_reference_and_oracle(hplai, oracle, torch_cuda):
    """n=1200, b=60, seed 42: hpl-harness < 16, the step-0 residual equals the
    reference's published value to 1e-13 (summation order differs), and x
    matches the oracle's x and a dense FP64 solve to 1e-12 relative."""
    g = json.load(open(os.path.join(HERE, "golden", "readme_step0.json")))
    n, b = g["n"], g["b"]
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.factor()
        r = s.iterative_refinement(50)
        x = s.x()
        log = s.ir_log()
        assert np.array_equal(s.rhs(), oracle.rhs(n))
        assert np.array_equal(s.diag(), oracle.diag(n))
        norma, normb = s.norms()
    assert r.status == hplai.HPLAI_OK and 0 <= r.hpl_harness < 16
    assert abs(log[0][0] - g["step0_residual"]) <= 1e-13 * g["step0_residual"]
    assert abs(log[0][1] - g["step0_harness"]) <= 1e-12 * g["step0_harness"]
    rc, xo, res, har, steps = oracle.solve(n, b, q=1)
    assert rc == 0
    assert np.abs(x - xo).max() <= 1e-12 * np.abs(xo).max()
    a = oracle.dense_matrix_f64(n)
    xr = np.linalg.solve(a, oracle.rhs(n))
    assert np.abs(x - xr).max() <= 1e-12 * np.abs(xr).max()
    assert norma == 2 * oracle.diag(n).max() and normb == np.abs(oracle.rhs(n)).max()


@pytest.mark.parametrize("flags", [0, 1])
def test_block_size_not_multiple_of_four(hplai, oracle, torch_cuda, flags):
    """b = 50 (as in the reference's sweep, tests/test.py) takes the plain
    Schur epilogue; the solve still converges to the oracle's x."""
    n, b = 1200, 50
    with hplai.Solver(n, b, flags=flags) as s:
        s.generate(42)
        s.factor()
        r = s.iterative_refinement(50)
        x = s.x()
    assert r.status == hplai.HPLAI_OK and 0 <= r.hpl_harness < 16
    rc, xo, _, _, _ = oracle.solve(n, b, q=1)
    assert rc == 0 and np.abs(x - xo).max() <= 1e-12 * np.abs(xo).max()


def _first_panels(hplai, n, b, flags):
    with hplai.Solver(n, b, flags=flags) as s:
        s.generate(42)
        s.factor()
        return s.lu()


@pytest.mark.parametrize("n,b", [(1200, 60), (4096, 512), (3072, 1024)])
def test_simt_panels_bit_exact_first_step(hplai, oracle, torch_cuda, n, b):
    """With HPLAI_FLAG_SIMT_PANELS the first step's diagonal block and both
    panels (final after step 0) equal the oracle's netlib-order TRSMs bit for
    bit; the rest differs only by the Schur update's summation order."""
    lu = _first_panels(hplai, n, b, hplai.FLAG_SIMT_PANELS)
    a = oracle.matrix(n)
    f = a[:b, :b].copy(order="F")
    d = oracle.getrf_nopiv(f)
    lcol = oracle.trsm_right_upper(np.triu(d), a[b:, :b])
    urow = oracle.trsm_left_lower_unit(np.tril(d, -1) + np.eye(b, dtype=np.float32), a[:b, b:])
    assert np.array_equal(lu[:b, :b].view(np.uint32), d.view(np.uint32))
    assert np.array_equal(lu[b:, :b].view(np.uint32), lcol.view(np.uint32))
    assert np.array_equal(lu[:b, b:].view(np.uint32), urow.view(np.uint32))
    if n <= 1200:
        ref = oracle.lu(a, b)
        rel = np.abs(lu.astype(np.float64) - ref) / (np.abs(ref) + 1e-3 * np.abs(ref).max())
        assert rel.max() < 1e-3


@pytest.mark.parametrize("n,b", [(1200, 60), (4096, 512), (3072, 1024)])
def test_tensor_core_panels_fp32_accurate(hplai, oracle, torch_cuda, n, b):
    """Default path: the panels come from the diagonal block's triangular
    inverses applied in 3xTF32 on tcgen05.  Against the FP64 products of the
    same (bit-exact) diagonal factors, every element is within
    2^-18 * (|A| |T^-1|) -- FP32-level, far below the FP16 of the Schur update."""
    lu = _first_panels(hplai, n, b, 0)
    a = oracle.matrix(n).astype(np.float64)
    d = oracle.getrf_nopiv(a[:b, :b].astype(np.float32)).astype(np.float64)
    assert np.array_equal(lu[:b, :b], d.astype(np.float32))
    uinv = np.linalg.inv(np.triu(d))
    linv = np.linalg.inv(np.tril(d, -1) + np.eye(b))
    lcol = a[b:, :b] @ uinv
    urow = linv @ a[:b, b:]
    bl = np.abs(a[b:, :b]) @ np.abs(uinv) * 2.0 ** -18
    bu = np.abs(linv) @ np.abs(a[:b, b:]) * 2.0 ** -18
    assert np.all(np.abs(lu[b:, :b] - lcol) <= bl + 1e-30)
    assert np.all(np.abs(lu[:b, b:] - urow) <= bu + 1e-30)


@pytest.mark.parametrize("n,b,flags", [(1200, 60, 0), (8192, 512, 0), (6144, 1024, 0), (4096, 256, 1), (1200, 50, 0)])
def test_lookahead_matches_serial_schedule(hplai, torch_cuda, n, b, flags):
    """The two-stream look-ahead (next panel formed on the side stream while
    the main stream updates the rest) computes exactly what the one-stream
    schedule computes: every element sees the same kernels in the same
    order, so the factors must be bit-identical."""
    def lu(f):
        with hplai.Solver(n, b, flags=f) as s:
            s.generate(42)
            s.factor()
            return s.lu()
    a = lu(flags | hplai.FLAG_LOOKAHEAD)
    z = lu(flags)
    assert np.array_equal(a.view(np.uint32), z.view(np.uint32))


@pytest.mark.parametrize("n,b", [(2048, 64), (3000, 100), (8192, 256), (16384, 512)])
def test_larger_solves_converge(hplai, oracle, torch_cuda, n, b):
    """Size-independent checks: hpl-harness < 16 (the FP64 backward-error
    criterion on the regenerated matrix) and the step-0 residual, which only
    involves the generator and the FP64 GEMV, against the oracle."""
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.factor()
        r = s.iterative_refinement(50)
        log = s.ir_log()
    assert r.status == hplai.HPLAI_OK and 0 <= r.hpl_harness < 16 and r.iters <= 6
    zero = np.zeros((n, n), dtype=np.float32, order="F") if n <= 4096 else None
    if zero is not None:
        _, _, _, _, steps = oracle.refine(zero, b, 42, oracle.rhs(n), oracle.diag(n), maxit=1)
        assert abs(log[0][0] - steps[0][0]) <= 1e-12 * steps[0][0]


def test_solve_host_matches_device_path(hplai, oracle, torch_cuda):
    n, b = 1200, 60
    a = oracle.matrix(n)
    with hplai.Solver(n, b) as s:
        x, r = s.solve_host(a, oracle.rhs(n), oracle.diag(n), 42, 50)
        assert r.status == hplai.HPLAI_OK and r.hpl_harness < 16
        s.generate(42)
        s.factor()
        s.iterative_refinement(50)
        assert np.array_equal(s.x(), x)


@pytest.mark.parametrize("precision,flags,n,b", [(0, 4, 4096, 256), (1, 4 | 8, 4096, 512), (1, 4 | 8 | 2, 8192, 1024)])
def test_streamed_host_solve_matches_device_path(hplai, oracle, torch_cuda, precision, flags, n, b):
    """hplai_solve_host with the FP16 deck and page-locked buffers copies the
    matrix panel by panel behind the factorisation: x equals the device
    path's bit for bit (the same kernels on the same values), twice in a row
    (the second solve overwrites the first one's factors)."""
    torch = torch_cuda
    with hplai.Solver(n, b, precision=precision, flags=flags) as s:
        s.generate(42)
        a_h = torch.empty(n * n, dtype=torch.float32, pin_memory=True)
        hplai.check(hplai._get_lu(s._h, a_h.data_ptr(), n), "hplai_get_lu")
        rhs_h = torch.from_numpy(s.rhs()).pin_memory()
        d_h = torch.from_numpy(s.diag()).pin_memory()
        x_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
        mode = hplai.GMRES if precision == hplai.F32_F8 else hplai.IR
        s.factor()
        s.iterative_refinement(50, mode=mode)
        x_dev = s.x()
        for _ in range(2):
            r = s.solve_host_ptrs(a_h.data_ptr(), n, rhs_h.data_ptr(), d_h.data_ptr(), 42, 50, x_h.data_ptr())
            assert r.status == hplai.HPLAI_OK and r.hpl_harness < 16
            assert np.array_equal(x_h.numpy(), x_dev)


def test_call_order_and_nonconvergence(hplai, torch_cuda):
    with hplai.Solver(480, 60) as s:
        with pytest.raises(hplai.HplaiError) as e:
            s.factor()
        assert e.value.status == hplai.HPLAI_ESTATE
        s.generate(42)
        with pytest.raises(hplai.HplaiError):
            s.iterative_refinement(5)          # before factor
        s.factor()
        r = s.iterative_refinement(1)          # one step cannot reach < 16: IRErrors {-1,-1}
        assert r.status == hplai.HPLAI_ENOTCONV and r.residual == -1 and r.hpl_harness == -1
        r = s.iterative_refinement(50)
        assert r.status == hplai.HPLAI_OK


def test_autotune_picks_a_schedule_and_solves(hplai, oracle, torch_cuda):
    """hplai_autotune leaves a valid schedule (serial, or look-ahead with a
    side-stream SM count) and a generated, unfactored context; the solve
    with that schedule converges to the same x as the serial one."""
    n, b = 4096, 512
    with hplai.Solver(n, b) as s:
        flags, side, ms = s.autotune(42)
        assert ms > 0.0 and (side in (16, 20, 24, 32, 48) or -24 <= side <= -8)
        assert flags & ~(hplai.FLAG_LOOKAHEAD | hplai.FLAG_GROUP2) == 0
        s.factor()
        res = s.iterative_refinement(50)
        x = s.x()
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0
    a = oracle.dense_matrix_f64(n, 42)
    xs = np.linalg.solve(a, oracle.rhs(n, 42))
    assert np.max(np.abs(x - xs)) / np.max(np.abs(xs)) < 1e-12


def test_checksum_after_lu_matches_oracle_and_driver(hplai, oracle, torch_cuda, tmp_path):
    """`--checksum` (panel_check.hpp:9-65, main.cpp:298-302) at n=1200, b=60:
    hplai_checksum over the factors equals the oracle's sums in the
    reference's block order to 1e-13 relative, repeats bit for bit, and
    driver.out prints the same three numbers on its `check` line.  The driver
    also writes the reference's Timerdump file (timer.hpp:174-218,
    main.cpp:470-478): 21 timer items, TOTAL at 100 %, the reference's
    operation counts, and the GEMM rate line."""
    import re
    import subprocess
    n, b = 1200, 60
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.factor()
        c1 = s.checksum()
        c2 = s.checksum()
        lu = s.lu()
    assert np.array_equal(c1, c2)
    want = oracle.panel_check(lu, b)
    assert np.all(np.abs(c1 - want) <= 1e-13 * want)
    exe = os.path.abspath(os.path.join(HERE, "..", "hpl-ai_b200", "driver.out"))
    out = subprocess.run([exe, str(n), str(b), "1", "--checksum", "--job-id", "7"], capture_output=True, text=True,
                         timeout=300, cwd=tmp_path)
    assert out.returncode == 0, out.stderr
    m = re.search(r"^check (\S+) (\S+), (\S+)$", out.stdout, re.M)
    assert m, out.stdout
    got = np.array([float(v) for v in m.groups()])
    assert np.all(np.abs(got - c1) <= 1e-15 * c1)
    assert re.search(r"GFlop/s resid = .* hpl-harness = ", out.stdout), out.stdout
    dump = (tmp_path / "Timerdump.000007.000001200.0060.00001.00000").read_text().splitlines()
    assert dump[0].startswith("# row=0, col=0, host=")
    items = {}
    for line in dump[1:22]:
        name, sec, pct, acc, _ = [f.strip() for f in line.split(":")]
        items[name] = (float(sec.split()[0]), float(pct.split()[0]), int(acc))
    assert len(items) == 21 and items["TOTAL"][1] == 100.0
    nb = n // b
    assert items["GEMM_UPDATE"][2] == 2 * b ** 3 * sum(k * k for k in range(nb))
    assert items["DIAG_LU"][2] == nb * (b * (b * (4 * b - 3) + 5) // 6)
    assert items["TRSM_L"][2] == items["TRSM_R"][2] == b ** 3 * nb * (nb - 1) // 2
    assert items["IR_GEMV"][2] > 0 and items["IR_GEMV"][2] % (2 * n * n) == 0
    assert items["GEMM_UPDATE"][0] > 0 and items["DIAG_BCAST"][0] == 0.0
    assert re.match(r"GEMM_TOTAL: \S+ Tflops$", dump[22])


def test_driver_warmup_and_l1est(hplai, torch_cuda, tmp_path):
    """driver.out -w (the first P + 2 panels, one refinement step, the
    skipped part taken off the flop count, a Warmup.* phase file) and
    --l1est (approximate factors, refinement to convergence), as the
    reference's driver (main.cpp:57,84,282-301,441-446,474)."""
    exe = os.path.abspath(os.path.join(HERE, "..", "hpl-ai_b200", "driver.out"))
    n, b, p = 1200, 60, 2
    out = subprocess.run([exe, str(n), str(b), str(p), "-w", "--job-id", "3"], capture_output=True, text=True,
                         timeout=300, cwd=tmp_path)
    assert out.returncode == 0, out.stderr
    m = re.search(r"^(\S+) sec\. (\S+) GFlop/s resid = (\S+) hpl-harness = (\S+)$", out.stdout, re.M)
    assert m and float(m.group(3)) == -1.0 and float(m.group(4)) == -1.0, out.stdout
    nn = n - (p + 2) * b
    flops = 2 / 3 * n ** 3 + 1.5 * n ** 2 - (2 / 3 * nn ** 3 + 1.5 * nn ** 2)
    assert abs(float(m.group(2)) - flops / float(m.group(1)) * 1e-9) <= 1e-6 * float(m.group(2))
    assert (tmp_path / "Warmup.000003.000001200.0060.00001.00000").exists()
    assert len(re.findall(r"# iterative refinement: step=", out.stdout)) == 1
    out = subprocess.run([exe, str(n), str(b), str(p), "--l1est"], capture_output=True, text=True, timeout=300,
                         cwd=tmp_path)
    assert out.returncode == 0, out.stderr
    m = re.search(r"resid = (\S+) hpl-harness = (\S+)$", out.stdout, re.M)
    assert m and 0 <= float(m.group(2)) < 16, out.stdout


def test_driver_ref_deck_reproduces_the_references_steps(hplai, torch_cuda, tmp_path):
    """driver.out ... -not -d -r --ref-deck: the reference's `-d` factors, so
    the refinement log has the reference's number of steps, its step-0
    residual to 1e-13 (the device GEMV's summation order) and its step-1
    residual to 1e-8 (tests/golden/ref_c1.json,
    the C1 command run by the reference's own driver)."""
    fix = json.load(open(os.path.join(HERE, "golden", "ref_c1.json")))["runs"]["netlib_not_d_r"]
    exe = os.path.abspath(os.path.join(HERE, "..", "hpl-ai_b200", "driver.out"))
    out = subprocess.run([exe, "1200", "60", "2", "-not", "-d", "-r", "--ref-deck"], capture_output=True, text=True,
                         timeout=300, cwd=tmp_path)
    assert out.returncode == 0, out.stderr
    assert "1gpu lazy full fp32/fp16 fp16-deck-ref" in out.stdout
    # the reference's settings lines for the same flags (main.cpp:214-232)
    assert "jobid=0\nn=1200 b=60 r=1 c=1\n2dbc lazy rdma full nopack nocheck noskiplu ddmat\n" in out.stdout
    assert "numasize=0 numamap=ROWDIST nbuf=2" in out.stdout
    steps = re.findall(r"# iterative refinement: step=\s*(\d+), residual=(\S+) hpl-harness=(\S+)", out.stdout)
    assert len(steps) == len(fix["steps"]), out.stdout
    assert abs(float(steps[0][1]) - fix["steps"][0]["residual"]) <= 1e-13 * fix["steps"][0]["residual"]
    assert abs(float(steps[1][1]) - fix["steps"][1]["residual"]) <= 1e-8 * fix["steps"][1]["residual"]
    m = re.search(r"resid = (\S+) hpl-harness = (\S+)$", out.stdout, re.M)
    assert m and 0 <= float(m.group(2)) < 16, out.stdout
