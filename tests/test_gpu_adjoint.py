"""The adjoint of the solve (a caller's right-hand side, the transposed
system, and the torch.autograd.Function) on the B200.

No reference counterpart: the checks are a dense FP64 solve of the same
matrix (numpy / torch linalg.solve with autograd), FP64 central differences
and the hpl-harness of the transposed system.  Tolerances: solutions and
the adjoint workload's gradients agree with the dense solve to 1e-12
relative (both are converged to a backward error near n*eps of a matrix
with cond_inf of a few units); the linear-loss gradients of the small
system to 1e-9.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_SMALL, B_SMALL = 2048, 256


@pytest.fixture(scope="module")
def small(hplai, oracle, torch_cuda):
    s = hplai.Solver(N_SMALL, B_SMALL)
    s.generate(42)
    s.factor()
    a = oracle.dense_matrix_f64(N_SMALL, 42)
    yield s, a
    s.close()


def rel(u, v):
    return float(np.max(np.abs(u - v)) / np.max(np.abs(v)))


def test_solve_rhs_matches_dense(hplai, small):
    s, a = small
    rng = np.random.default_rng(11)
    b = rng.uniform(-1.0, 1.0, N_SMALL)
    x, res = s.solve_rhs(b)
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0
    assert rel(x, np.linalg.solve(a, b)) < 1e-12


def test_solve_transpose_matches_dense(hplai, small):
    s, a = small
    rng = np.random.default_rng(12)
    g = rng.uniform(-1.0, 1.0, N_SMALL)
    lam, res = s.solve_transpose(g)
    assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0
    assert rel(lam, np.linalg.solve(a.T, g)) < 1e-12


def test_custom_solves_leave_context_solution(hplai, small):
    s, a = small
    res = s.iterative_refinement(50)
    x0 = s.x()
    s.solve_transpose(np.ones(N_SMALL))
    assert np.array_equal(s.x(), x0)
    assert res.status == hplai.HPLAI_OK


def test_autograd_matches_torch_fp64(hplai, small, torch_cuda):
    torch = torch_cuda
    import hplai_torch
    s, a = small
    rng = np.random.default_rng(13)
    bvec = rng.uniform(-1.0, 1.0, N_SMALL)
    xt = torch.from_numpy(rng.uniform(-1.0, 1.0, N_SMALL))
    # ours
    b1 = torch.tensor(bvec, requires_grad=True)
    x1 = hplai_torch.solve(b1, s)
    (xt * x1).sum().backward()
    # torch FP64 dense reference with autograd through linalg.solve
    at = torch.tensor(a, requires_grad=True)
    b2 = torch.tensor(bvec, requires_grad=True)
    x2 = torch.linalg.solve(at, b2)
    (xt * x2).sum().backward()
    assert rel(x1.detach().numpy(), x2.detach().numpy()) < 1e-12
    assert rel(b1.grad.numpy(), b2.grad.numpy()) < 1e-9
    # sampled matrix gradients dL/dA_ij = -lambda_i x_j
    rows = rng.integers(0, N_SMALL, 256)
    cols = rng.integers(0, N_SMALL, 256)
    ours = hplai_torch.matrix_grad_entries(b1.grad.numpy(), x1.detach().numpy(), rows, cols)
    ref = at.grad.numpy()[rows, cols]
    assert np.max(np.abs(ours - ref)) / np.max(np.abs(ref)) < 1e-9


def test_grad_b_central_differences(hplai, small):
    """L(b) = xt . A^{-1} b is linear in b, so central differences are exact
    up to rounding: dL/db_k = lambda_k."""
    s, _ = small
    rng = np.random.default_rng(14)
    b = rng.uniform(-1.0, 1.0, N_SMALL)
    xt = rng.uniform(-1.0, 1.0, N_SMALL)
    lam, _ = s.solve_transpose(xt)
    h = 1e-6
    for k in rng.integers(0, N_SMALL, 4):
        bp, bm = b.copy(), b.copy()
        bp[k] += h
        bm[k] -= h
        fd = (xt @ s.solve_rhs(bp)[0] - xt @ s.solve_rhs(bm)[0]) / (2 * h)
        assert abs(fd - lam[k]) <= 1e-6 * max(1.0, abs(lam[k]))


def test_adjoint_workload_n8192(hplai, oracle, torch_cuda):
    """C5 sizes (n = 8192, b = 256): the transposed system converges and its
    residual, checked on the host with the FP64 matrix, is at rounding level."""
    n, b = 8192, 256
    with hplai.Solver(n, b) as s:
        s.generate(42)
        s.factor()
        rng = np.random.default_rng(2024)
        g = rng.uniform(-1.0, 1.0, n)
        lam, res = s.solve_transpose(g)
        assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0, res
        a = oracle.dense_matrix_f64(n, 42)
        r = a.T @ lam - g
        norma = np.max(np.sum(np.abs(a), axis=1))
        harness = np.max(np.abs(r)) / (norma * np.max(np.abs(lam)) + np.max(np.abs(g))) / (n * 2.0 ** -53)
        assert harness < 16.0, harness


def test_c5_quadratic_loss_gradients(hplai, oracle, torch_cuda):
    """The adjoint workload: n = 8192, b = 256, L = 0.5 ||x - x_t||^2 with
    x_t ~ U[-1, 1).  x, grad_b = lambda = A^{-T}(x - x_t) and grad_A = -lambda x^T
    on 4096 sampled entries agree with torch's FP64 dense solve and its
    autograd to 1e-12 relative; central differences with step 1e-6 (in b, and
    in A through the Sherman-Morrison form of the perturbed solve, so that
    the difference is not lost to cancellation) agree with lambda_k and
    -lambda_i x_j to 1e-6."""
    torch = torch_cuda
    import hplai_torch
    n, bs = 8192, 256
    rng = np.random.default_rng(5)
    xt_np = rng.uniform(-1.0, 1.0, n)
    with hplai.Solver(n, bs) as s:
        s.generate(42)
        s.factor()
        bvec = s.rhs()
        b1 = torch.tensor(bvec, requires_grad=True)
        x1 = hplai_torch.solve(b1, s)
        xt = torch.from_numpy(xt_np)
        (0.5 * ((x1 - xt) ** 2).sum()).backward()
        x, lam = x1.detach().numpy(), b1.grad.numpy()
        rows = rng.integers(0, n, 4096)
        cols = rng.integers(0, n, 4096)
        ga = hplai_torch.matrix_grad_entries(lam, x, rows, cols)
        # central differences in b: L(b + h e_k) - L(b) = g . dx + 0.5 |dx|^2
        h = 1e-6
        g = x - xt_np
        for k in rng.integers(0, n, 3):
            def dl(sign):
                bp = bvec.copy()
                bp[k] += sign * h
                dx = s.solve_rhs(bp)[0] - x
                return g @ dx + 0.5 * dx @ dx
            fd = (dl(1.0) - dl(-1.0)) / (2 * h)
            assert abs(fd - lam[k]) <= 1e-6 * np.max(np.abs(lam)), (k, fd, lam[k])
        # central differences in A_ij: (A + t e_i e_j^T)^{-1} b = x - t x_j u / (1 + t u_j), u = A^{-1} e_i
        for q in range(3):
            i, j = int(rows[q]), int(cols[q])
            e = np.zeros(n)
            e[i] = 1.0
            u = s.solve_rhs(e)[0]

            def dla(t):
                dx = -t * x[j] * u / (1.0 + t * u[j])
                return g @ dx + 0.5 * dx @ dx
            fd = (dla(h) - dla(-h)) / (2 * h)
            assert abs(fd - ga[q]) <= 1e-6 * np.max(np.abs(ga)), (i, j, fd, ga[q])
    a = oracle.dense_matrix_f64(n, 42)
    at = torch.tensor(a, device="cuda", requires_grad=True)
    b2 = torch.tensor(bvec, device="cuda", requires_grad=True)
    x2 = torch.linalg.solve(at, b2)
    (0.5 * ((x2 - xt.cuda()) ** 2).sum()).backward()
    assert rel(x, x2.detach().cpu().numpy()) < 1e-12
    assert rel(lam, b2.grad.cpu().numpy()) < 1e-12
    ref = at.grad[torch.from_numpy(rows).cuda(), torch.from_numpy(cols).cuda()].cpu().numpy()
    assert np.max(np.abs(ga - ref)) / np.max(np.abs(ref)) < 1e-12
