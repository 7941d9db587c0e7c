"""Leaf kernels through the C ABI against the CPU oracle (B200).

The generator, the diagonal LU and both panel TRSMs are integer work or
apply every update in the oracle's order with the same FMA, so they must
match bit for bit.  The tensor-core Schur GEMM and the FP64 refinement
kernels sum in a different order and are checked against tolerances stated
per test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr)).cuda()


def colmajor_to_dev(torch, a):
    """Column-major numpy (F order) -> device buffer with the same layout (ld = rows)."""
    return torch.from_numpy(np.asfortranarray(a).T.copy()).cuda()   # rows of .T = columns of a


def dev_to_colmajor(t, rows, cols):
    return np.asfortranarray(t.cpu().numpy().reshape(cols, rows).T)


def test_fill_matrix_bit_exact(hplai, oracle, torch_cuda):
    torch = torch_cuda
    n = 1200
    a = torch.empty(n * n, dtype=torch.float32, device="cuda")
    hplai.check(hplai.fill_panel(n, 0, 0, n, n, a.data_ptr(), n, 42, 1, None))
    torch.cuda.synchronize()
    got = dev_to_colmajor(a, n, n)
    ref = oracle.matrix(n)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("n,i0,j0,nr,nc", [(65536, 65000, 12345, 300, 70), (131072, 0, 131000, 64, 72),
                                           (4096, 1024, 1024, 512, 512)])
def test_fill_panel_far_blocks_bit_exact(hplai, oracle, torch_cuda, n, i0, j0, nr, nc):
    torch = torch_cuda
    a = torch.empty(nr * nc, dtype=torch.float32, device="cuda")
    hplai.check(hplai.fill_panel(n, i0, j0, nr, nc, a.data_ptr(), nr, 42, 1, None))
    torch.cuda.synchronize()
    got = dev_to_colmajor(a, nr, nc)
    ref = oracle.fill_panel(n, i0, j0, nr, nc)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_rhs_and_diag_bit_exact(hplai, oracle, torch_cuda):
    torch = torch_cuda
    n = 3000
    r = torch.empty(n, dtype=torch.float64, device="cuda")
    d = torch.empty(n, dtype=torch.float64, device="cuda")
    hplai.check(hplai.gen_rhs(n, 42, r.data_ptr(), None))
    hplai.check(hplai.gen_diag(n, 42, 0, n, d.data_ptr(), None))
    torch.cuda.synchronize()
    assert np.array_equal(r.cpu().numpy(), oracle.rhs(n))
    assert np.array_equal(d.cpu().numpy(), oracle.diag(n))


def test_diag_large_n_sampled(hplai, oracle, torch_cuda):
    torch = torch_cuda
    n = 65536
    rows = [0, 1, 777, 40000, 65535]
    d = torch.empty(1, dtype=torch.float64, device="cuda")
    for i in rows:
        hplai.check(hplai.gen_diag(n, 42, i, 1, d.data_ptr(), None))
        torch.cuda.synchronize()
        assert d.item() == oracle.calc_diag(i, n, 42)


def dd_matrix(rng, n):
    m = rng.uniform(-0.5, 0.5, (n, n)).astype(np.float32)
    m[np.arange(n), np.arange(n)] = np.abs(m).sum(1)
    return np.asfortranarray(m)


@pytest.mark.parametrize("b", [16, 60, 64, 100, 256, 512, 640, 1000, 1024])
def test_getrf_bit_exact(hplai, oracle, torch_cuda, b):
    torch = torch_cuda
    m = dd_matrix(np.random.default_rng(b), b)
    lda = b + 3
    buf = np.zeros((lda, b), dtype=np.float32, order="F")
    buf[:b, :] = m
    t = colmajor_to_dev(torch, buf)
    hplai.check(hplai.getrf_nopiv(b, t.data_ptr(), lda, None))
    torch.cuda.synchronize()
    got = dev_to_colmajor(t, lda, b)[:b, :]
    ref = oracle.getrf_nopiv(m)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_getrf_on_generated_block(hplai, oracle, torch_cuda):
    torch = torch_cuda
    n, b = 4096, 512
    blk = oracle.fill_panel(n, 1024, 1024, b, b)
    t = colmajor_to_dev(torch, blk)
    hplai.check(hplai.getrf_nopiv(b, t.data_ptr(), b, None))
    torch.cuda.synchronize()
    assert np.array_equal(dev_to_colmajor(t, b, b).view(np.uint32), oracle.getrf_nopiv(blk).view(np.uint32))


@pytest.mark.parametrize("m,b", [(1140, 60), (1000, 100), (4000, 512), (333, 1024), (64, 16)])
def test_trsm_right_upper_bit_exact(hplai, oracle, torch_cuda, m, b):
    torch = torch_cuda
    rng = np.random.default_rng(m + b)
    lu = oracle.getrf_nopiv(dd_matrix(rng, b))
    x = np.asfortranarray(rng.uniform(-0.5, 0.5, (m, b)).astype(np.float32))
    u_d = colmajor_to_dev(torch, lu)
    a_d = colmajor_to_dev(torch, x)
    ldh = (b + 63) // 64 * 64
    lh = torch.zeros(m * ldh, dtype=torch.float16, device="cuda")
    hplai.check(hplai.trsm_right_upper(m, b, u_d.data_ptr(), b, a_d.data_ptr(), m, lh.data_ptr(), ldh, 1.0, None))
    torch.cuda.synchronize()
    got = dev_to_colmajor(a_d, m, b)
    ref = oracle.trsm_right_upper(np.triu(lu), x)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    lh_h = lh.cpu().numpy().reshape(m, ldh)[:, :b]
    assert np.array_equal(lh_h.view(np.uint16), ref.astype(np.float16).view(np.uint16))


@pytest.mark.parametrize("b,nc", [(60, 1140), (100, 1000), (512, 4000), (1024, 333), (16, 50)])
def test_trsm_left_lower_bit_exact(hplai, oracle, torch_cuda, b, nc):
    torch = torch_cuda
    rng = np.random.default_rng(3 * b + nc)
    lu = oracle.getrf_nopiv(dd_matrix(rng, b))
    y = np.asfortranarray(rng.uniform(-0.5, 0.5, (b, nc)).astype(np.float32))
    l_d = colmajor_to_dev(torch, lu)
    a_d = colmajor_to_dev(torch, y)
    ldh = (b + 63) // 64 * 64
    uh = torch.zeros(nc * ldh, dtype=torch.float16, device="cuda")
    hplai.check(hplai.trsm_left_lower(b, nc, l_d.data_ptr(), b, a_d.data_ptr(), b, uh.data_ptr(), ldh, 1.0, None))
    torch.cuda.synchronize()
    got = dev_to_colmajor(a_d, b, nc)
    lunit = np.tril(lu, -1) + np.eye(b, dtype=np.float32)
    ref = oracle.trsm_left_lower_unit(lunit, y)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    uh_h = uh.cpu().numpy().reshape(nc, ldh)[:, :b]          # row j = column j of U
    assert np.array_equal(uh_h.view(np.uint16), ref.T.astype(np.float16).view(np.uint16))


@pytest.mark.parametrize("m,n,k", [(1140, 1140, 60), (1000, 777, 100), (128, 256, 64), (4096, 4096, 512),
                                   (300, 5000, 1024), (2500, 129, 16), (1001, 777, 60), (333, 1200, 200)])
def test_shgemm_minus_vs_torch_fp32(hplai, oracle, torch_cuda, m, n, k):
    """C - L*U on tcgen05 vs a PyTorch FP32 reference of the same op on the
    same FP16 inputs (m % 4 != 0 exercises the plain epilogue, the others the
    TMA reduce-add epilogue).  Tolerance per element: 2^-19 * sum_k |l||u| + 2^-22 |C|.
    Both sides accumulate in FP32 but in different orders, and the tensor
    core's FP32 accumulation is not a sequence of IEEE round-to-nearest adds;
    measured on B200 the worst element sits near 2^-20.7 * sum|l||u|."""
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n + k)
    ldh = (k + 63) // 64 * 64
    l16 = (torch.rand(m, ldh, device="cuda", generator=g) - 0.5).half()
    u16 = (torch.rand(n, ldh, device="cuda", generator=g) - 0.5).half()
    c = torch.rand(n, m, device="cuda", generator=g) * 8 - 4      # column-major m x n: row j = column j
    c0 = c.clone()
    hplai.check(hplai.shgemm_minus(m, n, k, l16.data_ptr(), ldh, u16.data_ptr(), ldh, c.data_ptr(), m, None))
    torch.cuda.synchronize()
    lf, uf = l16[:, :k].float(), u16[:, :k].float()
    ref = c0 - (uf @ lf.T)                                       # (n x m) = (L U)^T
    bound = (uf.abs() @ lf.abs().T) * 2.0 ** -19 + c0.abs() * 2.0 ** -22 + 1e-30
    err = (c - ref).abs()
    assert bool((err <= bound).all()), float((err / bound).max())


@pytest.mark.parametrize("m,n,k", [(60, 300, 60), (200, 60, 60), (1000, 500, 512), (4, 4, 16)])
def test_shgemm_subregion_leaves_rest(hplai, torch_cuda, m, n, k):
    """C is an interior m x n block of a larger matrix: the update must touch
    exactly that block, even where a tensor-core tile reaches past its edge
    into the rest of the matrix (the trailing update is applied region by
    region)."""
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    ldh = (k + 63) // 64 * 64
    l16 = (torch.rand(m, ldh, device="cuda", generator=g) - 0.5).half()
    u16 = (torch.rand(n, ldh, device="cuda", generator=g) - 0.5).half()
    big_rows, big_cols = m + 300, n + 300
    big = torch.rand(big_cols, big_rows, device="cuda", generator=g)   # column-major, ld = big_rows
    big0 = big.clone()
    r0, c0 = 36, 20                                                     # interior offset, 16-byte aligned rows
    cptr = big.data_ptr() + 4 * (r0 + c0 * big_rows)
    hplai.check(hplai.shgemm_minus(m, n, k, l16.data_ptr(), ldh, u16.data_ptr(), ldh, cptr, big_rows, None))
    torch.cuda.synchronize()
    ref = big0.clone()
    lf, uf = l16[:, :k].float(), u16[:, :k].float()
    ref[c0:c0 + n, r0:r0 + m] -= uf @ lf.T
    mask = torch.ones_like(big, dtype=torch.bool)
    mask[c0:c0 + n, r0:r0 + m] = False
    assert torch.equal(big[mask], big0[mask])
    bound = (uf.abs() @ lf.abs().T) * 2.0 ** -19 + big0[c0:c0 + n, r0:r0 + m].abs() * 2.0 ** -22
    assert bool(((big[c0:c0 + n, r0:r0 + m] - ref[c0:c0 + n, r0:r0 + m]).abs() <= bound).all())


def test_shgemm_matches_oracle_at_c1_step(hplai, oracle, torch_cuda):
    """First C1 trailing update against the oracle's own Schur kernel."""
    torch = torch_cuda
    n, b = 1200, 60
    a = oracle.matrix(n)
    f = a.copy(order="F")
    f[:b, :b] = oracle.getrf_nopiv(a[:b, :b])
    f[b:, :b] = oracle.trsm_right_upper(np.triu(f[:b, :b]), f[b:, :b])
    lunit = np.tril(f[:b, :b], -1) + np.eye(b, dtype=np.float32)
    f[:b, b:] = oracle.trsm_left_lower_unit(lunit, f[:b, b:])
    l16 = f[b:, :b].astype(np.float16)
    u16 = f[:b, b:].astype(np.float16)
    ref = oracle.shgemm_minus(f[b:, b:], l16, u16)
    rem = n - b
    lh = torch.from_numpy(np.ascontiguousarray(np.pad(l16, ((0, 0), (0, 4))))).cuda()      # rem x 64
    uh = torch.from_numpy(np.ascontiguousarray(np.pad(u16.T, ((0, 0), (0, 4))))).cuda()    # rem x 64
    c = colmajor_to_dev(torch, f[b:, b:])
    hplai.check(hplai.shgemm_minus(rem, rem, b, lh.data_ptr(), 64, uh.data_ptr(), 64, c.data_ptr(), rem, None))
    torch.cuda.synchronize()
    got = dev_to_colmajor(c, rem, rem)
    scale = np.abs(l16.astype(np.float32)) @ np.abs(u16.astype(np.float32))
    assert np.all(np.abs(got - ref) <= scale * 2.0 ** -21 + np.abs(ref) * 2.0 ** -23)


@pytest.mark.parametrize("n", [1200, 4096, 5000])
def test_otf_gemv_vs_oracle(hplai, oracle, torch_cuda, n):
    """FP64 on-the-fly GEMV: relative to the row 1-norm of A times |x|, the
    GPU and the oracle agree to 1e-14 (both are FP64 sums of n terms)."""
    torch = torch_cuda
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, n)
    y0 = rng.uniform(-1, 1, n)
    d = oracle.diag(n)
    xd, yd, dd = dev(torch, x), dev(torch, y0), dev(torch, d)
    ws = hplai.otf_gemv_workspace(n)
    w = torch.empty(ws // 8 + 1, dtype=torch.float64, device="cuda")
    hplai.check(hplai.otf_gemv(n, -1.0, xd.data_ptr(), 1.0, yd.data_ptr(), 42, dd.data_ptr(), w.data_ptr(), ws, None))
    torch.cuda.synchronize()
    ref = oracle.otf_gemv(n, 60 if n % 60 == 0 else n, -1.0, x, y0, 42, d)
    scale = 2 * d.max() * np.abs(x).max()
    assert np.abs(yd.cpu().numpy() - ref).max() <= 1e-14 * scale


def test_otf_gemv_block(hplai, oracle, torch_cuda):
    """otf_gemv_kernel's contract: an off-diagonal sub-block from its (0,0) state."""
    torch = torch_cuda
    n, i0, j0, mb, nb = 4096, 2048, 512, 700, 900
    x = np.random.default_rng(5).uniform(-1, 1, nb)
    a = oracle.dense_matrix_f64(n)[i0:i0 + mb, j0:j0 + nb]
    s00 = oracle.state_at(n, i0, j0, 42)
    xd = dev(torch, x)
    yd = torch.zeros(mb, dtype=torch.float64, device="cuda")
    ws = hplai.otf_gemv_workspace(max(mb, nb))
    w = torch.empty(ws // 8 + 1, dtype=torch.float64, device="cuda")
    hplai.check(hplai.otf_gemv_block(n, mb, nb, 2.0, xd.data_ptr(), yd.data_ptr(), s00, w.data_ptr(), ws, None))
    torch.cuda.synchronize()
    ref = 2.0 * a @ x
    assert np.abs(yd.cpu().numpy() - ref).max() <= 1e-13 * np.abs(a).sum(1).max()


@pytest.mark.parametrize("n", [300, 1200, 4096])
def test_trsv_vs_oracle(hplai, oracle, torch_cuda, n):
    torch = torch_cuda
    rng = np.random.default_rng(n + 1)
    m = dd_matrix(rng, n)
    x = rng.uniform(-1, 1, n)
    md = colmajor_to_dev(torch, m)
    xd = dev(torch, x)
    ws = hplai.trsv_workspace(n)
    w = torch.zeros(ws // 4 + 1, dtype=torch.int32, device="cuda")
    hplai.check(hplai.trsv_lower(n, md.data_ptr(), n, xd.data_ptr(), w.data_ptr(), ws, None))
    torch.cuda.synchronize()
    y = xd.cpu().numpy()
    ref = oracle.trsv_lower(m, x, 60 if n % 60 == 0 else n)
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()
    hplai.check(hplai.trsv_upper(n, md.data_ptr(), n, xd.data_ptr(), w.data_ptr(), ws, None))
    torch.cuda.synchronize()
    z = xd.cpu().numpy()
    ref2 = oracle.trsv_upper(m, ref, 60 if n % 60 == 0 else n)
    assert np.abs(z - ref2).max() <= 1e-13 * np.abs(ref2).max()


def test_infnorm(hplai, torch_cuda):
    torch = torch_cuda
    v = torch.randn(100003, dtype=torch.float64, device="cuda")
    v[77777] = -123.5
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    hplai.check(hplai.infnorm(v.numel(), v.data_ptr(), out.data_ptr(), None))
    torch.cuda.synchronize()
    assert out.item() == 123.5
    v[5] = float("nan")
    hplai.check(hplai.infnorm(v.numel(), v.data_ptr(), out.data_ptr(), None))
    torch.cuda.synchronize()
    assert np.isnan(out.item())


@pytest.mark.parametrize("n,lda,off", [(4096, 4096, 0), (1030, 1032, 0), (1001, 1003, 0), (130, 132, 1), (5, 8, 0)])
def test_panel_check_leaf(hplai, torch_cuda, n, lda, off):
    """hplai_panel_check (panel_check.hpp:9-65) vs FP64 sums of |a_ij| over the
    diagonal and the strict triangles, 1e-13 relative (summation order only):
    float4 path with and without a row tail, lda not a multiple of 4, and a
    pointer off the 16-byte boundary (scalar path)."""
    torch = torch_cuda
    g = torch.Generator(device="cpu").manual_seed(n)
    buf = torch.rand(lda * n + off, generator=g, dtype=torch.float32) - 0.5
    dev = buf.cuda()
    ws = hplai.panel_check_workspace(n)
    work = torch.empty(ws // 8 + 1, dtype=torch.float64, device="cuda")
    sig = torch.empty(3, dtype=torch.float64, device="cuda")
    hplai.check(hplai.panel_check(n, dev.data_ptr() + 4 * off, lda, sig.data_ptr(), work.data_ptr(), ws, None),
                "hplai_panel_check")
    got = sig.cpu().numpy()
    # column-major: element (i, j) sits at j * lda + i
    a = np.abs(buf[off:].numpy().reshape(n, lda)[:, :n].astype(np.float64)).T
    want = np.array([np.trace(a), np.triu(a, 1).sum(), np.tril(a, -1).sum()])
    assert np.all(np.abs(got - want) <= 1e-13 * want)
    hplai.check(hplai.panel_check(0, None, 0, sig.data_ptr(), None, 0, None), "hplai_panel_check")
    assert np.array_equal(sig.cpu().numpy(), np.zeros(3))
