"""The FP16-deck trailing update on CTA pairs (tcgen05 cta_group::2, 256 x 256
tiles over two SMs) against the single-CTA kernel (128 x 256 tiles).

Both issue the same MMAs over the same K order into FP32 accumulators and the
same epilogue arithmetic, so the decks must agree bit for bit: for the leaf
calls (ragged n, m just above one 128-row half; K >= 2048, where the pairs
are used) and for whole
factorisations under the serial, look-ahead and two-panel schedules, with the
matrix stored or regenerated (HPLAI_FLAG_LAZY_A).
"""
import numpy as np
import pytest

from test_gpu_precision import panel_values

pytestmark = pytest.mark.gpu
DECK = 4   # HPLAI_FLAG_FP16_DECK


def _deck_leaf(hplai, oracle, torch, m, n, k, fp8, pairs):
    rng = np.random.default_rng(m * 7 + n + k)
    ldd = (m + 7) // 8 * 8 + 8
    deck0 = rng.uniform(-100, 100, (n + 1, ldd)).astype(np.float16)
    dd = torch.from_numpy(deck0.copy()).cuda()
    hplai.set_cta_pairs_default(pairs)
    try:
        if fp8:
            l8, sl = oracle.quantize_e4m3(panel_values(rng, m, k), col_major=True)
            u8, su = oracle.quantize_e4m3(panel_values(rng, n, k), col_major=False)
            l8d, u8d = torch.from_numpy(l8).cuda(), torch.from_numpy(u8).cuda()
            sld, sud = torch.from_numpy(sl).cuda(), torch.from_numpy(su).cuda()
            hplai.check(hplai.f8gemm_deck_minus(m, n, k, l8d.data_ptr(), l8.shape[1], sld.data_ptr(), u8d.data_ptr(),
                                                u8.shape[1], sud.data_ptr(), dd.data_ptr(), ldd, 2.0 ** -8, None))
        else:
            ld = (k + 7) // 8 * 8
            l16 = rng.uniform(-0.5, 0.5, (m, ld)).astype(np.float16)
            u16 = rng.uniform(-0.5, 0.5, (n, ld)).astype(np.float16)
            ld_, ud = torch.from_numpy(l16).cuda(), torch.from_numpy(u16).cuda()
            hplai.check(hplai.shgemm_deck_minus(m, n, k, ld_.data_ptr(), ld, ud.data_ptr(), ld, dd.data_ptr(), ldd,
                                                64.0, None))
        torch.cuda.synchronize()
    finally:
        hplai.set_cta_pairs_default(False)
    got = dd.cpu().numpy()
    # outside the m x n region nothing changes
    assert np.array_equal(got[:, m:], deck0[:, m:]) and np.array_equal(got[n], deck0[n])
    return got


@pytest.mark.parametrize("fp8", [True, False])
@pytest.mark.parametrize("m,n,k", [(136, 131, 2048), (392, 300, 2048), (1000, 777, 4096), (4096, 2600, 2048)])
def test_pair_deck_leaf_bit_identical(hplai, oracle, torch_cuda, m, n, k, fp8):
    one = _deck_leaf(hplai, oracle, torch_cuda, m, n, k, fp8, False)
    two = _deck_leaf(hplai, oracle, torch_cuda, m, n, k, fp8, True)
    assert np.array_equal(one.view(np.uint16), two.view(np.uint16))


@pytest.mark.parametrize("n,b,extra", [(4096, 512, 0), (8192, 1024, 8 | 2), (6144, 512, 8), (4096, 1024, 8 | 2 | 64)])
def test_pair_factors_bit_identical(hplai, torch_cuda, n, b, extra):
    lus = []
    for pairs in (0, 1):
        with hplai.Solver(n, b, precision=hplai.F32_F8, flags=DECK | extra) as s:
            s.set_cta_pairs(pairs)
            s.generate(42)
            s.factor()
            lus.append(s.lu())
    assert np.array_equal(lus[0].view(np.uint32), lus[1].view(np.uint32))


def test_pair_solve_converges(hplai, torch_cuda):
    with hplai.Solver(8192, 1024, precision=hplai.F32_F8, flags=DECK | 8 | 2) as s:
        s.set_cta_pairs(1)
        s.generate(42)
        s.factor()
        res = s.iterative_refinement(50, mode=hplai.GMRES)
        assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0


def test_pair_switch_arguments(hplai):
    with hplai.Solver(1024, 128, precision=hplai.F32_F8, flags=DECK) as s:
        for v in (-1, 0, 1):
            s.set_cta_pairs(v)
        with pytest.raises(hplai.HplaiError):
            s.set_cta_pairs(-2)


def test_autotune_tries_cta_pairs(hplai, torch_cuda):
    """For the deck with four-panel groups (K = 4096) the tuner times the
    chosen schedule once more on CTA pairs and keeps the faster tile shape;
    the chosen configuration solves."""
    with hplai.Solver(8192, 1024, precision=hplai.F32_F8, flags=DECK | 128) as s:
        flags, side, ms = s.autotune(42)
        trials = s.autotune_trials()
        paired = [t for t in trials if t[0] & hplai.TRIAL_CTA_PAIRS]
        if flags & (8 | 128):   # a grouped schedule: K >= 2048
            assert len(paired) == 2 and all(t[0] & (8 | 128) for t in paired)
        else:
            assert not paired
        assert s.cta_pairs() in (-1, 1)
        s.factor()
        res = s.iterative_refinement(50, mode=hplai.GMRES)
        assert res.status == hplai.HPLAI_OK and res.hpl_harness < 16.0
