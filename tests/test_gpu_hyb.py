"""DCSR -> HYB conversion and the HYB SpMV against the oracle's HYB
restatement (oracle.hyb_from_csr / hyb_spmv): the ELL and COO arrays bit-exact
for every ELL width (0, below, at and above the longest row), the SpMV within
1e-6 (FP32) / 1e-13 (FP64) of sum |a||x|, and HYB -> DCSR (dcsr_from_hyb) of
the result restores the matrix."""
import numpy as np
import pytest
import torch

from dcsr_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import assert_content_equal, make_pair, spmv_bound

pytestmark = pytest.mark.gpu

TOL = {0: 1e-6, 1: 1e-13}


@pytest.mark.parametrize("dtype", [0, 1])
def test_to_hyb_and_spmv(dcsr, dtype):
    n, rp, cols, vals, rounds = W.small_plain(6, n=2500, n_rounds=2, T=5000)
    dev, orc = make_pair(dcsr, n, n, dtype, 0)
    dev.from_csr(rp, cols, vals)
    assert orc.load_csr(rp, cols, vals.astype(np.float64)) == 0
    for r, c, v in rounds:  # chained rows
        assert dev.update(r, c, v) == orc.update_auto(r, c, v.astype(np.float64)) == 0
    orp, oc, ov = orc.export_csr()
    maxlen = int(np.max(np.diff(orp)))
    x = np.random.default_rng(1).uniform(-1, 1, n)
    xt = torch.tensor(x, dtype=dev.dtype).cuda()
    bound = spmv_bound(orc, xt.cpu().double().numpy()) + 1e-300
    for width in (0, 5, 12, maxlen, maxlen + 3):
        pitch = n + 7
        ec, ev, cr, cc, cv = dev.to_hyb(width, pitch)
        oec, oev, ocr, occ, ocv = O.hyb_from_csr(orp, oc, ov, width, pitch)
        np.testing.assert_array_equal(ec.cpu().numpy()[:, :n], oec[:, :n])
        np.testing.assert_array_equal(ev.cpu().double().numpy()[:, :n], oev[:, :n])
        np.testing.assert_array_equal(cr.cpu().numpy(), ocr)
        np.testing.assert_array_equal(cc.cpu().numpy(), occ)
        np.testing.assert_array_equal(cv.cpu().double().numpy(), ocv)
        y0 = torch.tensor(np.random.default_rng(2).uniform(-1, 1, n), dtype=dev.dtype).cuda()
        y = dcsr.hyb_spmv(ec, ev, cr, cc, cv, xt, y0.clone(), alpha=2.0, beta=0.5)
        y_ref = 2.0 * O.hyb_spmv(oec, oev, ocr, occ, ocv, xt.cpu().double().numpy(), n) + 0.5 * y0.cpu().double().numpy()
        err = np.abs(y.cpu().double().numpy() - y_ref)
        assert np.all(err <= TOL[dtype] * (2 * bound + 0.5 * np.abs(y0.cpu().double().numpy()))), width
        # HYB -> DCSR gives the matrix back
        back, borc = make_pair(dcsr, n, n, dtype, 0)
        back.from_hyb(ec, ev, cr, cc, cv)
        assert borc.load_csr(orp, oc, ov) == 0
        assert_content_equal(back, borc, f"hyb width {width} round trip")


def _hyb_update_case(dcsr, dtype, width, rows, cols, vals, extra_cap, n=600, seed=3):
    """dcsr_hyb_update on a HYB export against oracle.hyb_update (the
    reference's UpdateMatrix(hyb) restated): ELL and COO arrays bit-exact,
    the status and the COO count equal; returns the status."""
    n_, rp, c, v, _ = W.small_plain(seed, n=n, n_rounds=0, T=0)
    vt = np.float32 if dtype == 0 else np.float64
    dev, orc = make_pair(dcsr, n_, n_, dtype, 0)
    dev.from_csr(rp, c, v)
    assert orc.load_csr(rp, c, v.astype(np.float64)) == 0
    orp, oc, ov = orc.export_csr()
    pitch = n_ + 5
    ec, ev, cr0, cc0, cv0 = dev.to_hyb(width, pitch)
    oec, oev, ocr, occ, ocv = O.hyb_from_csr(orp, oc, ov, width, pitch)
    m = cr0.numel()
    cap = m + extra_cap
    cr = torch.zeros(max(cap, 1), dtype=torch.int32, device="cuda")
    cc = torch.zeros_like(cr)
    cv = torch.zeros(max(cap, 1), dtype=ev.dtype, device="cuda")
    cr[:m], cc[:m], cv[:m] = cr0, cc0, cv0
    r_t = torch.tensor(np.asarray(rows, np.int32), device="cuda")
    c_t = torch.tensor(np.asarray(cols, np.int32), device="cuda")
    v_t = torch.tensor(np.asarray(vals, vt), device="cuda")
    st, m2 = dcsr.hyb_update(ec, ev, cr[:cap] if cap else cr[:0], cc[:cap] if cap else cc[:0],
                             cv[:cap] if cap else cv[:0], m, r_t, c_t, v_t, n_, n_)
    ost, e_c, e_v, o_r, o_c, o_v = O.hyb_update(oec, oev, ocr, occ, ocv, rows, cols,
                                                np.asarray(vals, vt).astype(np.float64), n_, n_, cap)
    assert st == ost, (st, ost)
    assert m2 == o_r.size
    np.testing.assert_array_equal(ec.cpu().numpy()[:, :n_], e_c[:, :n_])
    np.testing.assert_array_equal(ev.cpu().double().numpy()[:, :n_], e_v[:, :n_])
    np.testing.assert_array_equal(cr[:m2].cpu().numpy(), o_r)
    np.testing.assert_array_equal(cc[:m2].cpu().numpy(), o_c)
    np.testing.assert_array_equal(cv[:m2].cpu().double().numpy(), o_v)
    if st == 0:  # the updated HYB multiplies like the oracle's
        x = np.random.default_rng(4).uniform(-1, 1, n_)
        xt = torch.tensor(x, dtype=ev.dtype, device="cuda")
        y = dcsr.hyb_spmv(ec, ev, cr[:m2], cc[:m2], cv[:m2], xt, torch.zeros(n_, dtype=ev.dtype, device="cuda"))
        y_ref = O.hyb_spmv(e_c, e_v, o_r, o_c, o_v, xt.cpu().double().numpy(), n_)
        scale = O.hyb_spmv(np.where(e_c >= 0, e_c, 0), np.abs(e_v), o_r, o_c, np.abs(o_v),
                           np.abs(xt.cpu().double().numpy()), n_)
        assert np.all(np.abs(y.cpu().double().numpy() - y_ref) <= TOL[dtype] * scale + 1e-300)
    return st


@pytest.mark.parametrize("dtype", [0, 1])
@pytest.mark.parametrize("width", [0, 3, 8, 64])
def test_hyb_update(dcsr, dtype, width):
    """Unsorted triples with repeated rows and repeated (row, column) pairs,
    rows with free ELL slots, full ones and ones that fill up mid-batch."""
    rng = np.random.default_rng(11 + width)
    n = 600
    T = 3000
    rows = np.concatenate([rng.integers(0, n, T - 200), np.full(100, 7), np.full(100, n - 1)])
    cols = rng.integers(0, n, T)
    cols[-50:] = cols[-51]  # duplicates appended, not merged
    perm = rng.permutation(T)
    assert _hyb_update_case(dcsr, dtype, width, rows[perm], cols[perm], rng.standard_normal(T), T) == 0


@pytest.mark.parametrize("dtype", [0, 1])
def test_hyb_update_errors_leave_matrix_unchanged(dcsr, dtype):
    rng = np.random.default_rng(12)
    n = 600
    rows, cols = rng.integers(0, n, 500), rng.integers(0, n, 500)
    # a row or column out of range: BAD_INDEX
    r_bad = rows.copy()
    r_bad[17] = n
    assert _hyb_update_case(dcsr, dtype, 4, r_bad, cols, rng.standard_normal(500), 500) == dcsr.BAD_INDEX
    c_bad = cols.copy()
    c_bad[3] = -1
    assert _hyb_update_case(dcsr, dtype, 4, rows, c_bad, rng.standard_normal(500), 500) == dcsr.BAD_INDEX
    # more overflow than the COO capacity: POOL_EXHAUSTED
    assert _hyb_update_case(dcsr, dtype, 0, rows, cols, rng.standard_normal(500), 499) == dcsr.POOL_EXHAUSTED


def test_hyb_update_large(dcsr):
    """200k triples (the multi-tile sort and scan) into a width-4 HYB."""
    rng = np.random.default_rng(13)
    n = 5000
    T = 200_000
    assert _hyb_update_case(dcsr, 1, 4, rng.integers(0, n, T), rng.integers(0, n, T), rng.standard_normal(T), T,
                            n=n) == 0
