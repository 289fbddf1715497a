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
