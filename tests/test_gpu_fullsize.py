"""Parity at the full sizes the measurements are quoted on.

* The power-law update stream: R-MAT 2^20 rows, (a,b,c,d) = (.57,.19,.19,.05),
  mean degree 16, FP32, 16 rounds of 1M triples with rows drawn by current
  row length (hot rows overflow their slack, chain segments and relocate;
  the repair policy compacts and grows the pool).  After rounds 1, 8 and 16:
  the layout (row_sizes, every segment pair, pool capacity) and the exported
  CSR bit-exact against the oracle; SpMV (k = 1 and k = 4) and row sums within
  1e-6 * sum_j |a_ij||x_j| of the FP64 oracle.
* SpGEMM on dynamic input: A 2^17 x 2^17 FP64, band half-width 2 plus 8
  random off-band columns per row; C = A*A; then 100k uniform update triples
  into A and C = A*A again.  C's layout and structure bit-exact, its values
  within 1e-12 relative of the oracle (they are compared bit for bit: both
  sum each entry's products in product order).
"""
import numpy as np
import pytest
import torch

from dcsr_b200 import workloads as W
from tests.helpers import assert_content_equal, assert_layout_equal, make_pair, oracle_opts, spmv_bound

pytestmark = pytest.mark.gpu


def _check_spmv(dev, orc, rng, k, tol):
    x = rng.uniform(-1, 1, (dev.n_cols, k))
    xt = torch.tensor(x if k > 1 else x[:, 0], dtype=dev.dtype).cuda()
    y = dev.spmv(xt).cpu().double().numpy()
    x64 = xt.cpu().double().numpy()
    y_ref = orc.spmv(x64.reshape(-1), k=k)
    bound = spmv_bound(orc, x64, k) + 1e-300
    err = np.abs(y.reshape(y_ref.shape) - y_ref)
    assert np.all(err <= tol * bound), f"spmv k={k}: max scaled err {np.max(err / bound):.3e}"


def _check_rowsum(dcsr, dev, orc, tol):
    y = dev.row_reduce(dcsr.REDUCE_SUM).cpu().double().numpy()
    y_ref = orc.row_reduce(dcsr.REDUCE_SUM)
    rp, c, v = orc.export_csr()
    b = np.zeros(orc.n_rows)
    np.add.at(b, np.repeat(np.arange(orc.n_rows), np.diff(rp)), np.abs(v))
    assert np.all(np.abs(y - y_ref) <= tol * b + 1e-300)


def test_rmat_stream_full_size(dcsr):
    n, rp, cols, vals, batches = W.rmat_stream(0, rounds=16)
    dev, orc = make_pair(dcsr, n, n, dcsr.F32, 0)
    dev.from_csr(rp, cols, vals)
    assert orc.load_csr(rp, cols, vals.astype(np.float64)) == 0
    rng = np.random.default_rng(7)
    for i, (r, c, v) in enumerate(batches, start=1):
        assert dev.update(r, c, v) == 0
        assert orc.update_auto(r, c, v.astype(np.float64)) == 0
        if i in (1, 8, 16):
            assert_layout_equal(dev, orc, f"round {i}")
            assert_content_equal(dev, orc, f"round {i}")
            _check_spmv(dev, orc, rng, 1, 1e-6)
            _check_rowsum(dcsr, dev, orc, 1e-6)
    _check_spmv(dev, orc, rng, 4, 1e-6)


def test_banded_spgemm_full_size(dcsr):
    n, rp, cols, vals, (ur, uc, uv) = W.banded_spgemm(0)
    dA, oA = make_pair(dcsr, n, n, dcsr.F64, 0)
    dA.from_csr(rp, cols, vals)
    assert oA.load_csr(rp, cols, vals) == 0
    for what in ("fresh A", "A after 100k updates"):
        dC = dA.spgemm(dA)
        oC = oA.spgemm(oA, oracle_opts(dC.opts))
        assert_layout_equal(dC, oC, f"C = A*A, {what}")
        assert_content_equal(dC, oC, f"C = A*A, {what}")  # bit-exact, within 1e-12 a fortiori
        _check_spmv(dA, oA, np.random.default_rng(3), 1, 1e-13)
        if what == "fresh A":
            assert dA.update(ur, uc, uv) == 0
            assert oA.update_auto(ur, uc, uv) == 0
            assert_content_equal(dA, oA, "A after updates")
