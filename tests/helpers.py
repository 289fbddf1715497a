"""Shared helpers for the parity tests: build the same matrix on the device
(through the C ABI) and in the CPU oracle, and compare them."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def oracle_opts(api_opts) -> "O.OrOpts":
    """The oracle's options struct with the same policy as a device handle."""
    o = O.OrOpts()
    for name, _ in O.OrOpts._fields_:
        setattr(o, name, getattr(api_opts, name))
    return o


def make_pair(api, n_rows, n_cols, dtype_code, mode, **kw):
    import torch
    opts = api.default_opts(mode, **kw)
    dt = torch.float32 if dtype_code == api.F32 else torch.float64
    dev = api.DcsrMatrix(n_rows, n_cols, dt, opts=opts)
    orc = O.OracleDcsr(n_rows, n_cols, dtype_code, oracle_opts(opts))
    return dev, orc


def assert_layout_equal(dev, orc, what=""):
    lay = dev.layout()
    rs_o = orc.row_sizes()
    seg_o = orc.seg()
    assert lay.pool_cap == orc.pool_cap, f"{what}: pool_cap {lay.pool_cap} != {orc.pool_cap}"
    np.testing.assert_array_equal(lay.row_sizes, rs_o, err_msg=f"{what}: row_sizes")
    np.testing.assert_array_equal(lay.seg, seg_o, err_msg=f"{what}: segment table")


def assert_content_equal(dev, orc, what="", exact=True):
    rp, c, v = dev.to_csr()
    rp_o, c_o, v_o = orc.export_csr()
    np.testing.assert_array_equal(rp.cpu().numpy(), rp_o, err_msg=f"{what}: row_ptr")
    np.testing.assert_array_equal(c.cpu().numpy(), c_o, err_msg=f"{what}: col_idx")
    vv = v.cpu().numpy().astype(np.float64)
    if exact:
        np.testing.assert_array_equal(vv, v_o, err_msg=f"{what}: values")
    else:
        np.testing.assert_allclose(vv, v_o, rtol=1e-12, atol=0, err_msg=f"{what}: values")


def spmv_bound(orc, x, k=1):
    """Per-entry magnitude bound sum_j |a_ij| |x_j| used to scale SpMV errors."""
    rp, c, v = orc.export_csr()
    ax = np.abs(v)
    xx = np.abs(np.asarray(x, np.float64)).reshape(orc.n_cols, k)
    out = np.zeros((orc.n_rows, k))
    rows = np.repeat(np.arange(orc.n_rows), np.diff(rp))
    for j in range(k):
        np.add.at(out[:, j], rows, ax * xx[c, j])
    return out if k > 1 else out[:, 0]
