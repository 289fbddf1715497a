"""Failure handling of the bounded look-back waits, without a GPU fault.

The single-pass scan waits on earlier tiles with an iteration limit.  The
debug hook lowers the limit and keeps the first tile of every single-pass
kernel from publishing, so the waits on it run out.  Each wait must give up
(no hang) and the operation must report DCSR_TIMEOUT; the context must stay
usable: with the hook off, the same handles load and compact correctly
(checked against the oracle).

Only operations whose host side reads the status before anything consumes
the scan's output run while the hook is on: a CSR load (its capacity scan is
read back before the layout is written) and a compaction (likewise).  A
stalled sort or an update would hand wrong offsets to later kernels on the
device before the host sees the status, so they are not run stalled.
"""
import numpy as np
import pytest
import torch

from helpers import assert_content_equal, assert_layout_equal, make_pair

pytestmark = pytest.mark.gpu

N = M = 20_000  # more rows than one scan block: the capacity scans are single-pass


def _csr(seed):
    from dcsr_b200 import workloads as W
    rng = np.random.default_rng(seed)
    rp, cols = W.poisson_matrix(rng, N, M, 6.0)
    vals = rng.uniform(-1, 1, cols.size).astype(np.float32)
    return rp, cols, vals


def _dev(a):
    return torch.from_numpy(a).cuda()


def test_load_and_compact_report_timeout_then_recover(dcsr):
    rp, cols, vals = _csr(1)
    dev, orc = make_pair(dcsr, N, M, dcsr.F32, 0)
    before = dcsr.spin_faults()
    dcsr.debug_lookback(2048, True)
    try:
        with pytest.raises(dcsr.DcsrError) as e:
            dev.from_csr(_dev(rp), _dev(cols), _dev(vals))
        assert e.value.status == dcsr.TIMEOUT
    finally:
        dcsr.debug_lookback(0, False)
    assert dcsr.spin_faults() > before
    # hook off: the same handle loads correctly
    dev.from_csr(_dev(rp), _dev(cols), _dev(vals))
    assert orc.load_csr(rp, cols, vals.astype(np.float64)) == 0
    assert_layout_equal(dev, orc, "load after timeout")
    assert_content_equal(dev, orc, "load after timeout")

    dev.bin_rows()  # the schedule is built before the stall: compaction runs only its capacity scan
    before = dcsr.spin_faults()
    dcsr.debug_lookback(2048, True)
    try:
        with pytest.raises(dcsr.DcsrError) as e:
            dev.compact()
        assert e.value.status == dcsr.TIMEOUT
    finally:
        dcsr.debug_lookback(0, False)
    assert dcsr.spin_faults() > before
    assert dev.get_status() == dcsr.TIMEOUT  # the status word holds it until read
    assert dev.get_status() == dcsr.OK
    dev.compact()
    orc.compact()
    assert_layout_equal(dev, orc, "compaction after timeout")
    assert_content_equal(dev, orc, "compaction after timeout")
