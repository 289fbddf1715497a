"""Matrices whose pools, schedules and scratch come from the reserved device
regions (dcsr_pool_reserve), worked on from two streams at once.

Each round updates matrix j on stream j (dcsr_update_sync), enqueues its
SpMV on the same stream and, every third round, compacts it (a new pool; the
old one goes back to the regions).  The other stream's calls run while that
work is still in flight, so they take blocks that this stream freed and
wait for them on the device.  Against the oracle: every SpMV within the
FP64 bound, and the final layouts and contents bit-exact.  No allocation
may leave the regions.
"""
import numpy as np
import pytest
import torch

from tests.helpers import assert_content_equal, assert_layout_equal, make_pair, spmv_bound

pytestmark = pytest.mark.gpu


def test_regions_shared_by_two_streams(dcsr):
    dcsr.pool_reserve(512 << 20)
    reserved, free, fb0 = dcsr.pool_usage()
    assert reserved >= 512 << 20 and free >= 512 << 20
    rng = np.random.default_rng(5)
    m = 40000
    ss = [torch.cuda.Stream(), torch.cuda.Stream()]
    mats = []
    for j in range(2):
        n = 3000 + 2000 * j
        lens = rng.integers(0, 300, n)
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        cols = np.concatenate([np.sort(rng.choice(m, L, replace=False)) for L in lens]).astype(np.int32)
        vals = rng.standard_normal(cols.size)
        dev, orc = make_pair(dcsr, n, m, 1, 0, max_segs=3)
        dev.from_csr(rp, cols, vals)
        orc.load_csr(rp, cols, vals)
        mats.append((dev, orc))
    x64 = rng.uniform(-1, 1, m)
    x = torch.tensor(x64, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    checks = []
    for it in range(6):
        for j, (dev, orc) in enumerate(mats):
            T = 20000 + 10000 * it
            r = rng.integers(0, dev.n_rows, T).astype(np.int32)
            c = rng.integers(0, m, T).astype(np.int32)
            v = rng.standard_normal(T)
            with torch.cuda.stream(ss[j]):
                assert dev.update(r, c, v, stream=ss[j]) == 0
                y = dev.spmv(x, stream=ss[j])
                if it % 3 == 2:
                    dev.compact(stream=ss[j])
            assert orc.update_auto(r, c, v) == 0
            checks.append((f"round {it} matrix {j}", y, orc.spmv(x64), spmv_bound(orc, x64)))
            if it % 3 == 2:
                orc.compact()
    torch.cuda.synchronize()
    for what, y, y_ref, bound in checks:
        err = np.abs(y.cpu().numpy() - y_ref)
        assert np.all(err <= 1e-13 * (bound + 1e-300)), f"{what}: spmv max scaled err {np.max(err / (bound + 1e-300)):.3e}"
    for j, (dev, orc) in enumerate(mats):
        assert_layout_equal(dev, orc, f"matrix {j}")
        assert_content_equal(dev, orc, f"matrix {j}")
    assert dcsr.pool_usage()[2] == fb0, "an allocation left the reserved regions"
