"""The single-pass scan and radix sort (decoupled look-back) at the sizes
where they take over from the one-block kernels (scans above 4096 values,
sorts above 8192 keys) and where sorts switch to three kernels per pass
(above 2^22 keys inside a stream capture, above 2^25 outside one), against
the oracle: COO loads (stable sort of (row,
column) keys, merge of duplicates), updates (a sort and four scans per
batch), reduce-by-key (a scan), in place and repeated on one handle so the
look-back epochs advance; and no look-back wait ever gave up."""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import assert_content_equal, assert_layout_equal, make_pair

pytestmark = pytest.mark.gpu


def spin_faults(dcsr):
    v = C.c_int64(-1)
    assert dcsr.lib().dcsr_spin_faults(C.byref(v)) == 0
    return v.value


@pytest.fixture(autouse=True)
def no_new_faults(dcsr):
    """No look-back wait gives up during the test (the counter is process-wide)."""
    before = spin_faults(dcsr)
    yield
    assert spin_faults(dcsr) == before


@pytest.mark.parametrize("T", [8193, 2048 * 37 + 5, 262_145, 1_500_000, 4_194_304, 4_194_305])
@pytest.mark.parametrize("mode", [0, 1])
def test_coo_load_sizes(dcsr, T, mode):
    rng = np.random.default_rng(T + mode)
    n, m = 50_000, 40_000
    r = rng.integers(0, n, T).astype(np.int32)
    c = rng.integers(0, m, T).astype(np.int32)
    v = rng.uniform(-1, 1, T)
    dev, orc = make_pair(dcsr, n, m, 1, mode)
    dev.from_coo(r, c, v)
    assert orc.load_coo(r, c, v) == 0
    assert_layout_equal(dev, orc, f"coo load T={T}")
    assert_content_equal(dev, orc, f"coo load T={T}")


def test_coo_load_three_kernel_sort(dcsr):
    """A COO load of 2^25 + 1 triples: its sort takes three kernels per pass
    (the single-pass tier stops at 2^25 keys outside a capture)."""
    T = (1 << 25) + 1
    rng = np.random.default_rng(25)
    n, m = 50_000, 40_000
    r = rng.integers(0, n, T).astype(np.int32)
    c = rng.integers(0, m, T).astype(np.int32)
    v = rng.uniform(-1, 1, T)
    dev, orc = make_pair(dcsr, n, m, 1, 0)
    dev.from_coo(r, c, v)
    assert orc.load_coo(r, c, v) == 0
    assert_layout_equal(dev, orc, "coo load T=2^25+1")
    assert_content_equal(dev, orc, "coo load T=2^25+1")


def test_update_sizes_repeated(dcsr):
    """Updates of changing size on one handle: every sort and scan reuses the
    handle's look-back area with a newer epoch."""
    rng = np.random.default_rng(5)
    n, m = 30_000, 30_000
    dev, orc = make_pair(dcsr, n, m, 1, 0)
    r = rng.integers(0, n, 200_000).astype(np.int32)
    c = rng.integers(0, m, 200_000).astype(np.int32)
    v = rng.uniform(-1, 1, 200_000)
    dev.from_coo(r, c, v)
    assert orc.load_coo(r, c, v) == 0
    for T in (9000, 5000, 100_000, 8193, 700_000, 4097, 250_000):
        r2 = rng.integers(0, n, T).astype(np.int32)
        c2 = rng.integers(0, m, T).astype(np.int32)
        v2 = rng.uniform(-1, 1, T)
        assert dev.update(r2, c2, v2) == orc.update_auto(r2, c2, v2) == 0
        assert_layout_equal(dev, orc, f"update T={T}")
        assert_content_equal(dev, orc, f"update T={T}")


@pytest.mark.parametrize("n", [4097, 2048 * 5 + 1, 2048 * 64, (1 << 20) + 77, 3_000_000])
def test_reduce_by_key_sizes(dcsr, n):
    rng = np.random.default_rng(n)
    keys = np.sort(rng.integers(0, max(n // 3, 1), n)).astype(np.int32)
    vals = rng.integers(-1000, 1000, n).astype(np.float64)  # integer-valued: every order of summation is exact
    ko, vo = dcsr.reduce_by_key(torch.tensor(keys, device="cuda"), torch.tensor(vals, device="cuda"))
    uk, start = np.unique(keys, return_index=True)
    np.testing.assert_array_equal(ko.cpu().numpy(), uk)
    np.testing.assert_array_equal(vo.cpu().numpy(), np.add.reduceat(vals, start))


@pytest.mark.parametrize("runs", ["one_key", "long_runs", "ragged"])
def test_reduce_by_key_long_runs(dcsr, runs):
    """Runs longer than a summation piece (256 keys), up to one run of 2^20
    keys: pieces are summed in parallel and combined in order."""
    rng = np.random.default_rng(11)
    if runs == "one_key":
        keys = np.full(1 << 20, 7, np.int32)
    elif runs == "long_runs":
        keys = np.repeat(np.arange(40, dtype=np.int32), rng.integers(200, 60_000, 40))
    else:
        keys = np.sort(np.concatenate([rng.integers(0, 50, 300_000), rng.integers(0, 200_000, 5_000)])).astype(np.int32)
    n = keys.size
    for dt in (torch.float32, torch.float64):
        vals = rng.integers(-100, 100, n).astype(np.float64)  # integer-valued: every order of summation is exact
        ko, vo = dcsr.reduce_by_key(torch.tensor(keys, device="cuda"), torch.tensor(vals, dtype=dt, device="cuda"))
        uk, start = np.unique(keys, return_index=True)
        np.testing.assert_array_equal(ko.cpu().numpy(), uk)
        np.testing.assert_array_equal(vo.cpu().double().numpy(), np.add.reduceat(vals, start))
