"""Parity of the CUDA DCSR path (through the C ABI) against the CPU oracle.

Structure (row_sizes, segment table, pool capacity, exported row_ptr and
col_idx) must be bit-exact; merged values are bit-exact too (same summation
order).  SpMV results are compared with the FP64 oracle with the tolerance
|y - y64| <= tol * sum_j |a_ij||x_j|, tol = 1e-6 (FP32) / 1e-13 (FP64), which
is tighter than the stated 1e-5 relative bound.
"""
import numpy as np
import pytest
import torch

from dcsr_b200 import workloads as W
from tests.helpers import assert_content_equal, assert_layout_equal, make_pair, spmv_bound

pytestmark = pytest.mark.gpu

TOL = {0: 1e-6, 1: 1e-13}


def check_spmv(dev, orc, rng, k=1, alpha=1.0, beta=0.0):
    dt = dev.dtype
    x = torch.tensor(rng.uniform(-1, 1, (dev.n_cols, k)), dtype=dt).cuda()
    y0 = torch.tensor(rng.uniform(-1, 1, (dev.n_rows, k)), dtype=dt).cuda()
    xs = x[:, 0].contiguous() if k == 1 else x
    y = (y0[:, 0].contiguous() if k == 1 else y0).clone()
    dev.spmv(xs, y, alpha=alpha, beta=beta)
    torch.cuda.synchronize()
    x64 = x.cpu().double().numpy()
    y_ref = orc.spmv(x64.reshape(-1), k=k, alpha=alpha, beta=beta,
                     y=y0.cpu().double().numpy().reshape(-1))
    bound = abs(alpha) * spmv_bound(orc, x64, k) + abs(beta) * np.abs(y0.cpu().double().numpy()).reshape(
        y_ref.shape) + 1e-300
    err = np.abs(y.cpu().double().numpy().reshape(y_ref.shape) - y_ref)
    assert np.all(err <= TOL[dev.dtype_code] * bound), f"spmv k={k}: max scaled err {np.max(err / bound):.3e}"


def check_reduce(dev, orc, api):
    for op in (api.REDUCE_SUM, api.REDUCE_MAX, api.REDUCE_MIN, api.REDUCE_COUNT):
        y = dev.row_reduce(op).cpu().double().numpy()
        y_ref = orc.row_reduce(op)
        if op == api.REDUCE_SUM:
            rp, c, v = orc.export_csr()
            b = np.zeros(orc.n_rows)
            np.add.at(b, np.repeat(np.arange(orc.n_rows), np.diff(rp)), np.abs(v))
            assert np.all(np.abs(y - y_ref) <= TOL[dev.dtype_code] * b + 1e-300)
        else:
            np.testing.assert_array_equal(y, y_ref)


@pytest.mark.parametrize("mode", [0, 1])
def test_small_plain_stream(dcsr, mode):
    """Small plain workload: CSR->DCSR with 2x slack, 4 update rounds of 8192
    triples, SpMV and DCSR->CSR after each round (MERGE and APPEND modes)."""
    n, rp, cols, vals, rounds = W.small_plain(0)
    dev, orc = make_pair(dcsr, n, n, dcsr.F32, mode)
    dev.from_csr(rp, cols, vals)
    assert orc.load_csr(rp, cols, vals.astype(np.float64)) == 0
    assert_layout_equal(dev, orc, "load")
    assert_content_equal(dev, orc, "load")
    rng = np.random.default_rng(5)
    for i, (r, c, v) in enumerate(rounds):
        st = dev.update(r, c, v)
        st_o = orc.update_auto(r, c, v.astype(np.float64))
        assert st == st_o == 0
        assert_layout_equal(dev, orc, f"round {i}")
        assert_content_equal(dev, orc, f"round {i}")
        check_spmv(dev, orc, rng)
    check_reduce(dev, orc, dcsr)
    assert orc.validate() == 0


@pytest.mark.parametrize("dtype", [0, 1])
@pytest.mark.parametrize("k", [1, 2, 3, 4, 8])
def test_spmv_multi_rhs(dcsr, dtype, k):
    n, rp, cols, vals, rounds = W.small_plain(1)
    dev, orc = make_pair(dcsr, n, n, dtype, 0)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    rng = np.random.default_rng(k)
    check_spmv(dev, orc, rng, k=k)
    check_spmv(dev, orc, rng, k=k, alpha=-0.5, beta=0.25)


def test_rows_in_every_bin(dcsr):
    """Rows whose lengths hit every bin boundary 0,1,2,3,4,7,8,15,16,31,32,
    511,512,2000 plus chained rows after updates."""
    rng = np.random.default_rng(3)
    lens = [0, 1, 2, 3, 4, 7, 8, 15, 16, 31, 32, 511, 512, 513, 2000, 0, 5, 4096, 4097, 9000, 65536, 65537,
            140000] + [3] * 40
    n, m = len(lens), 200000
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    cols = np.concatenate([np.sort(rng.choice(m, L, replace=False)) for L in lens]).astype(np.int32)
    vals = rng.uniform(-1, 1, cols.size).astype(np.float32)
    dev, orc = make_pair(dcsr, n, m, 0, 0)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    check_spmv(dev, orc, rng)
    for it in range(3):
        T = 3000
        r = rng.integers(0, n, T).astype(np.int32)
        c = rng.integers(0, m, T).astype(np.int32)
        v = rng.uniform(-1, 1, T).astype(np.float32)
        assert dev.update(r, c, v) == orc.update_auto(r, c, v.astype(np.float64)) == 0
        assert_layout_equal(dev, orc, f"it {it}")
        assert_content_equal(dev, orc, f"it {it}")
        check_spmv(dev, orc, rng)
        check_reduce(dev, orc, dcsr)


@pytest.mark.parametrize("reloc_min", [0, 8, 100000])
def test_relocation_and_chaining(dcsr, reloc_min):
    """Long rows take the out-of-place relocation path, short rows the
    in-place shift; both must give the oracle's layout bit for bit."""
    rng = np.random.default_rng(11)
    n, m = 64, 50000
    lens = rng.integers(0, 3000, n)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    cols = np.concatenate([np.sort(rng.choice(m, L, replace=False)) for L in lens]).astype(np.int32)
    vals = rng.standard_normal(cols.size)
    dev, orc = make_pair(dcsr, n, m, 1, 0, reloc_min=reloc_min, max_segs=3)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals)
    for it in range(4):
        T = 20000
        r = rng.integers(0, n, T).astype(np.int32)
        c = rng.integers(0, m, T).astype(np.int32)
        v = rng.standard_normal(T)
        assert dev.update(r, c, v) == orc.update_auto(r, c, v) == 0
        assert_layout_equal(dev, orc, f"it {it}")
        assert_content_equal(dev, orc, f"it {it}")
    check_spmv(dev, orc, rng)


def test_duplicates_only_batch(dcsr):
    """A batch of one (row, col) repeated: summed in batch order."""
    dev, orc = make_pair(dcsr, 8, 8, 0, 0)
    rp = np.array([0, 1, 1, 1, 1, 1, 1, 1, 1], np.int32)
    dev.from_csr(rp, np.array([3], np.int32), np.array([0.5], np.float32))
    orc.load_csr(rp, np.array([3], np.int32), np.array([0.5]))
    v = np.random.default_rng(0).uniform(-1, 1, 1000).astype(np.float32)
    for (rr, cc) in ((0, 3), (5, 5)):
        r = np.full(1000, rr, np.int32)
        c = np.full(1000, cc, np.int32)
        assert dev.update(r, c, v) == orc.update_auto(r, c, v.astype(np.float64)) == 0
    assert_layout_equal(dev, orc)
    assert_content_equal(dev, orc)


def test_bad_index_rejected(dcsr):
    n, rp, cols, vals, rounds = W.small_plain(2)
    dev, orc = make_pair(dcsr, n, n, 0, 0)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    r, c, v = rounds[0]
    c = c.copy()
    c[17] = n  # out of range
    assert dev.update(r, c, v) == dcsr.BAD_INDEX
    assert_layout_equal(dev, orc)
    assert_content_equal(dev, orc)


def test_pool_exhaustion_and_layer_overflow_repair(dcsr):
    """Tiny spare pool and 2 segment layers: the synchronous update compacts
    and grows exactly like the oracle's repair policy."""
    rng = np.random.default_rng(9)
    n, m = 300, 3000
    rp, cols = W.poisson_matrix(rng, n, m, 6.0)
    vals = rng.uniform(-1, 1, cols.size).astype(np.float32)
    dev, orc = make_pair(dcsr, n, m, 0, 0, max_segs=2, spare_x16=0, min_spare=16, factor_x16=16, min_cap=1,
                         align=1)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    assert_layout_equal(dev, orc, "load")
    for it in range(6):
        T = 2000
        r = rng.integers(0, n, T).astype(np.int32)
        c = rng.integers(0, m, T).astype(np.int32)
        v = rng.uniform(-1, 1, T).astype(np.float32)
        assert dev.update(r, c, v) == orc.update_auto(r, c, v.astype(np.float64)) == 0
        assert_layout_equal(dev, orc, f"it {it}")
        assert_content_equal(dev, orc, f"it {it}")


def test_async_update_rejection_is_atomic(dcsr):
    """dcsr_update (async) with a pool too small: POOL_EXHAUSTED, matrix unchanged."""
    rng = np.random.default_rng(4)
    n, m = 100, 1000
    rp, cols = W.poisson_matrix(rng, n, m, 5.0)
    vals = rng.uniform(-1, 1, cols.size).astype(np.float32)
    dev, orc = make_pair(dcsr, n, m, 0, 0, spare_x16=0, min_spare=8, factor_x16=16, min_cap=0, align=1)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    r = rng.integers(0, n, 5000).astype(np.int32)
    c = rng.integers(0, m, 5000).astype(np.int32)
    v = rng.uniform(-1, 1, 5000).astype(np.float32)
    assert dev.update(r, c, v, sync=False) == 0
    assert dev.get_status() == dcsr.POOL_EXHAUSTED
    st, need = orc.update(r, c, v.astype(np.float64))
    assert st == 1
    assert_layout_equal(dev, orc)
    assert_content_equal(dev, orc)


@pytest.mark.parametrize("mode", [0, 1])
def test_coo_load_and_compact(dcsr, mode):
    rng = np.random.default_rng(21)
    n, m, T = 1000, 800, 20000
    r = rng.integers(0, n, T).astype(np.int32)
    c = rng.integers(0, m, T).astype(np.int32)
    v = rng.uniform(-1, 1, T)
    dev, orc = make_pair(dcsr, n, m, 1, mode)
    dev.from_coo(r, c, v)
    assert orc.load_coo(r, c, v) == 0
    assert_layout_equal(dev, orc, "coo load")
    assert_content_equal(dev, orc, "coo load")
    for it in range(3):
        r2 = rng.integers(0, n, 5000).astype(np.int32)
        c2 = rng.integers(0, m, 5000).astype(np.int32)
        v2 = rng.uniform(-1, 1, 5000)
        assert dev.update(r2, c2, v2) == orc.update_auto(r2, c2, v2) == 0
    dev.compact()
    orc.compact()
    assert_layout_equal(dev, orc, "compact")
    assert_content_equal(dev, orc, "compact")
    rr, cc, vv = dev.to_coo()
    rp_o, c_o, v_o = orc.export_csr()
    np.testing.assert_array_equal(rr.cpu().numpy(), np.repeat(np.arange(n), np.diff(rp_o)))


def test_unsorted_csr_canonicalised(dcsr):
    rng = np.random.default_rng(8)
    n, m = 50, 40
    lens = rng.integers(0, 30, n)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    cols = rng.integers(0, m, rp[-1]).astype(np.int32)  # unsorted, with duplicates
    vals = rng.uniform(-1, 1, rp[-1]).astype(np.float32)
    dev, orc = make_pair(dcsr, n, m, 0, 0)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    assert_layout_equal(dev, orc)
    assert_content_equal(dev, orc)


def test_hyb_load(dcsr):
    rng = np.random.default_rng(12)
    n, m, width = 200, 300, 5
    ell_c = np.full((width, n), -1, np.int32)
    ell_v = np.zeros((width, n), np.float64)
    for r in range(n):
        k = rng.integers(0, width + 1)
        ell_c[:k, r] = np.sort(rng.choice(m, k, replace=False))
        ell_v[:k, r] = rng.standard_normal(k)
    T = 700
    cr = rng.integers(0, n, T).astype(np.int32)
    cc = rng.integers(0, m, T).astype(np.int32)
    cv = rng.standard_normal(T)
    dev, orc = make_pair(dcsr, n, m, 1, 0)
    dev.from_hyb(ell_c, ell_v, cr, cc, cv)
    rr = [(r, j) for r in range(n) for j in range(width) if ell_c[j, r] >= 0]
    er = np.array([r for r, _ in rr], np.int32)
    ec = np.array([ell_c[j, r] for r, j in rr], np.int32)
    ev = np.array([ell_v[j, r] for r, j in rr])
    orc.load_coo(np.concatenate([er, cr]), np.concatenate([ec, cc]), np.concatenate([ev, cv]))
    assert_layout_equal(dev, orc)
    assert_content_equal(dev, orc)


def test_empty_and_degenerate(dcsr):
    dev, orc = make_pair(dcsr, 10, 10, 0, 0)
    dev.from_csr(np.zeros(11, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    orc.load_csr(np.zeros(11, np.int32), np.zeros(0, np.int32), np.zeros(0))
    assert_layout_equal(dev, orc)
    assert dev.nnz() == 0
    y = dev.spmv(torch.ones(10, device="cuda"))
    assert torch.all(y == 0)
    assert dev.update(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32)) == 0
    r = np.array([9, 0, 9], np.int32)
    c = np.array([9, 0, 9], np.int32)
    v = np.array([1, 2, 3], np.float32)
    assert dev.update(r, c, v) == orc.update_auto(r, c, v.astype(np.float64)) == 0
    assert_layout_equal(dev, orc)
    assert_content_equal(dev, orc)


def test_count_sorted_and_reduce_by_key(dcsr, oracle_mod):
    rng = np.random.default_rng(2)
    I = np.sort(rng.integers(0, 500, 100000)).astype(np.int32)
    X0 = rng.integers(0, 5, 500).astype(np.int32)
    X = torch.tensor(X0).cuda()
    dcsr.count_sorted_indices(torch.tensor(I).cuda(), X)
    np.testing.assert_array_equal(X.cpu().numpy(), oracle_mod.count_sorted_indices(I, X0))
    vals = rng.standard_normal(I.size)
    k, v = dcsr.reduce_by_key(torch.tensor(I).cuda(), torch.tensor(vals).cuda())
    ko, vo = oracle_mod.reduce_by_key(I, vals, 1)
    np.testing.assert_array_equal(k.cpu().numpy(), ko)
    np.testing.assert_array_equal(v.cpu().numpy(), vo)


def test_launch_counter_moves(dcsr):
    n0 = dcsr.launch_count()
    dev = dcsr.DcsrMatrix(16, 16)
    dev.from_coo(np.arange(16, dtype=np.int32), np.arange(16, dtype=np.int32), np.ones(16, np.float32))
    dev.spmv(torch.ones(16, device="cuda"))
    torch.cuda.synchronize()
    assert dcsr.launch_count() > n0


def _spgemm_pair(dcsr, A_rp, A_c, A_v, B_rp, B_c, B_v, n, k, m, dtype):
    dA, oA = make_pair(dcsr, n, k, dtype, 0)
    dB, oB = make_pair(dcsr, k, m, dtype, 0)
    dA.from_csr(A_rp, A_c, A_v)
    oA.load_csr(A_rp, A_c, np.asarray(A_v, np.float64))
    dB.from_csr(B_rp, B_c, B_v)
    oB.load_csr(B_rp, B_c, np.asarray(B_v, np.float64))
    dC = dA.spgemm(dB)
    oC = oA.spgemm(oB, oracle_opts_of(dC))
    return dC, oC


def oracle_opts_of(dev):
    from tests.helpers import oracle_opts
    return oracle_opts(dev.opts)


@pytest.mark.parametrize("dtype", [0, 1])
def test_spgemm_banded(dcsr, dtype):
    """C = A*A on a small banded + random matrix: structure and values
    bit-exact with the oracle (products summed in product order)."""
    n, rp, cols, vals, _ = W.banded_spgemm(0, scale=11)
    v = vals.astype(np.float32) if dtype == 0 else vals
    dC, oC = _spgemm_pair(dcsr, rp, cols, v, rp, cols, v, n, n, n, dtype)
    assert_layout_equal(dC, oC, "C")
    assert_content_equal(dC, oC, "C")


def test_spgemm_all_size_classes(dcsr):
    """Rows with 0, <=256, <=4096 and >4096 products (warp, CTA and global
    paths) and rectangular shapes."""
    rng = np.random.default_rng(17)
    n, k, m = 40, 3000, 5000
    lensA = np.array([0, 1, 2, 5, 30, 100, 400, 1200] * 5)[:n]
    A_rp = np.concatenate([[0], np.cumsum(lensA)]).astype(np.int32)
    A_c = np.concatenate([np.sort(rng.choice(k, L, replace=False)) for L in lensA]).astype(np.int32)
    A_v = rng.standard_normal(A_c.size)
    lensB = rng.integers(0, 12, k)
    B_rp = np.concatenate([[0], np.cumsum(lensB)]).astype(np.int32)
    B_c = np.concatenate([np.sort(rng.choice(m, L, replace=False)) for L in lensB]).astype(np.int32)
    B_v = rng.standard_normal(B_c.size)
    dC, oC = _spgemm_pair(dcsr, A_rp, A_c, A_v, B_rp, B_c, B_v, n, k, m, 1)
    assert_layout_equal(dC, oC, "C")
    assert_content_equal(dC, oC, "C")


@pytest.mark.parametrize("dtype", [0, 1])
def test_spgemm_wide_columns(dcsr, dtype):
    """C's columns above 2^24 (the warp path's 64-bit sort keys) and at most
    2^24 (32-bit keys) give the same structure and values as the oracle;
    B's rows share columns so equal columns are summed."""
    rng = np.random.default_rng(23)
    n, k = 64, 64
    for m in ((1 << 24), (1 << 24) + 100):
        lensA = rng.integers(0, 12, n)
        A_rp = np.concatenate([[0], np.cumsum(lensA)]).astype(np.int32)
        A_c = np.concatenate([np.sort(rng.choice(k, L, replace=False)) for L in lensA]).astype(np.int32)
        A_v = rng.standard_normal(A_c.size)
        pool = np.concatenate([rng.choice(m, 40, replace=False), [m - 1, m - 2, 0]])  # shared columns
        lensB = rng.integers(0, 20, k)
        B_rp = np.concatenate([[0], np.cumsum(lensB)]).astype(np.int32)
        B_c = np.concatenate([np.sort(rng.choice(pool, L, replace=False)) for L in lensB]).astype(np.int32)
        B_v = rng.standard_normal(B_c.size)
        if dtype == 0:
            A_v, B_v = A_v.astype(np.float32), B_v.astype(np.float32)
        dC, oC = _spgemm_pair(dcsr, A_rp, A_c, A_v, B_rp, B_c, B_v, n, k, m, dtype)
        assert_layout_equal(dC, oC, f"C m={m}")
        assert_content_equal(dC, oC, f"C m={m}")


def test_spgemm_after_updates(dcsr):
    """SpGEMM reads chained (uncompacted) inputs correctly."""
    n, rp, cols, vals, upd = W.banded_spgemm(1, scale=10, n_updates=3000)
    dA, oA = make_pair(dcsr, n, n, 1, 0)
    dA.from_csr(rp, cols, vals)
    oA.load_csr(rp, cols, vals)
    assert dA.update(*upd) == oA.update_auto(*upd) == 0
    dC = dA.spgemm(dA)
    oC = oA.spgemm(oA, oracle_opts_of(dC))
    assert_layout_equal(dC, oC, "C")
    assert_content_equal(dC, oC, "C")


def test_pool_reserve(dcsr):
    """Pre-growing the device pool succeeds, rejects a negative size, and
    later matrices allocate from it as before (results unchanged)."""
    import ctypes as C
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert dcsr.lib().dcsr_pool_reserve(-1, s) == dcsr.BAD_ARG
    assert dcsr.lib().dcsr_pool_reserve(0, s) == 0
    dcsr.pool_reserve(256 << 20)
    dev = dcsr.DcsrMatrix(64, 64)
    dev.from_coo(np.arange(64, dtype=np.int32), np.arange(64, dtype=np.int32), np.full(64, 2.0, np.float32))
    y = dev.spmv(torch.ones(64, device="cuda"))
    assert torch.equal(y, torch.full((64,), 2.0, device="cuda"))


@pytest.mark.parametrize("n", [32768, 32769, 70000])
def test_spmv_k1_both_paths(dcsr, n):
    """k = 1 SpMV on both sides of the row threshold where a matrix moves from
    the row-group pass to the one-value stream (32768 rows), against the
    oracle, before and after an update."""
    rng = np.random.default_rng(n)
    lens = rng.poisson(9, n)
    m = 50000
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    cols = np.concatenate([np.sort(rng.choice(m, L, replace=False)) for L in lens]).astype(np.int32)
    vals = rng.uniform(-1, 1, cols.size).astype(np.float32)
    dev, orc = make_pair(dcsr, n, m, 0, 0)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    check_spmv(dev, orc, rng)
    check_spmv(dev, orc, rng, alpha=2.0, beta=-0.5)
    T = 20000
    r = rng.integers(0, n, T).astype(np.int32)
    c = rng.integers(0, m, T).astype(np.int32)
    v = rng.uniform(-1, 1, T).astype(np.float32)
    assert dev.update(r, c, v) == orc.update_auto(r, c, v.astype(np.float64)) == 0
    check_spmv(dev, orc, rng)


def test_full_chain_relocates_instead_of_overflowing(dcsr):
    """MERGE: a row that outgrows a chain already max_segs long is merged out
    of place into one fresh segment (no LAYER_OVERFLOW), exactly as the
    oracle restates; the asynchronous update is accepted."""
    rng = np.random.default_rng(31)
    n, m = 64, 5000
    rp, cols = W.poisson_matrix(rng, n, m, 4.0)
    vals = rng.uniform(-1, 1, cols.size).astype(np.float32)
    dev, orc = make_pair(dcsr, n, m, 0, 0, max_segs=2, factor_x16=16, min_cap=1, align=1, spare_x16=64)
    dev.from_csr(rp, cols, vals)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    for it in range(5):  # the same rows again and again: chains fill, then relocate
        r = np.repeat(np.arange(0, n, 4, dtype=np.int32), 6)
        c = rng.integers(0, m, r.size).astype(np.int32)
        v = rng.uniform(-1, 1, r.size).astype(np.float32)
        assert dev.update(r, c, v, sync=False) == 0
        assert dev.get_status() == dcsr.OK, f"round {it}"
        st, _ = orc.update(r, c, v.astype(np.float64))
        assert st == 0
        assert_layout_equal(dev, orc, f"round {it}")
        assert_content_equal(dev, orc, f"round {it}")
