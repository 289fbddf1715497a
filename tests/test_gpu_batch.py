"""The batched form (dcsr_batch_*) against the per-call path.

Every matrix gets the same update batch and SpMV through a batch and, on an
identical copy, through dcsr_update + dcsr_spmv.  Structure, values and the
SpMV output must agree bit for bit (the batched kernels are the per-call
kernels over descriptor arrays, so nothing may differ), for a direct run, for
CUDA-graph replays with new triples written in place, after a rejected update
repaired by dcsr_batch_repair, and in APPEND mode.  One SpMV result per batch
is also checked against the FP64 oracle.
"""
import numpy as np
import pytest
import torch

from tests.helpers import make_pair, spmv_bound

pytestmark = pytest.mark.gpu


def random_csr(rng, n, m, mean, long_rows=()):
    """Poisson row lengths (some rows forced long), distinct sorted columns."""
    lens = rng.poisson(mean, n).astype(np.int64)
    for r, L in long_rows:
        lens[r] = L
    lens = np.minimum(lens, m)
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    keys = np.unique(rows * m + rng.integers(0, m, rows.size))
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum(np.bincount(keys // m, minlength=n))
    cols = (keys % m).astype(np.int32)
    vals = rng.uniform(-1, 1, cols.size)
    return rp.astype(np.int32), cols, vals


def triples(rng, n, m, T):
    r = rng.integers(0, n, T).astype(np.int32)
    c = rng.integers(0, m, T).astype(np.int32)
    v = rng.uniform(-1, 1, T)
    return r, c, v


SHAPES = [  # (rows, cols, mean degree, long rows, update size, k)
    (1000, 1000, 4, (), 100, 1),
    (5000, 4000, 12, ((7, 3000), (100, 9000)), 3000, 2),
    (300, 300000, 8, ((0, 140000), (1, 65537), (2, 65536)), 20000, 1),
    (20000, 20000, 30, (), 50000, 4),
    (64, 64, 2, (), 0, 8),
    (7000, 7000, 60, ((5, 5000),), 40000, 8),
    (2500, 2500, 5, (), 9000, 4),
    (1, 1, 1, (), 3, 1),
    (40000, 10000, 3, ((1, 70000 // 7),), 100000, 2),
    (1200, 1200, 100, (), 5000, 1),
    (36000, 36000, 5, ((9, 700),), 4000, 1),  # k = 1 above the row-group threshold: the one-value stream
]


def build_set(dcsr, rng, dt, mode, shapes=SHAPES, **kw):
    mats, refs, work = [], [], []
    for (n, m, deg, long_rows, T, k) in shapes:
        rp, cols, vals = random_csr(rng, n, m, deg, long_rows)
        a = dcsr.DcsrMatrix(n, m, dt, mode=mode, **kw)
        b = dcsr.DcsrMatrix(n, m, dt, mode=mode, **kw)
        a.from_csr(rp, cols, vals)
        b.from_csr(rp, cols, vals)
        r, c, v = triples(rng, n, m, T)
        rows = torch.tensor(r, device="cuda")
        colt = torch.tensor(c, device="cuda")
        valt = torch.tensor(v, dtype=dt, device="cuda")
        x = torch.tensor(rng.uniform(-1, 1, (m, k)), dtype=dt, device="cuda")
        y0 = torch.tensor(rng.uniform(-1, 1, (n, k)), dtype=dt, device="cuda")
        w = dict(matrix=a, rows=rows, cols=colt, vals=valt, x=x, y=y0.clone(), alpha=1.5, beta=0.5)
        mats.append(a)
        refs.append((b, y0.clone()))
        work.append(w)
    return mats, refs, work


def per_call(dcsr, w, ref, sync=False):
    b, y = ref
    if w["rows"].numel():
        b.update(w["rows"], w["cols"], w["vals"], sync=sync)
    b.spmv(w["x"], y, alpha=w["alpha"], beta=w["beta"])


def assert_same(a, b, what):
    la, lb = a.layout(), b.layout()
    assert la.pool_cap == lb.pool_cap, f"{what}: pool_cap"
    np.testing.assert_array_equal(la.row_sizes, lb.row_sizes, err_msg=f"{what}: row_sizes")
    np.testing.assert_array_equal(la.seg, lb.seg, err_msg=f"{what}: segment table")
    for ta, tb, nm in zip(a.to_csr(), b.to_csr(), ("row_ptr", "cols", "vals")):
        assert torch.equal(ta, tb), f"{what}: {nm}"


def compare_all(work, refs, what):
    torch.cuda.synchronize()
    for i, (w, ref) in enumerate(zip(work, refs)):
        assert_same(w["matrix"], ref[0], f"{what} matrix {i}")
        assert torch.equal(w["y"], ref[1]), f"{what} matrix {i}: y differs"


def check_oracle(dcsr, w, y_before, mode):
    """The batch's SpMV of one matrix against the FP64 oracle."""
    a = w["matrix"]
    _, orc = make_pair(dcsr, a.n_rows, a.n_cols, a.dtype_code, mode)
    rp, c, v = a.to_csr()
    assert orc.load_csr(rp.cpu().numpy(), c.cpu().numpy(), v.cpu().double().numpy()) == 0
    x64 = w["x"].cpu().double().numpy()
    k = x64.shape[1]
    y_ref = orc.spmv(x64.reshape(-1), k=k, alpha=w["alpha"], beta=w["beta"],
                     y=y_before.cpu().double().numpy().reshape(-1)).reshape(-1, k)
    bound = abs(w["alpha"]) * spmv_bound(orc, x64, k).reshape(-1, k) + abs(w["beta"]) * np.abs(
        y_before.cpu().double().numpy()) + 1e-300
    err = np.abs(w["y"].cpu().double().numpy() - y_ref)
    tol = 1e-6 if a.dtype_code == dcsr.F32 else 1e-13
    assert np.all(err <= tol * bound), f"max scaled err {np.max(err / bound):.3e}"


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_batch_run_equals_per_call(dcsr, dt):
    rng = np.random.default_rng(11)
    mats, refs, work = build_set(dcsr, rng, dt, dcsr.MERGE)
    y_before = work[3]["y"].clone()
    batch = dcsr.DcsrBatch(work)
    batch.run()
    st = batch.status()
    statuses = []
    for w, ref in zip(work, refs):
        per_call(dcsr, w, ref)
        statuses.append(ref[0].get_status())
    np.testing.assert_array_equal(st, statuses)
    ok = [i for i in range(len(work)) if st[i] == 0]
    assert len(ok) >= len(work) - 2, st
    torch.cuda.synchronize()
    for i in ok:
        assert_same(work[i]["matrix"], refs[i][0], f"run matrix {i}")
        assert torch.equal(work[i]["y"], refs[i][1]), f"run matrix {i}: y differs"
    check_oracle(dcsr, work[3], y_before, dcsr.MERGE)
    batch.close()


def test_batch_graph_replay(dcsr):
    """Capture once, then replay with fresh triples and RHS written in place."""
    rng = np.random.default_rng(12)
    mats, refs, work = build_set(dcsr, rng, torch.float32, dcsr.MERGE)
    s = torch.cuda.Stream()
    batch = dcsr.DcsrBatch(work, stream=s)
    with torch.cuda.stream(s):
        batch.capture(s)
        for rnd in range(3):
            if rnd:
                for w in work:
                    n, m = w["matrix"].n_rows, w["matrix"].n_cols
                    T = w["rows"].numel()
                    r, c, v = triples(rng, n, m, T)
                    w["rows"].copy_(torch.tensor(r))
                    w["cols"].copy_(torch.tensor(c))
                    w["vals"].copy_(torch.tensor(v, dtype=w["vals"].dtype))
                    w["x"].copy_(torch.tensor(rng.uniform(-1, 1, tuple(w["x"].shape)), dtype=w["x"].dtype))
            batch.launch(s)
            batch.repair(batch.status(s), s)  # run + status + repair == update_sync + spmv
            for w, ref in zip(work, refs):
                per_call(dcsr, w, ref, sync=True)
    s.synchronize()
    compare_all(work, refs, "graph")
    batch.close()


def test_batch_rejection_and_repair(dcsr):
    """A matrix whose pool cannot take its update is rejected inside the
    batch (its y untouched), repaired by the repair policy, and then equals
    the per-call update_sync + spmv; the other matrices are unaffected."""
    rng = np.random.default_rng(13)
    shapes = [(2000, 2000, 6, (), 3000, 1), (3000, 3000, 4, (), 60000, 2), (500, 500, 3, (), 200, 4)]
    mats, refs, work = build_set(dcsr, rng, torch.float32, dcsr.MERGE, shapes, spare_x16=0, min_spare=16)
    y_keep = work[1]["y"].clone()
    batch = dcsr.DcsrBatch(work)
    batch.run()
    st = batch.status()
    assert st[1] == dcsr.POOL_EXHAUSTED, st
    assert torch.equal(work[1]["y"], y_keep), "a rejected matrix's y must stay untouched"
    assert batch.repair(st) == int((st != 0).sum())
    for w, ref in zip(work, refs):
        per_call(dcsr, w, ref, sync=True)
    compare_all(work, refs, "repair")
    # the batch keeps working after the repaired matrix's pool moved:
    # run + status + repair is the per-call update_sync + spmv
    for w in work:
        n, m, T = w["matrix"].n_rows, w["matrix"].n_cols, w["rows"].numel()
        r, c, v = triples(rng, n, m, min(T, 50))
        w["rows"][: len(r)].copy_(torch.tensor(r))
    batch.run()
    batch.repair(batch.status())
    for w, ref in zip(work, refs):
        per_call(dcsr, w, ref, sync=True)
    compare_all(work, refs, "after repair")
    batch.close()


def test_batch_append_mode(dcsr):
    rng = np.random.default_rng(14)
    shapes = [s for s in SHAPES if s[0] <= 20000]
    mats, refs, work = build_set(dcsr, rng, torch.float32, dcsr.APPEND, shapes)
    batch = dcsr.DcsrBatch(work)
    batch.run()
    st = batch.status()
    for w, ref in zip(work, refs):
        per_call(dcsr, w, ref)
    for i, ref in enumerate(refs):
        assert ref[0].get_status() == st[i]
    keep = [i for i in range(len(work)) if st[i] == 0]
    assert keep, st
    torch.cuda.synchronize()
    for i in keep:
        assert_same(work[i]["matrix"], refs[i][0], f"append {i}")
        assert torch.equal(work[i]["y"], refs[i][1])
    batch.close()


def test_batch_rejects_bad_items(dcsr):
    a = dcsr.DcsrMatrix(10, 10, torch.float32)
    b = dcsr.DcsrMatrix(10, 10, torch.float64)
    with pytest.raises(dcsr.DcsrError):
        dcsr.DcsrBatch([dict(matrix=a), dict(matrix=a)])  # a matrix twice
    with pytest.raises(dcsr.DcsrError):
        dcsr.DcsrBatch([dict(matrix=a), dict(matrix=b)])  # mixed dtypes


def test_batch_autotune(dcsr):
    """The autotuner picks row-class thresholds without touching the matrices
    or the items' outputs; with the same thresholds on the per-call copies,
    batched and per-call results stay bit-identical."""
    rng = np.random.default_rng(15)
    mats, refs, work = build_set(dcsr, rng, torch.float32, dcsr.MERGE)
    y_before = [w["y"].clone() for w in work]
    batch = dcsr.DcsrBatch(work)
    sm, lm, us = batch.autotune()
    assert (sm, lm) in {(a, b) for a in (32, 64, 128) for b in (512, 1024, 4096, 16384)} and us > 0
    # the chosen short-row split (if not the automatic rule) must not change
    # a result: the per-call copies below run under the automatic rule
    assert batch.short_split() in (0, 1, 2, 4, 8)
    torch.cuda.synchronize()
    for w, y0, ref in zip(work, y_before, refs):
        assert torch.equal(w["y"], y0), "autotune wrote an item's y"
        assert w["matrix"].row_classes() == (sm, lm)
        assert_same(w["matrix"], ref[0], "after autotune")
        ref[0].set_row_classes(sm, lm)
    batch.run()
    batch.repair(batch.status())
    for w, ref in zip(work, refs):
        per_call(dcsr, w, ref, sync=True)
    compare_all(work, refs, "tuned")
    batch.close()


def test_row_classes_api(dcsr):
    a = dcsr.DcsrMatrix(100, 100, torch.float32)
    assert a.row_classes() == (64, 512)
    a.set_row_classes(32, 4096)
    assert a.row_classes() == (32, 4096)
    for bad in ((0, 4096), (300, 4096), (64, 100), (64, 1 << 21)):
        with pytest.raises(dcsr.DcsrError):
            a.set_row_classes(*bad)


def test_grow_nearly_full_pools(dcsr):
    """dcsr_batch_grow after a status read grows the pools that the run left
    short of room (more than 7/8 full -- here every pool: 1/16 spare -- or
    with less room than two more runs of the last run's growth), and only
    their capacity: contents, row lengths and segments stay the per-call
    ones round after round."""
    rng = np.random.default_rng(31)
    shapes = [(3000, 3000, 6, (), 3000, 2), (2000, 2000, 4, (), 200, 1)]
    mats, refs, work = build_set(dcsr, rng, torch.float32, dcsr.MERGE, shapes=shapes, spare_x16=1, min_spare=16)
    batch = dcsr.DcsrBatch(work)
    grown_total = 0
    for rnd in range(4):
        for w in work:  # fresh triples in the batch's input buffers
            n, m, T = w["matrix"].n_rows, w["matrix"].n_cols, w["rows"].numel()
            w["rows"].copy_(torch.tensor(rng.integers(0, n, T).astype(np.int32)))
            w["cols"].copy_(torch.tensor(rng.integers(0, m, T).astype(np.int32)))
            w["vals"].copy_(torch.tensor(rng.uniform(-1, 1, T), dtype=w["vals"].dtype))
        batch.run()
        st = batch.status()
        batch.repair(st)
        caps_before = [w["matrix"].layout().pool_cap for w in work]
        grown = batch.grow()
        grown_total += grown
        torch.cuda.synchronize()
        caps_after = [w["matrix"].layout().pool_cap for w in work]
        assert sum(a > b for a, b in zip(caps_after, caps_before)) == grown
        for w, ref in zip(work, refs):
            per_call(dcsr, w, ref, sync=True)
            la, lb = w["matrix"].layout(), ref[0].layout()
            np.testing.assert_array_equal(la.row_sizes, lb.row_sizes)
            np.testing.assert_array_equal(la.seg, lb.seg)
            for ta, tb in zip(w["matrix"].to_csr(), ref[0].to_csr()):
                assert torch.equal(ta, tb)
            assert torch.equal(w["y"], ref[1])
            ref[0].reserve(la.pool_cap)  # the reference follows the growth
    assert grown_total >= 1
    batch.close()
