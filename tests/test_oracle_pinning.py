"""Pin the CPU oracle to the reference (CPU only, no GPU).

* Golden fixtures (tests/golden/*.npz, made by make_golden.py from the
  reference's own cusp host path) are checked on every machine.
* When oracle/_ref/ (the reference's cusp host path compiled from the
  reference tree) is present, the same comparisons run live on the full-size
  small workload, and on the reference's MTX fixtures when the reference tree
  itself is present.

Canonical-semantics notes enforced here: cusp::add drops entries whose sum is
exactly zero (cusp/system/detail/generic/elementwise.inl:212-231) while the
DCSR update keeps them, so the comparison uses the oracle's non-zero entries
and counts the zero ones separately; cusp's SpGEMM leaves rows unsorted and
drops zeros (csr_spgemm.h:129,147), so its rows are sorted before comparing.
"""
import os

import numpy as np
import pytest

from dcsr_b200 import mmio
from dcsr_b200 import workloads as W
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_TREE = O.reference_tree() or ""


def load(name):
    return np.load(os.path.join(GOLD, name))


def rows_of(rp):
    return np.repeat(np.arange(len(rp) - 1), np.diff(rp))


def check_merge_vs_add(orc, ref_rows, ref_cols, ref_vals):
    rp, c, v = orc.export_csr()
    r = rows_of(rp)
    nz = v != 0
    np.testing.assert_array_equal(r[nz], ref_rows)
    np.testing.assert_array_equal(c[nz], ref_cols)
    np.testing.assert_array_equal(v[nz], np.asarray(ref_vals, np.float64))
    return int((~nz).sum())


def test_golden_add_merge_semantics():
    g = load("add_small.npz")
    n = int(g["n"])
    orc = O.OracleDcsr(n, n, O.F32)
    assert orc.load_csr(g["rp"], g["cols"], g["vals"].astype(np.float64)) == 0
    for i in range(2):
        st = orc.update_auto(g[f"b{i}_rows"], g[f"b{i}_cols"], g[f"b{i}_vals"].astype(np.float64))
        assert st == 0
        assert orc.validate() == 0
        # cusp drops exact zeros; once a zero is dropped the two diverge, so
        # the fixtures are built on inputs that produce none
        assert check_merge_vs_add(orc, g[f"add{i}_rows"], g[f"add{i}_cols"], g[f"add{i}_vals"]) == 0


def test_golden_append_semantics():
    g = load("append_small.npz")
    n = int(g["n"])
    orc = O.OracleDcsr(n, n, O.F32, O.default_opts(O.APPEND))
    assert orc.load_csr(g["rp"], g["cols"], g["vals"].astype(np.float64)) == 0
    assert orc.update_auto(g["b_rows"], g["b_cols"], g["b_vals"].astype(np.float64)) == 0
    rp, c, v = orc.export_csr()
    np.testing.assert_array_equal(rows_of(rp), g["rows"])
    np.testing.assert_array_equal(c, g["out_cols"])
    np.testing.assert_array_equal(v, g["out_vals"].astype(np.float64))


def test_golden_spmv():
    g = load("spmv_small.npz")
    n = int(g["n"])
    orc = O.OracleDcsr(n, n, O.F32)
    orc.load_csr(g["rp"], g["cols"], g["vals"].astype(np.float64))
    y64 = orc.spmv(g["x"].astype(np.float64))
    # cusp accumulates in float: |y_f32 - y64| <= len * eps32 * sum|a||x|
    rp, c, v = orc.export_csr()
    bound = np.zeros(n)
    np.add.at(bound, rows_of(rp), np.abs(v) * np.abs(g["x"].astype(np.float64)[c]))
    lens = np.diff(rp)
    err = np.abs(g["y"].astype(np.float64) - y64)
    assert np.all(err <= (lens + 1) * 6e-8 * bound + 1e-30)


def test_golden_spgemm():
    g = load("spgemm_small.npz")
    n = int(g["n"])
    A = O.OracleDcsr(n, n, O.F64)
    A.load_csr(g["rp"], g["cols"], g["vals"])
    C = A.spgemm(A)
    assert C.validate() == 0
    rp, c, v = C.export_csr()
    crp, cc, cv = g["c_rp"], g["c_cols"], g["c_vals"]
    for i in range(n):
        mine_c, mine_v = c[rp[i]:rp[i + 1]], v[rp[i]:rp[i + 1]]
        nz = mine_v != 0
        o = np.argsort(cc[crp[i]:crp[i + 1]], kind="stable")
        np.testing.assert_array_equal(mine_c[nz], cc[crp[i]:crp[i + 1]][o])
        np.testing.assert_array_equal(mine_v[nz], cv[crp[i]:crp[i + 1]][o])


def test_oracle_policy_arithmetic():
    o = O.default_opts(O.MERGE)
    assert [O.policy_cap(o, n) for n in (0, 1, 2, 3, 7, 100)] == [4, 4, 4, 8, 16, 200]
    t = O.default_opts(O.APPEND)
    assert [O.policy_cap(t, n) for n in (0, 1, 5)] == [0, 1, 5]
    assert O.pool_capacity(o, 10) == 10 + 4096 and O.pool_capacity(o, 100000) == 200000


def test_oracle_repair_policy_and_invariants():
    rng = np.random.default_rng(1)
    n, m = 200, 1000
    rp, cols = W.poisson_matrix(rng, n, m, 5.0)
    o = O.default_opts(O.MERGE, max_segs=2, spare_x16=0, min_spare=8, factor_x16=16, min_cap=0, align=1)
    orc = O.OracleDcsr(n, m, O.F64, o)
    orc.load_csr(rp, cols, rng.standard_normal(cols.size))
    before = orc.export_csr()
    r = rng.integers(0, n, 3000).astype(np.int32)
    c = rng.integers(0, m, 3000).astype(np.int32)
    v = rng.standard_normal(3000)
    st, need = orc.update(r, c, v)
    assert st in (1, 2)  # rejected: pool or layers
    after = orc.export_csr()
    for a, b in zip(before, after):
        np.testing.assert_array_equal(a, b)  # all-or-nothing
    assert orc.update_auto(r, c, v) == 0
    assert orc.validate() == 0
    bad = c.copy()
    bad[0] = m
    assert orc.update(r, bad, v)[0] == 3


def test_oracle_count_and_reduce_by_key():
    I = np.array([0, 0, 1, 3, 3, 3, 7], np.int32)
    X = O.count_sorted_indices(I, np.zeros(8, np.int32))
    np.testing.assert_array_equal(X, [2, 1, 0, 3, 0, 0, 0, 1])
    k, v = O.reduce_by_key(I, np.arange(7, dtype=np.float64))
    np.testing.assert_array_equal(k, [0, 1, 3, 7])
    np.testing.assert_array_equal(v, [1, 2, 12, 6])


# ------------------------------------------------------------ live pinning

need_ref = pytest.mark.skipif(not O.Ref.available(True), reason="oracle/_ref not built")


@need_ref
def test_live_small_plain_full_size():
    ref = O.Ref(seq=True)
    n, rp, cols, vals, rounds = W.small_plain(0)
    orc = O.OracleDcsr(n, n, O.F32)
    orc.load_csr(rp, cols, vals.astype(np.float64))
    A = orc.export_csr()
    for r, c, v in rounds:
        R = ref.add(O.F32, n, n, *A, r, c, v.astype(np.float64))
        assert orc.update_auto(r, c, v.astype(np.float64)) == 0
        assert check_merge_vs_add(orc, *R) == 0
        A = orc.export_csr()


@need_ref
def test_live_append_vs_sort_by_row():
    ref = O.Ref(seq=True)
    n, rp, cols, vals, rounds = W.small_plain(3)
    orc = O.OracleDcsr(n, n, O.F32, O.default_opts(O.APPEND))
    orc.load_csr(rp, cols, vals.astype(np.float64))
    for r, c, v in rounds:
        rp0, c0, v0 = orc.export_csr()
        sr, sc, sv = ref.sort_by_row(O.F32, np.concatenate([rows_of(rp0), r]), np.concatenate([c0, c]),
                                     np.concatenate([v0, v.astype(np.float64)]))
        assert orc.update_auto(r, c, v.astype(np.float64)) == 0
        rp1, c1, v1 = orc.export_csr()
        np.testing.assert_array_equal(rows_of(rp1), sr)
        np.testing.assert_array_equal(c1, sc)
        np.testing.assert_array_equal(v1, sv)


@need_ref
def test_live_spgemm_banded():
    ref = O.Ref(seq=True)
    n, rp, cols, vals, _ = W.banded_spgemm(2, scale=12, n_updates=1)
    A = O.OracleDcsr(n, n, O.F64)
    A.load_csr(rp, cols, vals)
    crp, c, v = A.spgemm(A).export_csr()
    R = ref.spgemm(O.F64, n, n, n, rp, cols, vals, rp, cols, vals)
    for i in range(0, n, 7):
        nz = v[crp[i]:crp[i + 1]] != 0
        o = np.argsort(R[1][R[0][i]:R[0][i + 1]], kind="stable")
        np.testing.assert_array_equal(c[crp[i]:crp[i + 1]][nz], R[1][R[0][i]:R[0][i + 1]][o])
        np.testing.assert_array_equal(v[crp[i]:crp[i + 1]][nz], R[2][R[0][i]:R[0][i + 1]][o])


@need_ref
@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_TREE, "matrices")), reason="reference tree absent")
@pytest.mark.parametrize("name", ["can_256.mtx", "tols90.mtx"])
def test_reference_mtx_fixtures(name):
    """The reference's own MTX fixtures: load -> export equals the file's
    entries sorted by (row, col) (cusp::add with an empty batch merges the
    same way), and SpMV matches cusp's."""
    ref = O.Ref(seq=True)
    nr, nc, r, c, v = mmio.read_matrix_market(os.path.join(REF_TREE, "matrices", name))
    orc = O.OracleDcsr(nr, nc, O.F64)
    assert orc.load_coo(r, c, v) == 0
    rp = np.zeros(nr + 1, np.int32)
    R = ref.add(O.F64, nr, nc, rp, np.zeros(0, np.int32), np.zeros(0), r, c, v)
    assert check_merge_vs_add(orc, *R) == 0
    x = np.random.default_rng(0).uniform(-1, 1, nc)
    y = ref.spmv(O.F64, nr, nc, *orc.export_csr(), x)
    np.testing.assert_allclose(orc.spmv(x), y, rtol=1e-12, atol=1e-12)
