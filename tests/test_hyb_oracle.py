"""The oracle's HYB update (oracle.hyb_update) on hand-worked cases of the
reference's UpdateMatrix(hyb) rule (include/load.h:327-373, kernel
UpdateMatrix_hyb include/sparse_update.inl:321-366): a row's next free ELL
slot first, then the COO part, which ends up sorted by row with a row's
earlier COO entries first and its new ones in input order.  CPU only."""
import numpy as np

from oracle import oracle as O


def _base():
    # rows: 0 -> cols (0, 1); 1 -> empty; 2 -> cols (0, 1, 2); width 2, pitch 4
    rp, c, v = np.array([0, 2, 2, 5]), np.array([0, 1, 0, 1, 2]), np.arange(5.0)
    return O.hyb_from_csr(rp, c, v, 2, 4)


def test_slots_then_coo_in_row_order():
    ec, ev, cr, cc, cv = _base()
    assert cr.tolist() == [2] and cc.tolist() == [2]
    st, e_c, e_v, r2, c2, v2 = O.hyb_update(ec, ev, cr, cc, cv, [2, 1, 0, 1, 1], [3, 0, 2, 1, 2],
                                            [10.0, 11.0, 12.0, 13.0, 14.0], 3, 4, 10)
    assert st == 0
    # row 1's first two triples fill its ELL slots in input order
    assert e_c[:, 1].tolist() == [0, 1] and e_v[:, 1].tolist() == [11.0, 13.0]
    # rows 0 and 2 were full: their triples, and row 1's third, go to COO;
    # row 2's old COO entry stays ahead of its new one
    assert r2.tolist() == [0, 1, 2, 2]
    assert c2.tolist() == [2, 2, 2, 3]
    assert v2.tolist() == [12.0, 14.0, 4.0, 10.0]
    # rows without triples are untouched
    assert e_c[:, 3].tolist() == [-1, -1]


def test_duplicates_are_appended():
    ec, ev, cr, cc, cv = _base()
    st, e_c, e_v, r2, c2, v2 = O.hyb_update(ec, ev, cr, cc, cv, [1, 1, 1], [1, 1, 1], [1.0, 2.0, 3.0], 3, 4, 10)
    assert st == 0
    assert e_c[:, 1].tolist() == [1, 1] and e_v[:, 1].tolist() == [1.0, 2.0]
    assert r2.tolist() == [1, 2] and c2.tolist() == [1, 2] and v2.tolist() == [3.0, 4.0]


def test_errors_leave_everything_unchanged():
    ec, ev, cr, cc, cv = _base()
    for rows, cols, n_rows, cap, want in (([3], [0], 3, 10, 3), ([0], [4], 3, 10, 3), ([0, 0], [2, 3], 3, 2, 1)):
        st, e_c, e_v, r2, c2, v2 = O.hyb_update(ec, ev, cr, cc, cv, rows, cols, [9.0] * len(rows), n_rows, 4, cap)
        assert st == want
        np.testing.assert_array_equal(e_c, ec)
        np.testing.assert_array_equal(e_v, ev)
        assert r2.tolist() == cr.tolist() and c2.tolist() == cc.tolist() and v2.tolist() == cv.tolist()
