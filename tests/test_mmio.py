"""The Matrix Market reader against the reference's own ReadMatrixFile
(reference include/load_matrix.h:48-119).

Golden: tests/golden/mtx_values.npz holds what ReadMatrixFile returned for
the texts of tests/golden/mtx_corpus.py (values that end their line, values
followed by whitespace, zero / missing / unparsable values); the reader's
reference mode must return exactly that on every machine.  Live (where
oracle/_ref/libref_mtx.so was built from the reference tree): the same
comparison against the reference reader itself, also on the reference's own
fixtures (can_256, tols90) when the tree is present.
"""
import os

import numpy as np
import pytest

from dcsr_b200 import mmio
from oracle import oracle as O
from tests.golden.mtx_corpus import corpus

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mtx_values.npz")
REF_LIB = os.path.join(os.path.dirname(O.__file__), "_ref", "libref_mtx.so")


def _write(tmp_path, name, text):
    p = tmp_path / (name + ".mtx")
    with open(p, "w", newline="") as f:
        f.write(text)
    return str(p)


@pytest.mark.parametrize("name", sorted(corpus()))
def test_reference_values_match_golden(tmp_path, name):
    g = np.load(GOLD)
    nr, nc, r, c, v = mmio.read_matrix_market(_write(tmp_path, name, corpus()[name]))
    assert [nr, nc] == list(g[f"{name}_shape"])
    np.testing.assert_array_equal(r, g[f"{name}_rows"])
    np.testing.assert_array_equal(c, g[f"{name}_cols"])
    np.testing.assert_array_equal(v, g[f"{name}_vals"])


def test_value_rules():
    """The rule itself: a value ending the line becomes 1 in reference mode
    and is kept in file mode; whitespace after it keeps it in both."""
    assert mmio._value(" 2.5", True) == 1.0 and mmio._value(" 2.5", False) == 2.5
    assert mmio._value(" 2.5 ", True) == 2.5 and mmio._value(" 2.5\r", True) == 2.5
    for rest in ("", " ", " 0 ", " abc", " -0.0\t"):
        assert mmio._value(rest, True) == 1.0 and mmio._value(rest, False) == 1.0


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref/libref_mtx.so not built")
@pytest.mark.parametrize("name", sorted(corpus()))
def test_reference_values_live(tmp_path, name):
    path = _write(tmp_path, name, corpus()[name])
    got = mmio.read_matrix_market(path)
    want = O.ref_read_mtx(path)
    assert got[:2] == want[:2]
    for a, b in zip(got[2:], want[2:]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.skipif(not os.path.exists(REF_LIB) or not O.reference_tree(), reason="reference tree absent")
@pytest.mark.parametrize("name", ["can_256.mtx", "tols90.mtx"])
def test_reference_fixture_files_live(name):
    path = os.path.join(O.reference_tree(), "matrices", name)
    got = mmio.read_matrix_market(path)
    want = O.ref_read_mtx(path)
    assert got[:2] == want[:2]
    for a, b in zip(got[2:], want[2:]):
        np.testing.assert_array_equal(a, b)
    # file mode keeps the stored values (tols90 has non-unit values)
    if name == "tols90.mtx":
        assert np.any(mmio.read_matrix_market(path, values="file")[4] != 1.0)


def test_writer_round_trip(tmp_path):
    rng = np.random.default_rng(5)
    r = rng.integers(0, 50, 200).astype(np.int32)
    c = rng.integers(0, 60, 200).astype(np.int32)
    v = rng.standard_normal(200)
    path = str(tmp_path / "w.mtx")
    mmio.write_matrix_market(path, 50, 60, r, c, v)
    nr, nc, r2, c2, v2 = mmio.read_matrix_market(path, values="file")
    assert (nr, nc) == (50, 60)
    np.testing.assert_array_equal(r2, r)
    np.testing.assert_array_equal(c2, c)
    np.testing.assert_array_equal(v2, np.where(v == 0, 1.0, v))
    # the reference reader's rule turns every value that ends its line into 1
    assert np.all(mmio.read_matrix_market(path)[4] == 1.0)
