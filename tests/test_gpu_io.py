"""Matrix IO on the device: a Matrix Market file loaded into a handle
(through the reader's reference-value and file-value modes) against the
oracle loading the same entries; binary snapshots restore the layout bit for
bit (row lengths, every segment pair, pool capacity, contents) for loaded,
chained (after updates) and compacted matrices, through memory and a file;
corrupt images are rejected."""
import numpy as np
import pytest
import torch

from dcsr_b200 import mmio
from dcsr_b200 import workloads as W
from tests.helpers import assert_content_equal, assert_layout_equal, make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("values", ["reference", "file"])
def test_mtx_file_to_device(dcsr, tmp_path, values):
    rng = np.random.default_rng(4)
    n, m = 700, 900
    rp, cols = W.poisson_matrix(rng, n, m, 5.0)
    rows = np.repeat(np.arange(n), np.diff(rp)).astype(np.int32)
    vals = rng.uniform(-1, 1, cols.size)
    path = str(tmp_path / "a.mtx")
    mmio.write_matrix_market(path, n, m, rows, cols, vals)
    nr, nc, r, c, v = mmio.read_matrix_market(path, values=values)
    assert (nr, nc) == (n, m)
    if values == "reference":
        assert np.all(v == 1.0)  # every value ends its line
    else:
        np.testing.assert_array_equal(v, vals)
    dev, orc = make_pair(dcsr, nr, nc, dcsr.F64, 0)
    dev.from_coo(r, c, v)
    assert orc.load_coo(r, c, v) == 0
    assert_layout_equal(dev, orc, "mtx load")
    assert_content_equal(dev, orc, "mtx load")


def _assert_same_matrix(a, b):
    la, lb = a.layout(), b.layout()
    assert la.pool_cap == lb.pool_cap
    np.testing.assert_array_equal(la.row_sizes, lb.row_sizes)
    np.testing.assert_array_equal(la.seg, lb.seg)
    for x, y in zip(a.to_csr(), b.to_csr()):
        assert torch.equal(x, y)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_snapshot_roundtrip(dcsr, tmp_path, dtype):
    n, rp, cols, vals, rounds = W.small_plain(3, n=3000, n_rounds=3, T=6000)
    A = dcsr.DcsrMatrix(n, n, dtype)
    A.from_csr(rp, cols, vals.astype(np.float64))
    B = dcsr.DcsrMatrix.from_snapshot(A.snapshot())
    _assert_same_matrix(A, B)
    for r, c, v in rounds:  # chained rows, relocations
        assert A.update(r, c, v) == 0
    path = str(tmp_path / "a.dcsr")
    A.save(path)
    C = dcsr.DcsrMatrix.load(path)
    _assert_same_matrix(A, C)
    x = torch.rand(n, dtype=dtype, device="cuda")
    assert torch.equal(A.spmv(x), C.spmv(x))  # same layout, same results bit for bit
    # the restored matrix keeps working: updates land identically
    r, c, v = rounds[0]
    assert A.update(r, c, v) == C.update(r, c, v) == 0
    _assert_same_matrix(A, C)
    A.compact()
    D = dcsr.DcsrMatrix.from_snapshot(A.snapshot())
    _assert_same_matrix(A, D)


def test_snapshot_rejects_bad_images(dcsr):
    A = dcsr.DcsrMatrix(100, 100)
    A.from_coo(np.arange(100, dtype=np.int32), np.arange(100, dtype=np.int32), np.ones(100, np.float32))
    img = bytearray(A.snapshot())
    with pytest.raises(dcsr.DcsrError):
        dcsr.DcsrMatrix.from_snapshot(bytes(img[:50]))  # truncated header
    bad = bytearray(img)
    bad[0] ^= 0xFF
    with pytest.raises(dcsr.DcsrError):
        dcsr.DcsrMatrix.from_snapshot(bytes(bad))  # wrong magic
    with pytest.raises(dcsr.DcsrError):
        dcsr.DcsrMatrix.from_snapshot(bytes(img[:-4]))  # truncated pool
    import ctypes as C
    B = dcsr.DcsrMatrix(101, 100)  # wrong shape
    buf = C.create_string_buffer(bytes(img), len(img))
    assert dcsr.lib().dcsr_restore(B.h, buf, len(img), None) == dcsr.BAD_ARG
