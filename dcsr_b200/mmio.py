"""Matrix Market coordinate reader with the reference's conventions.

Follows ReadMatrixFile (reference include/load_matrix.h:48-119): '%' lines
are skipped, the size line gives rows, cols and the entry count, indices are
1-based, a missing, unparsable or zero value becomes 1, and symmetric storage
is NOT expanded (only the stored triangle is returned).  Entries are returned
in file order as COO arrays; load them with DcsrMatrix.from_coo.
"""
from __future__ import annotations

import numpy as np


def read_matrix_market(path: str, dtype=np.float64):
    """Returns (n_rows, n_cols, rows, cols, vals) as int32/int32/dtype arrays."""
    with open(path) as f:
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        parts = line.split()
        n_rows, n_cols, nnz = int(parts[0]), int(parts[1]), int(parts[2])
        rows = np.zeros(nnz, np.int32)
        cols = np.zeros(nnz, np.int32)
        vals = np.ones(nnz, dtype)
        for i in range(nnz):
            t = f.readline().split()
            rows[i] = int(t[0]) - 1
            cols[i] = int(t[1]) - 1
            if len(t) > 2:
                try:
                    v = float(t[2])
                except ValueError:
                    v = 0.0
                vals[i] = v if v != 0.0 else 1.0
    return n_rows, n_cols, rows, cols, vals


def write_matrix_market(path: str, n_rows: int, n_cols: int, rows, cols, vals):
    """Writes a general real coordinate file (1-based)."""
    rows, cols, vals = np.asarray(rows), np.asarray(cols), np.asarray(vals, np.float64)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n_rows} {n_cols} {rows.size}\n")
        for r, c, v in zip(rows, cols, vals):
            f.write(f"{r + 1} {c + 1} {v!r}\n")
