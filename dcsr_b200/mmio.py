"""Matrix Market coordinate reader/writer with the reference's conventions.

Follows ReadMatrixFile (reference include/load_matrix.h:48-119): '%' lines
are skipped, the size line gives rows, cols and the entry count, indices are
1-based, and symmetric storage is NOT expanded (only the stored triangle is
returned).  Entries are returned in file order as COO arrays; load them with
DcsrMatrix.from_coo.

Values, `values=`:

* "reference" (default, the drop-in behaviour): the reference's rule.  It
  reads a line with getline, parses row, col and value from a string stream
  and sets the value to 1 when the stream reached the end of the line, the
  parse failed, or the value is zero (load_matrix.h:88-93).  A value that
  ends its line (no trailing whitespace) therefore becomes 1 -- every value
  of a typical file -- while one followed by whitespace (a space, a tab, a
  carriage return) is kept.
* "file": the value as written (1 when missing, unparsable or zero), the
  canonical reading of the format.

Lines longer than 255 characters, which the reference's fixed 256-byte line
buffer does not read, are not reproduced.
"""
from __future__ import annotations

import re

import numpy as np

_WS = " \t\n\v\f\r"
_NUM = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")
_ENTRY = re.compile(r"[ \t\n\v\f\r]*([+-]?\d+)[ \t\n\v\f\r]+([+-]?\d+)(.*)\Z", re.S)


def _value(rest: str, reference: bool) -> float:
    s = rest.lstrip(_WS)
    m = _NUM.match(s) if s else None
    if m is None:
        return 1.0  # missing or unparsable
    if reference and m.end() == len(s):
        return 1.0  # the value ended the line: the reference's stream reached eof
    v = float(m.group(0))
    return 1.0 if v == 0.0 else v


def read_matrix_market(path: str, dtype=np.float64, values: str = "reference"):
    """Returns (n_rows, n_cols, rows, cols, vals) as int32/int32/dtype arrays."""
    if values not in ("reference", "file"):
        raise ValueError("values must be 'reference' or 'file'")
    reference = values == "reference"
    with open(path, newline="") as f:
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        parts = line.split()
        n_rows, n_cols, nnz = int(parts[0]), int(parts[1]), int(parts[2])
        rows = np.zeros(nnz, np.int32)
        cols = np.zeros(nnz, np.int32)
        vals = np.ones(nnz, dtype)
        for i in range(nnz):
            line = f.readline()
            if line.endswith("\n"):
                line = line[:-1]  # getline drops the newline only
            m = _ENTRY.match(line)
            if m is None:
                raise ValueError(f"{path}: entry {i + 1} has no row and column")
            rows[i] = int(m.group(1)) - 1
            cols[i] = int(m.group(2)) - 1
            vals[i] = _value(m.group(3), reference)
    return n_rows, n_cols, rows, cols, vals


def write_matrix_market(path: str, n_rows: int, n_cols: int, rows, cols, vals):
    """Writes a general real coordinate file (1-based)."""
    rows, cols, vals = np.asarray(rows), np.asarray(cols), np.asarray(vals, np.float64)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n_rows} {n_cols} {rows.size}\n")
        for r, c, v in zip(rows.tolist(), cols.tolist(), vals.tolist()):
            f.write(f"{r + 1} {c + 1} {v!r}\n")  # shortest repr that reads back exactly
