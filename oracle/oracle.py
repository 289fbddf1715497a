"""ctypes bindings for the CPU oracle and the reference's cusp host harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline leg -- never by the dcsr_b200 package.

* ``OracleDcsr`` wraps oracle/dcsr_oracle.c (the CPU restatement of the DCSR
  operators, see its header for the reference lines each function follows).
* ``Ref`` wraps oracle/ref_cusp.cpp built against the reference tree
  (oracle/_ref/libref_cusp_{seq,omp}.so): the reference's own cusp host
  SpMV / add / SpGEMM / sort_by_row.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REFDIR = os.path.join(HERE, "_ref")

F32, F64 = 0, 1
MERGE, APPEND = 0, 1
STATUS = {0: "OK", 1: "POOL_EXHAUSTED", 2: "LAYER_OVERFLOW", 3: "BAD_INDEX", 5: "BAD_ARG"}

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class OrOpts(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "max_segs", "factor_x16", "min_cap", "align", "alpha", "spare_x16", "min_spare", "mode",
        "reloc_min")]


class OrDcsr(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("n_cols", C.c_int32), ("dtype", C.c_int32),
                ("pitch", C.c_int32), ("o", OrOpts), ("pool_cap", C.c_int64),
                ("row_sizes", C.POINTER(C.c_int32)), ("seg", C.POINTER(C.c_int32)),
                ("cols", C.POINTER(C.c_int32)), ("vals", C.POINTER(C.c_double))]


def reference_tree() -> str | None:
    """The reference source tree: $DCSR_REFERENCE, else its conventional
    location in the build container when present; None elsewhere (the GPU
    box uses the prebuilt oracle/_ref only)."""
    p = os.environ.get("DCSR_REFERENCE") or "/root/reference"
    return p if os.path.isdir(p) else None


def build() -> None:
    """Compile the oracle (and oracle/_ref when the reference tree exists)."""
    ref = reference_tree()
    subprocess.run(["make", "-s", "-C", HERE] + ([f"REF={ref}"] if ref else []), check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(BUILD, "liboracle.so")
        build()  # make: rebuilds only when the oracle sources changed
        L = C.CDLL(path)
        P = C.POINTER(OrDcsr)
        L.or_default_opts.argtypes = [C.POINTER(OrOpts), C.c_int]
        L.or_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.POINTER(OrOpts)]
        L.or_create.restype = P
        L.or_destroy.argtypes = [P]
        L.or_policy_cap.argtypes = [C.POINTER(OrOpts), C.c_int64]
        L.or_policy_cap.restype = C.c_int64
        L.or_pool_capacity.argtypes = [C.POINTER(OrOpts), C.c_int64]
        L.or_pool_capacity.restype = C.c_int64
        L.or_load_csr.argtypes = [P, _i32p, _i32p, _f64p]
        L.or_load_coo.argtypes = [P, _i32p, _i32p, _f64p, C.c_int64]
        L.or_update.argtypes = [P, _i32p, _i32p, _f64p, C.c_int64, C.POINTER(C.c_int64)]
        L.or_update_auto.argtypes = [P, _i32p, _i32p, _f64p, C.c_int64]
        L.or_compact.argtypes = [P]
        L.or_grow.argtypes = [P, C.c_int64]
        L.or_nnz.argtypes = [P]
        L.or_nnz.restype = C.c_int64
        L.or_export_csr.argtypes = [P, _i32p, _i32p, _f64p]
        L.or_spmv.argtypes = [P, _f64p, C.c_int32, C.c_int64, _f64p, C.c_int64, C.c_double, C.c_double]
        L.or_row_reduce.argtypes = [P, C.c_int32, _f64p]
        L.or_spgemm.argtypes = [P, P, C.POINTER(OrOpts), C.POINTER(C.c_int)]
        L.or_spgemm.restype = P
        L.or_spgemm_counts.argtypes = [P, P, _i64p]
        L.or_count_sorted_indices.argtypes = [_i32p, C.c_int64, _i32p]
        L.or_reduce_by_key.argtypes = [_i32p, _f64p, C.c_int64, C.c_int32, _i32p, _f64p]
        L.or_reduce_by_key.restype = C.c_int64
        L.or_bin_counts.argtypes = [P, _i64p]
        L.or_validate.argtypes = [P]
        _lib = L
    return _lib


def default_opts(mode: int = MERGE, **kw) -> OrOpts:
    o = OrOpts()
    lib().or_default_opts(C.byref(o), mode)
    for k, v in kw.items():
        setattr(o, k, int(v))
    return o


def policy_cap(o: OrOpts, n: int) -> int:
    return lib().or_policy_cap(C.byref(o), n)


def pool_capacity(o: OrOpts, top: int) -> int:
    return lib().or_pool_capacity(C.byref(o), top)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OracleDcsr:
    """CPU restatement of one DCSR matrix (see oracle/dcsr_oracle.h)."""

    def __init__(self, n_rows, n_cols, dtype=F32, opts: OrOpts | None = None, _ptr=None):
        self.opts = opts if opts is not None else default_opts()
        self.p = _ptr if _ptr is not None else lib().or_create(n_rows, n_cols, dtype, C.byref(self.opts))
        if not self.p:
            raise ValueError("or_create failed")

    def __del__(self):
        if getattr(self, "p", None):
            lib().or_destroy(self.p)
            self.p = None

    @property
    def s(self) -> OrDcsr:
        return self.p.contents

    n_rows = property(lambda self: self.s.n_rows)
    n_cols = property(lambda self: self.s.n_cols)
    dtype = property(lambda self: self.s.dtype)
    pitch = property(lambda self: self.s.pitch)
    pool_cap = property(lambda self: self.s.pool_cap)

    def row_sizes(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.s.row_sizes, (self.n_rows + 1,)).copy()

    def seg(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.s.seg, (self.s.o.max_segs * self.pitch,)).copy()

    def load_csr(self, row_ptr, cols, vals) -> int:
        return lib().or_load_csr(self.p, _i32(row_ptr), _i32(cols), _f64(vals))

    def load_coo(self, rows, cols, vals) -> int:
        return lib().or_load_coo(self.p, _i32(rows), _i32(cols), _f64(vals), len(rows))

    def update(self, rows, cols, vals):
        need = C.c_int64(0)
        st = lib().or_update(self.p, _i32(rows), _i32(cols), _f64(vals), len(rows), C.byref(need))
        return st, need.value

    def update_auto(self, rows, cols, vals) -> int:
        return lib().or_update_auto(self.p, _i32(rows), _i32(cols), _f64(vals), len(rows))

    def compact(self):
        lib().or_compact(self.p)

    def grow(self, cap):
        lib().or_grow(self.p, cap)

    def nnz(self) -> int:
        return lib().or_nnz(self.p)

    def export_csr(self):
        nnz = self.nnz()
        rp = np.zeros(self.n_rows + 1, np.int32)
        c = np.zeros(max(nnz, 1), np.int32)
        v = np.zeros(max(nnz, 1), np.float64)
        lib().or_export_csr(self.p, rp, c, v)
        return rp, c[:nnz], v[:nnz]

    def spmv(self, x, k=1, alpha=1.0, beta=0.0, y=None):
        x = _f64(x).reshape(-1)
        y = np.zeros(self.n_rows * k, np.float64) if y is None else _f64(y).reshape(-1).copy()
        lib().or_spmv(self.p, x, k, k, y, k, alpha, beta)
        return y.reshape(self.n_rows, k) if k > 1 else y

    def row_reduce(self, op=0):
        y = np.zeros(self.n_rows, np.float64)
        lib().or_row_reduce(self.p, op, y)
        return y

    def cg(self, b, x0=None, max_iter=500, rel_tol=1e-5, abs_tol=0.0):
        """Unpreconditioned CG in FP64 over this matrix's SpMV: the steps of
        cusp::krylov::cg (reference cusp/krylov/detail/cg.inl:62-128) with
        cusp::monitor's stop rule (cusp/detail/monitor.inl: ||r||_2 <=
        abs_tol + rel_tol*||b||_2 tested before every iteration, at most
        max_iter iterations).  Returns (x, iterations, final residual norm)."""
        b = _f64(b)
        x = np.zeros(self.n_rows) if x0 is None else _f64(x0).copy()
        r = b - self.spmv(x)
        p = r.copy()
        rz = float(r @ r)
        tol = abs_tol + rel_tol * float(np.sqrt(b @ b))
        it = 0
        while not (np.sqrt(rz) <= tol or it >= max_iter):
            y = self.spmv(p)
            alpha = rz / float(y @ p)
            x += alpha * p
            r -= alpha * y
            rz_old, rz = rz, float(r @ r)
            p = r + (rz / rz_old) * p
            it += 1
        return x, it, float(np.sqrt(rz))

    def spgemm(self, B: "OracleDcsr", opts: OrOpts | None = None) -> "OracleDcsr":
        o = opts if opts is not None else default_opts()
        st = C.c_int(0)
        p = lib().or_spgemm(self.p, B.p, C.byref(o), C.byref(st))
        if st.value != 0:
            raise RuntimeError(f"or_spgemm: {STATUS.get(st.value, st.value)}")
        return OracleDcsr(0, 0, _ptr=p, opts=o)

    def spgemm_counts(self, B: "OracleDcsr") -> np.ndarray:
        out = np.zeros(self.n_rows, np.int64)
        lib().or_spgemm_counts(self.p, B.p, out)
        return out

    def bin_counts(self) -> np.ndarray:
        out = np.zeros(7, np.int64)
        lib().or_bin_counts(self.p, out)
        return out

    def validate(self) -> int:
        return lib().or_validate(self.p)


def count_sorted_indices(I, X):
    X = _i32(X).copy()
    lib().or_count_sorted_indices(_i32(I), len(I), X)
    return X


def reduce_by_key(keys, vals, dtype=F64):
    keys, vals = _i32(keys), _f64(vals)
    ok = np.zeros(max(len(keys), 1), np.int32)
    ov = np.zeros(max(len(keys), 1), np.float64)
    n = lib().or_reduce_by_key(keys, vals, len(keys), dtype, ok, ov)
    return ok[:n], ov[:n]


# ------------------------------------------------------------ cusp harness

def hyb_from_csr(rp, cols, vals, width, pitch):
    """The HYB layout restated: each row's first `width` entries in the ELL
    part (column-major, slot k of row r at [k, r]; unused slots column -1,
    value 0), the rest in the COO part in row order (the reference's
    hyb_matrix, include/dcsr_matrix.h:149-172, filled as LoadMatrix(hyb, csr)
    does, include/load.h:174-205, with a row-ordered COO part)."""
    rp = np.asarray(rp, np.int64)
    n = len(rp) - 1
    ec = np.full((width, pitch), -1, np.int32)
    ev = np.zeros((width, pitch), np.float64)
    cr, cc, cv = [], [], []
    for r in range(n):
        a, b = rp[r], rp[r + 1]
        k = min(width, b - a)
        ec[:k, r] = cols[a:a + k]
        ev[:k, r] = vals[a:a + k]
        if b - a > width:
            cr.append(np.full(b - a - width, r, np.int32))
            cc.append(np.asarray(cols[a + width:b], np.int32))
            cv.append(np.asarray(vals[a + width:b], np.float64))
    cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt)  # noqa: E731
    return ec, ev, cat(cr, np.int32), cat(cc, np.int32), cat(cv, np.float64)


def hyb_spmv(ec, ev, cr, cc, cv, x, n_rows):
    """FP64 y = A x over a HYB layout: a row's ELL slots in order, then its
    COO entries in order (reference spmv_hyb, include/spmv.inl:105-156)."""
    x = np.asarray(x, np.float64)
    width = ec.shape[0]
    y = np.zeros(n_rows)
    for k in range(width):
        c = ec[k, :n_rows]
        live = c >= 0
        y[live] += ev[k, :n_rows][live] * x[c[live]]
    np.add.at(y, cr, cv * x[cc])
    return y


def hyb_update(ec, ev, cr, cc, cv, rows, cols, vals, n_rows, n_cols, coo_cap):
    """The reference's HYB update restated (UpdateMatrix(hyb), include/load.h:
    327-373, kernel UpdateMatrix_hyb, include/sparse_update.inl:321-366):
    triples taken in row order (a stable sort by row; the reference needs its
    input sorted by row for indices_to_offsets), each appended to its row --
    the next free ELL slot while the row's ELL part has one (the slot after
    the row's current entries, sparse_update.inl:350-355), else the COO part
    (:357-363) -- with no duplicate check; the COO part then sorted by row
    (load.h:362-363, a stable sort: a row's earlier COO entries first, then
    its new ones in input order).  Returns (status, ec, ev, cr, cc, cv) as new
    arrays; status 3 (BAD_INDEX) for a row outside [0, n_rows) or a column
    outside [0, n_cols), 1 (POOL_EXHAUSTED) for a COO part beyond coo_cap,
    both with the inputs unchanged."""
    rows, cols = np.asarray(rows, np.int64), np.asarray(cols, np.int64)
    vals = np.asarray(vals, np.float64)
    width = ec.shape[0]
    unchanged = (ec.copy(), ev.copy(), cr.copy(), cc.copy(), cv.copy())
    if rows.size and (rows.min() < 0 or rows.max() >= n_rows or cols.min() < 0 or cols.max() >= n_cols):
        return (3,) + unchanged
    e_c, e_v = ec.copy(), ev.copy()
    fill = {}
    nr, nc, nv = [], [], []
    for i in np.argsort(rows, kind="stable"):
        r = int(rows[i])
        if r not in fill:
            fill[r] = int((e_c[:, r] >= 0).sum())
        f = fill[r]
        if f < width:
            e_c[f, r] = cols[i]
            e_v[f, r] = vals[i]
        else:
            nr.append(r)
            nc.append(int(cols[i]))
            nv.append(float(vals[i]))
        fill[r] = f + 1
    if cr.size + len(nr) > coo_cap:
        return (1,) + unchanged
    r2 = np.concatenate([cr, np.asarray(nr, np.int32)]).astype(np.int32)
    c2 = np.concatenate([cc, np.asarray(nc, np.int32)]).astype(np.int32)
    v2 = np.concatenate([cv, np.asarray(nv, np.float64)])
    o = np.argsort(r2, kind="stable")
    return 0, e_c, e_v, r2[o], c2[o], v2[o]


def ref_read_mtx(path: str, cap: int = 1 << 22):
    """The reference's own ReadMatrixFile<int, double> (oracle/_ref/libref_mtx.so):
    (n_rows, n_cols, rows, cols, vals) with 0-based indices, file order."""
    lib_path = os.path.join(REFDIR, "libref_mtx.so")
    if not os.path.exists(lib_path):
        raise FileNotFoundError(lib_path)
    L = C.CDLL(lib_path)
    L.ref_read_mtx.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_long, _i32p, _i32p, _f64p]
    L.ref_read_mtx.restype = C.c_int
    r = np.zeros(cap, np.int32)
    c = np.zeros(cap, np.int32)
    v = np.zeros(cap, np.float64)
    nr, nc = C.c_int(), C.c_int()
    nnz = L.ref_read_mtx(path.encode(), C.byref(nr), C.byref(nc), cap, r, c, v)
    return nr.value, nc.value, r[:nnz].copy(), c[:nnz].copy(), v[:nnz].copy()


class Ref:
    """The reference's own cusp host path (oracle/_ref); ``seq`` picks the
    sequential host system (bit-reproducible), else the OpenMP one."""

    def __init__(self, seq: bool = True):
        name = "libref_cusp_seq.so" if seq else "libref_cusp_omp.so"
        path = os.path.join(REFDIR, name)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.ref_threads.restype = C.c_int
        L.ref_spmv.argtypes = [C.c_int32, C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.ref_add.argtypes = [C.c_int32, C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p,
                              C.c_int64]
        L.ref_add.restype = C.c_void_p
        L.ref_spgemm.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _i32p,
                                 _i32p, _f64p]
        L.ref_spgemm.restype = C.c_void_p
        L.ref_sort_by_row.argtypes = [C.c_int32, _i32p, _i32p, _f64p, C.c_int64]
        L.ref_cg.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int32, C.c_double,
                             C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.ref_result_nnz.argtypes = [C.c_void_p]
        L.ref_result_nnz.restype = C.c_int64
        L.ref_result_rows_len.argtypes = [C.c_void_p]
        L.ref_result_rows_len.restype = C.c_int64
        L.ref_result_get.argtypes = [C.c_void_p, _i32p, _i32p, _f64p]
        L.ref_result_free.argtypes = [C.c_void_p]
        L.ref_stream_create.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _f64p]
        L.ref_stream_create.restype = C.c_void_p
        L.ref_stream_step.argtypes = [C.c_void_p, _i32p, _i32p, _f64p, C.c_int64,
                                      np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
                                      np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")]
        L.ref_stream_step.restype = C.c_int64
        L.ref_stream_free.argtypes = [C.c_void_p]
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        L.ref_res_create.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, f32p]
        L.ref_res_create.restype = C.c_void_p
        L.ref_res_update.argtypes = [C.c_void_p, _i32p, _i32p, f32p, C.c_int64]
        L.ref_res_update.restype = C.c_int64
        L.ref_res_spmv.argtypes = [C.c_void_p, f32p, C.c_int32, f32p]
        L.ref_res_export.argtypes = [C.c_void_p, _i32p, _i32p, f32p]
        L.ref_res_export.restype = C.c_int64
        L.ref_res_free.argtypes = [C.c_void_p]
        self.L = L

    @staticmethod
    def available(seq: bool = True) -> bool:
        return os.path.exists(os.path.join(REFDIR, "libref_cusp_seq.so" if seq else "libref_cusp_omp.so"))

    def threads(self) -> int:
        return self.L.ref_threads()

    def _take(self, h):
        nnz = self.L.ref_result_nnz(h)
        nr = self.L.ref_result_rows_len(h)
        r = np.zeros(max(nr, 1), np.int32)
        c = np.zeros(max(nnz, 1), np.int32)
        v = np.zeros(max(nnz, 1), np.float64)
        self.L.ref_result_get(h, r, c, v)
        self.L.ref_result_free(h)
        return r[:nr], c[:nnz], v[:nnz]

    def spmv(self, dtype, n, m, rp, ci, vv, x):
        y = np.zeros(n, np.float64)
        self.L.ref_spmv(dtype, n, m, _i32(rp), _i32(ci), _f64(vv), _f64(x), y)
        return y

    def add(self, dtype, n, m, rp, ci, vv, br, bc, bv):
        """cusp::add(A_coo, B_coo): returns COO (rows, cols, vals), zeros dropped."""
        h = self.L.ref_add(dtype, n, m, _i32(rp), _i32(ci), _f64(vv), _i32(br), _i32(bc), _f64(bv), len(br))
        return self._take(h)

    def spgemm(self, dtype, n, k, m, arp, aci, av, brp, bci, bv):
        """cusp::multiply(csr, csr): returns CSR (row_ptr, cols, vals); rows unsorted, zeros dropped."""
        h = self.L.ref_spgemm(dtype, n, k, m, _i32(arp), _i32(aci), _f64(av), _i32(brp), _i32(bci), _f64(bv))
        return self._take(h)

    def cg(self, dtype, n, rp, ci, vv, b, x0, max_iter=500, rel_tol=1e-5, abs_tol=0.0):
        """cusp::krylov::cg with a cusp::monitor(b, max_iter, rel_tol, abs_tol):
        (x, iterations, residual norm)."""
        x = _f64(x0).copy()
        it, res = C.c_int32(), C.c_double()
        self.L.ref_cg(dtype, n, _i32(rp), _i32(ci), _f64(vv), _f64(b), x, max_iter, rel_tol, abs_tol,
                      C.byref(it), C.byref(res))
        return x, it.value, res.value

    def sort_by_row(self, dtype, rows, cols, vals):
        r, c, v = _i32(rows).copy(), _i32(cols).copy(), _f64(vals).copy()
        self.L.ref_sort_by_row(dtype, r, c, v, len(r))
        return r, c, v
