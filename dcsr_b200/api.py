"""Python host binding of the DCSR C ABI (include/dcsr_b200.h).

Device memory is held in torch CUDA tensors; every call passes raw pointers
and the current torch CUDA stream to libdcsr_b200.so through ctypes.  There is
no CPU fallback: if the shared library is missing or fails to load, the first
call raises.

``DcsrMatrix`` is the handle class; ``dcsr_b200.device`` mirrors the
reference's free-function operator names on top of it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdcsr_b200.so")

F32, F64 = 0, 1
MERGE, APPEND = 0, 1
OK, POOL_EXHAUSTED, LAYER_OVERFLOW, BAD_INDEX, OOM, BAD_ARG, TIMEOUT, CUDA_ERROR, NOT_SUPPORTED = range(9)
REDUCE_SUM, REDUCE_MAX, REDUCE_MIN, REDUCE_COUNT = range(4)

_TORCH_DT = {F32: torch.float32, F64: torch.float64}


class DcsrError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


class Opts(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "max_segs", "factor_x16", "min_cap", "align", "alpha", "spare_x16", "min_spare", "mode", "reloc_min")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchItem(C.Structure):
    """dcsr_batch_item of the C ABI."""
    _fields_ = [("matrix", C.c_void_p), ("rows", C.c_void_p), ("cols", C.c_void_p), ("vals", C.c_void_p),
                ("nnz", C.c_int64), ("x", C.c_void_p), ("y", C.c_void_p), ("k", C.c_int32), ("ldx", C.c_int64),
                ("ldy", C.c_int64), ("alpha", C.c_double), ("beta", C.c_double)]


class ServerOpts(C.Structure):
    """dcsr_server_opts of the C ABI."""
    _fields_ = [("max_batch", C.c_int32), ("depth", C.c_int32), ("mem_budget", C.c_int64),
                ("mem_reserve", C.c_int64), ("plain", C.c_int32), ("workers", C.c_int32)]


class Request(C.Structure):
    """dcsr_request of the C ABI."""
    _fields_ = [("kind", C.c_int32), ("matrix", C.c_int32), ("rows", C.c_void_p), ("cols", C.c_void_p),
                ("vals", C.c_void_p), ("nnz", C.c_int64), ("x", C.c_void_p), ("y", C.c_void_p), ("k", C.c_int32),
                ("alpha", C.c_double), ("beta", C.c_double), ("row_ptr", C.c_void_p), ("out_cols", C.c_void_p),
                ("out_vals", C.c_void_p), ("cap", C.c_int64), ("on_device", C.c_int32)]


class Result(C.Structure):
    """dcsr_result of the C ABI."""
    _fields_ = [("status", C.c_int32), ("batch_size", C.c_int32), ("nnz", C.c_int64), ("queue_us", C.c_double),
                ("latency_us", C.c_double)]


REQ_UPDATE, REQ_SPMV, REQ_EXPORT = range(3)


class Info(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("n_cols", C.c_int32), ("dtype", C.c_int32), ("pitch", C.c_int32),
                ("pool_cap", C.c_int64), ("row_sizes", C.c_void_p), ("seg", C.c_void_p), ("cols", C.c_void_p),
                ("vals", C.c_void_p), ("opts", Opts)]


_lib = None
_vp, _i32, _i64, _dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double

_SIGS = {
    "dcsr_default_opts": (None, [C.POINTER(Opts), _i32]),
    "dcsr_create": (_i32, [C.POINTER(_vp), _i32, _i32, _i32, C.POINTER(Opts)]),
    "dcsr_destroy": (_i32, [_vp]),
    "dcsr_info": (_i32, [_vp, C.POINTER(Info)]),
    "dcsr_get_layout": (_i32, [_vp, _vp, _vp, _vp]),
    "dcsr_from_csr": (_i32, [_vp, _vp, _vp, _vp, _i64, _vp]),
    "dcsr_from_coo": (_i32, [_vp, _vp, _vp, _vp, _i64, _vp]),
    "dcsr_from_hyb": (_i32, [_vp, _vp, _vp, _i32, _i64, _vp, _vp, _vp, _i64, _vp]),
    "dcsr_nnz": (_i32, [_vp, C.POINTER(_i64), _vp]),
    "dcsr_to_csr": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "dcsr_to_coo": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "dcsr_update": (_i32, [_vp, _vp, _vp, _vp, _i64, _vp]),
    "dcsr_update_sync": (_i32, [_vp, _vp, _vp, _vp, _i64, _vp]),
    "dcsr_get_status": (_i32, [_vp, _vp, C.POINTER(_i32)]),
    "dcsr_compact": (_i32, [_vp, _vp]),
    "dcsr_reserve": (_i32, [_vp, _i64, _vp]),
    "dcsr_bin_rows": (_i32, [_vp, _vp]),
    "dcsr_spmv": (_i32, [_vp, _vp, _i32, _i64, _vp, _i64, _dbl, _dbl, _vp]),
    "dcsr_row_reduce": (_i32, [_vp, _i32, _vp, _vp]),
    "dcsr_spgemm": (_i32, [_vp, _vp, _vp, _vp]),
    "dcsr_count_sorted_indices": (_i32, [_vp, _i64, _vp, _vp]),
    "dcsr_reduce_by_key": (_i32, [_vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp]),
    "dcsr_batch_create": (_i32, [C.POINTER(_vp), _vp, _i32, _vp]),
    "dcsr_batch_run": (_i32, [_vp, _vp]),
    "dcsr_batch_capture": (_i32, [_vp, _vp]),
    "dcsr_batch_launch": (_i32, [_vp, _vp]),
    "dcsr_batch_status": (_i32, [_vp, _vp, _vp]),
    "dcsr_batch_repair": (_i32, [_vp, _vp, C.POINTER(_i32), _vp]),
    "dcsr_batch_grow": (_i32, [_vp, C.POINTER(_i32), _vp]),
    "dcsr_batch_destroy": (_i32, [_vp]),
    "dcsr_batch_autotune": (_i32, [_vp, _vp, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(C.c_float)]),
    "dcsr_batch_short_split": (_i32, [_vp, C.POINTER(_i32)]),
    "dcsr_set_row_classes": (_i32, [_vp, _i32, _i32]),
    "dcsr_get_row_classes": (_i32, [_vp, C.POINTER(_i32), C.POINTER(_i32)]),
    "dcsr_server_default_opts": (None, [_vp]),
    "dcsr_server_create": (_i32, [C.POINTER(_vp), _vp, _i32, _vp]),
    "dcsr_server_submit": (_i32, [_vp, _vp, C.POINTER(C.c_uint64)]),
    "dcsr_server_wait": (_i32, [_vp, C.c_uint64, _i64, _vp]),
    "dcsr_server_stats": (_i32, [_vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "dcsr_server_destroy": (_i32, [_vp]),
    "dcsr_server_replay": (_i32, [_vp, _vp, _vp, _i64, _vp, C.POINTER(_dbl)]),
    "dcsr_status_string": (C.c_char_p, [_i32]),
    "dcsr_launch_count": (C.c_uint64, []),
    "dcsr_spin_faults": (C.c_int, [C.POINTER(C.c_int64)]),
    "dcsr_debug_lookback": (_i32, [_i32, _i32]),
    "dcsr_snapshot_bytes": (_i32, [_vp, C.POINTER(_i64), _vp]),
    "dcsr_snapshot": (_i32, [_vp, _vp, _i64, _vp]),
    "dcsr_snapshot_header": (_i32, [_vp, _i64, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32), C.POINTER(Opts)]),
    "dcsr_restore": (_i32, [_vp, _vp, _i64, _vp]),
    "dcsr_hyb_overflow": (_i32, [_vp, _i32, C.POINTER(_i64), _vp]),
    "dcsr_to_hyb": (_i32, [_vp, _i32, _i64, _vp, _vp, _vp, _vp, _vp, _i64, C.POINTER(_i64), _vp]),
    "dcsr_hyb_spmv": (_i32, [_i32, _i32, _i32, _i64, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _dbl, _dbl, _vp]),
    "dcsr_hyb_update": (_i32, [_i32, _i32, _i32, _i32, _i64, _vp, _vp, _vp, _vp, _vp, _i64, C.POINTER(_i64), _vp,
                               _vp, _vp, _i64, _vp]),
    "dcsr_measure_gather": (_i32, [_vp, _vp, _i64, _vp, _vp, _i32, _vp]),
    "dcsr_cg": (_i32, [_vp, _vp, _vp, _i32, _dbl, _dbl, C.POINTER(_i32), C.POINTER(_dbl), _vp]),
    "dcsr_pool_reserve": (C.c_int, [C.c_int64, C.c_void_p]),
    "dcsr_pool_usage": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dcsr_version": (C.c_char_p, []),
}


def lib():
    """Load libdcsr_b200.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m dcsr_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(st: int) -> str:
    return lib().dcsr_status_string(st).decode()


def launch_count() -> int:
    return int(lib().dcsr_launch_count())


def spin_faults() -> int:
    """Look-back waits that gave up since the library was loaded (synchronises)."""
    v = C.c_int64(-1)
    _check(lib().dcsr_spin_faults(C.byref(v)), "dcsr_spin_faults")
    return v.value


def debug_lookback(spin_limit: int = 0, stall_first_tile: bool = False):
    """Test hook: look-back wait limit (0: default) and the first-tile stall switch."""
    _check(lib().dcsr_debug_lookback(spin_limit, 1 if stall_first_tile else 0), "dcsr_debug_lookback")


def pool_reserve(nbytes: int, stream=None):
    """Make sure `nbytes` of device memory reserved for the library are free
    (mapped up front; later growth of matrices, scratch and staging is carved
    from it with no driver allocation)."""
    _check(lib().dcsr_pool_reserve(int(nbytes), _stream(stream)), "dcsr_pool_reserve")


def pool_usage():
    """(reserved bytes, free bytes, allocations made outside the reserve) of
    the current device."""
    r, f, n = C.c_int64(), C.c_int64(), C.c_int64()
    _check(lib().dcsr_pool_usage(C.byref(r), C.byref(f), C.byref(n)), "dcsr_pool_usage")
    return r.value, f.value, n.value


def _check(st: int, what: str):
    if st != OK:
        raise DcsrError(st, what)


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("device tensor expected")
    if not t.is_contiguous():
        raise ValueError("contiguous tensor expected")
    return C.c_void_p(t.data_ptr())


def default_opts(mode: int = MERGE, **kw) -> Opts:
    o = Opts()
    lib().dcsr_default_opts(C.byref(o), mode)
    for k, v in kw.items():
        setattr(o, k, int(v))
    return o


def _dtype_code(dtype) -> int:
    if dtype in (torch.float32, F32, "f32", "float32"):
        return F32
    if dtype in (torch.float64, F64, "f64", "float64"):
        return F64
    raise ValueError(f"unsupported dtype {dtype}")


@dataclass
class Layout:
    row_sizes: np.ndarray
    seg: np.ndarray
    pitch: int
    max_segs: int
    pool_cap: int


class DcsrMatrix:
    """A DCSR matrix resident on the current CUDA device."""

    def __init__(self, n_rows: int, n_cols: int, dtype=torch.float32, mode: int = MERGE, opts: Opts | None = None,
                 **kw):
        self.h = None
        o = opts if opts is not None else default_opts(mode, **kw)
        self.opts = o
        self.n_rows, self.n_cols = int(n_rows), int(n_cols)
        self.dtype_code = _dtype_code(dtype)
        self.dtype = _TORCH_DT[self.dtype_code]
        h = C.c_void_p()
        _check(lib().dcsr_create(C.byref(h), self.n_rows, self.n_cols, self.dtype_code, C.byref(o)), "dcsr_create")
        self.h = h

    def close(self):
        if self.h is not None and _lib is not None:
            lib().dcsr_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------- loading
    def from_csr(self, row_ptr, cols, vals, stream=None):
        row_ptr, cols, vals = self._i(row_ptr), self._i(cols), self._v(vals)
        _check(lib().dcsr_from_csr(self.h, _ptr(row_ptr), _ptr(cols), _ptr(vals), cols.numel(), _stream(stream)),
               "dcsr_from_csr")
        return self

    def from_coo(self, rows, cols, vals, stream=None):
        rows, cols, vals = self._i(rows), self._i(cols), self._v(vals)
        _check(lib().dcsr_from_coo(self.h, _ptr(rows), _ptr(cols), _ptr(vals), rows.numel(), _stream(stream)),
               "dcsr_from_coo")
        return self

    def from_hyb(self, ell_cols, ell_vals, coo_rows, coo_cols, coo_vals, stream=None):
        """ell_cols/ell_vals: [width, pitch] column-major ELL (-1 = padding)."""
        ell_cols, ell_vals = self._i(ell_cols), self._v(ell_vals)
        coo_rows, coo_cols, coo_vals = self._i(coo_rows), self._i(coo_cols), self._v(coo_vals)
        width = ell_cols.shape[0] if ell_cols.dim() == 2 else 0
        pitch = ell_cols.shape[1] if ell_cols.dim() == 2 else self.n_rows
        _check(lib().dcsr_from_hyb(self.h, _ptr(ell_cols), _ptr(ell_vals), width, pitch, _ptr(coo_rows),
                                   _ptr(coo_cols), _ptr(coo_vals), coo_rows.numel(), _stream(stream)),
               "dcsr_from_hyb")
        return self

    # ---------------------------------------------------------- updates
    def update(self, rows, cols, vals, sync: bool = True, stream=None) -> int:
        """Batch update; sync=True applies the repair policy and returns the
        final status, sync=False enqueues only (status via get_status())."""
        rows, cols, vals = self._i(rows), self._i(cols), self._v(vals)
        fn = lib().dcsr_update_sync if sync else lib().dcsr_update
        st = fn(self.h, _ptr(rows), _ptr(cols), _ptr(vals), rows.numel(), _stream(stream))
        if st in (BAD_ARG, OOM, CUDA_ERROR):
            raise DcsrError(st, "dcsr_update")
        return st

    def get_status(self, stream=None) -> int:
        s = C.c_int32()
        _check(lib().dcsr_get_status(self.h, _stream(stream), C.byref(s)), "dcsr_get_status")
        return s.value

    def compact(self, stream=None):
        _check(lib().dcsr_compact(self.h, _stream(stream)), "dcsr_compact")

    def reserve(self, cap: int, stream=None):
        _check(lib().dcsr_reserve(self.h, cap, _stream(stream)), "dcsr_reserve")

    def set_row_classes(self, short_max: int, long_min: int):
        _check(lib().dcsr_set_row_classes(self.h, short_max, long_min), "dcsr_set_row_classes")

    def row_classes(self):
        sm, lm = _i32(), _i32()
        _check(lib().dcsr_get_row_classes(self.h, C.byref(sm), C.byref(lm)), "dcsr_get_row_classes")
        return sm.value, lm.value

    def bin_rows(self, stream=None):
        _check(lib().dcsr_bin_rows(self.h, _stream(stream)), "dcsr_bin_rows")

    # ----------------------------------------------------------- export
    def nnz(self, stream=None) -> int:
        v = C.c_int64()
        _check(lib().dcsr_nnz(self.h, C.byref(v), _stream(stream)), "dcsr_nnz")
        return v.value

    def to_csr(self, stream=None):
        nnz = self.nnz(stream)
        dev = torch.device("cuda", torch.cuda.current_device())
        rp = torch.empty(self.n_rows + 1, dtype=torch.int32, device=dev)
        c = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        v = torch.empty(max(nnz, 1), dtype=self.dtype, device=dev)
        _check(lib().dcsr_to_csr(self.h, _ptr(rp), _ptr(c), _ptr(v), _stream(stream)), "dcsr_to_csr")
        return rp, c[:nnz], v[:nnz]

    def to_hyb(self, ell_width: int, ell_pitch: int | None = None, stream=None):
        """DCSR -> HYB: returns (ell_cols [width, pitch], ell_vals, coo_rows, coo_cols, coo_vals)."""
        pitch = self.n_rows if ell_pitch is None else int(ell_pitch)
        n = _i64()
        _check(lib().dcsr_hyb_overflow(self.h, ell_width, C.byref(n), _stream(stream)), "dcsr_hyb_overflow")
        dev = torch.device("cuda", torch.cuda.current_device())
        ec = torch.empty((ell_width, pitch), dtype=torch.int32, device=dev)
        ev = torch.empty((ell_width, pitch), dtype=self.dtype, device=dev)
        m = max(n.value, 1)
        cr = torch.empty(m, dtype=torch.int32, device=dev)
        cc = torch.empty(m, dtype=torch.int32, device=dev)
        cv = torch.empty(m, dtype=self.dtype, device=dev)
        got = _i64()
        _check(lib().dcsr_to_hyb(self.h, ell_width, pitch, _ptr(ec), _ptr(ev), _ptr(cr), _ptr(cc), _ptr(cv), m,
                                 C.byref(got), _stream(stream)), "dcsr_to_hyb")
        k = got.value
        return ec, ev, cr[:k], cc[:k], cv[:k]

    def to_coo(self, stream=None):
        nnz = self.nnz(stream)
        dev = torch.device("cuda", torch.cuda.current_device())
        r = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        c = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        v = torch.empty(max(nnz, 1), dtype=self.dtype, device=dev)
        _check(lib().dcsr_to_coo(self.h, _ptr(r), _ptr(c), _ptr(v), _stream(stream)), "dcsr_to_coo")
        return r[:nnz], c[:nnz], v[:nnz]

    def layout(self, stream=None) -> Layout:
        info = self.info()
        rs = np.zeros(self.n_rows + 1, np.int32)
        seg = np.zeros(info.pitch * info.opts.max_segs, np.int32)
        _check(lib().dcsr_get_layout(self.h, C.c_void_p(rs.ctypes.data), C.c_void_p(seg.ctypes.data),
                                     _stream(stream)), "dcsr_get_layout")
        return Layout(rs, seg, info.pitch, info.opts.max_segs, info.pool_cap)

    def info(self) -> Info:
        i = Info()
        _check(lib().dcsr_info(self.h, C.byref(i)), "dcsr_info")
        return i

    # ---------------------------------------------------------- snapshot
    def snapshot(self, stream=None) -> bytes:
        """Binary image of the layout (dcsr_snapshot); restores bit-exact."""
        nb = _i64()
        _check(lib().dcsr_snapshot_bytes(self.h, C.byref(nb), _stream(stream)), "dcsr_snapshot_bytes")
        buf = (C.c_char * nb.value)()
        _check(lib().dcsr_snapshot(self.h, buf, nb.value, _stream(stream)), "dcsr_snapshot")
        return bytes(buf)

    def save(self, path: str, stream=None):
        with open(path, "wb") as f:
            f.write(self.snapshot(stream))

    @classmethod
    def from_snapshot(cls, data: bytes, stream=None) -> "DcsrMatrix":
        nr, nc, dt, o = _i32(), _i32(), _i32(), Opts()
        buf = C.create_string_buffer(data, len(data))
        _check(lib().dcsr_snapshot_header(buf, len(data), C.byref(nr), C.byref(nc), C.byref(dt), C.byref(o)),
               "dcsr_snapshot_header")
        A = cls(nr.value, nc.value, _TORCH_DT[dt.value], opts=o)
        _check(lib().dcsr_restore(A.h, buf, len(data), _stream(stream)), "dcsr_restore")
        return A

    @classmethod
    def load(cls, path: str, stream=None) -> "DcsrMatrix":
        with open(path, "rb") as f:
            return cls.from_snapshot(f.read(), stream)

    # -------------------------------------------------------- operators
    def spmv(self, x: torch.Tensor, y: torch.Tensor | None = None, alpha: float = 1.0, beta: float = 0.0,
             stream=None) -> torch.Tensor:
        """y = alpha*A@x + beta*y; x is [n_cols] or [n_cols, k] (row-major)."""
        x = self._v(x)
        k = 1 if x.dim() == 1 else x.shape[1]
        if y is None:
            y = torch.empty((self.n_rows,) if x.dim() == 1 else (self.n_rows, k), dtype=self.dtype, device=x.device)
            beta = 0.0
        _check(lib().dcsr_spmv(self.h, _ptr(x), k, k, _ptr(y), k, alpha, beta, _stream(stream)), "dcsr_spmv")
        return y

    def cg(self, b: torch.Tensor, x0: torch.Tensor | None = None, max_iter: int = 500, rel_tol: float = 1e-5,
           abs_tol: float = 0.0, stream=None):
        """Conjugate gradient (dcsr_cg, cusp::krylov::cg's iteration and stop
        rule): returns (x, iterations, final residual norm)."""
        b = self._v(b)
        x = torch.zeros_like(b) if x0 is None else self._v(x0).clone()
        it, res = _i32(), _dbl()
        _check(lib().dcsr_cg(self.h, _ptr(b), _ptr(x), max_iter, rel_tol, abs_tol, C.byref(it), C.byref(res),
                             _stream(stream)), "dcsr_cg")
        return x, it.value, res.value

    def row_reduce(self, op: int = REDUCE_SUM, y: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        if y is None:
            y = torch.empty(self.n_rows, dtype=self.dtype, device=torch.device("cuda", torch.cuda.current_device()))
        _check(lib().dcsr_row_reduce(self.h, op, _ptr(y), _stream(stream)), "dcsr_row_reduce")
        return y

    def spgemm(self, B: "DcsrMatrix", C_out: "DcsrMatrix | None" = None, stream=None, **kw) -> "DcsrMatrix":
        if C_out is None:
            C_out = DcsrMatrix(self.n_rows, B.n_cols, self.dtype, **kw)
        _check(lib().dcsr_spgemm(self.h, B.h, C_out.h, _stream(stream)), "dcsr_spgemm")
        return C_out

    # ---------------------------------------------------------- helpers
    def _i(self, t):
        t = torch.as_tensor(t)
        if not t.is_cuda:
            t = t.cuda()
        return t.to(torch.int32).contiguous()

    def _v(self, t):
        t = torch.as_tensor(t)
        if not t.is_cuda:
            t = t.cuda()
        return t.to(self.dtype).contiguous()


def hyb_spmv(ell_cols, ell_vals, coo_rows, coo_cols, coo_vals, x, y=None, alpha=1.0, beta=0.0, stream=None):
    """y = alpha * A x + beta * y for a HYB matrix (dcsr_hyb_spmv); ell_* are [width, pitch]."""
    width, pitch = (ell_cols.shape[0], ell_cols.shape[1]) if ell_cols.dim() == 2 else (0, x.numel())
    n_rows = pitch if y is None else y.numel()
    if y is None:
        y = torch.empty(n_rows, dtype=ell_vals.dtype, device=ell_vals.device)
        beta = 0.0
    _check(lib().dcsr_hyb_spmv(n_rows, _dtype_code(ell_vals.dtype), width, pitch, _ptr(ell_cols), _ptr(ell_vals),
                               coo_rows.numel(), _ptr(coo_rows), _ptr(coo_cols), _ptr(coo_vals), _ptr(x), _ptr(y),
                               alpha, beta, _stream(stream)), "dcsr_hyb_spmv")
    return y


def hyb_update(ell_cols, ell_vals, coo_rows, coo_cols, coo_vals, coo_nnz: int, rows, cols, vals, n_rows: int,
               n_cols: int, stream=None):
    """Append triples to a HYB matrix in place (dcsr_hyb_update).  The COO
    arrays' length is their capacity and their first coo_nnz entries the
    COO part.  Returns (status, new coo_nnz): DCSR_BAD_INDEX or
    DCSR_POOL_EXHAUSTED leave the matrix unchanged."""
    width, pitch = (ell_cols.shape[0], ell_cols.shape[1]) if ell_cols.dim() == 2 else (0, n_rows)
    n = _i64(int(coo_nnz))
    st = lib().dcsr_hyb_update(n_rows, n_cols, _dtype_code(ell_vals.dtype), width, pitch, _ptr(ell_cols),
                               _ptr(ell_vals), _ptr(coo_rows), _ptr(coo_cols), _ptr(coo_vals), coo_rows.numel(),
                               C.byref(n), _ptr(rows), _ptr(cols), _ptr(vals), rows.numel(), _stream(stream))
    if st not in (OK, POOL_EXHAUSTED, BAD_INDEX):
        _check(st, "dcsr_hyb_update")
    return st, int(n.value)


def count_sorted_indices(I: torch.Tensor, X: torch.Tensor, stream=None) -> torch.Tensor:
    """X[I[n]] += 1 (in place) for a sorted int32 index tensor I."""
    _check(lib().dcsr_count_sorted_indices(_ptr(I), I.numel(), _ptr(X), _stream(stream)),
           "dcsr_count_sorted_indices")
    return X


def reduce_by_key(keys: torch.Tensor, vals: torch.Tensor, stream=None):
    """Unique sorted keys and their left-to-right sums."""
    n = keys.numel()
    ko = torch.empty(max(n, 1), dtype=torch.int32, device=keys.device)
    vo = torch.empty(max(n, 1), dtype=vals.dtype, device=keys.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=keys.device)
    _check(lib().dcsr_reduce_by_key(_ptr(keys), _ptr(vals), n, _dtype_code(vals.dtype), _ptr(ko), _ptr(vo),
                                    _ptr(cnt), _stream(stream)), "dcsr_reduce_by_key")
    m = int(cnt.item())
    return ko[:m], vo[:m]


class DcsrBatch:
    """Batched update + SpMV over many matrices (dcsr_batch_* of the C ABI).

    ``work`` is a list of dicts with keys ``matrix`` (DcsrMatrix), optional
    ``rows``/``cols``/``vals`` (the update triples, device tensors) and optional
    ``x``/``y`` ([n_cols, k] / [n_rows, k] or 1-D device tensors), ``alpha``,
    ``beta``.  The tensors are referenced for the batch's lifetime: write new
    triples or right-hand sides into them in place between runs.
    """

    def __init__(self, work, stream=None):
        items = (BatchItem * len(work))()
        self._keep = []
        for i, w in enumerate(work):
            m = w["matrix"]
            it = items[i]
            it.matrix = m.h.value
            r, c, v = w.get("rows"), w.get("cols"), w.get("vals")
            if r is not None and r.numel() > 0:
                it.rows, it.cols, it.vals = _ptr(r).value, _ptr(c).value, _ptr(v).value
                it.nnz = r.numel()
            x, y = w.get("x"), w.get("y")
            if x is not None:
                k = 1 if x.dim() == 1 else x.shape[1]
                it.x, it.y, it.k, it.ldx, it.ldy = _ptr(x).value, _ptr(y).value, k, k, k
                it.alpha, it.beta = float(w.get("alpha", 1.0)), float(w.get("beta", 0.0))
            self._keep += [m, r, c, v, x, y]
        self.count = len(work)
        self.h = C.c_void_p()
        _check(lib().dcsr_batch_create(C.byref(self.h), items, len(work), _stream(stream)), "dcsr_batch_create")

    def run(self, stream=None):
        _check(lib().dcsr_batch_run(self.h, _stream(stream)), "dcsr_batch_run")

    def capture(self, stream=None):
        _check(lib().dcsr_batch_capture(self.h, _stream(stream)), "dcsr_batch_capture")

    def launch(self, stream=None):
        _check(lib().dcsr_batch_launch(self.h, _stream(stream)), "dcsr_batch_launch")

    def status(self, stream=None) -> np.ndarray:
        st = np.zeros(self.count, dtype=np.int32)
        _check(lib().dcsr_batch_status(self.h, st.ctypes.data_as(C.c_void_p), _stream(stream)), "dcsr_batch_status")
        return st

    def autotune(self, stream=None):
        """Pick the row-class thresholds of the batch's matrices and the
        short-row split of its k >= 2 passes by timing their SpMV passes;
        returns (short_max, long_min, us per run).  Capture after this."""
        sm, lm, us = _i32(), _i32(), C.c_float()
        _check(lib().dcsr_batch_autotune(self.h, _stream(stream), C.byref(sm), C.byref(lm), C.byref(us)),
               "dcsr_batch_autotune")
        return sm.value, lm.value, us.value

    def short_split(self) -> int:
        """Warps per 32-row short-row block chosen by autotune (0: automatic)."""
        v = _i32(0)
        _check(lib().dcsr_batch_short_split(self.h, C.byref(v)), "dcsr_batch_short_split")
        return int(v.value)

    def grow(self, stream=None) -> int:
        """After status(): grow pools that the last run left more than 7/8
        full (returns how many)."""
        n = _i32(0)
        _check(lib().dcsr_batch_grow(self.h, C.byref(n), _stream(stream)), "dcsr_batch_grow")
        return int(n.value)

    def repair(self, statuses: np.ndarray, stream=None) -> int:
        st = np.ascontiguousarray(statuses, dtype=np.int32)
        n = _i32(0)
        _check(lib().dcsr_batch_repair(self.h, st.ctypes.data_as(C.c_void_p), C.byref(n), _stream(stream)),
               "dcsr_batch_repair")
        return int(n.value)

    def close(self):
        if self.h:
            lib().dcsr_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _buf(*ts):
    """Pointers of a request's tensors and whether they are device memory
    (all of a request's tensors must be on the same side; host tensors
    should be pinned so the server's copies stay asynchronous)."""
    ts = [t for t in ts if t is not None]
    dev = {t.is_cuda for t in ts}
    if len(dev) > 1:
        raise ValueError("a request's tensors must all be host or all be device tensors")
    for t in ts:
        if not t.is_contiguous():
            raise ValueError("contiguous tensor expected")
    return dev == {True}


class DcsrServer:
    """Request server over resident matrices (dcsr_server_* of the C ABI).

    Requests carry host tensors (allocate them with ``pin_memory()``); they are
    referenced until their result is taken with ``wait``.
    """

    def __init__(self, matrices, max_batch=256, depth=8, mem_budget=0, mem_reserve=1 << 30, plain=False, workers=2):
        o = ServerOpts()
        lib().dcsr_server_default_opts(C.byref(o))
        o.max_batch, o.depth, o.mem_budget, o.mem_reserve, o.plain = max_batch, depth, mem_budget, mem_reserve, int(plain)
        o.workers = workers
        self.matrices = list(matrices)
        arr = (C.c_void_p * len(self.matrices))(*[m.h.value for m in self.matrices])
        self.h = C.c_void_p()
        _check(lib().dcsr_server_create(C.byref(self.h), arr, len(self.matrices), C.byref(o)), "dcsr_server_create")
        self._keep = {}

    def _submit(self, req, keep):
        t = C.c_uint64()
        _check(lib().dcsr_server_submit(self.h, C.byref(req), C.byref(t)), "dcsr_server_submit")
        self._keep[t.value] = keep
        return t.value

    def submit_update(self, i, rows, cols, vals):
        r = Request(kind=REQ_UPDATE, matrix=i, nnz=rows.numel(), on_device=int(_buf(rows, cols, vals)))
        if rows.numel():
            r.rows, r.cols, r.vals = rows.data_ptr(), cols.data_ptr(), vals.data_ptr()
        return self._submit(r, (rows, cols, vals))

    def submit_spmv(self, i, x, y, alpha=1.0, beta=0.0):
        """y ([n_rows] or [n_rows, k]) = alpha*A@x + beta*y."""
        k = 1 if x.dim() == 1 else x.shape[1]
        r = Request(kind=REQ_SPMV, matrix=i, x=x.data_ptr(), y=y.data_ptr(), k=k, alpha=alpha, beta=beta,
                    on_device=int(_buf(x, y)))
        return self._submit(r, (x, y))

    def submit_export(self, i, row_ptr, cols, vals):
        """CSR of the matrix into row_ptr [n_rows+1] and cols/vals (capacity = their length)."""
        r = Request(kind=REQ_EXPORT, matrix=i, row_ptr=row_ptr.data_ptr(), cap=cols.numel(),
                    on_device=int(_buf(row_ptr, cols, vals)))
        if cols.numel():
            r.out_cols, r.out_vals = cols.data_ptr(), vals.data_ptr()
        return self._submit(r, (row_ptr, cols, vals))

    def wait(self, ticket, timeout_us=-1) -> dict:
        res = Result()
        _check(lib().dcsr_server_wait(self.h, ticket, timeout_us, C.byref(res)), "dcsr_server_wait")
        self._keep.pop(ticket, None)
        return {"status": res.status, "batch_size": res.batch_size, "nnz": res.nnz, "queue_us": res.queue_us,
                "latency_us": res.latency_us}

    def stats(self):
        c, b, m = _i64(), _i64(), _i64()
        _check(lib().dcsr_server_stats(self.h, C.byref(c), C.byref(b), C.byref(m)), "dcsr_server_stats")
        return {"completed": c.value, "batches": b.value, "mem_in_use": m.value}

    def close(self):
        if self.h:
            lib().dcsr_server_destroy(self.h)
            self.h = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
