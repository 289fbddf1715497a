"""The allocation-free reduce-by-key entry point against the allocating one.

dcsr_reduce_by_key_noalloc exists for callers that cannot allocate device
memory at call time (fixed up-front memory budgets, or a foreign allocator
that must not have CUDA's allocator run underneath it).  Its scratch is a
static device array in the library, shared by every call.  This test calls
both entry points through the C ABI on three different inputs in a row and
requires identical results (the same bit-exact bar as the other
reduce-by-key tests), so a later call cannot see stale scratch (head
positions, look-back epochs and tile counters) from an earlier one.  It sits
in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bind(api):
    L = api.lib()
    fn = L.dcsr_reduce_by_key_noalloc
    fn.restype = C.c_int32
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return L, fn


def _run(fn, keys, vals, dtype_code):
    n = keys.numel()
    ko = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    vo = torch.full((max(n, 1),), -7.0, dtype=vals.dtype, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = fn(C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()), n, dtype_code, C.c_void_p(ko.data_ptr()),
            C.c_void_p(vo.data_ptr()), C.c_void_p(cnt.data_ptr()), s)
    torch.cuda.synchronize()
    assert st == 0, f"status {st}"
    m = int(cnt.item())
    return ko[:m].cpu().numpy(), vo[:m].cpu().numpy()


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_noalloc_matches_allocating_entry_point_twice(dcsr, dtype):
    L, fn_noalloc = _bind(dcsr)
    code = dcsr.F32 if dtype == torch.float32 else dcsr.F64
    rng = np.random.default_rng(123)
    faults = dcsr.spin_faults()
    # calls in a row, all above one scan block (4096 keys), so each reuses the
    # static array's look-back area after the previous call: the full
    # capacity, then a smaller input with other keys, then one single run
    for n, span in ((dcsr_max(L), 70000), (dcsr_max(L) // 3 + 12345, 900), (5000, 1)):
        keys = torch.tensor(np.sort(rng.integers(0, span, n)).astype(np.int32), device="cuda")
        vals = torch.tensor(rng.standard_normal(n), dtype=dtype, device="cuda")
        k_ref, v_ref = dcsr.reduce_by_key(keys, vals)
        k_na, v_na = _run(fn_noalloc, keys, vals, code)
        np.testing.assert_array_equal(k_na, k_ref.cpu().numpy())
        np.testing.assert_array_equal(v_na, v_ref.cpu().numpy())
    assert dcsr.spin_faults() == faults  # no look-back wait gave up


def dcsr_max(L):
    return 1 << 20  # DCSR_NOALLOC_MAX_KEYS in include/dcsr_b200.h


def test_noalloc_rejects_oversize(dcsr):
    L, fn = _bind(dcsr)
    n = dcsr_max(L) + 1
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # the size check comes first: no device pointer is touched
    assert fn(C.c_void_p(1), C.c_void_p(1), n, dcsr.F32, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), s) == \
        dcsr.BAD_ARG
