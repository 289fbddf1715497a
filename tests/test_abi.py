"""The C-ABI library loads and exports every function include/*.h declares
(no compute: runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(dcsr_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def so():
    from dcsr_b200.build import LIB, build
    build()
    return ctypes.CDLL(LIB)


def test_header_parses():
    names = declared_functions()
    assert "dcsr_create" in names and "dcsr_spmv" in names and "dcsr_update" in names
    assert len(names) >= 20


def test_every_declared_symbol_is_exported(so):
    missing = [n for n in declared_functions() if not hasattr(so, n)]
    assert not missing, f"not exported: {missing}"


def test_host_only_entry_points(so):
    so.dcsr_status_string.restype = ctypes.c_char_p
    assert so.dcsr_status_string(0) == b"OK"
    assert so.dcsr_status_string(1) == b"POOL_EXHAUSTED"
    so.dcsr_version.restype = ctypes.c_char_p
    assert b"sm_100a" in so.dcsr_version()


def test_default_opts_match_oracle(so):
    from dcsr_b200 import api
    from oracle import oracle as O
    for mode in (0, 1):
        a = api.Opts()
        so.dcsr_default_opts(ctypes.byref(a), mode)
        b = O.default_opts(mode)
        assert a.as_dict() == {n: getattr(b, n) for n, _ in O.OrOpts._fields_}


def test_bad_args_rejected_without_device(so):
    # null handle / null output: argument checks happen before any CUDA call
    assert so.dcsr_destroy(None) == 5
    assert so.dcsr_info(None, None) == 5
    assert so.dcsr_compact(None, None) == 5
