"""The Python binding's ctypes structures have the C ABI's layout: sizes and
field offsets of every struct in include/dcsr_b200.h, compiled with gcc."""
import ctypes as C
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "dcsr_opts": ("Opts", ["max_segs", "factor_x16", "min_cap", "align", "alpha", "spare_x16", "min_spare", "mode",
                           "reloc_min"]),
    "dcsr_info_t": ("Info", ["n_rows", "n_cols", "dtype", "pitch", "pool_cap", "row_sizes", "seg", "cols", "vals",
                             "opts"]),
    "dcsr_batch_item": ("BatchItem", ["matrix", "rows", "cols", "vals", "nnz", "x", "y", "k", "ldx", "ldy", "alpha",
                                      "beta"]),
    "dcsr_server_opts": ("ServerOpts", ["max_batch", "depth", "mem_budget", "mem_reserve", "plain", "workers"]),
    "dcsr_request": ("Request", ["kind", "matrix", "rows", "cols", "vals", "nnz", "x", "y", "k", "alpha", "beta",
                                 "row_ptr", "out_cols", "out_vals", "cap", "on_device"]),
    "dcsr_result": ("Result", ["status", "batch_size", "nnz", "queue_us", "latency_us"]),
}


def c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dcsr_b200.h"', "int main(void) {"]
    for cname, (_, fields) in STRUCTS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        name, field, val = line.split()
        res[(name, field)] = int(val)
    return res


def test_ctypes_match_c_layout(tmp_path):
    from dcsr_b200 import api
    ref = c_layout(tmp_path)
    for cname, (pyname, fields) in STRUCTS.items():
        cls = getattr(api, pyname)
        assert C.sizeof(cls) == ref[(cname, "sizeof")], f"{cname}: size"
        for f in fields:
            assert getattr(cls, f).offset == ref[(cname, f)], f"{cname}.{f}: offset"


@pytest.mark.parametrize("name", ["dcsr_batch_autotune", "dcsr_batch_short_split", "dcsr_batch_grow", "dcsr_server_replay", "dcsr_set_row_classes",
                                  "dcsr_pool_reserve", "dcsr_pool_usage", "dcsr_spin_faults"])
def test_new_entry_points_declared(name):
    text = open(os.path.join(ROOT, "include", "dcsr_b200.h")).read()
    assert f" {name}(" in text
