"""Generate the golden fixtures in this folder from the reference's own code.

Run in a container that has the reference tree (it builds oracle/_ref from
it): ``python tests/golden/make_golden.py``.  Every fixture stores seeded
synthetic inputs and the outputs of the reference's cusp host path
(oracle/ref_cusp.cpp, sequential system):

  add_small.npz      cusp::add(A, batch) for 2 update rounds (merge semantics)
  append_small.npz   cusp::sort_by_row(A entries ++ batch) (append semantics)
  spmv_small.npz     cusp::multiply(A, x) in FP32
  spgemm_small.npz   cusp::multiply(A, A) in FP64 (rows unsorted, zeros dropped)
  mtx_values.npz     ReadMatrixFile (the reference's Matrix Market reader) on
                     the texts of mtx_corpus.py
  cg_small.npz       cusp::krylov::cg (cusp::monitor defaults) on an SPD matrix
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from dcsr_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def csr_rows(rp):
    return np.repeat(np.arange(len(rp) - 1), np.diff(rp)).astype(np.int32)


def main():
    O.build()
    ref = O.Ref(seq=True)
    n, rp, cols, vals, rounds = W.small_plain(7, n=512, n_rounds=2, T=1024)
    v64 = vals.astype(np.float64)
    out = dict(n=n, rp=rp, cols=cols, vals=vals)
    A = (rp, cols, v64)
    for i, (r, c, v) in enumerate(rounds):
        out[f"b{i}_rows"], out[f"b{i}_cols"], out[f"b{i}_vals"] = r, c, v
        R = ref.add(O.F32, n, n, *A, r, c, v.astype(np.float64))
        out[f"add{i}_rows"], out[f"add{i}_cols"], out[f"add{i}_vals"] = R[0], R[1], R[2].astype(np.float32)
        # the next round adds to cusp's result (zeros dropped by cusp)
        rr, cc, vv = R
        rp2 = np.zeros(n + 1, np.int32)
        np.cumsum(np.bincount(rr, minlength=n), out=rp2[1:])
        A = (rp2, cc, vv)
    np.savez_compressed(os.path.join(HERE, "add_small.npz"), **out)

    # append semantics: existing entries then the batch, stably by row
    r, c, v = rounds[0]
    cat_r = np.concatenate([csr_rows(rp), r])
    cat_c = np.concatenate([cols, c])
    cat_v = np.concatenate([v64, v.astype(np.float64)])
    sr, sc, sv = ref.sort_by_row(O.F32, cat_r, cat_c, cat_v)
    np.savez_compressed(os.path.join(HERE, "append_small.npz"), n=n, rp=rp, cols=cols, vals=vals, b_rows=r,
                        b_cols=c, b_vals=v, rows=sr, out_cols=sc, out_vals=sv.astype(np.float32))

    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    y = ref.spmv(O.F32, n, n, rp, cols, v64, x.astype(np.float64))
    np.savez_compressed(os.path.join(HERE, "spmv_small.npz"), n=n, rp=rp, cols=cols, vals=vals, x=x,
                        y=y.astype(np.float32))

    m, grp, gcols, gvals, _ = W.banded_spgemm(5, scale=9, off_band=3, n_updates=1)
    C = ref.spgemm(O.F64, m, m, m, grp, gcols, gvals, grp, gcols, gvals)
    np.savez_compressed(os.path.join(HERE, "spgemm_small.npz"), n=m, rp=grp, cols=gcols, vals=gvals, c_rp=C[0],
                        c_cols=C[1], c_vals=C[2])
    import tempfile
    from mtx_corpus import corpus
    mtx = {}
    with tempfile.TemporaryDirectory() as d:
        for name, text in corpus().items():
            path = os.path.join(d, name + ".mtx")
            with open(path, "w", newline="") as f:
                f.write(text)
            nr, nc, r, c, v = O.ref_read_mtx(path)
            mtx.update({f"{name}_shape": np.array([nr, nc]), f"{name}_rows": r, f"{name}_cols": c,
                        f"{name}_vals": v})
    np.savez_compressed(os.path.join(HERE, "mtx_values.npz"), **mtx)
    n = 600
    rp, cg_c, cg_v = W.spd_matrix(21, n)
    b = np.random.default_rng(22).uniform(-1, 1, n)
    x, it, res = ref.cg(O.F64, n, rp, cg_c, cg_v, b, np.zeros(n))
    np.savez_compressed(os.path.join(HERE, "cg_small.npz"), rp=rp, cols=cg_c, vals=cg_v, b=b, x=x, iters=it,
                        resid=res, max_iter=500, rel_tol=1e-5)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
