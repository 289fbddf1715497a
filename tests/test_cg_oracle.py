"""The oracle's CG (oracle/oracle.py OracleDcsr.cg) against the reference's
own solver, cusp::krylov::cg with cusp::monitor (built into
oracle/_ref from the reference tree): the same iterates, iteration counts and
residuals on SPD matrices, before and after SPD-preserving updates.  Golden:
tests/golden/cg_small.npz (cusp's result, made by make_golden.py) on every
machine; live where oracle/_ref is built."""
import os

import numpy as np
import pytest

from dcsr_b200 import workloads as W
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cg_small.npz")


def _oracle(rp, c, v):
    n = len(rp) - 1
    o = O.OracleDcsr(n, n, O.F64)
    assert o.load_csr(rp, c, v) == 0
    return o


def test_cg_matches_golden():
    g = np.load(GOLD)
    o = _oracle(g["rp"], g["cols"], g["vals"])
    x, it, res = o.cg(g["b"], max_iter=int(g["max_iter"]), rel_tol=float(g["rel_tol"]))
    assert it == int(g["iters"])
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=1e-12 * np.max(np.abs(g["x"])))
    assert abs(res - float(g["resid"])) <= 1e-12 * float(g["resid"]) + 1e-300


@pytest.mark.skipif(not O.Ref.available(seq=True), reason="oracle/_ref not built")
@pytest.mark.parametrize("n,seed", [(500, 1), (4000, 2)])
def test_cg_matches_cusp_live(n, seed):
    rp, c, v = W.spd_matrix(seed, n)
    o = _oracle(rp, c, v)
    ref = O.Ref(seq=True)
    b = np.random.default_rng(seed).uniform(-1, 1, n)
    for rnd in range(2):
        rp2, c2, v2 = o.export_csr()
        x, it, res = o.cg(b)
        xr, itr, resr = ref.cg(O.F64, n, rp2, c2, v2, b, np.zeros(n))
        assert it == itr
        np.testing.assert_allclose(x, xr, rtol=0, atol=1e-12 * np.max(np.abs(xr)))
        assert abs(res - resr) <= 1e-10 * resr
        ur, uc, uv = W.spd_updates(seed + 10 + rnd, n, n // 4)
        assert o.update_auto(ur, uc, uv) == 0
