"""The device CG (dcsr_cg) against the oracle's CG, itself pinned to the
reference's cusp::krylov::cg (tests/test_cg_oracle.py): an SPD matrix, a
solve, SPD-preserving update batches applied to both, and a solve after each
(the reference tree's included solver over a dynamic matrix).

FP64: the same iteration count (+-1 where the residual lands on the
threshold: the device sums its dot products in another order) and the
iterate within 1e-9 relative.  FP32 matrices: the iteration runs in FP32
with FP64 dot products; it converges to the same tolerance, its true
residual is checked in FP64, and the iterate agrees with the FP64 one within
1e-3 relative.
"""
import numpy as np
import pytest
import torch

from dcsr_b200 import workloads as W
from tests.helpers import make_pair

pytestmark = pytest.mark.gpu


def _true_residual(orc, b, x):
    return float(np.linalg.norm(b - orc.spmv(np.asarray(x, np.float64))))


@pytest.mark.parametrize("n", [3000, 70_000])
def test_cg_fp64_with_updates(dcsr, n):
    rp, c, v = W.spd_matrix(5, n)
    dev, orc = make_pair(dcsr, n, n, dcsr.F64, 0)
    dev.from_csr(rp, c, v)
    assert orc.load_csr(rp, c, v) == 0
    b = np.random.default_rng(6).uniform(-1, 1, n)
    for rnd in range(3):
        x, it, res = dev.cg(torch.from_numpy(b).cuda())
        xo, ito, reso = orc.cg(b)
        assert abs(it - ito) <= 1, (it, ito)
        xd = x.cpu().numpy()
        assert np.linalg.norm(xd - xo) <= 1e-9 * np.linalg.norm(xo)
        assert _true_residual(orc, b, xd) <= 1.01e-5 * np.linalg.norm(b)
        ur, uc, uv = W.spd_updates(7 + rnd, n, n // 3)
        assert dev.update(ur, uc, uv) == 0
        assert orc.update_auto(ur, uc, uv) == 0


def test_cg_fp32_and_initial_guess(dcsr):
    n = 20_000
    rp, c, v = W.spd_matrix(8, n)
    dev, orc = make_pair(dcsr, n, n, dcsr.F32, 0)
    dev.from_csr(rp, c, v.astype(np.float32))
    assert orc.load_csr(rp, c, v.astype(np.float32).astype(np.float64)) == 0
    b = np.random.default_rng(9).uniform(-1, 1, n)
    bt = torch.from_numpy(b.astype(np.float32)).cuda()
    x, it, res = dev.cg(bt)
    xo, ito, _ = orc.cg(b.astype(np.float32).astype(np.float64))
    xd = x.cpu().double().numpy()
    assert abs(it - ito) <= 2
    assert np.linalg.norm(xd - xo) <= 1e-3 * np.linalg.norm(xo)
    # starting from the solution: stops before the first iteration
    x2, it2, _ = dev.cg(bt, x0=x, rel_tol=1e-3)
    assert it2 == 0 and torch.equal(x2, x)
    # the iteration limit holds
    _, it3, _ = dev.cg(bt, max_iter=3)
    assert it3 == 3
