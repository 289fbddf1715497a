"""Host-side helpers of bench.py that shape the reported numbers: the
median-p99 pick of a served load point over repeated replays, the median
capacity over closed-loop replays, Poisson arrivals, and the roofline
traffic taken from the committed ncu summary."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class _FakeApi:
    def __init__(self):
        self.n = 0

    def launch_count(self):
        self.n += 10
        return self.n


def test_replay_point_takes_the_median_p99_run(monkeypatch):
    p99s = iter([3.0, 1.0, 2.0])

    def fake_replay(api, srv, trace, arrivals, lo=0, hi=None):
        p = next(p99s)
        return {"requests": 100, "wall_ms": 10.0, "req_s": 1000.0 / p, "p50_ms": p / 2, "p99_ms": p,
                "errors": 0, "mean_batch": 1.0}

    monkeypatch.setattr(bench, "replay", fake_replay)
    r = bench.replay_point(_FakeApi(), None, None, 5000.0, 100, 7, 3)
    assert r["p99_ms"] == 2.0 and r["p50_ms"] == 1.0  # the median run, whole
    assert r["p99_ms_runs"] == [3.0, 1.0, 2.0]
    assert r["offered_req_s"] == 5000.0
    assert r["kernel_launches"] == 10


def test_capacity_takes_the_median_replay(monkeypatch):
    """One replay slowed by an allocation stall does not set the capacity."""
    rates = iter([12000.0, 4000.0, 11800.0])
    seen = []

    def fake_replay(api, srv, trace, arrivals, lo=0, hi=None):
        assert np.all(np.asarray(arrivals) == 0)  # closed loop: all queued at once
        seen.append((lo, hi))
        return {"requests": 100, "wall_ms": 1.0, "req_s": next(rates), "p50_ms": 1.0, "p99_ms": 2.0,
                "errors": 0, "mean_batch": 3.0}

    monkeypatch.setattr(bench, "replay", fake_replay)
    r = bench.capacity(_FakeApi(), None, None, 100, 0, 100)
    assert r["req_s"] == 11800.0
    assert r["req_s_runs"] == [4000.0, 11800.0, 12000.0]
    assert seen == [(0, 100)] * 3


def test_poisson_arrivals_rate_and_seed():
    a = bench.poisson_arrivals(10_000.0, 20_000, 3)
    assert np.all(np.diff(a) >= 0)
    rate = len(a) / (a[-1] / 1e6)
    assert abs(rate - 10_000.0) / 10_000.0 < 0.03
    assert np.array_equal(a, bench.poisson_arrivals(10_000.0, 20_000, 3))


def test_spmv_traffic_is_keyed_by_matrix_state():
    """The SpMV's DRAM traffic comes from an ncu capture of the same matrix
    state (same stored-entry count) or is not reported: never scaled from
    another state."""
    for nnz, t in bench.SPMV_TRAFFIC.items():
        assert isinstance(nnz, int) and nnz > 0 and t > 0
    assert bench.SPMV_TRAFFIC.get(-1) is None
