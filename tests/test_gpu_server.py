"""The serving form (dcsr_server_*).

* alone vs in the mix: the same request stream served one request at a time
  (each waited for before the next is submitted) and all at once (coalesced
  into batches, several batches in flight) gives bit-identical results for
  every request -- SpMV outputs, exported CSRs, statuses -- and identical
  final matrices;
* the plain per-call server (no coalescing) agrees bit for bit when no pool
  runs short (with a pool running short the batched server grows it ahead of
  time, so its layout -- and the rounding of segment-split rows -- can
  differ from the per-call history);
* per-matrix order: an update followed by an SpMV of the same matrix sees the
  update; an SpMV followed by an update does not;
* admission: a small memory budget still serves everything; a request larger
  than the whole budget fails with OOM instead of blocking the queue.
"""
import numpy as np
import pytest
import torch

from tests.test_gpu_batch import random_csr

pytestmark = pytest.mark.gpu

SHAPES = [(3000, 3000, 8), (800, 5000, 20), (12000, 12000, 4), (200, 200, 40), (5000, 2000, 6), (64, 64, 3),
          (20000, 20000, 12), (1500, 1500, 70)]


def make_mats(dcsr, seed, dt=torch.float32, **kw):
    rng = np.random.default_rng(seed)
    out = []
    for n, m, d in SHAPES:
        rp, c, v = random_csr(rng, n, m, d, ((0, min(m, 6000)),) if n > 1000 else ())
        A = dcsr.DcsrMatrix(n, m, dt, **kw)
        A.from_csr(rp, c, v)
        out.append(A)
    return out


def make_requests(seed, mats, count=160):
    """(kind, matrix, payload) with host tensors, seeded; 40% update, 50% SpMV, 10% export."""
    rng = np.random.default_rng(seed)
    reqs = []
    bound = [m.nnz() for m in mats]  # entries a matrix can hold at each point of the stream
    for _ in range(count):
        i = int(rng.integers(0, len(mats)))
        A = mats[i]
        u = rng.random()
        if u < 0.4:
            T = int(np.exp(rng.uniform(np.log(10), np.log(20000))))
            bound[i] += T
            reqs.append(("update", i, (rng.integers(0, A.n_rows, T).astype(np.int32),
                                        rng.integers(0, A.n_cols, T).astype(np.int32),
                                        rng.uniform(-1, 1, T).astype(np.float32))))
        elif u < 0.9:
            k = int(rng.choice([1, 2, 4, 8]))
            beta = float(rng.choice([0.0, 0.5]))
            reqs.append(("spmv", i, (rng.uniform(-1, 1, (A.n_cols, k)).astype(np.float32),
                                      rng.uniform(-1, 1, (A.n_rows, k)).astype(np.float32), 1.25, beta)))
        else:
            reqs.append(("export", i, bound[i]))
    return reqs


def pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def submit(srv, mats, req):
    kind, i, p = req
    if kind == "update":
        bufs = tuple(pinned(a) for a in p)
        return srv.submit_update(i, *bufs), bufs
    if kind == "spmv":
        x, y = pinned(p[0]), pinned(p[1])
        return srv.submit_spmv(i, x, y, p[2], p[3]), (x, y)
    A = mats[i]
    cap = p
    rp = torch.empty(A.n_rows + 1, dtype=torch.int32).pin_memory()
    c = torch.empty(cap, dtype=torch.int32).pin_memory()
    v = torch.empty(cap, dtype=torch.float32).pin_memory()
    return srv.submit_export(i, rp, c, v), (rp, c, v)


def outputs(res, bufs, req):
    kind = req[0]
    if kind == "update":
        return (res["status"],)
    if kind == "spmv":
        return (res["status"], bufs[1].clone())
    n = int(res["nnz"])
    return (res["status"], bufs[0].clone(), bufs[1][:n].clone(), bufs[2][:n].clone())


def serve(dcsr, mats, reqs, mode, **kw):
    srv = dcsr.DcsrServer(mats, **kw)
    outs = [None] * len(reqs)
    sizes = []
    if mode == "alone":
        for j, r in enumerate(reqs):
            t, b = submit(srv, mats, r)
            res = srv.wait(t)
            outs[j] = outputs(res, b, r)
            sizes.append(res["batch_size"])
    else:
        pend = [submit(srv, mats, r) for r in reqs]
        for j, ((t, b), r) in enumerate(zip(pend, reqs)):
            res = srv.wait(t, 60_000_000)
            outs[j] = outputs(res, b, r)
            sizes.append(res["batch_size"])
    stats = srv.stats()
    srv.close()
    return outs, sizes, stats


def test_alone_equals_mix(dcsr):
    mats_a = make_mats(dcsr, 1)
    mats_m = make_mats(dcsr, 1)
    reqs = make_requests(2, mats_a)
    alone, sz_a, _ = serve(dcsr, mats_a, reqs, "alone", max_batch=64, depth=2)
    mix, sz_m, st = serve(dcsr, mats_m, reqs, "mix", max_batch=64, depth=3)
    assert all(o[0] == 0 for o in alone)
    assert max(sz_a) == 1
    assert max(sz_m) > 4, f"requests were not coalesced: {st}"
    for j, (a, m) in enumerate(zip(alone, mix)):
        assert len(a) == len(m)
        for x, y in zip(a, m):
            if isinstance(x, torch.Tensor):
                assert torch.equal(x, y), f"request {j} ({reqs[j][0]} on matrix {reqs[j][1]}) differs"
            else:
                assert x == y, f"request {j}: status {x} != {y}"
    for i, (A, B) in enumerate(zip(mats_a, mats_m)):
        la, lb = A.layout(), B.layout()
        assert la.pool_cap == lb.pool_cap
        np.testing.assert_array_equal(la.row_sizes, lb.row_sizes, err_msg=f"matrix {i}")
        np.testing.assert_array_equal(la.seg, lb.seg, err_msg=f"matrix {i}")


def test_plain_server_agrees(dcsr):
    """With pools roomy enough that no update is rejected and no pool is grown
    ahead, the plain server (per-call operators, one request at a time) and
    the batched server leave identical layouts, so every result is identical."""
    mats_p = make_mats(dcsr, 3, spare_x16=64)
    mats_s = make_mats(dcsr, 3, spare_x16=64)
    reqs = make_requests(4, mats_p, count=100)
    plain, sz_p, _ = serve(dcsr, mats_p, reqs, "mix", plain=True)
    served, sz_s, _ = serve(dcsr, mats_s, reqs, "mix", max_batch=32, depth=2)
    assert max(sz_p) == 1 and max(sz_s) > 1
    for j, (a, b) in enumerate(zip(plain, served)):
        for x, y in zip(a, b):
            if isinstance(x, torch.Tensor):
                assert torch.equal(x, y), f"request {j} ({reqs[j][0]}) differs"
            else:
                assert x == y, f"request {j}: status {x} != {y}"
    for A, B in zip(mats_p, mats_s):
        la, lb = A.layout(), B.layout()
        np.testing.assert_array_equal(la.seg, lb.seg)


def test_per_matrix_order(dcsr):
    rng = np.random.default_rng(5)
    rp, c, v = random_csr(rng, 1000, 1000, 10)
    A = dcsr.DcsrMatrix(1000, 1000, torch.float32)
    A.from_csr(rp, c, v)
    B = dcsr.DcsrMatrix(1000, 1000, torch.float32)
    B.from_csr(rp, c, v)
    r = rng.integers(0, 1000, 5000).astype(np.int32)
    cc = rng.integers(0, 1000, 5000).astype(np.int32)
    vv = rng.uniform(-1, 1, 5000).astype(np.float32)
    x = rng.uniform(-1, 1, (1000, 1)).astype(np.float32)
    srv = dcsr.DcsrServer([A], max_batch=16)
    y_before = torch.zeros(1000, 1).pin_memory()
    y_after = torch.zeros(1000, 1).pin_memory()
    t0 = srv.submit_spmv(0, pinned(x), y_before)
    t1 = srv.submit_update(0, pinned(r), pinned(cc), pinned(vv))
    t2 = srv.submit_spmv(0, pinned(x), y_after)
    for t in (t0, t1, t2):
        assert srv.wait(t)["status"] == 0
    srv.close()
    xb = torch.tensor(x).cuda()
    ref_before = B.spmv(xb).cpu()
    B.update(torch.tensor(r).cuda(), torch.tensor(cc).cuda(), torch.tensor(vv).cuda())
    ref_after = B.spmv(xb).cpu()
    assert torch.equal(y_before, ref_before)
    assert torch.equal(y_after, ref_after)


def test_admission_by_memory(dcsr):
    mats = make_mats(dcsr, 6)
    reqs = make_requests(7, mats, count=60)
    outs, sizes, st = serve(dcsr, mats, reqs, "mix", max_batch=64, mem_budget=64 << 20)
    assert all(o[0] == 0 for o in outs)
    assert st["completed"] == len(reqs) and st["mem_in_use"] == 0
    srv = dcsr.DcsrServer(mats, mem_budget=1 << 20)
    big = pinned(np.zeros(200000, np.int32))
    t = srv.submit_update(0, big, big, pinned(np.zeros(200000, np.float32)))
    assert srv.wait(t, 30_000_000)["status"] == dcsr.OOM
    t = srv.submit_spmv(5, pinned(np.ones((64, 1), np.float32)), torch.zeros(64, 1).pin_memory())
    assert srv.wait(t, 30_000_000)["status"] == 0
    srv.close()


def test_export_capacity_bound(dcsr):
    """An export whose buffers are too small reports BAD_ARG with the entry
    count and writes nothing past its capacity (device buffers are written
    directly with a device-side bound; host buffers get exactly min(nnz, cap)
    entries); full-size exports equal the per-call export."""
    mats = make_mats(dcsr, 8)
    A = mats[0]
    rp_ref, c_ref, v_ref = A.to_csr()
    nnz = c_ref.numel()
    cap, guard = nnz // 2, 1000
    srv = dcsr.DcsrServer(mats)
    rp = torch.empty(A.n_rows + 1, dtype=torch.int32, device="cuda")
    c = torch.full((cap + guard,), -7, dtype=torch.int32, device="cuda")
    v = torch.full((cap + guard,), -7.0, device="cuda")
    res = srv.wait(srv.submit_export(0, rp, c[:cap], v[:cap]))
    assert res["status"] == dcsr.BAD_ARG and res["nnz"] == nnz
    assert torch.equal(rp, rp_ref)
    assert torch.equal(c[:cap], c_ref[:cap]) and torch.equal(v[:cap], v_ref[:cap])
    assert bool((c[cap:] == -7).all()) and bool((v[cap:] == -7.0).all())
    rph = torch.empty(A.n_rows + 1, dtype=torch.int32).pin_memory()
    ch = torch.full((cap + guard,), -7, dtype=torch.int32).pin_memory()
    vh = torch.full((cap + guard,), -7.0).pin_memory()
    res = srv.wait(srv.submit_export(0, rph, ch[:cap], vh[:cap]))
    assert res["status"] == dcsr.BAD_ARG and res["nnz"] == nnz
    assert torch.equal(ch[:cap], c_ref[:cap].cpu()) and bool((ch[cap:] == -7).all())
    c2 = torch.empty(nnz, dtype=torch.int32, device="cuda")
    v2 = torch.empty(nnz, device="cuda")
    res = srv.wait(srv.submit_export(0, rp, c2, v2))
    assert res["status"] == 0 and torch.equal(c2, c_ref) and torch.equal(v2, v_ref)
    srv.close()


def test_device_requests_match_host_requests(dcsr):
    """The same requests with device buffers and with pinned host buffers
    give identical results."""
    mats_h = make_mats(dcsr, 9)
    mats_d = make_mats(dcsr, 9)
    reqs = make_requests(10, mats_h, count=60)
    host, _, _ = serve(dcsr, mats_h, reqs, "mix", max_batch=16)
    srv = dcsr.DcsrServer(mats_d, max_batch=16)
    pend = []
    for kind, i, p in reqs:
        A = mats_d[i]
        if kind == "update":
            bufs = tuple(torch.from_numpy(a).cuda() for a in p)
            pend.append((srv.submit_update(i, *bufs), bufs))
        elif kind == "spmv":
            bufs = (torch.from_numpy(p[0]).cuda(), torch.from_numpy(p[1]).cuda())
            pend.append((srv.submit_spmv(i, bufs[0], bufs[1], p[2], p[3]), bufs))
        else:
            bufs = (torch.empty(A.n_rows + 1, dtype=torch.int32, device="cuda"),
                    torch.empty(p, dtype=torch.int32, device="cuda"), torch.empty(p, device="cuda"))
            pend.append((srv.submit_export(i, *bufs), bufs))
    for j, ((t, b), r) in enumerate(zip(pend, reqs)):
        res = srv.wait(t)
        out = outputs(res, tuple(x.cpu() for x in b), r)
        for x, y in zip(out, host[j]):
            if isinstance(x, torch.Tensor):
                assert torch.equal(x, y), f"request {j} ({r[0]}) differs"
            else:
                assert x == y
    srv.close()
