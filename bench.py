"""DCSR benchmark: one JSON line on rank 0.

Three workloads, all seeded synthetic data (no public dataset exists for
them):

served (headline)  2000 resident matrices (rows log-uniform [1k, 256k], mean
        degree U[4, 64], Poisson row lengths, FP32; ~60 GB of HBM) and a
        request stream: 40% updates (log-uniform 10..100k triples), 50% SpMV
        (k uniform in 1..8), 10% DCSR->CSR exports, matrices uniform.  At
        set-up the batch autotuner picks the matrices' row-class thresholds
        (both servers then use them).  The plain per-call server (each request alone through dcsr_update_sync /
        dcsr_spmv / dcsr_to_csr) is measured first: its capacity (all requests
        queued at once; the median of three such replays) and its p99 latency under Poisson arrivals at 50, 70
        and 90% of that capacity; the 90% point (its best sustained
        throughput) sets the latency target.  The batched server (continuous
        batching, memory admission) then runs Poisson arrivals at fractions of
        its own capacity; `value` = its request throughput at the highest load
        whose p99 stays at or below the plain path's p99.  Every load point
        of both servers is replayed three times with different arrival seeds
        and stands as its median-p99 run (one run's p99 rests on its 1%
        slowest requests and moved by +-30% between runs).  Throughput = requests / wall time
        from the first scheduled arrival to the last completion (the GPU is
        idle before and after); latency = scheduled arrival -> result visible
        to the caller.  `value` uses device-resident request buffers; `e2e`
        applies the same rule with pinned host buffers (inputs copied in,
        results copied out, inside each request; exports move whole matrices
        over the host link, which bounds that mode).
stream  the power-law update stream: R-MAT 2^20 rows, (a,b,c,d) =
        (.57,.19,.19,.05), mean degree 16, FP32; 16 batches of 1M triples with
        rows drawn by current row length; a step = dcsr_update_sync (merge,
        slack insertion / chaining / relocation, repair) + SpMV + row sums +
        DCSR->CSR export, CUDA events on the stream.  The SpMV of this matrix is
        the roofline kernel (timed alone, L2 flushed before each launch).
batched 512 matrices like the served ones, each with an update batch
        (log-uniform 100..100k triples) and an SpMV (k in {1,2,4,8}): one
        captured graph launch (+ status read) vs 512 plain per-call sequences
        (dcsr_update_sync + dcsr_spmv), CUDA events.

--impl reference runs the reference's own CPU path (its cusp host operators,
OpenMP, all host threads) on a bounded sample of the served workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "served update+SpMV req/s & p99 ms vs plain per-call DCSR; SpMV HBM GB/s"
L2_BYTES = 126 << 20


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one k = 1
# SpMV call (its two launches, k_rows1 + k_rows1_blocks) on the update-stream
# matrix, from one ncu capture of the same seeded workload in the same state
# (this file's stream part with --skip-batched --skip-spgemm --skip-served,
# the 4th roofline call): keyed by the matrix's stored-entry count, so a run
# on another state reports no traffic rather than a scaled one.
SPMV_TRAFFIC = {32832123: 235237120 + 3247104 + 118304256 + 560384}


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, tag: str):
        self.index = index
        self.proc = None
        # raw samples: $DCSR_BENCH_OUT if set, else the temp directory (the
        # JSON line carries their summary)
        out = os.environ.get("DCSR_BENCH_OUT") or tempfile.gettempdir()
        self.path = os.path.join(out, f"clocks_{tag}_rank{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def spmv_bytes(nnz, n, m, segs, k=1, sv=4):
    """Algorithmic SpMV bytes: entries (col+val), x and y, row lengths, segment pairs."""
    return nnz * (4 + sv) + k * sv * (m + n) + 4 * n + 8 * segs


def pct(a, q):
    return float(np.percentile(np.asarray(a), q)) if len(a) else None


# ------------------------------------------------------------ stream part

def stream_part(args, dev, world):
    import torch
    import torch.distributed as dist
    from dcsr_b200 import api
    from dcsr_b200 import workloads as W

    sc = args.stream_scale
    n, rp, cols, vals, batches = W.rmat_stream(args.seed, scale=sc, rounds=16, batch=1 << sc)
    nnz0 = int(rp[-1])
    A = api.DcsrMatrix(n, n, torch.float32)
    A.from_csr(torch.from_numpy(rp).to(dev), torch.from_numpy(cols).to(dev), torch.from_numpy(vals).to(dev))
    dbatch = [tuple(torch.from_numpy(a).to(dev) for a in b) for b in batches]
    # set-up: room in the device pool for the matrix to grow into (compaction
    # and repair allocate new pools; mapping new memory during the stream
    # would time the driver, not the library)
    api.pool_reserve(8 << 30)
    rng = np.random.default_rng(args.seed + 1)
    x = torch.from_numpy(rng.uniform(-1, 1, n).astype(np.float32)).to(dev)
    y = torch.empty(n, dtype=torch.float32, device=dev)
    rs = torch.empty(n, dtype=torch.float32, device=dev)
    cap = nnz0 + (2 * args.steps + args.warmup + 8) * len(batches[0][0]) + 1024
    out_rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    out_c = torch.empty(cap, dtype=torch.int32, device=dev)
    out_v = torch.empty(cap, dtype=torch.float32, device=dev)
    L = api.lib()
    h = A.h
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    def step(i, src=None):
        br, bc, bv = src if src is not None else dbatch[i % len(dbatch)]
        st = L.dcsr_update_sync(h, P(br), P(bc), P(bv), br.numel(), sp)
        if st != 0:
            raise RuntimeError(f"update failed: {api.status_string(st)}")
        assert L.dcsr_spmv(h, P(x), 1, 1, P(y), 1, 1.0, 0.0, sp) == 0
        assert L.dcsr_row_reduce(h, 0, P(rs), sp) == 0
        assert L.dcsr_to_csr(h, P(out_rp), P(out_c), P(out_v), sp) == 0

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    total_ms = evs[0].elapsed_time(evs[-1])
    per_step = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())

    # roofline: SpMV alone, L2 flushed before each launch
    lay = A.layout()
    segs = int((lay.seg.reshape(lay.max_segs, -1)[:, 0:2 * n:2] >= 0).sum())
    nnz = int(lay.row_sizes[:n].sum())
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    A.bin_rows()
    times = []
    for rep in range(args.spmv_reps + 3):
        flush.fill_(float(rep))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        assert L.dcsr_spmv(h, P(x), 1, 1, P(y), 1, 1.0, 0.0, sp) == 0
        e1.record(stream)
        torch.cuda.synchronize()
        if rep >= 3:
            times.append(e0.elapsed_time(e1))
    spmv_ms = statistics.mean(times)
    sb = spmv_bytes(nnz, n, n, segs)
    achieved = sb / (spmv_ms / 1e3) / 1e9

    def timed(fn, reps):
        """Mean device time (ms) of fn over reps launches, L2 flushed before each."""
        ts = []
        for rep in range(reps + 3):
            flush.fill_(float(rep))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            if rep >= 3:
                ts.append(e0.elapsed_time(e1))
        return statistics.mean(ts)

    hbm, _ = peaks()
    frac = lambda b, ms: round(b / (ms / 1e3) / 1e9 / hbm, 4)  # noqa: E731
    # gather floor: the same entries (this matrix's CSR export) read coalesced
    # with x gathered at every column, no row bookkeeping (dcsr_measure_gather)
    assert L.dcsr_to_csr(h, P(out_rp), P(out_c), P(out_v), sp) == 0
    gsum = torch.empty(148 * 8, dtype=torch.float32, device=dev)
    gather_ms = timed(lambda: L.dcsr_measure_gather(P(out_c), P(out_v), nnz, P(x), P(gsum), gsum.numel(), sp), 10)
    gather_bytes = nnz * 8 + 4 * n  # entries + x
    ops = {}
    # row sums alone (no gathers): nnz*sV + 4n + 8*segs + n*sV
    rs_ms = timed(lambda: L.dcsr_row_reduce(h, 0, P(rs), sp), 10)
    b = nnz * 4 + 4 * n + 8 * segs + 4 * n
    ops["row_sum"] = {"ms": round(rs_ms, 4), "bytes": b, "hbm_frac": frac(b, rs_ms)}
    # DCSR -> CSR export alone: 2*nnz*(4+sV) + 4(n+1) (+ the row lengths and segment table read)
    ex_ms = timed(lambda: L.dcsr_to_csr(h, P(out_rp), P(out_c), P(out_v), sp), 5)
    b = 2 * nnz * 8 + 4 * (n + 1)
    ops["export_csr"] = {"ms": round(ex_ms, 4), "bytes": b, "hbm_frac": frac(b, ex_ms)}
    # one update alone (1M skewed triples): T(8+sV) read + T_new(4+sV) written + 4*sum of touched rows' lengths
    br, bc, bv = dbatch[(args.warmup + args.steps) % len(dbatch)]
    touched = np.unique(br.cpu().numpy())
    nnz_before = nnz
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.fill_(0.5)
    e0.record(stream)
    st = L.dcsr_update_sync(h, P(br), P(bc), P(bv), br.numel(), sp)
    e1.record(stream)
    torch.cuda.synchronize()
    assert st == 0
    up_ms = e0.elapsed_time(e1)
    nnz_after = A.nnz()
    b = br.numel() * 12 + (nnz_after - nnz_before) * 8 + 4 * int(lay.row_sizes[touched].sum())
    ops["update"] = {"ms": round(up_ms, 4), "triples": int(br.numel()), "updates_per_s": round(br.numel() / (up_ms / 1e3), 1),
                     "bytes": b, "hbm_frac": frac(b, up_ms),
                     "note": "includes the batch sort and plan (their traffic is not in the algorithmic bytes)"}
    # compaction (defragmentation into a fresh pool): 2*nnz*(4+sV) + 16n
    e0.record(stream)
    A.compact()
    e1.record(stream)
    torch.cuda.synchronize()
    cp_ms = e0.elapsed_time(e1)
    b = 2 * nnz_after * 8 + 16 * n
    ops["compact"] = {"ms": round(cp_ms, 4), "bytes": b, "hbm_frac": frac(b, cp_ms),
                      "note": "includes its one synchronisation (pool size)"}
    # COO load of the initial matrix (unsorted triples): T(8+sV) in, nnz(4+sV) out, 16n layout
    rows0 = torch.repeat_interleave(torch.arange(n, dtype=torch.int32, device=dev),
                                    torch.from_numpy(np.diff(rp)).to(dev))
    perm = torch.randperm(nnz0, device=dev)
    r0, c0, v0 = rows0[perm], torch.from_numpy(cols).to(dev)[perm], torch.from_numpy(vals).to(dev)[perm]
    B = api.DcsrMatrix(n, n, torch.float32)
    B.from_coo(r0, c0, v0)
    torch.cuda.synchronize()
    e0.record(stream)
    B.from_coo(r0, c0, v0)
    e1.record(stream)
    torch.cuda.synchronize()
    ld_ms = e0.elapsed_time(e1)
    b = nnz0 * 12 + nnz0 * 8 + 16 * n
    ops["coo_load"] = {"ms": round(ld_ms, 4), "triples": nnz0, "bytes": b, "hbm_frac": frac(b, ld_ms),
                       "note": "unsorted triples; includes the radix sort and the load's one synchronisation"}
    del B, rows0, perm, r0, c0, v0

    # the same steps through host buffers (pinned), copies inside the timed region
    hb = [tuple(torch.from_numpy(a).pin_memory() for a in b) for b in batches]
    y_h = torch.empty(n, dtype=torch.float32).pin_memory()
    rs_h = torch.empty(n, dtype=torch.float32).pin_memory()
    stage = tuple(torch.empty_like(a, device=dev) for a in dbatch[0])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        src = hb[(args.warmup + args.steps + i) % len(hb)]
        for d, s_ in zip(stage, src):
            d.copy_(s_, non_blocking=True)
        step(0, stage)
        y_h.copy_(y, non_blocking=True)
        rs_h.copy_(rs, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    del A
    torch.cuda.synchronize()
    return {
        "workload": f"R-MAT 2^{sc} rows, (a,b,c,d)=(.57,.19,.19,.05), mean degree 16, FP32; 16 batches x "
                    f"2^{sc} triples, rows ~ current row length; step = update_sync + SpMV + row-sum + DCSR->CSR export",
        "req_s": round(world * args.steps / (total_ms / 1e3), 3),
        "req_s_host_buffers": round(args.steps / (e2e_ms / 1e3), 3),
        "ms_per_step": round(total_ms / args.steps, 4),
        "p50_ms": round(statistics.median(per_step), 4),
        "p99_ms": round(pct(per_step, 99), 4),
        "step_ms": [round(t, 3) for t in per_step],
        "updates_per_s": round(world * args.steps * len(batches[0][0]) / (total_ms / 1e3), 1),
        "nnz_initial": nnz0, "nnz_final": nnz, "rows": n,
        "spmv": {"ms": round(spmv_ms, 4), "bytes": int(sb), "gbs": round(achieved, 1),
                 "gather_floor_ms": round(gather_ms, 4), "gather_floor_bytes": gather_bytes},
        "ops": ops,
        "_host": (n, rp, cols, vals, batches),
    }


# ----------------------------------------------------------- SpGEMM part

def spgemm_part(args, dev):
    """C = A*A for the banded FP64 workload (2^17 rows, band half-width 2 +
    8 random off-band columns per row), then 100k update triples into A and
    C = A*A again; output entries per second, CUDA events."""
    import torch
    from dcsr_b200 import api
    from dcsr_b200 import workloads as W

    n, rp, cols, vals, (ur, uc, uv) = W.banded_spgemm(args.seed)
    api.pool_reserve(4 << 30)  # set-up: C's pools come from mapped memory, not fresh mappings inside the timing
    A = api.DcsrMatrix(n, n, torch.float64)
    A.from_csr(torch.from_numpy(rp).to(dev), torch.from_numpy(cols).to(dev), torch.from_numpy(vals).to(dev))
    C = api.DcsrMatrix(n, n, torch.float64)
    stream = torch.cuda.current_stream()
    for _ in range(2):  # warm-up
        A.spgemm(A, C)
    torch.cuda.synchronize()
    times, outs = [], []
    for rep in range(args.spgemm_reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        A.spgemm(A, C)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    nnz_c = C.nnz()
    A.update(torch.from_numpy(ur).to(dev), torch.from_numpy(uc).to(dev), torch.from_numpy(uv).to(dev))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    A.spgemm(A, C)
    e1.record(stream)
    torch.cuda.synchronize()
    after_ms = e0.elapsed_time(e1)
    nnz_c2 = C.nnz()
    ms = statistics.median(times)
    del A, C
    torch.cuda.synchronize()
    # algorithmic bytes: read A, the B rows its entries select (products x
    # (4 + sV)), write C (nnz_C x (4 + sV))
    lens = np.diff(rp).astype(np.int64)
    products = int((np.bincount(cols, minlength=n).astype(np.int64) * lens).sum())
    alg = int(rp[-1]) * 12 + 4 * n + products * 12 + nnz_c * 12
    hbm, _ = peaks()
    return {"workload": f"C = A*A, A 2^17 x 2^17 FP64, band half-width 2 + 8 random off-band columns per row "
                        f"({int(rp[-1])} nnz); then 100k update triples into A and C = A*A again",
            "ms": round(ms, 3), "nnz_c": int(nnz_c), "output_nnz_per_s": round(nnz_c / (ms / 1e3), 1),
            "products": products, "bytes": alg, "hbm_frac": round(alg / (ms / 1e3) / 1e9 / hbm, 4),
            "after_update_ms": round(after_ms, 3), "after_update_nnz_c": int(nnz_c2),
            "after_update_output_nnz_per_s": round(nnz_c2 / (after_ms / 1e3), 1),
            "note": "includes the operator's two host synchronisations (product count, C's pool top)",
            "_host": (n, rp, cols, vals)}


# ----------------------------------------------------------- batched part

def batched_part(args, dev):
    import torch
    from dcsr_b200 import api
    from dcsr_b200 import workloads as W

    specs = W.batched_specs(args.seed + 3, count=args.batched_mats)
    reps, warm = args.batched_reps, 3
    mats, work, per_mat = [], [], []
    nnz = 0
    for sp in specs:
        r, c, v = W.device_matrix(sp, dev)
        A = api.DcsrMatrix(sp["n"], sp["n"], torch.float32)
        A.from_coo(r, c, v)
        nnz += r.numel()
        del r, c, v
        k = sp["k"]
        x = torch.rand(sp["n"], k, device=dev) * 2 - 1
        y = torch.zeros(sp["n"], k, device=dev)
        per_mat.append([W.device_updates(sp, dev, i) for i in range(warm + reps)])
        mats.append(A)
        work.append(dict(matrix=A, x=x, y=y))
    # every round's triples of all matrices in one buffer per array (the way
    # a feed delivers a round); the batch reads them from one live buffer,
    # matrix i at its fixed offset, refilled by one copy per array per round
    sizes = [mr[0][0].numel() for mr in per_mat]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    rounds = [tuple(torch.cat([mr[i][a] for mr in per_mat]) for a in range(3)) for i in range(warm + reps)]
    per_mat.clear()
    live = tuple(t.clone() for t in rounds[0])
    for w, o0, o1 in zip(work, offs[:-1], offs[1:]):
        w["rows"], w["cols"], w["vals"] = (t[o0:o1] for t in live)
    torch.cuda.synchronize()
    api.pool_reserve(32 << 30)  # set-up: room for pool growth and repairs (mapped memory, not fresh mappings)
    s = torch.cuda.Stream()
    batch = api.DcsrBatch(work, stream=s)
    tuned = batch.autotune(s)  # row-class thresholds + short-row split for this set (outputs untouched)
    split = batch.short_split()
    batch.capture(s)
    T = sum(sp["updates"] for sp in specs)

    repaired = [0]
    grown = [0]
    repair_s = [0.0]
    grow_s = [0.0]
    rejected = np.zeros(9, np.int64)  # rejections by status code, timed rounds

    def batched_round(i):
        for dst, src in zip(live, rounds[i]):
            dst.copy_(src, non_blocking=True)
        batch.launch(s)
        st = batch.status(s)  # synchronises: the graph's work is done here
        t0 = time.perf_counter()
        rejected[:] += np.bincount(np.asarray(st), minlength=9)[:9]
        if (st != 0).any():
            repaired[0] += batch.repair(st, s)
            s.synchronize()
        t1 = time.perf_counter()
        grown[0] += batch.grow(s)  # pools left short of room, grown ahead of the next round
        s.synchronize()
        repair_s[0] += t1 - t0
        grow_s[0] += time.perf_counter() - t1

    with torch.cuda.stream(s):
        for i in range(warm):
            batched_round(i)
        s.synchronize()
        launches0 = api.launch_count()
        fallback0 = api.pool_usage()[2]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        repaired[0] = grown[0] = 0
        repair_s[0] = grow_s[0] = 0.0
        rejected[:] = 0
        for i in range(reps):
            batched_round(warm + i)
        e1.record(s)
        s.synchronize()
        batched_ms = e0.elapsed_time(e1) / reps
        repairs_per_round = repaired[0] / reps
        repair_ms_per_round = 1e3 * repair_s[0] / reps
        batched_launches = (api.launch_count() - launches0) / reps
        regions = api.pool_usage()
        fallback_allocs = regions[2] - fallback0
        # plain per-call sequences on the same matrices (fresh update rounds)
        L = api.lib()
        sp_ = C.c_void_p(s.cuda_stream)
        P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        e0.record(s)
        launches0 = api.launch_count()
        for i in range(reps):
            rd = rounds[(warm + i) % len(rounds)]
            for w, o0, o1 in zip(work, offs[:-1], offs[1:]):
                r, c, v = (t[o0:o1] for t in rd)
                st = L.dcsr_update_sync(w["matrix"].h, P(r), P(c), P(v), r.numel(), sp_)
                assert st == 0, api.status_string(st)
                k = w["x"].shape[1]
                assert L.dcsr_spmv(w["matrix"].h, P(w["x"]), k, k, P(w["y"]), k, 1.0, 0.0, sp_) == 0
        e1.record(s)
        s.synchronize()
        plain_ms = e0.elapsed_time(e1) / reps
        plain_launches = (api.launch_count() - launches0) / reps
    batch.close()
    del work, rounds, live, per_mat, mats
    torch.cuda.synchronize()
    return {
        "workload": f"{len(specs)} matrices, rows log-uniform [1k,256k], mean degree U[4,64], FP32, "
                    f"{nnz / 1e6:.0f}M nnz; per matrix an update (log-uniform 100..100k, {T / 1e6:.2f}M triples "
                    "in all) + SpMV with k in {1,2,4,8}",
        "autotuned_row_classes": {"short_max": tuned[0], "long_min": tuned[1], "short_split": split,
                                  "spmv_pass_us": round(tuned[2], 1)},
        "batched_ms": round(batched_ms, 3), "plain_ms": round(plain_ms, 3),
        "speedup": round(plain_ms / batched_ms, 2),
        "batched_kernel_launches": round(batched_launches, 1), "plain_kernel_launches": round(plain_launches, 1),
        "repairs_per_round": repairs_per_round, "repair_ms_per_round": round(repair_ms_per_round, 3),
        "pools_grown_ahead_per_round": grown[0] / reps, "grow_ms_per_round": round(1e3 * grow_s[0] / reps, 3),
        "reserved_regions_gib": round(regions[0] / 2**30, 1),
        "allocations_outside_regions_timed": int(fallback_allocs),
        "rejections_per_round": {"pool_exhausted": round(float(rejected[1]) / reps, 2),
                                 "layer_overflow": round(float(rejected[2]) / reps, 2)},
        "updates_per_s_batched": round(T / (batched_ms / 1e3), 1),
    }


# ------------------------------------------------------------ served part

class ServedTrace:
    """Request arrays (ctypes dcsr_request) over device or pinned host buffers."""

    def __init__(self, api, torch, dev, specs, kind, mat, size, seed, export_cap, on_device):
        n_of = np.array([sp["n"] for sp in specs], np.int64)
        self.count = len(kind)
        upd = np.nonzero(kind == 0)[0]
        Ts = size[upd].astype(np.int64)
        off = np.zeros(len(upd) + 1, np.int64)
        off[1:] = np.cumsum(Ts)
        total = int(off[-1])
        g = torch.Generator(device=dev)
        g.manual_seed(seed)
        lim = torch.from_numpy(np.repeat(n_of[mat[upd]], Ts)).to(dev)
        rows = (torch.rand(total, device=dev, generator=g, dtype=torch.float64) * lim).to(torch.int32)
        cols = (torch.rand(total, device=dev, generator=g, dtype=torch.float64) * lim).to(torch.int32)
        vals = torch.rand(total, device=dev, generator=g) * 2 - 1
        del lim
        max_n = int(n_of.max())
        if on_device:
            self.rows, self.cols, self.vals = rows, cols, vals
            self.x = torch.rand(max_n * 8, device=dev, generator=g) * 2 - 1
            self.y = torch.empty(64, max_n * 8, device=dev)
            self.erp = torch.empty(4, max_n + 1, dtype=torch.int32, device=dev)
            self.ec = torch.empty(4, export_cap, dtype=torch.int32, device=dev)
            self.ev = torch.empty(4, export_cap, device=dev)
        else:
            self.rows, self.cols, self.vals = (t.cpu().pin_memory() for t in (rows, cols, vals))
            self.x = (torch.rand(max_n * 8, device=dev, generator=g) * 2 - 1).cpu().pin_memory()
            self.y = torch.empty(64, max_n * 8).pin_memory()
            self.erp = torch.empty(4, max_n + 1, dtype=torch.int32).pin_memory()
            self.ec = torch.empty(4, export_cap, dtype=torch.int32).pin_memory()
            self.ev = torch.empty(4, export_cap).pin_memory()
        reqs = (api.Request * self.count)()
        ui = {int(j): q for q, j in enumerate(upd)}
        rb, cb, vb = self.rows.data_ptr(), self.cols.data_ptr(), self.vals.data_ptr()
        n_spmv = n_exp = 0
        for j in range(self.count):
            r = reqs[j]
            r.kind, r.matrix, r.on_device = int(kind[j]), int(mat[j]), int(on_device)
            if kind[j] == 0:
                q = ui[j]
                o = int(off[q])
                r.rows, r.cols, r.vals, r.nnz = rb + 4 * o, cb + 4 * o, vb + 4 * o, int(Ts[q])
            elif kind[j] == 1:
                r.x, r.y, r.k = self.x.data_ptr(), self.y[n_spmv % 64].data_ptr(), int(size[j])
                r.alpha, r.beta = 1.0, 0.0
                n_spmv += 1
            else:
                e = n_exp % 4
                r.row_ptr, r.out_cols, r.out_vals = self.erp[e].data_ptr(), self.ec[e].data_ptr(), self.ev[e].data_ptr()
                r.cap = export_cap
                n_exp += 1
        self.reqs = reqs
        self.triples = total


def replay(api, srv, trace, arrivals, lo=0, hi=None):
    hi = trace.count if hi is None else hi
    n = hi - lo
    res = (api.Result * n)()
    arr = np.ascontiguousarray(arrivals[:n], dtype=np.float64)
    wall = C.c_double()
    base = C.addressof(trace.reqs) + lo * C.sizeof(api.Request)
    st = api.lib().dcsr_server_replay(srv.h, C.c_void_p(base), arr.ctypes.data_as(C.c_void_p), n, C.byref(res),
                                      C.byref(wall))
    assert st == 0, api.status_string(st)
    lat = np.array([r.latency_us for r in res]) / 1e3
    bad = sum(1 for r in res if r.status != 0)
    sizes = np.array([r.batch_size for r in res])
    return {"requests": n, "wall_ms": wall.value / 1e3, "req_s": n / (wall.value / 1e6), "p50_ms": pct(lat, 50),
            "p99_ms": pct(lat, 99), "errors": bad, "mean_batch": float(sizes.mean())}


def capacity(api, srv, trace, n, lo=0, hi=None, runs=3):
    """A server's capacity: `runs` closed-loop replays (all requests queued at
    once), the median-throughput run standing for it.  A single replay can
    take a stall of the device pool mapping new memory (tens to hundreds of
    ms) and would then set every load point of the sweep too low."""
    rs = sorted((replay(api, srv, trace, np.zeros(n), lo, hi) for _ in range(runs)), key=lambda r: r["req_s"])
    pick = dict(rs[len(rs) // 2])
    pick["req_s_runs"] = [round(r["req_s"], 1) for r in rs]
    return pick


def replay_point(api, srv, trace, rate, n, seed, repeats, lo=0, hi=None):
    """`repeats` Poisson replays at one offered rate (different arrival seeds);
    the run with the median p99 stands for the point (a single run's p99 rests
    on its 1% slowest requests), with every run's p99 listed beside it."""
    runs = []
    for j in range(repeats):
        launches0 = api.launch_count()
        r = replay(api, srv, trace, poisson_arrivals(rate, n, seed + 1000 * j), lo, hi)
        r["kernel_launches"] = api.launch_count() - launches0
        runs.append(r)
    order = sorted(range(len(runs)), key=lambda j: runs[j]["p99_ms"])
    pick = dict(runs[order[len(runs) // 2]])
    pick["p99_ms_runs"] = [round(r["p99_ms"], 3) for r in runs]
    pick["offered_req_s"] = rate
    return pick


def host_link_gbs(torch, dev, nbytes=1 << 30):
    """Pinned host <-> device copy bandwidth (GB/s), best of 3 each way."""
    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    out = {}
    for name, dst, src in (("h2d_gbs", d, h), ("d2h_gbs", h, d)):
        best = None
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dst.copy_(src, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name] = round(nbytes / (best / 1e3) / 1e9, 1)
    del h, d
    return out


def poisson_arrivals(rate_per_s, n, seed):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1e6 / rate_per_s, n))


def served_part(args, dev, rank, local_rank):
    import torch
    from dcsr_b200 import api
    from dcsr_b200 import workloads as W

    from dcsr_b200 import shard
    world = int(os.environ.get("WORLD_SIZE", 1))
    # one global table of served_mats matrices per GPU, sharded by device bytes
    specs_all = W.batched_specs(args.seed + 5, count=args.served_mats * world)
    owner = shard.partition([shard.matrix_bytes(sp["n"], sp["n"], int(sp["n"] * sp["degree"])) for sp in specs_all],
                            world)
    mine, _ = shard.local_view(owner, rank)
    specs = [specs_all[i] for i in mine]
    mats, nnz, resident = [], 0, 0
    for sp in specs:
        r, c, v = W.device_matrix(sp, dev)
        A = api.DcsrMatrix(sp["n"], sp["n"], torch.float32)
        A.from_coo(r, c, v)
        nnz += r.numel()
        del r, c, v
        inf = A.info()
        resident += inf.pool_cap * 8 + (sp["n"] + 1) * 4 + inf.pitch * 4 * inf.opts.max_segs
        mats.append(A)
    torch.cuda.synchronize()
    # set-up: row-class thresholds of the served matrices from the batch
    # autotuner (an SpMV of every matrix, k = 4; both servers use the result)
    tuned = None
    if not args.no_served_autotune:
        xs = [torch.zeros(sp["n"], 4, device=dev) for sp in specs]
        ys = [torch.zeros(sp["n"], 4, device=dev) for sp in specs]
        tb = api.DcsrBatch([dict(matrix=A, x=x, y=y) for A, x, y in zip(mats, xs, ys)])
        tuned = tb.autotune()
        tb.close()
        del xs, ys
        torch.cuda.synchronize()
    # the global trace; this rank serves the requests addressed to its matrices
    kind_g, mat_g, size_g = W.served_trace(args.seed + 6, len(specs_all), args.served_requests * world)
    sel, local = shard.route(mat_g, owner, rank)
    kind, mat, size = kind_g[sel], local.astype(np.int32), size_g[sel]
    N = len(kind)
    passes = 12  # replays of the trace below (bounds the growth of every matrix)
    grow = np.bincount(mat[kind == 0], weights=size[kind == 0], minlength=len(mats))
    export_cap = int(max(sp["n"] * sp["degree"] * 1.2 + 64 * np.sqrt(sp["n"] * sp["degree"]) + passes * g
                         for sp, g in zip(specs, grow)))
    tr_dev = ServedTrace(api, torch, dev, specs, kind, mat, size, args.seed + 7, export_cap, True)
    tr_host = ServedTrace(api, torch, dev, specs, kind, mat, size, args.seed + 7, export_cap, False)
    torch.cuda.synchronize()
    # set-up: free reserved regions for the pools that grow during the trace
    api.pool_reserve(16 << 30)
    fallback0 = api.pool_usage()[2]
    out = {"workload": f"{len(specs)} resident matrices like the batched ones ({nnz / 1e9:.2f}G nnz, "
                       f"{resident / 2**30:.1f} GiB resident); {N} requests: 40% update (log-uniform 10..100k "
                       "triples), 50% SpMV (k uniform 1..8), 10% DCSR->CSR export; matrices uniform"}
    # plain per-call server: capacity, then Poisson loads; its p99 at the
    # highest load is the latency target both servers are compared at (with
    # device buffers for `value`, with host buffers for `e2e`)
    Np = min(N, args.plain_requests)

    def plain_sweep(tr):
        srv = api.DcsrServer(mats, plain=True)
        replay(api, srv, tr, np.zeros(Np), 0, Np)  # warm-up: one full pass (first-touch schedules, pool growth)
        cap = capacity(api, srv, tr, Np, 0, Np)
        pts = []
        for f in args.plain_fracs:
            r = replay_point(api, srv, tr, f * cap["req_s"], Np, args.seed + 8, args.repeats, 0, Np)
            pts.append({k: (round(v, 3) if not isinstance(v, list) else v) for k, v in r.items()})
        srv.close()
        ref = pts[-1]
        return {"capacity_req_s": round(cap["req_s"], 1), "capacity_runs": cap["req_s_runs"], "sweep": pts,
                "slo_point": {"load_frac": args.plain_fracs[-1], "req_s": ref["req_s"], "p99_ms": ref["p99_ms"]}}

    out["plain"] = plain_sweep(tr_dev)
    out["plain_host_buffers"] = plain_sweep(tr_host)
    fallback1 = api.pool_usage()[2]
    ref_p = out["plain"]["slo_point"]
    cap_p = {"req_s": out["plain"]["capacity_req_s"]}
    p99_plain = ref_p["p99_ms"]
    # batched server; the clock sampler starts before the warm-up pass (its
    # start-up queries the driver, which must not fall in a measured sweep)
    sampler = ClockSampler(local_rank, "served")
    sampler.start()

    def sweep_at(tr, p99_plain):
        """Capacity, then Poisson loads; the highest throughput whose p99 is at
        or below the plain path's target (else the lowest-p99 point, flagged)."""
        replay(api, srv, tr, np.zeros(N))  # warm-up: one full pass
        cap = capacity(api, srv, tr, N)
        pts, best, best_f = [], None, None
        for f in args.load_fracs:
            r = replay_point(api, srv, tr, f * cap["req_s"], N, args.seed + 9, args.repeats)
            pts.append({k: (round(v, 3) if not isinstance(v, list) else v) for k, v in r.items()})
            if r["p99_ms"] <= p99_plain and r["errors"] == 0 and (best is None or r["req_s"] > best["req_s"]):
                best, best_f = r, f
        met = best is not None
        if not met:
            best, best_f = min(((s_, f) for s_, f in zip(pts, args.load_fracs)), key=lambda t: t[0]["p99_ms"])
        return cap, pts, best, best_f, met

    srv = api.DcsrServer(mats, max_batch=args.max_batch, depth=args.depth, workers=args.workers)
    cap_s, sweep, best, best_f, met = sweep_at(tr_dev, p99_plain)
    clocks = sampler.stop()
    # end to end: the same rule with pinned host buffers (inputs copied in,
    # results copied out per request; exports move whole matrices to the host)
    cap_h, sweep_h, e2e, e2e_f, e2e_met = sweep_at(tr_host, out["plain_host_buffers"]["slo_point"]["p99_ms"])
    st = srv.stats()
    fallback2 = api.pool_usage()[2]
    srv.close()
    # bytes each request of the host-buffer run moved (mean over the trace)
    n_of = np.array([sp["n"] for sp in specs], np.int64)
    nnz_now = np.array([m.nnz() for m in mats], np.int64)
    nm = n_of[mat]
    h2d = np.where(kind == 0, 12 * size, np.where(kind == 1, 4 * nm * size, 0)).sum()
    d2h = np.where(kind == 1, 4 * nm * size, np.where(kind == 2, 4 * (nm + 1) + 8 * nnz_now[mat], 0)).sum()
    del tr_dev, tr_host, mats
    torch.cuda.synchronize()
    out["served"] = {"capacity_req_s": round(cap_s["req_s"], 1), "capacity_runs": cap_s["req_s_runs"],
                     "mean_batch_at_capacity": round(cap_s["mean_batch"], 1),
                     "sweep": sweep, "chosen_load_frac": best_f, "p99_constraint_met": met,
                     "batches": st["batches"], "max_batch": args.max_batch, "depth": args.depth,
                     "workers": args.workers,
                     "allocations_outside_regions": {"plain": int(fallback1 - fallback0),
                                                     "batched": int(fallback2 - fallback1)},
                     "row_classes": None if tuned is None else {"short_max": tuned[0], "long_min": tuned[1]}}
    out["value"] = best["req_s"]
    out["chosen"] = {"requests": best["requests"], "wall_ms": best["wall_ms"]}
    out["p50_ms"] = best["p50_ms"]
    out["p99_ms"] = best["p99_ms"]
    out["speedup_at_equal_p99"] = round(best["req_s"] / ref_p["req_s"], 2)
    out["speedup_vs_plain_capacity"] = round(best["req_s"] / cap_p["req_s"], 2)
    out["e2e"] = {k: (round(v, 3) if not isinstance(v, list) else v) for k, v in e2e.items()}
    out["e2e"].update({"capacity_req_s": round(cap_h["req_s"], 1), "capacity_runs": cap_h["req_s_runs"],
                       "chosen_load_frac": e2e_f,
                       "p99_constraint_met": e2e_met, "sweep": sweep_h,
                       "speedup_at_equal_p99": round(e2e["req_s"] / out["plain_host_buffers"]["slo_point"]["req_s"], 2)})
    out["e2e"]["h2d_bytes_per_request"] = int(h2d / N)
    out["e2e"]["d2h_bytes_per_request"] = int(d2h / N)
    # the host link: pinned copies of 1 GiB each way, and the request rate it
    # bounds the host-buffer form to (bytes per request / bandwidth, the two
    # directions overlapping)
    link = host_link_gbs(torch, dev)
    bound = min(link["h2d_gbs"] * 1e9 / max(h2d / N, 1), link["d2h_gbs"] * 1e9 / max(d2h / N, 1))
    out["e2e"]["host_link"] = {**link, "req_s_bound": round(bound, 1),
                               "capacity_frac_of_bound": round(cap_h["req_s"] / bound, 3)}
    out["launches"] = int(best["kernel_launches"])
    out["clocks"] = clocks
    return out


# ------------------------------------------------------------ CPU (reference) leg

class RefServed:
    """The reference's cusp host path (oracle/_ref, OpenMP on all host
    threads) serving a sample of the served workload: the first n_mats matrix
    specs, generated on the host once, and the trace's requests mapped onto
    them, one at a time (update = cusp::add of the triples, SpMV = one
    cusp::multiply per right-hand side, export = a copy of the CSR arrays)."""

    def __init__(self, args, n_mats=64):
        from dcsr_b200 import workloads as W
        from oracle import oracle as O
        self.ref = O.Ref(seq=False)
        self.specs = W.batched_specs(args.seed + 5, count=args.served_mats)[:n_mats]
        self.hs = []
        for sp in self.specs:
            rng = np.random.default_rng(sp["seed"])
            rp, cols = W.poisson_matrix(rng, sp["n"], sp["n"], sp["degree"])
            vals = rng.uniform(-1, 1, cols.size).astype(np.float32)
            self.hs.append(self.ref.L.ref_res_create(sp["n"], sp["n"], rp, cols, vals))
        self.kind, self.mat, self.size = W.served_trace(args.seed + 6, args.served_mats, 1 << 16)
        self.rng = np.random.default_rng(args.seed + 7)
        self.next = 0

    def serve(self, n_req):
        """Serve the trace's next n_req requests; returns their latencies (ms) and the wall time (s)."""
        lat = []
        t0 = time.perf_counter()
        for _ in range(n_req):
            j = self.next % len(self.kind)
            self.next += 1
            i = int(self.mat[j]) % len(self.hs)
            n = self.specs[i]["n"]
            ts = time.perf_counter()
            if self.kind[j] == 0:
                T = int(self.size[j])
                self.ref.L.ref_res_update(self.hs[i], self.rng.integers(0, n, T).astype(np.int32),
                                          self.rng.integers(0, n, T).astype(np.int32),
                                          self.rng.uniform(-1, 1, T).astype(np.float32), T)
            elif self.kind[j] == 1:
                k = int(self.size[j])
                x = self.rng.uniform(-1, 1, n * k).astype(np.float32)
                y = np.empty(n * k, np.float32)
                self.ref.L.ref_res_spmv(self.hs[i], x, k, y)
            else:
                cap = int(self.specs[i]["n"] * self.specs[i]["degree"] * 2 + 200000)
                self.ref.L.ref_res_export(self.hs[i], np.empty(n + 1, np.int32), np.empty(cap, np.int32),
                                          np.empty(cap, np.float32))
            lat.append(1e3 * (time.perf_counter() - ts))
        return lat, time.perf_counter() - t0

    def close(self):
        for h in self.hs:
            self.ref.L.ref_res_free(h)
        self.hs = []

    def sample_text(self, n_req):
        return (f"{n_req} requests of the served trace on its first {len(self.specs)} matrices (host-generated), "
                "served one at a time by cusp::add / cusp::multiply / CSR copy (OpenMP)")


def reference_served_sample(args, n_req=400):
    srv = RefServed(args)
    srv.serve(8)  # warm-up
    lat, dt = srv.serve(n_req)
    out = {"value": round(n_req / dt, 3), "unit": "req/s", "cores": srv.ref.threads(), "kind": "reference",
           "p50_ms": round(pct(lat, 50), 3), "p99_ms": round(pct(lat, 99), 3), "sample": srv.sample_text(n_req)}
    srv.close()
    return out


def cpu_ops_baseline(args, stream_host, spgemm_host):
    """The reference's cusp host path on the update stream's step (cusp::add
    of a 1M-triple batch, then SpMV, row sums -- SpMV with x = 1 -- and the
    CSR copy) and on the SpGEMM workload (cusp::multiply), once on one thread
    (the sequential host system) and once on all host threads (OpenMP)."""
    from oracle import oracle as O
    out = {}
    if stream_host is not None:
        n, rp, cols, vals, batches = stream_host
        x = np.random.default_rng(args.seed + 1).uniform(-1, 1, n)
        rows = {}
        for seq in (True, False):
            ref = O.Ref(seq=seq)
            h = ref.L.ref_stream_create(n, n, rp, cols, vals.astype(np.float64), x)
            y, rsum = np.empty(n), np.empty(n)
            ts = []
            for b in batches[:2]:
                t0 = time.perf_counter()
                ref.L.ref_stream_step(h, b[0], b[1], b[2].astype(np.float64), len(b[0]), y, rsum)
                ts.append(time.perf_counter() - t0)
            ref.L.ref_stream_free(h)
            rows["1_thread" if seq else f"{ref.threads()}_threads"] = {"step_s": round(statistics.mean(ts), 4)}
        out["stream_step"] = {"workload": "R-MAT 2^20 update-stream step: cusp::add of 1M triples + SpMV + row "
                                          "sums + CSR copy (first two batches)", **rows}
    if spgemm_host is not None:
        n, rp, cols, vals = spgemm_host
        rows = {}
        for seq in (True, False):
            ref = O.Ref(seq=seq)
            t0 = time.perf_counter()
            R = ref.spgemm(O.F64, n, n, n, rp, cols, vals, rp, cols, vals)
            dt = time.perf_counter() - t0
            rows["1_thread" if seq else f"{ref.threads()}_threads"] = {
                "s": round(dt, 4), "output_nnz_per_s": round(len(R[1]) / dt, 1)}
        out["spgemm"] = {"workload": "C = A*A, banded 2^17 FP64 (cusp::multiply)", **rows}
    return out


def run_reference(args):
    from oracle import oracle as O
    if not O.Ref.available(seq=False):
        return {"impl": "reference", "unavailable": "oracle/_ref (the reference's cusp host path) is not built"}
    srv = RefServed(args)
    for _ in range(args.warmup):
        srv.serve(4)
    # the sample (ref_requests requests) split across the timed steps
    per = max(1, args.ref_requests // max(args.steps, 1))
    lat, wall = [], 0.0
    for _ in range(args.steps):
        l_, dt = srv.serve(per)
        lat += l_
        wall += dt
    value = len(lat) / wall
    sample = srv.sample_text(len(lat))
    cores = srv.ref.threads()
    srv.close()
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "req/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * wall / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded served workload sample, generated on the host)",
        "config": {"workload": "served: matrices like the batched ones, 40/50/10 update/SpMV/export requests",
                   "sample": sample, "parallelism": "host OpenMP"},
        "p50_ms": round(pct(lat, 50), 3), "p99_ms": round(pct(lat, 99), 3),
        "cpu_baseline": {"value": round(value, 3), "unit": "req/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "req/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------------- main

def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    hbm, peak_kind = peaks()

    stream = stream_part(args, dev, world) if not args.skip_stream else None
    spgemm = spgemm_part(args, dev) if not args.skip_spgemm else None
    batched = batched_part(args, dev) if not args.skip_batched else None
    if args.skip_served:  # profiling runs of the other parts only
        strip = lambda d: None if d is None else {k: v for k, v in d.items() if not k.startswith("_")}  # noqa: E731
        return {"stream": strip(stream), "batched": batched, "spgemm": strip(spgemm)}
    served = served_part(args, dev, rank, local_rank)

    # aggregate over ranks: requests of all ranks / the slowest rank's wall time
    from dcsr_b200 import shard
    value, _, _ = shard.aggregate(served["chosen"]["requests"], served["chosen"]["wall_ms"] / 1e3)
    e2e_value, _, _ = shard.aggregate(served["e2e"]["requests"], served["e2e"]["wall_ms"] / 1e3)
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "req/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 / served["value"], 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; served/batched matrices generated on the device, R-MAT stream on the host)",
        "config": {"workload": "served: " + served["workload"],
                   "headline": "batched-server req/s at the highest Poisson load whose p99 <= the plain per-call "
                               "server's p99 at its highest load (90% of its capacity); device-resident request "
                               f"buffers; each load point the median-p99 of {args.repeats} replays",
                   "parallelism": f"matrix shards x{world} (no data-path collective)",
                   "step": f"one served request (ms_per_step = 1/value); `steps`/`warmup` are the update-stream "
                           f"part's; the served sweep replays {args.served_requests} requests per load point, "
                           f"{len(args.load_fracs)} load points x {args.repeats} replays, after a warm-up pass",
                   "l2": "working sets > L2 (60 GB resident; SpMV roofline flushes L2 between launches)"},
        "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"],
        "plain": served["plain"], "plain_host_buffers": served["plain_host_buffers"], "served": served["served"],
        "speedup_at_equal_p99": served["speedup_at_equal_p99"],
        "speedup_at_equal_p99_host_buffers": served["e2e"]["speedup_at_equal_p99"],
        "speedup_vs_plain_capacity": served["speedup_vs_plain_capacity"],
        "e2e": {"value": round(e2e_value, 3), "unit": "req/s", "p99_ms": served["e2e"]["p99_ms"],
                "capacity_req_s": served["e2e"]["capacity_req_s"], "p99_constraint_met": served["e2e"]["p99_constraint_met"],
                "speedup_at_equal_p99": served["e2e"]["speedup_at_equal_p99"],
                "sweep": served["e2e"]["sweep"],
                "host_link": served["e2e"].get("host_link"),
                "h2d_bytes_per_step": served["e2e"]["h2d_bytes_per_request"],
                "d2h_bytes_per_step": served["e2e"]["d2h_bytes_per_request"],
                "note": "a step is one request: its triples or x copied in from pinned host memory, its y or CSR "
                        "copied out (means over the trace)"},
        "gpu_launches": served["launches"],
        "clocks": served["clocks"],
    }
    if stream is not None:
        sp = stream["spmv"]
        traffic = SPMV_TRAFFIC.get(stream["nnz_final"])
        out["spmv_gbs"] = sp["gbs"]
        out["roofline"] = {"kernel": "k_rows1 (DCSR SpMV, k=1, FP32: one launch over long-row chunks, medium rows "
                                     "and short-row blocks; R-MAT 2^20 after the update stream)",
                           "bound": "hbm", "achieved": sp["gbs"], "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                           "frac": round(sp["gbs"] / hbm, 4), "traffic": traffic, "bytes_per_launch": sp["bytes"],
                           "avg_ms": sp["ms"],
                           "gather_floor": {
                               "ms": sp["gather_floor_ms"],
                               "frac_of_hbm": round(sp["bytes"] / (sp["gather_floor_ms"] / 1e3) / 1e9 / hbm, 4),
                               "note": "dcsr_measure_gather over the same entries (CSR export: int32 columns, FP32 "
                                       "values, coalesced) gathering x at each column, no row bookkeeping: the "
                                       "SpMV's data movement at best on this GPU; frac_of_hbm = the SpMV's "
                                       "algorithmic bytes over that time"}}
        out["stream"] = {k: v for k, v in stream.items() if not k.startswith("_")}
    if batched is not None:
        out["batched"] = batched
    if spgemm is not None:
        out["spgemm"] = {k: v for k, v in spgemm.items() if not k.startswith("_")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = reference_served_sample(args, n_req=args.ref_requests)
            out["cpu_ops"] = cpu_ops_baseline(args, stream["_host"] if stream is not None else None,
                                              spgemm["_host"] if spgemm is not None else None)
        except FileNotFoundError as e:
            out["cpu_baseline"] = {"unavailable": str(e)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--spmv-reps", type=int, default=20)
    ap.add_argument("--served-mats", type=int, default=2000)
    ap.add_argument("--served-requests", type=int, default=20000)
    ap.add_argument("--plain-requests", type=int, default=6000)
    ap.add_argument("--max-batch", type=int, default=256)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--repeats", type=int, default=3, help="Poisson replays per served load point (median p99)")
    ap.add_argument("--load-fracs", type=float, nargs="+",
                    default=[0.3, 0.4, 0.5, 0.55, 0.6, 0.625, 0.65, 0.675, 0.7, 0.725, 0.75, 0.8, 0.85])
    ap.add_argument("--plain-fracs", type=float, nargs="+", default=[0.5, 0.7, 0.9])
    ap.add_argument("--batched-mats", type=int, default=512)
    ap.add_argument("--batched-reps", type=int, default=5)
    ap.add_argument("--ref-requests", type=int, default=400)
    ap.add_argument("--skip-stream", action="store_true")
    ap.add_argument("--stream-scale", type=int, default=20, help="profiling: log2 rows of the update-stream matrix")
    ap.add_argument("--skip-batched", action="store_true")
    ap.add_argument("--skip-spgemm", action="store_true")
    ap.add_argument("--spgemm-reps", type=int, default=5)
    ap.add_argument("--skip-served", action="store_true", help="profiling: no headline line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-served-autotune", action="store_true", help="served matrices keep the default row classes")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", local_rank))
    out = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
