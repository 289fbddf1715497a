"""DCSR update-stream benchmark (one JSON line on rank 0).

Workload (per GPU, weak scaling, independent replicas -- no collective on the
data path): the power-law update stream -- an R-MAT graph with 2^20 rows,
(a,b,c,d) = (.57,.19,.19,.05), mean degree 16, FP32 U(0,1) values, and 16
pre-generated batches of 1M update triples whose rows follow the current row
lengths.  One step = one request = one batch merged into the DCSR matrix
(dcsr_update_sync: sort, duplicate merge, slack insertion / chaining /
relocation, compaction when the pool or layers run out), then y = A x,
row sums, and DCSR -> CSR export.  Batches cycle through the 16 rounds.

value   requests/s with inputs resident in HBM, CUDA events on the launching
        stream, max over ranks; the working set (pool >= 250 MB) exceeds the
        126 MB L2, so no flush is needed between steps.
e2e     the same requests through the C ABI with host buffers: batch copied
        from pinned host memory, y and row sums copied back, each step.
roofline the top kernel of the step (SpMV), timed alone with an L2 flush.

--impl reference times the reference's own CPU implementation (its cusp
host path, OpenMP, all host threads: cusp::add + SpMV + row sums + CSR copy)
on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
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


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{index}.csv")

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


# ------------------------------------------------------------------ ours

def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from dcsr_b200 import api
    from dcsr_b200 import workloads as W

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n, rp, cols, vals, batches = W.rmat_stream(args.seed, rounds=16)
    nnz0 = int(rp[-1])
    A = api.DcsrMatrix(n, n, torch.float32)
    A.from_csr(torch.from_numpy(rp).to(dev), torch.from_numpy(cols).to(dev), torch.from_numpy(vals).to(dev))
    dbatch = [tuple(torch.from_numpy(a).to(dev) for a in b) for b in batches]
    rng = np.random.default_rng(args.seed + 1)
    x = torch.from_numpy(rng.uniform(-1, 1, n).astype(np.float32)).to(dev)
    y = torch.empty(n, dtype=torch.float32, device=dev)
    rs = torch.empty(n, dtype=torch.float32, device=dev)
    cap = nnz0 + (args.steps + args.warmup + args.e2e_steps + 8) * len(batches[0][0]) + 1024
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
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    launches0 = api.launch_count()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    torch.cuda.synchronize()
    evs[0].record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    launches = api.launch_count() - launches0
    clocks = sampler.stop()
    total_ms = evs[0].elapsed_time(evs[-1])
    per_step = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)

    # --- roofline: SpMV alone, L2 flushed before each launch
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
    hbm, peak_kind = peaks()
    achieved = sb / (spmv_ms / 1e3) / 1e9

    # --- e2e: host buffers through the C ABI, copies inside the timed region
    hb = [tuple(torch.from_numpy(a).pin_memory() for a in b) for b in batches]
    y_h = torch.empty(n, dtype=torch.float32).pin_memory()
    rs_h = torch.empty(n, dtype=torch.float32).pin_memory()
    stage = tuple(torch.empty_like(a, device=dev) for a in dbatch[0])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_t0 = torch.cuda.Event(enable_timing=True)
    e2e_t1 = torch.cuda.Event(enable_timing=True)
    e2e_t0.record(stream)
    for i in range(args.e2e_steps):
        src = hb[(args.warmup + args.steps + i) % len(hb)]
        for d, s_ in zip(stage, src):
            d.copy_(s_, non_blocking=True)
        step(0, stage)
        y_h.copy_(y, non_blocking=True)
        rs_h.copy_(rs, non_blocking=True)
    e2e_t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e2e_t0.elapsed_time(e2e_t1)
    t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
    h2d = sum(a.numel() * a.element_size() for a in hb[0])
    d2h = 2 * n * 4

    out = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "req/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded R-MAT + update stream, generated on the host)",
        "config": {
            "workload": "rmat_stream: R-MAT 2^20 rows, (a,b,c,d)=(.57,.19,.19,.05), mean degree 16, FP32; "
                        "16 batches x 1M triples, rows ~ current row length",
            "request": "1M-triple merged update + SpMV + row-sum + DCSR->CSR export",
            "rows": n, "nnz_initial": nnz0, "nnz_final": nnz, "batch": len(batches[0][0]),
            "parallelism": f"replicas x{world} (no collective)",
            "l2": "working set > L2 (no flush needed between steps)",
        },
        "p50_ms": round(statistics.median(per_step), 4),
        "p99_ms": round(float(np.percentile(per_step, 99)), 4),
        "updates_per_s": round(value * len(batches[0][0]), 1),
        "spmv_gbs": round(achieved, 1),
        "e2e": {"value": round(world * args.e2e_steps / (e2e_ms / 1e3), 3), "unit": "req/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "k_spmv (DCSR SpMV, k=1, FP32)", "bound": "hbm", "achieved": round(achieved, 1),
                     "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "traffic": None, "bytes_per_launch": int(sb), "avg_ms": round(spmv_ms, 4)},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, n, rp, cols, vals, batches)
    return out


def cpu_baseline(args, n, rp, cols, vals, batches, steps=2):
    """The reference's cusp host path (OpenMP, all host threads) on the same
    matrix: `steps` update rounds, each cusp::add + SpMV + row sums + CSR copy."""
    from oracle import oracle as O
    try:
        ref = O.Ref(seq=False)
    except FileNotFoundError as e:
        return {"unavailable": str(e)}
    hnd = ref.L.ref_stream_create(n, n, rp, cols, vals.astype(np.float64), np.ones(n))
    y = np.zeros(n)
    rs = np.zeros(n)
    t0 = time.perf_counter()
    for i in range(steps):
        b = batches[i % len(batches)]
        ref.L.ref_stream_step(hnd, b[0], b[1], b[2].astype(np.float64), len(b[0]), y, rs)
    dt = time.perf_counter() - t0
    ref.L.ref_stream_free(hnd)
    return {"value": round(steps / dt, 4), "unit": "req/s", "cores": ref.threads(), "kind": "reference",
            "sample": f"{steps} full update rounds of the same workload (cusp::add + SpMV + row-sum + CSR copy)"}


def run_reference(args):
    from dcsr_b200 import workloads as W
    from oracle import oracle as O
    try:
        ref = O.Ref(seq=False)
    except FileNotFoundError as e:
        return {"impl": "reference", "unavailable": f"oracle/_ref not built: {e}"}
    n, rp, cols, vals, batches = W.rmat_stream(args.seed, rounds=16)
    hnd = ref.L.ref_stream_create(n, n, rp, cols, vals.astype(np.float64), np.ones(n))
    y = np.zeros(n)
    rs = np.zeros(n)
    for i in range(args.warmup):
        b = batches[i % 16]
        ref.L.ref_stream_step(hnd, b[0], b[1], b[2].astype(np.float64), len(b[0]), y, rs)
    times = []
    t0 = time.perf_counter()
    for i in range(args.steps):
        b = batches[(args.warmup + i) % 16]
        ts = time.perf_counter()
        ref.L.ref_stream_step(hnd, b[0], b[1], b[2].astype(np.float64), len(b[0]), y, rs)
        times.append(time.perf_counter() - ts)
    dt = time.perf_counter() - t0
    ref.L.ref_stream_free(hnd)
    value = args.steps / dt
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "req/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded R-MAT + update stream, generated on the host)",
        "config": {"workload": "rmat_stream: R-MAT 2^20 rows, mean degree 16, FP32; 16 batches x 1M triples",
                   "request": "cusp::add(A, batch) + SpMV + row-sum (SpMV with x=1) + CSR copy",
                   "parallelism": "host OpenMP"},
        "p50_ms": round(1e3 * statistics.median(times), 3),
        "p99_ms": round(1e3 * float(np.percentile(times, 99)), 3),
        "cpu_baseline": {"value": round(value, 4), "unit": "req/s", "cores": ref.threads(), "kind": "reference",
                         "sample": f"{args.steps} full update rounds"},
        "e2e": {"value": round(value, 4), "unit": "req/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--spmv-reps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
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
