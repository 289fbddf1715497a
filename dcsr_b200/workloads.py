"""Seeded synthetic DCSR workloads (host-side numpy generators).

No public dataset is used: every matrix and update stream here is generated
from a fixed seed with the shapes and value distributions of the five DCSR
workloads:

* ``small_plain``      n=4096 square FP32, diagonal + Poisson(12) distinct
                       uniform columns per row; 4 rounds x 8192 update
                       triples (row uniform, column 50% an existing entry /
                       50% uniform, value U(-1,1)).
* ``rmat_stream``      R-MAT 2^20 rows, (a,b,c,d)=(.57,.19,.19,.05), mean
                       degree 16, FP32 U(0,1); 16 rounds x 1M triples whose
                       rows are drawn proportional to the row's current length.
* ``banded_spgemm``    2^17 square FP64, band half-width 2 plus 8 distinct
                       uniform off-band columns per row, N(0,1); 100k uniform
                       update triples.
* ``batched``          512 matrices, rows log-uniform [1k, 256k], mean degree
                       U[4, 64] with Poisson row lengths, FP32 U(-1,1); update
                       batches log-uniform [100, 100k]; SpMV with k in {1,2,4,8}.
* ``served``           2000 resident matrices drawn like ``batched``.
* ``spd_matrix``       a symmetric, strictly diagonally dominant (so positive
                       definite) matrix for the CG solver, and update batches
                       that keep it so.

Generators return CSR (row_ptr, cols, vals) with rows sorted and unique, and
update batches as COO (rows, cols, vals) in batch order.
"""
from __future__ import annotations

import numpy as np


def _csr_from_keys(keys: np.ndarray, n_rows: int, n_cols: int):
    keys = np.sort(keys, kind="stable")
    if keys.size:
        keep = np.empty(keys.size, bool)
        keep[0] = True
        np.not_equal(keys[1:], keys[:-1], out=keep[1:])
        keys = keys[keep]
    rows = (keys // n_cols).astype(np.int32)
    cols = (keys % n_cols).astype(np.int32)
    counts = np.bincount(rows, minlength=n_rows)
    row_ptr = np.zeros(n_rows + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return row_ptr.astype(np.int32), cols, rows


def poisson_matrix(rng, n_rows, n_cols, mean_deg, diag=False):
    """Rows with Poisson(mean_deg) distinct uniform columns (+ the diagonal)."""
    lens = rng.poisson(mean_deg, n_rows).astype(np.int64)
    lens = np.minimum(lens, n_cols)
    rows = np.repeat(np.arange(n_rows, dtype=np.int64), lens)
    cols = rng.integers(0, n_cols, rows.size, dtype=np.int64)
    keys = rows * n_cols + cols
    if diag:
        d = np.arange(min(n_rows, n_cols), dtype=np.int64)
        keys = np.concatenate([keys, d * n_cols + d])
    row_ptr, c, r = _csr_from_keys(keys, n_rows, n_cols)
    return row_ptr, c


def small_plain(seed: int = 0, n: int = 4096, n_rounds: int = 4, T: int = 8192):
    """Small plain workload: returns (n, row_ptr, cols, vals, rounds)."""
    rng = np.random.default_rng(seed)
    row_ptr, cols = poisson_matrix(rng, n, n, 12.0, diag=True)
    vals = rng.uniform(-1.0, 1.0, cols.size).astype(np.float32)
    rounds = []
    lens = np.diff(row_ptr)
    for _ in range(n_rounds):
        r = rng.integers(0, n, T).astype(np.int32)
        existing = rng.random(T) < 0.5
        pick = (rng.random(T) * lens[r]).astype(np.int64)
        c_exist = cols[row_ptr[r] + pick]
        c_new = rng.integers(0, n, T)
        c = np.where(existing, c_exist, c_new).astype(np.int32)
        v = rng.uniform(-1.0, 1.0, T).astype(np.float32)
        rounds.append((r, c, v))
    return n, row_ptr, cols, vals, rounds


def rmat_edges(rng, scale: int, n_edges: int, probs=(0.57, 0.19, 0.19, 0.05)):
    """R-MAT edge list (rows, cols) with 2^scale vertices, before dedup."""
    a, b, c, _ = probs
    rows = np.zeros(n_edges, np.int64)
    cols = np.zeros(n_edges, np.int64)
    for level in range(scale):
        u = rng.random(n_edges, dtype=np.float32)
        rbit = u >= (a + b)
        cbit = ((u >= a) & (u < a + b)) | (u >= (a + b + c))
        rows |= rbit.astype(np.int64) << level
        cols |= cbit.astype(np.int64) << level
    return rows, cols


def rmat_stream(seed: int = 0, scale: int = 20, degree: int = 16, rounds: int = 16,
                batch: int = 1 << 20):
    """Power-law update stream: returns (n, row_ptr, cols, vals, batches).

    Batch rows are drawn proportional to the row's current length, tracked on
    the host as (initial length + triples drawn for the row so far), which
    bounds the true length from above and needs no device round trip."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    r, c = rmat_edges(rng, scale, degree * n)
    row_ptr, cols, _ = _csr_from_keys(r * n + c, n, n)
    vals = rng.random(cols.size, dtype=np.float32)
    cur = np.diff(row_ptr).astype(np.float64)
    batches = []
    for _ in range(rounds):
        cdf = np.cumsum(cur)
        cdf /= cdf[-1]
        br = np.searchsorted(cdf, rng.random(batch), side="right").astype(np.int32)
        br = np.minimum(br, n - 1)
        bc = rng.integers(0, n, batch).astype(np.int32)
        bv = rng.random(batch, dtype=np.float32)
        cur += np.bincount(br, minlength=n)
        batches.append((br, bc, bv))
    return n, row_ptr, cols, vals, batches


def banded_spgemm(seed: int = 0, scale: int = 17, half_width: int = 2, off_band: int = 8,
                  n_updates: int = 100_000):
    """SpGEMM workload: returns (n, row_ptr, cols, vals[f64], update batch)."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    rr = np.arange(n, dtype=np.int64)
    keys = []
    for d in range(-half_width, half_width + 1):
        cc = rr + d
        ok = (cc >= 0) & (cc < n)
        keys.append(rr[ok] * n + cc[ok])
    band = np.concatenate(keys)
    # off-band columns: draw with replacement, then keep distinct off-band ones
    extra_r = np.repeat(rr, off_band * 2)
    extra_c = rng.integers(0, n, extra_r.size)
    off = np.abs(extra_c - extra_r) > half_width
    ek = np.unique(extra_r[off] * n + extra_c[off])
    er = ek // n
    # keep the first `off_band` distinct off-band columns of each row
    first = np.searchsorted(er, rr)
    rank = np.arange(ek.size) - first[er]
    ek = ek[rank < off_band]
    row_ptr, cols, _ = _csr_from_keys(np.concatenate([band, ek]), n, n)
    vals = rng.standard_normal(cols.size)
    ur = rng.integers(0, n, n_updates).astype(np.int32)
    uc = rng.integers(0, n, n_updates).astype(np.int32)
    uv = rng.standard_normal(n_updates)
    return n, row_ptr, cols, vals, (ur, uc, uv)


def batched_specs(seed: int = 0, count: int = 512, min_rows: int = 1000, max_rows: int = 256_000,
                  min_upd: int = 100, max_upd: int = 100_000):
    """Per-matrix specs for the batched / served workloads: list of dicts
    with rows, mean degree, update-batch size and RHS count."""
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(np.log(min_rows), np.log(max_rows), count)).astype(np.int64)
    deg = rng.uniform(4.0, 64.0, count)
    upd = np.exp(rng.uniform(np.log(min_upd), np.log(max_upd), count)).astype(np.int64)
    k = rng.choice([1, 2, 4, 8], count)
    return [dict(index=i, n=int(rows[i]), degree=float(deg[i]), updates=int(upd[i]), k=int(k[i]),
                 seed=int(seed * 1_000_003 + i)) for i in range(count)]


def batched_matrix(spec):
    """Matrix + update batch + RHS block for one batched/served spec."""
    rng = np.random.default_rng(spec["seed"])
    n = spec["n"]
    row_ptr, cols = poisson_matrix(rng, n, n, spec["degree"])
    vals = rng.uniform(-1.0, 1.0, cols.size).astype(np.float32)
    T = spec["updates"]
    ur = rng.integers(0, n, T).astype(np.int32)
    uc = rng.integers(0, n, T).astype(np.int32)
    uv = rng.uniform(-1.0, 1.0, T).astype(np.float32)
    x = rng.uniform(-1.0, 1.0, (n, spec["k"])).astype(np.float32)
    return row_ptr, cols, vals, (ur, uc, uv), x


def device_matrix(spec, dev, dtype=None):
    """One batched/served matrix generated on the device (seeded torch
    generator): COO (rows, cols, vals) with Poisson(degree) entries per row,
    uniform columns (duplicate pairs are summed by a MERGE-mode load) and
    U(-1,1) values."""
    import torch
    dtype = dtype or torch.float32
    g = torch.Generator(device=dev)
    g.manual_seed(spec["seed"])
    n = spec["n"]
    lens = torch.poisson(torch.full((n,), float(spec["degree"]), device=dev), generator=g).to(torch.int64)
    lens.clamp_(max=n)
    rows = torch.repeat_interleave(torch.arange(n, device=dev, dtype=torch.int32), lens)
    cols = torch.randint(0, n, (rows.numel(),), device=dev, dtype=torch.int32, generator=g)
    vals = torch.rand(rows.numel(), device=dev, dtype=dtype, generator=g) * 2 - 1
    return rows, cols, vals


def device_updates(spec, dev, rnd=0, dtype=None):
    """Update batch `rnd` of a batched/served spec, on the device: uniform
    rows and columns, U(-1,1) values."""
    import torch
    dtype = dtype or torch.float32
    g = torch.Generator(device=dev)
    g.manual_seed(spec["seed"] * 7919 + 1 + rnd)
    n, T = spec["n"], spec["updates"]
    r = torch.randint(0, n, (T,), device=dev, dtype=torch.int32, generator=g)
    c = torch.randint(0, n, (T,), device=dev, dtype=torch.int32, generator=g)
    v = torch.rand(T, device=dev, dtype=dtype, generator=g) * 2 - 1
    return r, c, v


def served_trace(seed: int, n_mats: int, count: int, min_upd: int = 10, max_upd: int = 100_000):
    """Request mix of the served workload: (kind, matrix, size) with kind 0 =
    update (40%, log-uniform [10, 100k] triples), 1 = SpMV (50%, k uniform in
    1..8), 2 = export (10%); matrices uniform."""
    rng = np.random.default_rng(seed)
    u = rng.random(count)
    kind = np.where(u < 0.4, 0, np.where(u < 0.9, 1, 2)).astype(np.int32)
    mat = rng.integers(0, n_mats, count).astype(np.int32)
    upd = np.exp(rng.uniform(np.log(min_upd), np.log(max_upd), count)).astype(np.int64)
    k = rng.integers(1, 9, count).astype(np.int32)
    size = np.where(kind == 0, upd, np.where(kind == 1, k, 0))
    return kind, mat, size


def spd_matrix(seed: int = 0, n: int = 4096, degree: float = 6.0):
    """Symmetric, strictly diagonally dominant matrix with a positive diagonal
    (hence positive definite): returns CSR (row_ptr, cols, vals[f64]) with
    rows sorted and unique."""
    rng = np.random.default_rng(seed)
    rp, cols = poisson_matrix(rng, n, n, degree / 2)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    off = rows != cols
    rows, cols = rows[off], cols[off].astype(np.int64)
    v = rng.uniform(-1.0, 1.0, rows.size)
    # symmetric: (i, j) and (j, i) with the same value, duplicates summed
    keys = np.concatenate([rows * n + cols, cols * n + rows])
    vals = np.concatenate([v, v])
    order = np.argsort(keys, kind="stable")
    keys, vals = keys[order], vals[order]
    uk, start = np.unique(keys, return_index=True)
    sv = np.add.reduceat(vals, start) if keys.size else vals
    r, c = uk // n, uk % n
    absrow = np.bincount(r, weights=np.abs(sv), minlength=n)
    keys = np.concatenate([uk, np.arange(n, dtype=np.int64) * (n + 1)])
    vals = np.concatenate([sv, absrow + 1.0])
    order = np.argsort(keys, kind="stable")
    keys, vals = keys[order], vals[order]
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(keys // n, minlength=n), out=row_ptr[1:])
    return row_ptr.astype(np.int32), (keys % n).astype(np.int32), vals


def spd_updates(seed: int, n: int, pairs: int):
    """COO update batch that keeps spd_matrix's properties: each pair (i, j),
    i != j, adds v at (i, j) and (j, i) and 2|v| at (i, i) and (j, j)."""
    rng = np.random.default_rng(seed)
    i = rng.integers(0, n, pairs)
    j = (i + rng.integers(1, n, pairs)) % n
    v = rng.uniform(-1.0, 1.0, pairs)
    rows = np.concatenate([i, j, i, j]).astype(np.int32)
    cols = np.concatenate([j, i, i, j]).astype(np.int32)
    vals = np.concatenate([v, v, 2 * np.abs(v), 2 * np.abs(v)])
    return rows, cols, vals
