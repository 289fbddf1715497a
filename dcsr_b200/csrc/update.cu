// update.cu -- in-place batch updates of a DCSR matrix and COO grouping.
//
// Pipeline (all on the caller's stream, no host synchronisation):
//   keys     (row,col) keys with an index check            k_make_keys
//   sort     stable LSD radix sort of (key, batch index)    radix_sort_pairs
//   bucket   sorted columns/values + per-row batch ranges   k_gather_sorted, scan, k_touched
//   plan     per touched row: duplicate search, new length, capacity, new
//            segment size and layer (no mutation)           k_plan_merge / k_plan_append
//   alloc    exclusive scan of new segment sizes (deterministic, row order)
//   check    pool / layer / index verdict -> go flag         k_check
//   apply    warp per row: merge in place (or append)       k_apply_merge / k_apply_append
//   relocate rows whose in-place shift would exceed reloc_min are merged out
//            of place into a fresh segment, tile-parallel   k_relocate
//   finish   chain reset of relocated rows, new pool top    k_finish
// A rejected batch (status != OK) leaves the matrix untouched.
//
// Reference: device::UpdateMatrix include/load.h:258-325 and UpdateMatrix_dcsr
// include/sparse_update.inl:16-130 (segment walk, bump allocation, layer
// linking).  The reference appends without merging and allocates with
// atomicAdd; here MERGE mode keeps rows sorted and unique (duplicates summed
// in batch order) and the allocation is a row-ordered scan, so layouts are
// reproducible bit for bit.
#include "internal.cuh"

namespace dcsr {

constexpr int UPD_THREADS = 256;
constexpr int RT_TILE = 1024;  // relocation: outputs per tile
constexpr int RT_THREADS = 256;
constexpr int RT_ITEMS = RT_TILE / RT_THREADS;

enum { AUX_BAD_INDEX = 1, AUX_LAYER_OVF = 2 };

__device__ __forceinline__ unsigned lanemask_lt_u() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ int32_t key_row(unsigned long long k, int cb, int merge) {
  return merge ? (int32_t)(k >> cb) : (int32_t)k;
}

__global__ void k_make_keys(const int32_t *rows, const int32_t *cols, int64_t n, int32_t n_rows, int32_t n_cols,
                            int cb, int merge, unsigned long long *keys, unsigned *perm, long long *stat) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    int32_t r = rows[i], c = cols[i];
    if (r < 0 || r >= n_rows || c < 0 || c >= n_cols) {
      atomicOr((unsigned long long *)&stat[ST_AUX], (unsigned long long)AUX_BAD_INDEX);
      r = 0;
      c = 0;
    }
    keys[i] = merge ? (((unsigned long long)r << cb) | (unsigned long long)c) : (unsigned long long)r;
    perm[i] = (unsigned)i;
  }
}

template <typename V>
__global__ void k_gather_sorted(const unsigned long long *keys, const unsigned *perm, const int32_t *cols,
                                const V *vals, int64_t n, int cb, int merge, int32_t n_cols, int32_t *bcol,
                                V *bval, long long *hflag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const unsigned long long cmask = (1ull << cb) - 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    unsigned long long k = keys[i];
    unsigned p = perm[i];
    int32_t c = merge ? (int32_t)(k & cmask) : cols[p];
    if (c < 0 || c >= n_cols) c = 0;  // rejected batch; keeps later reads in range
    bcol[i] = c;
    bval[i] = vals[p];
    hflag[i] = (i == 0 || key_row(keys[i - 1], cb, merge) != key_row(k, cb, merge)) ? 1 : 0;
  }
}

__global__ void k_touched(const unsigned long long *keys, int64_t n, int cb, int merge, const long long *hpos,
                          int32_t *trow, int32_t *tb0) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    int32_t r = key_row(keys[i], cb, merge);
    bool head = i == 0 || key_row(keys[i - 1], cb, merge) != r;
    if (head) {
      trow[hpos[i]] = r;
      tb0[hpos[i]] = (int32_t)i;
    }
    if (i == n - 1) tb0[hpos[i] + (head ? 1 : 0)] = (int32_t)n;
  }
}

// --------------------------------------------------------------- planning

// Sub-warp of S lanes (S divides 32): lane-local mask, ballot and helpers.
template <int S>
struct Sub {
  int sl, sw;
  unsigned mask;
  __device__ __forceinline__ Sub() {
    const int lane = lane_id();
    sl = lane & (S - 1);
    sw = lane / S;
    mask = S == 32 ? FULL : (((1u << S) - 1u) << (sw * S));
  }
  __device__ __forceinline__ unsigned ballot(bool p) const {
    const unsigned b = __ballot_sync(mask, p);
    return S == 32 ? b : (b >> (sw * S)) & ((1u << S) - 1u);
  }
  __device__ __forceinline__ unsigned full() const { return S == 32 ? FULL : (1u << S) - 1u; }
  template <typename T>
  __device__ __forceinline__ T shfl(T v, int src) const { return __shfl_sync(mask, v, src, S); }
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  __device__ __forceinline__ int incl_scan(int v) const {
#pragma unroll
    for (int o = 1; o < S; o <<= 1) {
      const int w = __shfl_up_sync(mask, v, o, S);
      if (sl >= o) v += w;
    }
    return v;
  }
  // consecutive set bits of a lane-local ballot starting at bit 0
  __device__ __forceinline__ int leading(unsigned bm) const { return bm == full() ? S : __ffs(~bm) - 1; }
};

constexpr int PLAN_S = 8;     // lanes per touched row in the plan
constexpr int SMALL_AFF = 96; // apply: rows shifting <= this many entries use 8-lane sub-warps

// MERGE plan, step 1 (thread per batch entry): every (row, col) group head
// binary-searches its column in the row: bpos = position (existing) or
// ~insertion point (new); nflag = 1 for new columns.
template <typename V>
__global__ void k_head_search(Mat<V> m, const unsigned long long *keys, int64_t T, int cb, const int32_t *bcol,
                              int32_t *bpos, long long *nflag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= T; i += stride) {
    if (i == T) {
      nflag[T] = 0;
      continue;
    }
    const unsigned long long k = keys[i];
    long long isnew = 0;
    if (i == 0 || keys[i - 1] != k) {
      const int32_t r = (int32_t)(k >> cb);
      const int32_t c = bcol[i];
      const int64_t L = m.row_sizes[r];
      const Chain ch = load_chain(m, r);
      int64_t lo = 0, hi = L;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(m.cols + ch.phys(mid)) < c) lo = mid + 1;
        else hi = mid;
      }
      isnew = !(lo < L && __ldg(m.cols + ch.phys(lo)) == c);
      bpos[i] = isnew ? ~(int32_t)lo : (int32_t)lo;
    }
    nflag[i] = isnew;
  }
}

// MERGE plan, step 2 (thread per batch entry): new groups are written, in
// column order, to slot b0 + k of their row (k from the scan of nflag), with
// their batch-order sum.
template <typename V>
__global__ void k_new_compact(const unsigned long long *keys, int64_t T, int cb, const int32_t *bcol, const V *bval,
                              const int32_t *bpos, const long long *nflag_excl, const long long *hpos,
                              const int32_t *tb0, int32_t *ncol, V *nval, int32_t *nins) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T; i += stride) {
    const unsigned long long k = keys[i];
    if (i > 0 && keys[i - 1] == k) continue;
    if (bpos[i] >= 0) continue;  // existing column
    const bool rowhead = i == 0 || (keys[i - 1] >> cb) != (k >> cb);
    const int64_t t = hpos[i] - (rowhead ? 0 : 1);
    const int32_t b0 = tb0[t];
    const int64_t slot = b0 + (nflag_excl[i] - nflag_excl[b0]);
    V v = bval[i];
    for (int64_t j = i + 1; j < T && keys[j] == k; j++) v = v + bval[j];
    ncol[slot] = bcol[i];
    nval[slot] = v;
    nins[slot] = ~bpos[i];
  }
}

// MERGE plan, step 3 (thread per touched row): new length, capacity, layer,
// relocation decision and apply width class.
template <typename V>
__global__ void k_row_plan(Mat<V> m, int64_t T, const int32_t *trow, const int32_t *tb0, const long long *nflag_excl,
                           const int32_t *nins, long long *tcap, long long *ttiles, int32_t *tmnew, int32_t *tinfo) {
  const int64_t nt = m.stat[ST_TOUCHED];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= T; t += stride) {
    if (t >= nt) {
      tcap[t] = 0;
      ttiles[t] = 0;
      continue;
    }
    const int32_t r = trow[t];
    const int32_t b0 = tb0[t], b1 = tb0[t + 1];
    const int64_t L = m.row_sizes[r];
    const int64_t mnew = nflag_excl[b1] - nflag_excl[b0];
    const int64_t ins0 = mnew > 0 ? nins[b0] : L;
    const Chain ch = load_chain(m, r);
    const int64_t nl = L + mnew;
    int64_t cap = 0;
    int layer = -1, reloc = 0, big = 0;
    if (mnew > 0 && L - ins0 > m.o.reloc_min) {
      reloc = 1;
      layer = 0;
      cap = policy_cap(m.o, nl);
    } else {
      big = mnew > 0 && L - ins0 > SMALL_AFF;
      if (nl > ch.total) {
        cap = align_up(policy_cap(m.o, nl) - ch.total, m.o.align);
        layer = ch.total == 0 ? 0 : ch.ns;
        if (layer >= m.max_segs) atomicOr((unsigned long long *)&m.stat[ST_AUX], (unsigned long long)AUX_LAYER_OVF);
      }
    }
    tcap[t] = cap;
    ttiles[t] = reloc ? div_up(nl, RT_TILE) : 0;
    tmnew[t] = (int32_t)mnew;
    tinfo[t] = (layer & 0xff) | (reloc << 8) | (big << 9) | ((mnew > 0 || cap > 0) ? (1 << 10) : 0);
  }
}

// Apply, step 1 (thread per batch group): existing columns take their batch
// values in batch order, in place, before any shift or relocation reads them.
template <typename V>
__global__ void k_apply_existing(Mat<V> m, const unsigned long long *keys, int64_t T, int cb, const V *bval,
                                 const int32_t *bpos) {
  if (!m.stat[ST_GO]) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T; i += stride) {
    const unsigned long long k = keys[i];
    if (i > 0 && keys[i - 1] == k) continue;
    const int32_t p = bpos[i];
    if (p < 0) continue;
    const Chain ch = load_chain(m, (int32_t)(k >> cb));
    const int64_t q = ch.phys(p);
    V v = m.vals[q];
    for (int64_t j = i; j < T && keys[j] == k; j++) v = v + bval[j];
    m.vals[q] = v;
  }
}

template <typename V>
__global__ void __launch_bounds__(UPD_THREADS) k_plan_merge(Mat<V> m, int64_t T, const int32_t *trow,
                                                            const int32_t *tb0, const int32_t *bcol, const V *bval,
                                                            int32_t *bpos, long long *tcap, long long *ttiles,
                                                            int32_t *tmnew, int32_t *tinfo, int32_t *ncol, V *nval,
                                                            int32_t *nins) {
  constexpr int S = PLAN_S;
  const int64_t nt = m.stat[ST_TOUCHED];
  const int64_t gthreads = (int64_t)gridDim.x * blockDim.x;
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t t = gtid; t <= T; t += gthreads)
    if (t >= nt) {
      tcap[t] = 0;
      ttiles[t] = 0;
    }
  const Sub<S> sub;
  const unsigned lt = (1u << sub.sl) - 1u;
  for (int64_t t = gtid / S; t < nt; t += gthreads / S) {
    const int32_t r = trow[t];
    const int32_t b0 = tb0[t], b1 = tb0[t + 1];
    const int64_t L = m.row_sizes[r];
    const Chain ch = load_chain(m, r);
    int32_t mnew = 0;
    int64_t ins0 = L;
    for (int32_t base = b0; base < b1; base += S) {
      const int32_t i = base + sub.sl;
      const bool valid = i < b1;
      const int32_t c = valid ? bcol[i] : 0;
      const bool head = valid && (i == b0 || bcol[i - 1] != c);
      int64_t pos = 0;
      bool isnew = false;
      if (head) {
        int64_t lo = 0, hi = L;
        while (lo < hi) {
          const int64_t mid = (lo + hi) >> 1;
          if (__ldg(m.cols + ch.phys(mid)) < c) lo = mid + 1;
          else hi = mid;
        }
        pos = lo;
        isnew = !(lo < L && __ldg(m.cols + ch.phys(lo)) == c);
        bpos[i] = isnew ? ~(int32_t)pos : (int32_t)pos;
      }
      const unsigned nm = sub.ballot(isnew);
      if (nm) {
        if (isnew) {
          const int32_t k = mnew + __popc(nm & lt);
          V v = bval[i];
          for (int32_t j = i + 1; j < b1 && bcol[j] == c; j++) v = v + bval[j];
          ncol[b0 + k] = c;
          nval[b0 + k] = v;
          nins[b0 + k] = (int32_t)pos;
        }
        const int64_t p0 = sub.shfl(pos, __ffs(nm) - 1);
        if (mnew == 0) ins0 = p0;
        mnew += __popc(nm);
      }
    }
    if (sub.sl == 0) {
      const int64_t nl = L + mnew;
      int64_t cap = 0;
      int layer = -1, reloc = 0, big = 0;
      if (mnew > 0 && L - ins0 > m.o.reloc_min) {
        reloc = 1;
        layer = 0;
        cap = policy_cap(m.o, nl);
      } else {
        big = mnew > 0 && L - ins0 > SMALL_AFF;
        if (nl > ch.total) {
          cap = align_up(policy_cap(m.o, nl) - ch.total, m.o.align);
          layer = ch.total == 0 ? 0 : ch.ns;
          if (layer >= m.max_segs)
            atomicOr((unsigned long long *)&m.stat[ST_AUX], (unsigned long long)AUX_LAYER_OVF);
        }
      }
      tcap[t] = cap;
      ttiles[t] = reloc ? div_up(nl, RT_TILE) : 0;
      tmnew[t] = mnew;
      tinfo[t] = (layer & 0xff) | (reloc << 8) | (big << 9);
    }
  }
}

// APPEND mode: the reference's segment walk and allocation size.
template <typename V>
__global__ void k_plan_append(Mat<V> m, int64_t T, const int32_t *trow, const int32_t *tb0, long long *tcap,
                              long long *ttiles, int32_t *tmnew, int32_t *tinfo) {
  const int64_t nt = m.stat[ST_TOUCHED];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= T; t += stride) {
    if (t >= nt) {
      tcap[t] = 0;
      ttiles[t] = 0;
      continue;
    }
    const int32_t r = trow[t];
    const int64_t rlB = tb0[t + 1] - tb0[t];
    const int64_t rlA = m.row_sizes[r];
    const int2 l0 = *reinterpret_cast<const int2 *>(m.seg + 2 * (int64_t)r);
    int64_t cap = 0;
    int layer = -1;
    if (rlA == 0 && l0.x == l0.y) {
      cap = rlB + m.o.alpha;
      layer = 0;
    } else {
      // segment holding position rlA (reference walk :77-88): the first
      // whose cumulative capacity reaches rlA; free = that capacity - rlA
      const Chain ch = load_chain(m, r);
      int off = 0;
      int64_t before = 0, after = 0;
      bool found = false;
#pragma unroll
      for (int i = 0; i < MAX_SEGS; i++) {
        if (!found && i < ch.ns) {
          after = before + ch.cp[i];
          off = i;
          if (after >= rlA || i + 1 >= ch.ns) found = true;
          else before = after;
        }
      }
      const int64_t fr = after - rlA;
      if (fr < rlB) {
        cap = rlB - fr + m.o.alpha;
        layer = off + 1;
        if (layer >= m.max_segs) atomicOr((unsigned long long *)&m.stat[ST_AUX], (unsigned long long)AUX_LAYER_OVF);
      }
    }
    tcap[t] = cap;
    ttiles[t] = 0;
    tmnew[t] = (int32_t)rlB;
    tinfo[t] = layer & 0xff;
  }
}

__global__ void k_check(long long *stat, const int32_t *row_sizes, int32_t n_rows, int64_t pool_cap) {
  const long long aux = stat[ST_AUX];
  const long long top = row_sizes[n_rows];
  const long long need = top + stat[ST_TOTAL];
  stat[ST_NEED] = need;
  int st = DCSR_OK;
  if (aux & AUX_BAD_INDEX) st = DCSR_BAD_INDEX;
  else if (aux & AUX_LAYER_OVF) st = DCSR_LAYER_OVERFLOW;
  else if (need > pool_cap || need > 0x7fffffffLL) st = DCSR_POOL_EXHAUSTED;
  stat[ST_GO] = st == DCSR_OK ? 1 : 0;
  if (st != DCSR_OK && stat[ST_STATUS] == 0) stat[ST_STATUS] = st;
  stat[ST_AUX] = 0;
}

// --------------------------------------------------------------- applying

// Old pool top of the running update (row_sizes[n] is only rewritten by k_finish).
__device__ __forceinline__ long long old_top(const long long *stat) { return stat[ST_NEED] - stat[ST_TOTAL]; }

// Apply for the rows of one width class: S = 8 takes rows shifting at most
// SMALL_AFF entries (and rows without shifts), S = 32 takes the larger ones.
template <typename V, int S>
__global__ void __launch_bounds__(UPD_THREADS) k_apply_merge(Mat<V> m, const int32_t *trow, const int32_t *tb0,
                                                             const int32_t *bcol, const V *bval,
                                                             const int32_t *bpos, const long long *addr,
                                                             const int32_t *tmnew, const int32_t *tinfo,
                                                             const int32_t *ncol, const V *nval,
                                                             const int32_t *nins) {
  if (!m.stat[ST_GO]) return;
  __shared__ int hist[UPD_THREADS / S][S];
  const int64_t nt = m.stat[ST_TOUCHED];
  const long long top = old_top(m.stat);
  const Sub<S> sub;
  int *h = hist[threadIdx.x / S];
  const int64_t gthreads = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / S; t < nt; t += gthreads / S) {
    const int info = tinfo[t];
    if (!((info >> 10) & 1) || ((info >> 9) & 1) != (S == 32 ? 1 : 0) || ((info >> 8) & 1)) continue;
    const int32_t r = trow[t];
    const int32_t b0 = tb0[t], b1 = tb0[t + 1];
    const int64_t L = m.row_sizes[r];
    const bool reloc = (info >> 8) & 1;
    const int layer = (int8_t)(info & 0xff);
    const int32_t mnew = tmnew[t];
    const long long cap = addr[t + 1] - addr[t];
    Chain ch = load_chain(m, r);
    if (!reloc && cap > 0) {
      const int32_t st = (int32_t)(top + addr[t]);
      ch.append(st, (int32_t)cap, layer == 0);
      if (sub.sl == 0)
        *reinterpret_cast<int2 *>(m.seg + (int64_t)layer * m.pitch + 2 * (int64_t)r) =
            make_int2(st, (int32_t)(st + cap));
    }
    // (existing columns were updated by k_apply_existing)
    if (!reloc && mnew > 0) {
      // 2. shift the entries after the first insertion point, back to front,
      //    S per step; shift(i) = #{new k : nins[k] <= i}
      const int32_t *ins = nins + b0;
      const int64_t lo_a = ins[0];
      int32_t khi = mnew;
      for (;;) {
        const int32_t k = khi - 1 - sub.sl;
        const int cnt = sub.leading(sub.ballot(k >= 0 && ins[k] >= L));
        khi -= cnt;
        if (cnt < S) break;
      }
      int64_t c1 = L;
      while (c1 > lo_a) {
        const int64_t c0 = c1 - S > lo_a ? c1 - S : lo_a;
        int32_t klo = khi;
        for (;;) {
          const int32_t k = klo - 1 - sub.sl;
          const int cnt = sub.leading(sub.ballot(k >= 0 && ins[k] >= c0));
          klo -= cnt;
          if (cnt < S) break;
        }
        h[sub.sl] = 0;
        sub.sync();
        for (int32_t k = klo + sub.sl; k < khi; k += S) atomicAdd(&h[ins[k] - c0], 1);
        sub.sync();
        const int inc = sub.incl_scan(h[sub.sl]);
        const int64_t i = c0 + sub.sl;
        const bool act = i < c1;
        int32_t col = 0;
        V val = V(0);
        int64_t dst = 0;
        if (act) {
          const int64_t src = ch.phys(i);
          col = m.cols[src];
          val = m.vals[src];
          dst = ch.phys(i + klo + inc);
        }
        sub.sync();
        if (act) {
          m.cols[dst] = col;
          m.vals[dst] = val;
        }
        sub.sync();
        c1 = c0;
        khi = klo;
      }
      // 3. new columns at nins[k] + k
      for (int32_t k = sub.sl; k < mnew; k += S) {
        const int64_t q = ch.phys((int64_t)ins[k] + k);
        m.cols[q] = ncol[b0 + k];
        m.vals[q] = nval[b0 + k];
      }
    }
    if (!reloc && sub.sl == 0) m.row_sizes[r] = (int32_t)(L + mnew);
    sub.sync();
  }
}

// Relocation: merge-path over (old row, new columns) into a fresh segment.
template <typename V>
__global__ void __launch_bounds__(RT_THREADS) k_relocate(Mat<V> m, const int32_t *trow, const int32_t *tb0,
                                                         const long long *addr, const long long *toff,
                                                         const int32_t *tmnew, const int32_t *ncol,
                                                         const V *nval) {
  if (!m.stat[ST_GO]) return;
  const int64_t nt = m.stat[ST_TOUCHED];
  const int64_t ntiles = m.stat[ST_TILES];
  const long long top = old_top(m.stat);
  for (int64_t q = blockIdx.x; q < ntiles; q += gridDim.x) {
    int64_t lo = 0, hi = nt;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (toff[mid] <= q) lo = mid + 1;
      else hi = mid;
    }
    const int64_t t = lo - 1;
    const int64_t j = q - toff[t];
    const int32_t r = trow[t];
    const int32_t b0 = tb0[t];
    const int64_t mn = tmnew[t];
    const int64_t L = m.row_sizes[r];
    const Chain ch = load_chain(m, r);
    const int64_t nl = L + mn;
    const int64_t start = top + addr[t];
    const int64_t o1 = (j + 1) * RT_TILE < nl ? (j + 1) * RT_TILE : nl;
    const int64_t o = j * RT_TILE + (int64_t)threadIdx.x * RT_ITEMS;
    if (o >= o1) continue;
    const int32_t *B = ncol + b0;
    const V *BV = nval + b0;
    int64_t a = o - mn > 0 ? o - mn : 0, b = o < L ? o : L;
    while (a < b) {
      int64_t mid = (a + b) >> 1;
      if (m.cols[ch.phys(mid)] < B[o - mid - 1]) a = mid + 1;
      else b = mid;
    }
    int64_t ia = a, ib = o - a;
    for (int e = 0; e < RT_ITEMS && o + e < o1; e++) {
      int32_t col;
      V val;
      bool takeA;
      if (ib >= mn) takeA = true;
      else if (ia >= L) takeA = false;
      else takeA = m.cols[ch.phys(ia)] < B[ib];
      if (takeA) {
        const int64_t p = ch.phys(ia++);
        col = m.cols[p];
        val = m.vals[p];
      } else {
        col = B[ib];
        val = BV[ib];
        ib++;
      }
      m.cols[start + o + e] = col;
      m.vals[start + o + e] = val;
    }
  }
}

template <typename V>
__global__ void k_finish(Mat<V> m, const int32_t *trow, const long long *addr, const int32_t *tmnew,
                         const int32_t *tinfo) {
  if (!m.stat[ST_GO]) return;
  const int64_t nt = m.stat[ST_TOUCHED];
  const long long top = old_top(m.stat);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t t = tid; t < nt; t += stride) {
    if (!((tinfo[t] >> 8) & 1)) continue;
    const int32_t r = trow[t];
    const int32_t st = (int32_t)(top + addr[t]);
    const int32_t cap = (int32_t)(addr[t + 1] - addr[t]);
    for (int l = 1; l < m.max_segs; l++)
      *reinterpret_cast<int2 *>(m.seg + (int64_t)l * m.pitch + 2 * (int64_t)r) = make_int2(-1, -1);
    *reinterpret_cast<int2 *>(m.seg + 2 * (int64_t)r) = make_int2(st, st + cap);
    m.row_sizes[r] = m.row_sizes[r] + tmnew[t];
  }
  if (tid == 0) m.row_sizes[m.n_rows] = (int32_t)m.stat[ST_NEED];
}

template <typename V>
__global__ void __launch_bounds__(UPD_THREADS) k_apply_append(Mat<V> m, const int32_t *trow, const int32_t *tb0,
                                                              const int32_t *bcol, const V *bval,
                                                              const long long *addr, const int32_t *tinfo) {
  if (!m.stat[ST_GO]) return;
  const int64_t nt = m.stat[ST_TOUCHED];
  const long long top = old_top(m.stat);
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t t = gw; t < nt; t += nwarps) {
    const int32_t r = trow[t];
    const int32_t b0 = tb0[t], b1 = tb0[t + 1];
    const int64_t L = m.row_sizes[r];
    const int layer = (int8_t)(tinfo[t] & 0xff);
    const long long cap = addr[t + 1] - addr[t];
    Chain ch = load_chain(m, r);
    if (cap > 0) {
      const int32_t st = (int32_t)(top + addr[t]);
      ch.append(st, (int32_t)cap, layer == 0);
      if (lane == 0)
        *reinterpret_cast<int2 *>(m.seg + (int64_t)layer * m.pitch + 2 * (int64_t)r) =
            make_int2(st, (int32_t)(st + cap));
    }
    for (int32_t j = lane; j < b1 - b0; j += 32) {
      const int64_t q = ch.phys(L + j);
      m.cols[q] = bcol[b0 + j];
      m.vals[q] = bval[b0 + j];
    }
    if (lane == 0) m.row_sizes[r] = (int32_t)(L + (b1 - b0));
    __syncwarp();
  }
}

// ------------------------------------------------------------ host driver

static int grid_for(int64_t n, int block) {
  int64_t g = div_up(n, block);
  int64_t cap = (int64_t)sm_count() * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

template <typename V>
static int update_impl(dcsr_handle h, const int32_t *rows, const int32_t *cols, const V *vals, int64_t T,
                       cudaStream_t s) {
  const bool merge = h->o.mode == DCSR_MERGE;
  const int cb = bits_for(h->n_cols), rb = bits_for(h->n_rows);
  const int bits = merge ? rb + cb : rb;
  Arena &ar = h->scratch;
  size_t need = 2 * arena_bytes(T, 8) + 2 * arena_bytes(T, 4) + 5 * arena_bytes(T + 2, 4) +
                2 * arena_bytes(T, sizeof(V)) + 4 * arena_bytes(T + 2, 8) + radix_scratch_bytes(T) +
                scan_scratch_bytes(T + 2);
  DCSR_TRY(ar.reserve(need, s));
  unsigned long long *k0 = ar.take<unsigned long long>(T), *k1 = ar.take<unsigned long long>(T);
  unsigned *p0 = ar.take<unsigned>(T), *p1 = ar.take<unsigned>(T);
  int32_t *bcol = ar.take<int32_t>(T + 2), *bpos = ar.take<int32_t>(T + 2), *trow = ar.take<int32_t>(T + 2);
  int32_t *tb0 = ar.take<int32_t>(T + 2), *tmnew = ar.take<int32_t>(T + 2);
  V *bval = ar.take<V>(T), *nval = ar.take<V>(T);
  long long *hflag = ar.take<long long>(T + 2), *tcap = ar.take<long long>(T + 2);
  long long *ttiles = ar.take<long long>(T + 2);
  long long *nflag = ar.take<long long>(T + 2);
  // tinfo / ncol / nins reuse the sort buffers once the sort is done
  Mat<V> m = h->view<V>();

  DCSR_CUDA(cudaMemsetAsync(h->stat + ST_AUX, 0, sizeof(long long), s));
  DCSR_LAUNCH(k_make_keys, grid_for(T, 256), 256, 0, s, rows, cols, T, h->n_rows, h->n_cols, cb, merge ? 1 : 0, k0,
              p0, h->stat);
  DCSR_TRY(radix_sort_pairs(&k0, &p0, &k1, &p1, T, bits, ar, s));
  DCSR_LAUNCH(k_gather_sorted<V>, grid_for(T, 256), 256, 0, s, k0, p0, cols, vals, T, cb, merge ? 1 : 0, h->n_cols,
              bcol, bval, hflag);
  DCSR_TRY(scan_i64(hflag, hflag, T, h->stat + ST_TOUCHED, ar, s));
  DCSR_LAUNCH(k_touched, grid_for(T, 256), 256, 0, s, k0, T, cb, merge ? 1 : 0, hflag, trow, tb0);
  // k1 / p1 are free after the sort: carve tinfo, ncol, nins from them
  int32_t *tinfo = (int32_t *)p1;
  int32_t *ncol = (int32_t *)k1;
  int32_t *nins = ncol + T;
  static int g_plan = 0, g_apply = 0, g_apply8 = 0, g_reloc = 0;
  if (!g_plan) {
    g_plan = persistent_grid((const void *)k_plan_merge<double>, UPD_THREADS, 0);
    g_apply = persistent_grid((const void *)k_apply_merge<double, 32>, UPD_THREADS, 0);
    g_apply8 = persistent_grid((const void *)k_apply_merge<double, 8>, UPD_THREADS, 0);
    g_reloc = persistent_grid((const void *)k_relocate<double>, RT_THREADS, 0);
  }
  if (merge) {
    const int gT = grid_for(T + 1, 256);
    DCSR_LAUNCH(k_head_search<V>, gT, 256, 0, s, m, k0, T, cb, bcol, bpos, nflag);
    DCSR_TRY(scan_i64(nflag, nflag, T + 1, nullptr, ar, s));
    DCSR_LAUNCH(k_new_compact<V>, gT, 256, 0, s, k0, T, cb, bcol, bval, bpos, nflag, hflag, tb0, ncol, nval, nins);
    DCSR_LAUNCH(k_row_plan<V>, gT, 256, 0, s, m, T, trow, tb0, nflag, nins, tcap, ttiles, tmnew, tinfo);
  } else {
    DCSR_LAUNCH(k_plan_append<V>, grid_for(T + 1, 256), 256, 0, s, m, T, trow, tb0, tcap, ttiles, tmnew, tinfo);
  }
  DCSR_TRY(scan_i64(tcap, tcap, T + 1, h->stat + ST_TOTAL, ar, s));
  if (merge) DCSR_TRY(scan_i64(ttiles, ttiles, T + 1, h->stat + ST_TILES, ar, s));
  DCSR_LAUNCH(k_check, 1, 1, 0, s, h->stat, h->row_sizes, h->n_rows, h->pool_cap);
  if (merge) {
    DCSR_LAUNCH(k_apply_existing<V>, grid_for(T, 256), 256, 0, s, m, k0, T, cb, bval, bpos);
    DCSR_LAUNCH((k_apply_merge<V, 8>), g_apply8, UPD_THREADS, 0, s, m, trow, tb0, bcol, bval, bpos, tcap, tmnew,
                tinfo, ncol, nval, nins);
    DCSR_LAUNCH((k_apply_merge<V, 32>), g_apply, UPD_THREADS, 0, s, m, trow, tb0, bcol, bval, bpos, tcap, tmnew,
                tinfo, ncol, nval, nins);
    DCSR_LAUNCH(k_relocate<V>, g_reloc, RT_THREADS, 0, s, m, trow, tb0, tcap, ttiles, tmnew, ncol, nval);
  } else {
    DCSR_LAUNCH(k_apply_append<V>, g_apply, UPD_THREADS, 0, s, m, trow, tb0, bcol, bval, tcap, tinfo);
  }
  DCSR_LAUNCH(k_finish<V>, grid_for(T, 256), 256, 0, s, m, trow, tcap, tmnew, tinfo);
  h->bins_valid = false;
  return DCSR_OK;
}

int update_async(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                 cudaStream_t s) {
  if (nnz == 0) return DCSR_OK;
  if (nnz > 0x7ffffff0LL) return DCSR_BAD_ARG;
  if (!h->vals) DCSR_TRY(reserve(h, 0, s));
  if (h->dtype == DCSR_F32) return update_impl<float>(h, rows, cols, (const float *)vals, nnz, s);
  return update_impl<double>(h, rows, cols, (const double *)vals, nnz, s);
}

// ------------------------------------------------------------- COO -> CSR

template <typename V>
__global__ void k_group(const unsigned long long *keys, const unsigned *perm, const int32_t *cols, const V *vals,
                        int64_t n, int cb, int merge, int32_t n_cols, long long *flag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    flag[i] = (!merge || i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

template <typename V>
__global__ void k_group_emit(const unsigned long long *keys, const unsigned *perm, const int32_t *cols,
                             const V *vals, int64_t n, int cb, int merge, int32_t n_cols, const long long *pos,
                             int32_t *ocols, V *ovals, long long *rowcnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const unsigned long long cmask = (1ull << cb) - 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long k = keys[i];
    if (merge && i > 0 && keys[i - 1] == k) continue;
    V v = vals[perm[i]];
    if (merge)
      for (int64_t j = i + 1; j < n && keys[j] == k; j++) v = v + vals[perm[j]];
    int32_t c = merge ? (int32_t)(k & cmask) : cols[perm[i]];
    if (c < 0 || c >= n_cols) c = 0;
    ocols[pos[i]] = c;
    ovals[pos[i]] = v;
    atomicAdd((unsigned long long *)&rowcnt[key_row(k, cb, merge)], 1ull);
  }
}

size_t coo_to_csr_scratch(dcsr_handle h, int64_t T) {
  return 2 * arena_bytes(T, 8) + 2 * arena_bytes(T, 4) + arena_bytes(T + 1, 8) + arena_bytes(T, 4) +
         arena_bytes(T, 8) + arena_bytes(h->n_rows + 2, 8) + radix_scratch_bytes(T) +
         scan_scratch_bytes(std::max<int64_t>(T, h->n_rows + 1));
}

template <typename V>
static int coo_impl(dcsr_handle h, const int32_t *rows, const int32_t *cols, const V *vals, int64_t T, bool merge,
                    Arena &ar, long long **rp, int32_t **ocols, void **ovals, cudaStream_t s) {
  const int cb = bits_for(h->n_cols), rb = bits_for(h->n_rows);
  unsigned long long *k0 = ar.take<unsigned long long>(T), *k1 = ar.take<unsigned long long>(T);
  unsigned *p0 = ar.take<unsigned>(T), *p1 = ar.take<unsigned>(T);
  long long *flag = ar.take<long long>(T + 1);
  int32_t *oc = ar.take<int32_t>(T);
  V *ov = (V *)ar.take<double>(T);
  long long *cnt = ar.take<long long>(h->n_rows + 2);
  DCSR_CUDA(cudaMemsetAsync(cnt, 0, sizeof(long long) * (h->n_rows + 2), s));
  if (T > 0) {
    DCSR_LAUNCH(k_make_keys, grid_for(T, 256), 256, 0, s, rows, cols, T, h->n_rows, h->n_cols, cb, merge ? 1 : 0,
                k0, p0, h->stat);
    DCSR_TRY(radix_sort_pairs(&k0, &p0, &k1, &p1, T, merge ? rb + cb : rb, ar, s));
    DCSR_LAUNCH(k_group<V>, grid_for(T, 256), 256, 0, s, k0, p0, cols, vals, T, cb, merge ? 1 : 0, h->n_cols, flag);
    DCSR_TRY(scan_i64(flag, flag, T, nullptr, ar, s));
    DCSR_LAUNCH(k_group_emit<V>, grid_for(T, 256), 256, 0, s, k0, p0, cols, vals, T, cb, merge ? 1 : 0, h->n_cols,
                flag, oc, ov, cnt);
  }
  DCSR_TRY(scan_i64(cnt, cnt, h->n_rows + 1, nullptr, ar, s));
  *rp = cnt;
  *ocols = oc;
  *ovals = ov;
  return DCSR_OK;
}

int coo_to_csr64(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz, bool merge,
                 Arena &ar, long long **rp, int32_t **ocols, void **ovals, int *bad, cudaStream_t s) {
  (void)bad;
  if (h->dtype == DCSR_F32)
    return coo_impl<float>(h, rows, cols, (const float *)vals, nnz, merge, ar, rp, ocols, ovals, s);
  return coo_impl<double>(h, rows, cols, (const double *)vals, nnz, merge, ar, rp, ocols, ovals, s);
}

}  // namespace dcsr
