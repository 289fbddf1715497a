// update.cu -- in-place batch updates of one DCSR matrix or of a set of
// matrices at once, and COO grouping for loads.
//
// Pipeline (all on the caller's stream, no host synchronisation); every
// kernel runs over the union of all matrices' triples / touched rows:
//   keys     (matrix, row, col) keys with an index check        k_make_keys
//   sort     stable LSD radix sort of (key, global triple index) radix_sort_pairs
//   bucket   sorted columns/values + per-row batch ranges        k_gather_sorted, scan, k_touched
//   plan     MERGE: each (row, col) group binary-searches its row
//            (thread per group), new groups are placed by a scan, then
//            per touched row: new length, capacity, layer, relocation
//            APPEND: the reference's segment walk per touched row
//   alloc    exclusive scan of new segment sizes (row order, per matrix
//            offsets taken relative to its first touched row)
//   check    per matrix: pool / layer / index status -> go flag   k_check
//   apply    existing columns in place (thread per group), then per row
//            the in-place shift + inserts (8- or 32-lane sub-warps)
//   relocate rows whose in-place shift would exceed reloc_min, and rows
//            that outgrow a chain already max_segs long, are merged out
//            of place into a fresh segment, tile-parallel          k_relocate
//   finish   chain reset of relocated rows, new pool tops          k_finish
// A rejected matrix (status != OK) is left untouched; the others proceed.
//
// Reference: device::UpdateMatrix include/load.h:258-325 and UpdateMatrix_dcsr
// include/sparse_update.inl:16-130 (segment walk, bump allocation, layer
// linking).  The reference appends without merging and allocates with
// atomicAdd; here MERGE mode keeps rows sorted and unique (duplicates summed
// in batch order) and the allocation is a row-ordered scan, so layouts are
// reproducible bit for bit, alone or in a batch.
#include "internal.cuh"

namespace dcsr {

constexpr int UPD_THREADS = 256;
constexpr int RT_TILE = 1024;  // relocation: outputs per tile
constexpr int RT_THREADS = 256;
constexpr int RT_ITEMS = RT_TILE / RT_THREADS;
constexpr int SMALL_AFF = 96;  // apply: rows shifting <= this many entries use 8-lane sub-warps

enum { AUX_BAD_INDEX = 1, AUX_LAYER_OVF = 2 };

// Key layout: [matrix | row | col] (MERGE) or [matrix | row] (APPEND).
struct KeyFmt {
  int cb, rb, merge;
  __device__ __forceinline__ int32_t row(unsigned long long k) const {
    const unsigned long long rk = merge ? (k >> cb) : k;
    return (int32_t)(rk & ((1ull << rb) - 1));
  }
  __device__ __forceinline__ int item(unsigned long long k) const { return (int)(k >> (rb + (merge ? cb : 0))); }
  __device__ __forceinline__ unsigned long long rowkey(unsigned long long k) const { return merge ? (k >> cb) : k; }
  __device__ __forceinline__ int32_t col(unsigned long long k) const { return (int32_t)(k & ((1ull << cb) - 1)); }
};

// ------------------------------------------------------------ matrix sources

// One matrix, passed by value.
template <typename V>
struct UpdOne {
  Mat<V> m;
  const int32_t *rows, *cols;
  const V *vals;
  __device__ __forceinline__ const Mat<V> &mat(int) const { return m; }
  __device__ __forceinline__ long long *st(int) const { return m.stat; }
  __device__ __forceinline__ int item_of_g(int64_t) const { return 0; }
  __device__ __forceinline__ int64_t local(int, int64_t g) const { return g; }
  __device__ __forceinline__ const int32_t *urows(int) const { return rows; }
  __device__ __forceinline__ const int32_t *ucols(int) const { return cols; }
  __device__ __forceinline__ const V *uvals(int) const { return vals; }
};

// A set of matrices: device array of batch items.
template <typename V>
struct UpdMany {
  const BatchItem<V> *it;
  int count;
  __device__ __forceinline__ const Mat<V> &mat(int i) const { return it[i].m; }
  __device__ __forceinline__ long long *st(int i) const { return it[i].m.stat; }
  __device__ __forceinline__ int item_of_g(int64_t g) const {
    int lo = 0, hi = count;  // largest i with toff <= g
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (it[mid].toff <= g) lo = mid;
      else hi = mid;
    }
    return lo;
  }
  __device__ __forceinline__ int64_t local(int i, int64_t g) const { return g - it[i].toff; }
  __device__ __forceinline__ const int32_t *urows(int i) const { return it[i].rows; }
  __device__ __forceinline__ const int32_t *ucols(int i) const { return it[i].cols; }
  __device__ __forceinline__ const V *uvals(int i) const { return (const V *)it[i].vals; }
};

// ------------------------------------------------------------------ keys

template <typename V, typename Src>
__global__ void k_item_init(Src src, int count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    long long *st = src.st(i);
    st[ST_AUX] = 0;
    st[ST_T0] = 0;
    st[ST_T1] = 0;
    st[ST_GO] = 0;
  }
}

template <typename V, typename Src>
__global__ void k_make_keys(Src src, int64_t n, KeyFmt f, unsigned long long *keys, unsigned *perm) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += stride) {
    const int i = src.item_of_g(g);
    const int64_t l = src.local(i, g);
    const Mat<V> &m = src.mat(i);
    int32_t r = src.urows(i)[l], c = src.ucols(i)[l];
    if (r < 0 || r >= m.n_rows || c < 0 || c >= m.n_cols) {
      atomicOr((unsigned long long *)&src.st(i)[ST_AUX], (unsigned long long)AUX_BAD_INDEX);
      r = 0;
      c = 0;
    }
    const unsigned long long it = (unsigned long long)i << (f.rb + (f.merge ? f.cb : 0));
    keys[g] = f.merge ? (it | ((unsigned long long)r << f.cb) | (unsigned long long)c) : (it | (unsigned long long)r);
    perm[g] = (unsigned)g;
  }
}

template <typename V, typename Src>
__global__ void k_gather_sorted(Src src, const unsigned long long *keys, const unsigned *perm, int64_t n, KeyFmt f,
                                int32_t *bcol, V *bval, long long *hflag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += stride) {
    const unsigned long long k = keys[g];
    const unsigned p = perm[g];
    const int i = f.item(k);
    const int64_t l = src.local(i, p);
    int32_t c = f.merge ? f.col(k) : src.ucols(i)[l];
    if (c < 0 || c >= src.mat(i).n_cols) c = 0;  // rejected matrix; keeps later reads in range
    bcol[g] = c;
    bval[g] = src.uvals(i)[l];
    hflag[g] = (g == 0 || f.rowkey(keys[g - 1]) != f.rowkey(k)) ? 1 : 0;
  }
}

template <typename V, typename Src>
__global__ void k_touched(Src src, const unsigned long long *keys, int64_t n, KeyFmt f, const long long *hpos,
                          const long long *gstat, int32_t *trow, int32_t *tb0, int32_t *tmat) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += stride) {
    const unsigned long long k = keys[g];
    const bool head = g == 0 || f.rowkey(keys[g - 1]) != f.rowkey(k);
    if (head) {
      const int64_t t = hpos[g];
      const int i = f.item(k);
      trow[t] = f.row(k);
      tb0[t] = (int32_t)g;
      tmat[t] = i;
      const int prev = g == 0 ? -1 : f.item(keys[g - 1]);
      if (prev != i) {
        src.st(i)[ST_T0] = t;
        if (prev >= 0) src.st(prev)[ST_T1] = t;
      }
    }
    if (g == n - 1) {
      const int64_t nt = hpos[g] + (head ? 1 : 0);
      tb0[nt] = (int32_t)n;
      src.st(f.item(k))[ST_T1] = nt;
    }
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

// MERGE plan, step 1 (thread per batch entry): every (row, col) group head
// binary-searches its column in the row: bpos = position (existing) or
// ~insertion point (new); nflag = 1 for new columns.
template <typename V, typename Src>
__global__ void k_head_search(Src src, const unsigned long long *keys, int64_t T, KeyFmt f, const int32_t *bcol,
                              int32_t *bpos, long long *nflag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g <= T; g += stride) {
    if (g == T) {
      nflag[T] = 0;
      continue;
    }
    const unsigned long long k = keys[g];
    long long isnew = 0;
    if (g == 0 || keys[g - 1] != k) {
      const Mat<V> &m = src.mat(f.item(k));
      const int32_t r = f.row(k);
      const int32_t c = bcol[g];
      const int64_t L = m.row_sizes[r];
      const Chain ch = load_chain(m, r);
      int64_t lo = 0, hi = L;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(m.cols + ch.phys(mid)) < c) lo = mid + 1;
        else hi = mid;
      }
      isnew = !(lo < L && __ldg(m.cols + ch.phys(lo)) == c);
      bpos[g] = isnew ? ~(int32_t)lo : (int32_t)lo;
    }
    nflag[g] = isnew;
  }
}

// MERGE plan, step 2 (thread per batch entry): new groups are written, in
// column order, to slot b0 + k of their row (k from the scan of nflag), with
// their batch-order sum.
template <typename V>
__global__ void k_new_compact(const unsigned long long *keys, int64_t T, KeyFmt f, const int32_t *bcol,
                              const V *bval, const int32_t *bpos, const long long *nflag_excl, const long long *hpos,
                              const int32_t *tb0, int32_t *ncol, V *nval, int32_t *nins) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < T; g += stride) {
    const unsigned long long k = keys[g];
    if (g > 0 && keys[g - 1] == k) continue;
    if (bpos[g] >= 0) continue;  // existing column
    const bool rowhead = g == 0 || f.rowkey(keys[g - 1]) != f.rowkey(k);
    const int64_t t = hpos[g] - (rowhead ? 0 : 1);
    const int32_t b0 = tb0[t];
    const int64_t slot = b0 + (nflag_excl[g] - nflag_excl[b0]);
    V v = bval[g];
    for (int64_t j = g + 1; j < T && keys[j] == k; j++) v = v + bval[j];
    ncol[slot] = bcol[g];
    nval[slot] = v;
    nins[slot] = ~bpos[g];
  }
}

// MERGE plan, step 3 (thread per touched row): new length, capacity, layer,
// relocation decision and apply width class.
template <typename V, typename Src>
__global__ void k_row_plan(Src src, int64_t T, const long long *gstat, const int32_t *trow, const int32_t *tb0,
                           const int32_t *tmat, const long long *nflag_excl, const int32_t *nins, long long *tcap,
                           long long *ttiles, int32_t *tmnew, int32_t *tinfo) {
  const int64_t nt = gstat[ST_TOUCHED];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= T; t += stride) {
    if (t >= nt) {
      tcap[t] = 0;
      ttiles[t] = 0;
      continue;
    }
    const int i = tmat[t];
    const Mat<V> &m = src.mat(i);
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
        layer = ch.total == 0 ? 0 : ch.ns;
        if (layer >= m.max_segs) {
          // every layer in use: the row is merged out of place into one
          // fresh segment of policy_cap(nl) (chain reset), as a relocation
          reloc = 1;
          layer = 0;
          big = 0;
          cap = policy_cap(m.o, nl);
        } else {
          cap = align_up(policy_cap(m.o, nl) - ch.total, m.o.align);
        }
      }
    }
    tcap[t] = cap;
    ttiles[t] = reloc ? div_up(nl, RT_TILE) : 0;
    tmnew[t] = (int32_t)mnew;
    tinfo[t] = (layer & 0xff) | (reloc << 8) | (big << 9) | ((mnew > 0 || cap > 0) ? (1 << 10) : 0);
  }
}

// APPEND mode: the reference's segment walk and allocation size.
template <typename V, typename Src>
__global__ void k_plan_append(Src src, int64_t T, const long long *gstat, const int32_t *trow, const int32_t *tb0,
                              const int32_t *tmat, long long *tcap, long long *ttiles, int32_t *tmnew,
                              int32_t *tinfo) {
  const int64_t nt = gstat[ST_TOUCHED];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= T; t += stride) {
    if (t >= nt) {
      tcap[t] = 0;
      ttiles[t] = 0;
      continue;
    }
    const int i = tmat[t];
    const Mat<V> &m = src.mat(i);
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
      for (int q = 0; q < MAX_SEGS; q++) {
        if (!found && q < ch.ns) {
          after = before + ch.cp[q];
          off = q;
          if (after >= rlA || q + 1 >= ch.ns) found = true;
          else before = after;
        }
      }
      const int64_t fr = after - rlA;
      if (fr < rlB) {
        cap = rlB - fr + m.o.alpha;
        layer = off + 1;
        if (layer >= m.max_segs)
          atomicOr((unsigned long long *)&src.st(i)[ST_AUX], (unsigned long long)AUX_LAYER_OVF);
      }
    }
    tcap[t] = cap;
    ttiles[t] = 0;
    tmnew[t] = (int32_t)rlB;
    tinfo[t] = (layer & 0xff) | (1 << 10);
  }
}

// Per matrix: requirement from the scanned capacities, status and go flag.
template <typename V, typename Src>
__global__ void k_check(Src src, int count, const long long *addr) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    long long *st = src.st(i);
    const Mat<V> &m = src.mat(i);
    const long long aux = st[ST_AUX];
    const long long top = m.row_sizes[m.n_rows];
    const long long need = top + (addr[st[ST_T1]] - addr[st[ST_T0]]);
    st[ST_TOP] = top;
    st[ST_NEED] = need;
    int s = DCSR_OK;
    if (aux & AUX_BAD_INDEX) s = DCSR_BAD_INDEX;
    else if (aux & AUX_LAYER_OVF) s = DCSR_LAYER_OVERFLOW;
    else if (need > m.pool_cap || need > 0x7fffffffLL) s = DCSR_POOL_EXHAUSTED;
    st[ST_GO] = s == DCSR_OK ? 1 : 0;
    if (s != DCSR_OK && st[ST_STATUS] == 0) st[ST_STATUS] = s;
    st[ST_AUX] = 0;
  }
}

// --------------------------------------------------------------- applying

// Apply, step 1 (thread per batch group): existing columns take their batch
// values in batch order, in place, before any shift or relocation reads them.
template <typename V, typename Src>
__global__ void k_apply_existing(Src src, const unsigned long long *keys, int64_t T, KeyFmt f, const V *bval,
                                 const int32_t *bpos) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < T; g += stride) {
    const unsigned long long k = keys[g];
    if (g > 0 && keys[g - 1] == k) continue;
    const int32_t p = bpos[g];
    if (p < 0) continue;
    const int i = f.item(k);
    if (!src.st(i)[ST_GO]) continue;
    const Mat<V> &m = src.mat(i);
    const Chain ch = load_chain(m, f.row(k));
    const int64_t q = ch.phys(p);
    V v = m.vals[q];
    for (int64_t j = g; j < T && keys[j] == k; j++) v = v + bval[j];
    m.vals[q] = v;
  }
}

// Apply, step 2, for the rows of one width class: S = 8 takes rows shifting
// at most SMALL_AFF entries (and rows without shifts), S = 32 the larger ones.
// Links a new segment when planned, shifts entries after the first insertion
// point back to front (S per step; shift(i) = #{new k : nins[k] <= i}, from a
// histogram of the insertion points in the window), then writes new columns.
template <typename V, typename Src, int S>
__global__ void __launch_bounds__(UPD_THREADS) k_apply_merge(Src src, const long long *gstat, const int32_t *trow,
                                                             const int32_t *tb0, const int32_t *tmat,
                                                             const long long *addr, const int32_t *tmnew,
                                                             const int32_t *tinfo, const int32_t *ncol,
                                                             const V *nval, const int32_t *nins) {
  __shared__ int hist[UPD_THREADS / S][S];
  const int64_t nt = gstat[ST_TOUCHED];
  const Sub<S> sub;
  int *h = hist[threadIdx.x / S];
  const int64_t gthreads = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / S; t < nt; t += gthreads / S) {
    const int info = tinfo[t];
    if (!((info >> 10) & 1) || ((info >> 9) & 1) != (S == 32 ? 1 : 0) || ((info >> 8) & 1)) continue;
    const int i = tmat[t];
    const long long *st = src.st(i);
    if (!st[ST_GO]) continue;
    const Mat<V> &m = src.mat(i);
    const int32_t r = trow[t];
    const int32_t b0 = tb0[t];
    const int64_t L = m.row_sizes[r];
    const int layer = (int8_t)(info & 0xff);
    const int32_t mnew = tmnew[t];
    const long long cap = addr[t + 1] - addr[t];
    Chain ch = load_chain(m, r);
    if (cap > 0) {
      const int32_t stp = (int32_t)(st[ST_TOP] + (addr[t] - addr[st[ST_T0]]));
      ch.append(stp, (int32_t)cap, layer == 0);
      if (sub.sl == 0)
        *reinterpret_cast<int2 *>(m.seg + (int64_t)layer * m.pitch + 2 * (int64_t)r) =
            make_int2(stp, (int32_t)(stp + cap));
    }
    if (mnew > 0) {
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
        const int64_t e = c0 + sub.sl;
        const bool act = e < c1;
        int32_t col = 0;
        V val = V(0);
        int64_t dst = 0;
        if (act) {
          const int64_t srcq = ch.phys(e);
          col = m.cols[srcq];
          val = m.vals[srcq];
          dst = ch.phys(e + klo + inc);
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
      for (int32_t k = sub.sl; k < mnew; k += S) {
        const int64_t q = ch.phys((int64_t)ins[k] + k);
        m.cols[q] = ncol[b0 + k];
        m.vals[q] = nval[b0 + k];
      }
    }
    if (sub.sl == 0) m.row_sizes[r] = (int32_t)(L + mnew);
    sub.sync();
  }
}

// Relocation: merge-path over (old row, new columns) into a fresh segment.
template <typename V, typename Src>
__global__ void __launch_bounds__(RT_THREADS) k_relocate(Src src, const long long *gstat, const int32_t *trow,
                                                         const int32_t *tb0, const int32_t *tmat,
                                                         const long long *addr, const long long *toff,
                                                         const int32_t *tmnew, const int32_t *ncol,
                                                         const V *nval) {
  const int64_t nt = gstat[ST_TOUCHED];
  const int64_t ntiles = gstat[ST_TILES];
  for (int64_t q = blockIdx.x; q < ntiles; q += gridDim.x) {
    int64_t lo = 0, hi = nt;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (toff[mid] <= q) lo = mid + 1;
      else hi = mid;
    }
    const int64_t t = lo - 1;
    const int i = tmat[t];
    const long long *st = src.st(i);
    if (!st[ST_GO]) continue;
    const Mat<V> &m = src.mat(i);
    const int64_t j = q - toff[t];
    const int32_t r = trow[t];
    const int32_t b0 = tb0[t];
    const int64_t mn = tmnew[t];
    const int64_t L = m.row_sizes[r];
    const Chain ch = load_chain(m, r);
    const int64_t nl = L + mn;
    const int64_t start = st[ST_TOP] + (addr[t] - addr[st[ST_T0]]);
    const int64_t o1 = (j + 1) * RT_TILE < nl ? (j + 1) * RT_TILE : nl;
    const int64_t o = j * RT_TILE + (int64_t)threadIdx.x * RT_ITEMS;
    if (o >= o1) continue;
    const int32_t *B = ncol + b0;
    const V *BV = nval + b0;
    int64_t a = o - mn > 0 ? o - mn : 0, b = o < L ? o : L;
    while (a < b) {
      const int64_t mid = (a + b) >> 1;
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

template <typename V, typename Src>
__global__ void k_finish(Src src, int count, const long long *gstat, const int32_t *trow, const int32_t *tmat,
                         const long long *addr, const int32_t *tmnew, const int32_t *tinfo) {
  const int64_t nt = gstat[ST_TOUCHED];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t t = tid; t < nt; t += stride) {
    if (!((tinfo[t] >> 8) & 1)) continue;
    const int i = tmat[t];
    const long long *st = src.st(i);
    if (!st[ST_GO]) continue;
    const Mat<V> &m = src.mat(i);
    const int32_t r = trow[t];
    const int32_t stp = (int32_t)(st[ST_TOP] + (addr[t] - addr[st[ST_T0]]));
    const int32_t cap = (int32_t)(addr[t + 1] - addr[t]);
    for (int l = 1; l < m.max_segs; l++)
      *reinterpret_cast<int2 *>(m.seg + (int64_t)l * m.pitch + 2 * (int64_t)r) = make_int2(-1, -1);
    *reinterpret_cast<int2 *>(m.seg + 2 * (int64_t)r) = make_int2(stp, stp + cap);
    m.row_sizes[r] = m.row_sizes[r] + tmnew[t];
  }
  for (int64_t i = tid; i < count; i += stride) {
    const long long *st = src.st((int)i);
    if (st[ST_GO]) {
      const Mat<V> &m = src.mat((int)i);
      m.row_sizes[m.n_rows] = (int32_t)st[ST_NEED];
    }
  }
}

template <typename V, typename Src>
__global__ void __launch_bounds__(UPD_THREADS) k_apply_append(Src src, const long long *gstat, const int32_t *trow,
                                                              const int32_t *tb0, const int32_t *tmat,
                                                              const int32_t *bcol, const V *bval,
                                                              const long long *addr, const int32_t *tinfo) {
  const int64_t nt = gstat[ST_TOUCHED];
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t t = gw; t < nt; t += nwarps) {
    const int i = tmat[t];
    const long long *st = src.st(i);
    if (!st[ST_GO]) continue;
    const Mat<V> &m = src.mat(i);
    const int32_t r = trow[t];
    const int32_t b0 = tb0[t], b1 = tb0[t + 1];
    const int64_t L = m.row_sizes[r];
    const int layer = (int8_t)(tinfo[t] & 0xff);
    const long long cap = addr[t + 1] - addr[t];
    Chain ch = load_chain(m, r);
    if (cap > 0) {
      const int32_t stp = (int32_t)(st[ST_TOP] + (addr[t] - addr[st[ST_T0]]));
      ch.append(stp, (int32_t)cap, layer == 0);
      if (lane == 0)
        *reinterpret_cast<int2 *>(m.seg + (int64_t)layer * m.pitch + 2 * (int64_t)r) =
            make_int2(stp, (int32_t)(stp + cap));
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

size_t update_scratch_bytes(int64_t T, size_t vsize) {
  return 2 * arena_bytes(T, 8) + 2 * arena_bytes(T, 4) + 6 * arena_bytes(T + 2, 4) + 2 * arena_bytes(T, vsize) +
         4 * arena_bytes(T + 2, 8) + radix_scratch_bytes(T) + scan_scratch_bytes(T + 2);
}

// The update of `count` matrices (one Src) with T triples in total.
// gstat: batch-global status words (ST_TOUCHED, ST_TILES, ST_TOTAL).
template <typename V, typename Src>
static int update_pipeline(const Src &src, int count, int64_t T, bool merge, int rb, int cb, long long *gstat,
                           Arena &ar, cudaStream_t s) {
  const int ib = count > 1 ? bits_for(count) : 0;
  const KeyFmt f{cb, rb, merge ? 1 : 0};
  const int bits = ib + rb + (merge ? cb : 0);
  if (bits > 63) return DCSR_NOT_SUPPORTED;
  DCSR_TRY(ar.reserve(update_scratch_bytes(T, sizeof(V)), s));
  unsigned long long *k0 = ar.take<unsigned long long>(T), *k1 = ar.take<unsigned long long>(T);
  unsigned *p0 = ar.take<unsigned>(T), *p1 = ar.take<unsigned>(T);
  int32_t *bcol = ar.take<int32_t>(T + 2), *bpos = ar.take<int32_t>(T + 2), *trow = ar.take<int32_t>(T + 2);
  int32_t *tb0 = ar.take<int32_t>(T + 2), *tmnew = ar.take<int32_t>(T + 2), *tmat = ar.take<int32_t>(T + 2);
  V *bval = ar.take<V>(T), *nval = ar.take<V>(T);
  long long *hflag = ar.take<long long>(T + 2), *tcap = ar.take<long long>(T + 2);
  long long *ttiles = ar.take<long long>(T + 2), *nflag = ar.take<long long>(T + 2);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  const int gT = grid_for(T + 1, 256);
  const int gI = grid_for(count, 256);

  DCSR_LAUNCH((k_item_init<V, Src>), gI, 256, 0, s, src, count);
  DCSR_LAUNCH((k_make_keys<V, Src>), gT, 256, 0, s, src, T, f, k0, p0);
  DCSR_TRY(radix_sort_pairs(&k0, &p0, &k1, &p1, T, bits, ar, s));
  DCSR_LAUNCH((k_gather_sorted<V, Src>), gT, 256, 0, s, src, k0, p0, T, f, bcol, bval, hflag);
  DCSR_TRY(scan_i64(hflag, hflag, T, gstat + ST_TOUCHED, ar, s));
  DCSR_LAUNCH((k_touched<V, Src>), gT, 256, 0, s, src, k0, T, f, hflag, gstat, trow, tb0, tmat);
  // k1 / p1 are free after the sort: carve tinfo, ncol, nins from them
  int32_t *tinfo = (int32_t *)p1;
  int32_t *ncol = (int32_t *)k1;
  int32_t *nins = ncol + T;
  static const int g_apply = persistent_grid((const void *)k_apply_merge<double, UpdOne<double>, 32>, UPD_THREADS, 0);
  static const int g_apply8 = persistent_grid((const void *)k_apply_merge<double, UpdOne<double>, 8>, UPD_THREADS, 0);
  static const int g_reloc = persistent_grid((const void *)k_relocate<double, UpdOne<double>>, RT_THREADS, 0);
  if (merge) {
    DCSR_LAUNCH((k_head_search<V, Src>), gT, 256, 0, s, src, k0, T, f, bcol, bpos, nflag);
    DCSR_TRY(scan_i64(nflag, nflag, T + 1, nullptr, ar, s));
    DCSR_LAUNCH(k_new_compact<V>, gT, 256, 0, s, k0, T, f, bcol, bval, bpos, nflag, hflag, tb0, ncol, nval, nins);
    DCSR_LAUNCH((k_row_plan<V, Src>), gT, 256, 0, s, src, T, gstat, trow, tb0, tmat, nflag, nins, tcap, ttiles,
                tmnew, tinfo);
  } else {
    DCSR_LAUNCH((k_plan_append<V, Src>), gT, 256, 0, s, src, T, gstat, trow, tb0, tmat, tcap, ttiles, tmnew, tinfo);
  }
  if (merge)
    DCSR_TRY(scan2_i64(tcap, tcap, gstat + ST_TOTAL, ttiles, ttiles, gstat + ST_TILES, T + 1, ar, s));
  else
    DCSR_TRY(scan_i64(tcap, tcap, T + 1, gstat + ST_TOTAL, ar, s));
  DCSR_LAUNCH((k_check<V, Src>), gI, 256, 0, s, src, count, tcap);
  if (merge) {
    DCSR_LAUNCH((k_apply_existing<V, Src>), gT, 256, 0, s, src, k0, T, f, bval, bpos);
    DCSR_LAUNCH((k_apply_merge<V, Src, 8>), g_apply8, UPD_THREADS, 0, s, src, gstat, trow, tb0, tmat, tcap, tmnew,
                tinfo, ncol, nval, nins);
    DCSR_LAUNCH((k_apply_merge<V, Src, 32>), g_apply, UPD_THREADS, 0, s, src, gstat, trow, tb0, tmat, tcap, tmnew,
                tinfo, ncol, nval, nins);
    DCSR_LAUNCH((k_relocate<V, Src>), g_reloc, RT_THREADS, 0, s, src, gstat, trow, tb0, tmat, tcap, ttiles, tmnew,
                ncol, nval);
  } else {
    DCSR_LAUNCH((k_apply_append<V, Src>), g_apply, UPD_THREADS, 0, s, src, gstat, trow, tb0, tmat, bcol, bval, tcap,
                tinfo);
  }
  DCSR_LAUNCH((k_finish<V, Src>), gT, 256, 0, s, src, count, gstat, trow, tmat, tcap, tmnew, tinfo);
  return DCSR_OK;
}

template <typename V>
static int update_one(dcsr_handle h, const int32_t *rows, const int32_t *cols, const V *vals, int64_t T,
                      cudaStream_t s, Arena &ar) {
  UpdOne<V> src{h->view<V>(), rows, cols, vals};
  DCSR_TRY(update_pipeline<V>(src, 1, T, h->o.mode == DCSR_MERGE, bits_for(h->n_rows), bits_for(h->n_cols), h->stat,
                              ar, s));
  h->bins_valid = false;
  return DCSR_OK;
}

int update_async(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                 cudaStream_t s, Arena *ar) {
  if (nnz == 0) return DCSR_OK;
  if (nnz > 0x7ffffff0LL) return DCSR_BAD_ARG;
  Arena &a = ar ? *ar : h->scratch;
  a.status = h->stat + ST_STATUS;  // a look-back wait that gives up reports DCSR_TIMEOUT here
  if (h->dtype == DCSR_F32) return update_one<float>(h, rows, cols, (const float *)vals, nnz, s, a);
  return update_one<double>(h, rows, cols, (const double *)vals, nnz, s, a);
}

template <typename V>
static int update_many_t(const BatchItem<V> *items_dev, int count, int64_t T, bool merge, int rb, int cb,
                         long long *gstat, Arena &ar, cudaStream_t s) {
  UpdMany<V> src{items_dev, count};
  return update_pipeline<V>(src, count, T, merge, rb, cb, gstat, ar, s);
}

int update_many(const void *items_dev, int dtype, int count, int64_t T, bool merge, int rb, int cb, long long *gstat,
                Arena &ar, cudaStream_t s) {
  if (T == 0 || count == 0) return DCSR_OK;
  ar.status = gstat + ST_STATUS;  // a look-back wait that gives up reports DCSR_TIMEOUT for the batch
  if (dtype == DCSR_F32)
    return update_many_t<float>((const BatchItem<float> *)items_dev, count, T, merge, rb, cb, gstat, ar, s);
  return update_many_t<double>((const BatchItem<double> *)items_dev, count, T, merge, rb, cb, gstat, ar, s);
}

// ------------------------------------------------------------- COO -> CSR

__global__ void k_coo_keys(const int32_t *rows, const int32_t *cols, int64_t n, int32_t n_rows, int32_t n_cols,
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

__global__ void k_group(const unsigned long long *keys, int64_t n, int merge, long long *flag) {
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
  const int lane = threadIdx.x & 31;
  // block-uniform trip count, so whole warps take part in the count below
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
    const int64_t i = i0 + threadIdx.x;
    int32_t r = -1;  // the row of the entry this thread emits
    if (i < n) {
      const unsigned long long k = keys[i];
      if (!(merge && i > 0 && keys[i - 1] == k)) {
        V v = vals[perm[i]];
        if (merge)
          for (int64_t j = i + 1; j < n && keys[j] == k; j++) v = v + vals[perm[j]];
        int32_t c = merge ? (int32_t)(k & cmask) : cols[perm[i]];
        if (c < 0 || c >= n_cols) c = 0;
        ocols[pos[i]] = c;
        ovals[pos[i]] = v;
        r = merge ? (int32_t)(k >> cb) : (int32_t)k;
      }
    }
    // row counts, one atomic per row and warp: the keys are sorted, so a
    // warp's entries are a few runs of one row each (a power-law graph's
    // hottest rows otherwise took one atomic per entry on a single word)
    const unsigned peers = __match_any_sync(FULL, r);
    if (r >= 0 && __ffs(peers) - 1 == lane) atomicAdd((unsigned long long *)&rowcnt[r], (unsigned long long)__popc(peers));
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
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  DCSR_CUDA(cudaMemsetAsync(cnt, 0, sizeof(long long) * (h->n_rows + 2), s));
  if (T > 0) {
    DCSR_LAUNCH(k_coo_keys, grid_for(T, 256), 256, 0, s, rows, cols, T, h->n_rows, h->n_cols, cb, merge ? 1 : 0, k0,
                p0, h->stat);
    DCSR_TRY(radix_sort_pairs(&k0, &p0, &k1, &p1, T, merge ? rb + cb : rb, ar, s));
    DCSR_LAUNCH(k_group, grid_for(T, 256), 256, 0, s, k0, T, merge ? 1 : 0, flag);
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
