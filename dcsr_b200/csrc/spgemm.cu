// spgemm.cu -- C = A*B for DCSR matrices (expand - sort - reduce).
//
// 1. count   products per row P_i = sum_{k in A_i} |B_k| and a size class
//            (reference CalcSortSizes_SPMM / SetBins_SPMM include/spmm.inl:951-1061)
// 2. bucket  rows by class (one radix pass), scan P_i -> per-row staging offsets
// 3. numeric per row: expand products a_ik*b_kj tagged with their product
//            index p, sort by (column, p), sum equal columns left to right,
//            write unique columns to the staging area:
//              P_i <= 256   warp per row, bitonic sort in shared memory
//              P_i <= 4096  CTA per row, bitonic sort in shared memory
//              P_i >  4096  all such rows together: global stable radix sort
//                           of (row, column) keys (no row is skipped; the
//                           reference left rows > 2048 products uncomputed,
//                           include/spmm.h:368-389)
// 4. layout  C's rows placed straight from the staging area into C's pool
//            with C's slack policy; the pool is allocated at an upper bound
//            (the policy capacity of P_i per row) so nothing waits for the
//            unique counts.  Two synchronisations: the product counts (to size
//            the staging area) and C's pool top.
// Sorting by (column, p) makes every sum run in product order, so values are
// reproducible and match the CPU oracle bit for bit; explicit zeros are kept
// (reference include/spmm.inl:215-218).
#include <algorithm>

#include "internal.cuh"

namespace dcsr {

constexpr int SG_THREADS = 256;
constexpr int SG_WARP_MAX = 256;   // products per warp-row
constexpr int SG_CTA_MAX = 4096;   // products per CTA-row
enum { SG_EMPTY = 0, SG_WARP = 1, SG_CTA = 2, SG_GLOBAL = 3 };

// Per row: its product count P_i, its size class, and the capacity C's
// layout policy gives a row of P_i entries (an upper bound of the row's
// capacity, whatever its unique columns); the products of the rows of the
// global class are added up in *gtotal.
template <typename V>
__global__ void k_sg_count(Mat<V> A, Mat<V> B, dcsr_opts co, long long *cnt, long long *capub,
                           unsigned long long *cls, unsigned *rows, unsigned long long *gtotal) {
  constexpr int G = 8;  // lanes per row: a warp has four rows' loads in flight
  const int lane = threadIdx.x & 31, j = lane & (G - 1);
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32 / G); i0 < A.n_rows;
       i0 += nw * (32 / G)) {
    const int64_t i = i0 + lane / G;
    long long s = 0;
    if (i < A.n_rows) {
      const Chain ch = load_chain(A, (int32_t)i);
      const int64_t L = A.row_sizes[i];
      for (int64_t p = j; p < L; p += G) s += B.row_sizes[A.cols[ch.phys(p)]];
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if (j == 0 && i < A.n_rows) {
      cnt[i] = s;
      capub[i] = policy_cap(co, s);
      const int c = s == 0 ? SG_EMPTY : s <= SG_WARP_MAX ? SG_WARP : s <= SG_CTA_MAX ? SG_CTA : SG_GLOBAL;
      cls[i] = c;
      rows[i] = (unsigned)i;
      if (c == SG_GLOBAL) atomicAdd(gtotal, (unsigned long long)s);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    cnt[A.n_rows] = 0;
    capub[A.n_rows] = 0;
  }
}

// class starts [0..4] from the sorted class keys
__global__ void k_sg_classes(const unsigned long long *keys, int32_t n, long long *starts) {
  const int c = threadIdx.x;
  if (c <= 4) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < (unsigned long long)c) lo = mid + 1;
      else hi = mid;
    }
    starts[c] = c == 4 ? n : lo;
  }
}

// Expand row i's products into (key = col<<32 | p, prod[p]) over `nthr`
// cooperating threads (tid in [0, nthr)); returns the product count.
template <typename V>
__device__ __forceinline__ int64_t sg_expand(const Mat<V> &A, const Mat<V> &B, int64_t i, int tid, int nthr,
                                             unsigned long long *key, V *prod) {
  const Chain ca = load_chain(A, (int32_t)i);
  const int64_t LA = A.row_sizes[i];
  int64_t pos = 0;
  for (int64_t e = 0; e < LA; e++) {
    const int64_t qa = ca.phys(e);
    const int32_t k = A.cols[qa];
    const V a = A.vals[qa];
    const Chain cb = load_chain(B, k);
    const int64_t LB = B.row_sizes[k];
    for (int64_t j = tid; j < LB; j += nthr) {
      const int64_t qb = cb.phys(j);
      key[pos + j] = ((unsigned long long)(uint32_t)B.cols[qb] << 32) | (unsigned long long)(pos + j);
      V pr;
      if constexpr (sizeof(V) == 4) pr = __fmul_rn(a, B.vals[qb]);
      else pr = __dmul_rn(a, B.vals[qb]);
      prod[pos + j] = pr;
    }
    pos += LB;
  }
  return pos;
}

// Sort keys of the warp class: (column, product index p < 256) packed into
// 32 bits when columns fit in 24 bits, else into 64.
template <typename K>
struct SgKey {
  static constexpr int S = sizeof(K) == 4 ? 8 : 32;
  __device__ __forceinline__ static K make(int32_t col, int p) { return ((K)(uint32_t)col << S) | (K)p; }
  __device__ __forceinline__ static int32_t col(K k) { return (int32_t)(k >> S); }
  __device__ __forceinline__ static uint32_t idx(K k) { return (uint32_t)(k & ((K(1) << S) - 1)); }
};

// The warp class's expand (P_i <= 256): row i's A entries are taken 32 at
// a time, one per lane, each lane loading its entry's column k and value,
// then B row k's length and segments, side by side (no load waits on another
// entry's); the B-row lengths are scanned into product offsets, and lane l
// produces products q = l, l + 32, ... of the group: the entry owning q is
// found by a binary search over the lanes' offsets, and all B loads of the
// group are issued before the first is used.  Same keys and products as
// sg_expand (product p = the row's p-th product in A-entry-major order).
template <typename V, typename K>
__device__ __forceinline__ int sg_expand_warp(const Mat<V> &A, const Mat<V> &B, int64_t i, int lane, K *key,
                                              V *prod) {
  constexpr int H = 4;
  const int32_t LA = A.row_sizes[i];
  const Chain ca = load_chain_used(A, (int32_t)i, LA);
  int base = 0;
  for (int32_t e0 = 0; e0 < LA; e0 += 32) {
    const int nE = LA - e0 < 32 ? LA - e0 : 32;
    int32_t kb = 0, lb = 0;
    V a = V(0);
    if (lane < nE) {
      const int64_t qa = ca.phys(e0 + lane);
      kb = A.cols[qa];
      a = A.vals[qa];
      lb = B.row_sizes[kb];
    }
    const Chain cb = load_chain_used(B, kb, lb);
    const bool flat = __all_sync(FULL, cb.ns <= 1);  // every B row in its first segment (the common case)
    const int incl = warp_incl_scan(lb);
    const int pos = incl - lb;
    const int tot = __shfl_sync(FULL, incl, 31);  // base + tot <= P_i <= SG_WARP_MAX
    // products in groups of H per lane: every B load of a group in flight at once
    for (int t0 = 0; t0 * 32 < tot; t0 += H) {
      int own[H];
      int32_t bc[H];
      V bv[H];
#pragma unroll
      for (int h = 0; h < H; h++) {
        const int q = (t0 + h) * 32 + lane;
        own[h] = 0;
        bc[h] = 0;
        bv[h] = V(0);
        if ((t0 + h) * 32 < tot) {  // warp-uniform
          int lo = 0;  // the last entry (< nE) whose offset is <= q: it owns q
#pragma unroll
          for (int st = 16; st > 0; st >>= 1) {
            const int c = lo + st;  // <= 31
            const int pc = __shfl_sync(FULL, pos, c);
            if (c < nE && pc <= q) lo = c;
          }
          own[h] = lo;
          const int pj = __shfl_sync(FULL, pos, lo);
          int64_t qb;
          if (flat) {
            qb = (int64_t)__shfl_sync(FULL, cb.st[0], lo) + (q - pj);
          } else {
            const Chain co = shfl_chain(cb, lo);
            qb = co.phys(q - pj);
          }
          if (q < tot) {
            bc[h] = B.cols[qb];
            bv[h] = B.vals[qb];
          }
        }
      }
#pragma unroll
      for (int h = 0; h < H; h++) {
        const int q = (t0 + h) * 32 + lane;
        if ((t0 + h) * 32 < tot) {
          const V ao = __shfl_sync(FULL, a, own[h]);
          if (q < tot) {
            key[base + q] = SgKey<K>::make(bc[h], base + q);
            V pr;
            if constexpr (sizeof(V) == 4) pr = __fmul_rn(ao, bv[h]);
            else pr = __dmul_rn(ao, bv[h]);
            prod[base + q] = pr;
          }
        }
      }
    }
    base += tot;
  }
  return base;
}

__device__ __forceinline__ int next_pow2(int x) {
  int p = 32;
  while (p < x) p <<= 1;
  return p;
}

// Bitonic sort of n2 (power of two) keys by `nthr` threads; sync() between steps.
template <typename K, typename Sync>
__device__ __forceinline__ void bitonic(K *key, int n2, int tid, int nthr, Sync sync) {
  for (int k = 2; k <= n2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < (n2 >> 1); t += nthr) {
        const int i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
        const int l = i + j;
        const bool up = (i & k) == 0;
        const K a = key[i], b = key[l];
        if ((a > b) == up) {
          key[i] = b;
          key[l] = a;
        }
      }
      sync();
    }
}

// Bitonic sort of the 32*E keys held by a warp, E per lane: key i = lane*E + t
// in v[t].  Steps with partner distance j < E swap within a lane's
// registers, the others exchange with lane ^ (j / E) by shuffle; nothing
// goes through shared memory.
template <int E, typename K>
__device__ __forceinline__ void warp_bitonic(K (&v)[E], int lane) {
  constexpr int N = 32 * E;
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= E) {
#pragma unroll
        for (int t = 0; t < E; t++) {
          const int i = lane * E + t;
          const K o = __shfl_xor_sync(FULL, v[t], j / E);
          // the lower index of a pair keeps the smaller key in an ascending
          // block (i & k == 0) and the larger in a descending one
          const bool keep_min = ((i & k) == 0) == ((i & j) == 0);
          v[t] = keep_min ? (o < v[t] ? o : v[t]) : (o > v[t] ? o : v[t]);
        }
      } else {
#pragma unroll
        for (int t = 0; t < E; t++) {
          const int q = t ^ j;
          if (q > t) {
            const bool up = ((lane * E + t) & k) == 0;
            const K a = v[t], b = v[q];
            const bool sw = up ? (a > b) : (a < b);
            v[t] = sw ? b : a;
            v[q] = sw ? a : b;
          }
        }
      }
    }
  }
}

// A warp-row's P keys (in key[0, P), P <= 32*E) sorted in place through
// registers; slots past P take the largest key and end up past P.
template <int E, typename K>
__device__ __forceinline__ void sort_row_keys(K *key, int P, int lane) {
  K v[E];
#pragma unroll
  for (int t = 0; t < E; t++) v[t] = lane * E + t < P ? key[lane * E + t] : ~K(0);
  warp_bitonic<E>(v, lane);
#pragma unroll
  for (int t = 0; t < E; t++) key[lane * E + t] = v[t];
}

// Warp per row, P_i <= 256.
template <typename V, typename K>
__global__ void __launch_bounds__(SG_THREADS, 3) k_sg_warp(Mat<V> A, Mat<V> B, const unsigned *rows,
                                                        const long long *starts, const long long *ub, int32_t *tcol,
                                                        V *tval, long long *ucnt) {
  using KO = SgKey<K>;
  __shared__ K skey[SG_THREADS / 32][SG_WARP_MAX];
  __shared__ V sprod[SG_THREADS / 32][SG_WARP_MAX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t b = starts[SG_WARP], e = starts[SG_WARP + 1];
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lt = (1u << lane) - 1u;
  K *key = skey[w];
  V *prod = sprod[w];
  for (int64_t it = b + (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); it < e; it += nw) {
    const int64_t i = rows[it];
    const int P = sg_expand_warp(A, B, i, lane, key, prod);
    __syncwarp();
    if (P <= 32) sort_row_keys<1>(key, P, lane);
    else if (P <= 64) sort_row_keys<2>(key, P, lane);
    else if (P <= 128) sort_row_keys<4>(key, P, lane);
    else sort_row_keys<8>(key, P, lane);
    __syncwarp();
    const int64_t base = ub[i];
    int heads = 0;
    for (int c0 = 0; c0 < P; c0 += 32) {
      const int idx = c0 + lane;
      const bool valid = idx < P;
      const K k = valid ? key[idx] : K(0);
      const bool head = valid && (idx == 0 || KO::col(key[idx - 1]) != KO::col(k));
      const unsigned hm = __ballot_sync(FULL, head);
      if (head) {
        V v = prod[KO::idx(k)];
        for (int j = idx + 1; j < P && KO::col(key[j]) == KO::col(k); j++) v = v + prod[KO::idx(key[j])];
        const int64_t o = base + heads + __popc(hm & lt);
        tcol[o] = KO::col(k);
        tval[o] = v;
      }
      heads += __popc(hm);
    }
    if (lane == 0) ucnt[i] = heads;
    __syncwarp();
  }
}

// The CTA class's expand (256 < P_i <= 4096): row i's A entries are taken
// 256 at a time, one per thread (column, value, B row length and first
// segment loaded side by side), the lengths scanned across the block into
// product offsets, then each thread produces products q = tid, tid + 256,
// ... of the group -- the owning entry found by a binary search over the
// offsets in shared memory, four products' B loads in flight at a time.  A
// B row that does not lie in its first segment is read through its chain.
// Same keys and products as the warp class (product p = the row's p-th
// product in A-entry-major order).
template <typename V>
__device__ __forceinline__ int sg_expand_cta(const Mat<V> &A, const Mat<V> &B, int64_t i, int tid,
                                             unsigned long long *key, V *prod, int *soff, int32_t *sk, V *sa,
                                             int32_t *sst, int *wsum) {
  constexpr int H = 4;
  const int32_t LA = A.row_sizes[i];
  const Chain ca = load_chain_used(A, (int32_t)i, LA);
  int base = 0;
  for (int32_t e0 = 0; e0 < LA; e0 += SG_THREADS) {
    const int nE = LA - e0 < SG_THREADS ? LA - e0 : SG_THREADS;
    int32_t kb = 0, lb = 0, st0 = -1;
    V a = V(0);
    if (tid < nE) {
      const int64_t qa = ca.phys(e0 + tid);
      kb = A.cols[qa];
      a = A.vals[qa];
      lb = B.row_sizes[kb];
      const int2 s0 = __ldg(reinterpret_cast<const int2 *>(B.seg + 2 * (int64_t)kb));
      st0 = s0.x >= 0 && s0.y - s0.x >= lb ? s0.x : -1;  // all of the row in its first segment
    }
    const int incl = warp_incl_scan(lb);
    if ((tid & 31) == 31) wsum[tid >> 5] = incl;
    __syncthreads();
    int pre = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < SG_THREADS / 32; q++) {
      if (q < (tid >> 5)) pre += wsum[q];
      tot += wsum[q];
    }
    soff[tid] = pre + incl - lb;
    sk[tid] = kb;
    sa[tid] = a;
    sst[tid] = st0;
    __syncthreads();
    for (int q0 = tid; q0 < tot; q0 += H * SG_THREADS) {
      int own[H];
      int32_t bc[H];
      V bv[H];
#pragma unroll
      for (int h = 0; h < H; h++) {
        const int q = q0 + h * SG_THREADS;
        own[h] = 0;
        bc[h] = 0;
        bv[h] = V(0);
        if (q < tot) {
          int lo = 0, hi = nE - 1;  // the last entry whose offset is <= q owns q
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (soff[mid] <= q) lo = mid;
            else hi = mid - 1;
          }
          own[h] = lo;
          const int32_t j = q - soff[lo];
          const int64_t qb = sst[lo] >= 0 ? (int64_t)sst[lo] + j : load_chain(B, sk[lo]).phys(j);
          bc[h] = B.cols[qb];
          bv[h] = B.vals[qb];
        }
      }
#pragma unroll
      for (int h = 0; h < H; h++) {
        const int q = q0 + h * SG_THREADS;
        if (q < tot) {
          key[base + q] = ((unsigned long long)(uint32_t)bc[h] << 32) | (unsigned long long)(base + q);
          V pr;
          if constexpr (sizeof(V) == 4) pr = __fmul_rn(sa[own[h]], bv[h]);
          else pr = __dmul_rn(sa[own[h]], bv[h]);
          prod[base + q] = pr;
        }
      }
    }
    base += tot;
    __syncthreads();  // the group's tables are reused by the next group
  }
  return base;
}

// CTA per row, 256 < P_i <= 4096 (dynamic shared memory).
template <typename V>
__global__ void __launch_bounds__(SG_THREADS) k_sg_cta(Mat<V> A, Mat<V> B, const unsigned *rows,
                                                       const long long *starts, const long long *ub, int32_t *tcol,
                                                       V *tval, long long *ucnt) {
  extern __shared__ unsigned long long sg_smem[];
  unsigned long long *key = sg_smem;
  V *prod = reinterpret_cast<V *>(sg_smem + SG_CTA_MAX);
  __shared__ int wheads[SG_THREADS / 32 + 1];
  __shared__ int soff[SG_THREADS], wsum[SG_THREADS / 32];
  __shared__ int32_t sk[SG_THREADS], sst[SG_THREADS];
  __shared__ V sa[SG_THREADS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t b = starts[SG_CTA], e = starts[SG_CTA + 1];
  for (int64_t it = b + blockIdx.x; it < e; it += gridDim.x) {
    const int64_t i = rows[it];
    const int P = sg_expand_cta(A, B, i, threadIdx.x, key, prod, soff, sk, sa, sst, wsum);
    const int n2 = next_pow2(P);
    for (int t = P + threadIdx.x; t < n2; t += SG_THREADS) key[t] = ~0ull;
    __syncthreads();
    bitonic(key, n2, threadIdx.x, SG_THREADS, []() { __syncthreads(); });
    const int64_t base = ub[i];
    int heads = 0;  // running total (uniform across the block)
    for (int c0 = 0; c0 < P; c0 += SG_THREADS) {
      const int idx = c0 + threadIdx.x;
      const bool valid = idx < P;
      const unsigned long long k = valid ? key[idx] : 0;
      const bool head = valid && (idx == 0 || (key[idx - 1] >> 32) != (k >> 32));
      const unsigned hm = __ballot_sync(FULL, head);
      if (lane == 0) wheads[w] = __popc(hm);
      __syncthreads();
      int before = 0, total = 0;
      for (int q = 0; q < SG_THREADS / 32; q++) {
        if (q < w) before += wheads[q];
        total += wheads[q];
      }
      if (head) {
        V v = prod[(uint32_t)k];
        for (int j = idx + 1; j < P && (key[j] >> 32) == (k >> 32); j++) v = v + prod[(uint32_t)key[j]];
        const int64_t o = base + heads + before + __popc(hm & ((1u << lane) - 1u));
        tcol[o] = (int32_t)(k >> 32);
        tval[o] = v;
      }
      heads += total;
      __syncthreads();
    }
    if (threadIdx.x == 0) ucnt[i] = heads;
    __syncthreads();
  }
}

// Global path: expand rows with P_i > 4096 into (key = slot<<cb | col, value = global product index).
template <typename V>
__global__ void k_sg_global_expand(Mat<V> A, Mat<V> B, const unsigned *rows, const long long *starts,
                                   const long long *goff, int cb, unsigned long long *gkey, unsigned *gidx,
                                   V *gprod) {
  const int lane = threadIdx.x & 31;
  const int64_t b = starts[SG_GLOBAL], e = starts[SG_GLOBAL + 1];
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t it = b + (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); it < e; it += nw) {
    const int64_t i = rows[it];
    const int64_t slot = it - b;
    const int64_t o = goff[slot];
    const Chain ca = load_chain(A, (int32_t)i);
    const int64_t LA = A.row_sizes[i];
    int64_t pos = 0;
    for (int64_t ea = 0; ea < LA; ea++) {
      const int64_t qa = ca.phys(ea);
      const int32_t k = A.cols[qa];
      const V a = A.vals[qa];
      const Chain ck = load_chain(B, k);
      const int64_t LB = B.row_sizes[k];
      for (int64_t j = lane; j < LB; j += 32) {
        const int64_t qb = ck.phys(j);
        gkey[o + pos + j] = ((unsigned long long)slot << cb) | (unsigned long long)(uint32_t)B.cols[qb];
        gidx[o + pos + j] = (unsigned)(o + pos + j);
        V pr;
        if constexpr (sizeof(V) == 4) pr = __fmul_rn(a, B.vals[qb]);
        else pr = __dmul_rn(a, B.vals[qb]);
        gprod[o + pos + j] = pr;
      }
      pos += LB;
    }
  }
}

// Heads of equal keys after the sort.
__global__ void k_sg_global_flags(const unsigned long long *gkey, int64_t n, long long *flag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride)
    flag[q] = (q == 0 || gkey[q] != gkey[q - 1]) ? 1 : 0;
}

template <typename V>
__global__ void k_sg_global_emit(const unsigned long long *gkey, const unsigned *gidx, const V *gprod, int64_t n,
                                 const long long *hpos, const unsigned *rows, const long long *starts,
                                 const long long *goff, const long long *ub, int cb, int32_t *tcol, V *tval,
                                 long long *ucnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const unsigned long long cmask = (1ull << cb) - 1;
  const int64_t b = starts[SG_GLOBAL];
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    const unsigned long long k = gkey[q];
    if (q > 0 && gkey[q - 1] == k) continue;
    const int64_t slot = (int64_t)(k >> cb);
    const int64_t i = rows[b + slot];
    V v = gprod[gidx[q]];
    for (int64_t j = q + 1; j < n && gkey[j] == k; j++) v = v + gprod[gidx[j]];
    const int64_t first = hpos[goff[slot]];  // head rank of the row's first product
    const int64_t o = ub[i] + (hpos[q] - first);
    tcol[o] = (int32_t)(k & cmask);
    tval[o] = v;
    atomicAdd((unsigned long long *)&ucnt[i], 1ull);
  }
}

// slot products for the global class: goff[slot] = ub-like offsets of the
// large rows in a dense staging array
__global__ void k_sg_global_sizes(const unsigned *rows, const long long *starts, const long long *ub,
                                  long long *gsz) {
  const int64_t b = starts[SG_GLOBAL], e = starts[SG_GLOBAL + 1];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t it = b + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it <= e; it += stride)
    gsz[it - b] = it < e ? ub[rows[it] + 1] - ub[rows[it]] : 0;
}

static int grid_for(int64_t n, int block) {
  int64_t g = div_up(n, block);
  int64_t cap = (int64_t)sm_count() * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

template <typename V>
static int spgemm_impl(dcsr_handle hA, dcsr_handle hB, dcsr_handle hC, cudaStream_t s) {
  const int32_t n = hA->n_rows;
  Mat<V> A = hA->view<V>(), B = hB->view<V>();
  Arena ar;
  ar.status = hC->stat + ST_STATUS;  // look-back timeouts reach C's status
  DCSR_TRY(ar.reserve(arena_bytes(n + 2, 8) * 4 + arena_bytes(n + 2, 4) * 2 + arena_bytes(8, 8) +
                          radix_scratch_bytes(n) + scan_scratch_bytes(n + 2), s));
  long long *cnt = ar.take<long long>(n + 2), *capub = ar.take<long long>(n + 2);
  unsigned long long *k0 = ar.take<unsigned long long>(n + 2), *k1 = ar.take<unsigned long long>(n + 2);
  unsigned *r0 = ar.take<unsigned>(n + 2), *r1 = ar.take<unsigned>(n + 2);
  long long *starts = ar.take<long long>(8);  // [0..4] class starts, [5] products of the global class
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  long long *ub = cnt;  // scanned in place
  DCSR_CUDA(cudaMemsetAsync(starts, 0, sizeof(long long) * 8, s));
  if (n > 0) {
    DCSR_LAUNCH(k_sg_count<V>, grid_for((int64_t)n * 8, SG_THREADS), SG_THREADS, 0, s, A, B, hC->o, cnt, capub, k0,
                r0, (unsigned long long *)(starts + 5));
    if (n > 1) DCSR_TRY(radix_sort_pairs(&k0, &r0, &k1, &r1, n, 2, ar, s));
  }
  DCSR_LAUNCH(k_sg_classes, 1, 32, 0, s, k0, n, starts);
  DCSR_TRY(scan2_i64(cnt, ub, hC->stat + ST_TOTAL, capub, capub, hC->stat + ST_AUX + 1, n + 1, ar, s));
  // the one read before the numeric pass: staging and C's pool are sized here
  long long host[8];
  DCSR_CUDA(cudaMemcpyAsync(host, starts, sizeof(long long) * 6, cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaMemcpyAsync(host + 6, hC->stat + ST_TOTAL, sizeof(long long), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaMemcpyAsync(host + 7, hC->stat + ST_AUX + 1, sizeof(long long), cudaMemcpyDeviceToHost, s));
  long long st_word = 0;
  DCSR_CUDA(cudaMemcpyAsync(&st_word, hC->stat + ST_STATUS, sizeof(long long), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  if (st_word == DCSR_TIMEOUT) {
    DCSR_CUDA(cudaMemsetAsync(hC->stat + ST_STATUS, 0, sizeof(long long), s));
    ar.release(s);
    return DCSR_TIMEOUT;
  }
  const int64_t Pg = host[5], P = host[6], cap_bound = pool_capacity(hC->o, host[7]);
  const int64_t n_global = host[SG_GLOBAL + 1] - host[SG_GLOBAL];
  if (Pg > 0xffffffffLL) return DCSR_NOT_SUPPORTED;
  // staging: row i's unique columns at ub[i]
  int32_t *tcol = nullptr;
  V *tval = nullptr;
  long long *ucnt = nullptr;
  DCSR_CUDA(dcsr::dev_alloc((void **)&tcol, sizeof(int32_t) * (P + 1), s));
  DCSR_CUDA(dcsr::dev_alloc((void **)&tval, sizeof(V) * (P + 1), s));
  DCSR_CUDA(dcsr::dev_alloc((void **)&ucnt, sizeof(long long) * (n + 2), s));
  DCSR_CUDA(cudaMemsetAsync(ucnt, 0, sizeof(long long) * (n + 2), s));
  const size_t cta_smem = SG_CTA_MAX * (sizeof(unsigned long long) + sizeof(V));
  static const int g_warp = persistent_grid((const void *)k_sg_warp<double, unsigned long long>, SG_THREADS, 0);
  static const int g_cta = [] {  // once, thread-safely: the CTA kernels' shared-memory limit, then their grid
    cudaFuncSetAttribute(k_sg_cta<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(SG_CTA_MAX * (sizeof(unsigned long long) + sizeof(float))));
    cudaFuncSetAttribute(k_sg_cta<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(SG_CTA_MAX * (sizeof(unsigned long long) + sizeof(double))));
    return persistent_grid((const void *)k_sg_cta<double>, SG_THREADS,
                           SG_CTA_MAX * (sizeof(unsigned long long) + sizeof(double)));
  }();
  if (host[SG_WARP + 1] > host[SG_WARP]) {
    if (hB->n_cols <= (1 << 24))  // (column, p) in 32-bit keys
      DCSR_LAUNCH((k_sg_warp<V, unsigned>), g_warp, SG_THREADS, 0, s, A, B, r0, starts, ub, tcol, tval, ucnt);
    else
      DCSR_LAUNCH((k_sg_warp<V, unsigned long long>), g_warp, SG_THREADS, 0, s, A, B, r0, starts, ub, tcol, tval,
                  ucnt);
  }
  if (host[SG_CTA + 1] > host[SG_CTA])
    DCSR_LAUNCH(k_sg_cta<V>, g_cta, SG_THREADS, cta_smem, s, A, B, r0, starts, ub, tcol, tval, ucnt);
  Arena gg;
  if (n_global > 0) {
    // products of all large rows, laid out densely by slot, then one stable
    // radix sort by (slot, column) keeps every column's products in p order
    gg.status = hC->stat + ST_STATUS;  // look-back timeouts reach C's status
    DCSR_TRY(gg.reserve(arena_bytes(n_global + 2, 8) + 2 * arena_bytes(Pg, 8) + 2 * arena_bytes(Pg, 4) +
                            arena_bytes(Pg, sizeof(V)) + arena_bytes(Pg + 1, 8) + radix_scratch_bytes(Pg) +
                            scan_scratch_bytes(Pg + 1) + scan_scratch_bytes(n_global + 2), s));
    long long *goff = gg.take<long long>(n_global + 2);
    unsigned long long *gk0 = gg.take<unsigned long long>(Pg), *gk1 = gg.take<unsigned long long>(Pg);
    unsigned *gi0 = gg.take<unsigned>(Pg), *gi1 = gg.take<unsigned>(Pg);
    V *gprod = (V *)gg.take<double>(Pg);
    long long *hpos = gg.take<long long>(Pg + 1);
    if (gg.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
    DCSR_LAUNCH(k_sg_global_sizes, grid_for(n_global + 1, 256), 256, 0, s, r0, starts, ub, goff);
    DCSR_TRY(scan_i64(goff, goff, n_global + 1, nullptr, gg, s));
    const int cb = bits_for(hB->n_cols);
    DCSR_LAUNCH(k_sg_global_expand<V>, grid_for(n_global * 32, 256), 256, 0, s, A, B, r0, starts, goff, cb, gk0, gi0,
                gprod);
    DCSR_TRY(radix_sort_pairs(&gk0, &gi0, &gk1, &gi1, Pg, bits_for(n_global) + cb, gg, s));
    DCSR_LAUNCH(k_sg_global_flags, grid_for(Pg, 256), 256, 0, s, gk0, Pg, hpos);
    DCSR_TRY(scan_i64(hpos, hpos, Pg, nullptr, gg, s));
    DCSR_LAUNCH(k_sg_global_emit<V>, grid_for(Pg, 256), 256, 0, s, gk0, gi0, gprod, Pg, hpos, r0, starts, goff, ub,
                cb, tcol, tval, ucnt);
  }
  // C's rows go straight from the staging area into C's pool (policy
  // capacities); the second and last synchronisation reads C's pool top
  const int st = load_from_rows(hC, ub, ucnt, tcol, tval, cap_bound, s);
  gg.release(s);
  ar.release(s);
  dcsr::dev_free(tcol, s);
  dcsr::dev_free(tval, s);
  dcsr::dev_free(ucnt, s);
  return st;
}

}  // namespace dcsr

using namespace dcsr;

extern "C" int dcsr_spgemm(dcsr_handle A, dcsr_handle B, dcsr_handle C, void *stream) {
  if (!A || !B || !C) return DCSR_BAD_ARG;
  if (A->n_cols != B->n_rows || C->n_rows != A->n_rows || C->n_cols != B->n_cols || A->dtype != B->dtype ||
      C->dtype != A->dtype || C == A || C == B)
    return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (A->dtype == DCSR_F32) return spgemm_impl<float>(A, B, C, s);
  return spgemm_impl<double>(A, B, C, s);
}
