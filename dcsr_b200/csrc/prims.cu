// prims.cu -- device-wide primitives: exclusive scan, stable LSD radix sort of
// (key, value) pairs, and the public segmented primitives
// (count_sorted_indices, reduce_by_key).  All hand-written for sm_100a.
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace dcsr {

std::atomic<uint64_t> g_launches{0};

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

int persistent_grid(const void *kernel, int block, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm * sm_count();
}

// ------------------------------------------------------------------ scan

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// Block-wide exclusive scan of one value per thread; returns the block total.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *total) {
  __shared__ T wsum[33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T inc = warp_incl_scan(v);
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < nw ? wsum[lane] : T(0);
    T wi = warp_incl_scan(w);
    if (lane < nw) wsum[lane] = wi - w;
    if (lane == nw - 1) wsum[32] = wi;
  }
  __syncthreads();
  T out = inc - v + wsum[warp];
  *total = wsum[32];
  __syncthreads();
  return out;
}

__global__ void k_scan_reduce(const long long *in, int64_t n, long long *partial) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  long long s = 0;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    int64_t i = base + j * SCAN_THREADS + threadIdx.x;
    if (i < n) s += in[i];
  }
  s = warp_sum(s);
  __shared__ long long ws[SCAN_THREADS / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < SCAN_THREADS / 32; w++) t += ws[w];
    partial[blockIdx.x] = t;
  }
}

// Single block: exclusive scan of the tile partials in place; total -> *total.
__global__ void k_scan_partials(long long *partial, int64_t ntiles, long long *total) {
  long long carry = 0;
  for (int64_t b = 0; b < ntiles; b += blockDim.x) {
    int64_t i = b + threadIdx.x;
    long long v = i < ntiles ? partial[i] : 0;
    long long bt;
    long long ex = block_excl_scan(v, &bt);
    if (i < ntiles) partial[i] = ex + carry;
    carry += bt;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_down(const long long *in, long long *out, int64_t n, const long long *partial) {
  __shared__ long long tile[SCAN_TILE];
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    int64_t i = base + j * SCAN_THREADS + threadIdx.x;
    tile[j * SCAN_THREADS + threadIdx.x] = i < n ? in[i] : 0;
  }
  __syncthreads();
  long long loc[SCAN_ITEMS];
  long long s = 0;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    loc[j] = tile[threadIdx.x * SCAN_ITEMS + j];
    s += loc[j];
  }
  long long bt;
  long long ex = block_excl_scan(s, &bt) + partial[blockIdx.x];
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    tile[threadIdx.x * SCAN_ITEMS + j] = ex;
    ex += loc[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    int64_t i = base + j * SCAN_THREADS + threadIdx.x;
    if (i < n) out[i] = tile[j * SCAN_THREADS + threadIdx.x];
  }
}

// Small inputs: one block; coalesced loads into shared memory, each thread
// scans 4 consecutive values, one block scan, coalesced stores.
constexpr int SCAN_SMALL = 1024 * 4;
__global__ void __launch_bounds__(1024) k_scan_small(const long long *in, long long *out, int64_t n,
                                                      long long *total) {
  __shared__ long long tile[SCAN_SMALL];
  for (int i = threadIdx.x; i < SCAN_SMALL; i += 1024) tile[i] = i < n ? in[i] : 0;
  __syncthreads();
  long long loc[4], sum = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    loc[j] = tile[threadIdx.x * 4 + j];
    sum += loc[j];
  }
  long long bt;
  long long ex = block_excl_scan(sum, &bt);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    tile[threadIdx.x * 4 + j] = ex;
    ex += loc[j];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += 1024) out[i] = tile[i];
  if (threadIdx.x == 0 && total) *total = bt;
}

size_t scan_scratch_bytes(int64_t n) { return arena_bytes(div_up(n, SCAN_TILE) + 1, 8); }

int scan_i64(const long long *in, long long *out, int64_t n, long long *total, Arena &ar, cudaStream_t s) {
  if (n <= 0) {
    if (total) DCSR_CUDA(cudaMemsetAsync(total, 0, sizeof(long long), s));
    return DCSR_OK;
  }
  if (n <= SCAN_SMALL) {
    DCSR_LAUNCH(k_scan_small, 1, 1024, 0, s, in, out, n, total);
    return DCSR_OK;
  }
  int64_t nt = div_up(n, SCAN_TILE);
  const size_t mark = ar.used;  // partials are stream-ordered scratch: released on return
  long long *partial = ar.take<long long>(nt + 1);
  DCSR_LAUNCH(k_scan_reduce, (unsigned)nt, SCAN_THREADS, 0, s, in, n, partial);
  DCSR_LAUNCH(k_scan_partials, 1, 1024, 0, s, partial, nt, total);
  DCSR_LAUNCH(k_scan_down, (unsigned)nt, SCAN_THREADS, 0, s, in, out, n, partial);
  ar.used = mark;
  return DCSR_OK;
}

// ------------------------------------------------------------ radix sort
//
// Stable LSD radix sort, 8-bit digits.  Per pass: (1) per-tile digit
// histograms, (2) exclusive scan over the digit-major histogram table, (3) a
// stable scatter: each warp ranks its 512 consecutive items with match_any
// (ties keep input order), warps are ordered by a per-digit prefix across the
// block, and the block's global digit offsets come from the scanned table.

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_BINS = 256;
// items per lane: 16 for large inputs, 4 below RS_MID items (more, shorter tiles)
constexpr int64_t RS_MID = 1 << 18;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <int RS_ITEMS>
__global__ void __launch_bounds__(RS_THREADS) k_radix_hist(const unsigned long long *keys, int64_t n, int shift,
                                                            long long *ghist, int64_t ntiles) {
  constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
  __shared__ unsigned h[RS_BINS];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * RS_TILE + (int64_t)warp * (32 * RS_ITEMS);
#pragma unroll 4
  for (int j = 0; j < RS_ITEMS; j++) {
    int64_t i = base + j * 32 + lane;
    unsigned d = i < n ? (unsigned)((keys[i] >> shift) & 0xff) : 0x100u;
    unsigned peers = __match_any_sync(FULL, d);
    if (d < 0x100u && (__ffs(peers) - 1) == lane) atomicAdd(&h[d], (unsigned)__popc(peers));
  }
  __syncthreads();
  ghist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

template <int RS_ITEMS>
__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const unsigned long long *keys, const unsigned *vals,
                                                               unsigned long long *keys_out, unsigned *vals_out,
                                                               int64_t n, int shift, const long long *goff,
                                                               int64_t ntiles) {
  constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
  __shared__ unsigned wcnt[RS_WARPS][RS_BINS];
  __shared__ long long boff[RS_BINS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int w = 0; w < RS_WARPS; w++) wcnt[w][threadIdx.x] = 0;
  boff[threadIdx.x] = goff[(int64_t)threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * RS_TILE + (int64_t)warp * (32 * RS_ITEMS);
  unsigned long long k[RS_ITEMS];
  unsigned rank[RS_ITEMS];
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int j = 0; j < RS_ITEMS; j++) {
    int64_t i = base + j * 32 + lane;
    k[j] = i < n ? keys[i] : ~0ull;
    unsigned d = i < n ? (unsigned)((k[j] >> shift) & 0xff) : 0x100u;
    unsigned peers = __match_any_sync(FULL, d);
    unsigned pre = d < 0x100u ? wcnt[warp][d] : 0u;
    rank[j] = pre + __popc(peers & lt);
    __syncwarp();
    if (d < 0x100u && (__ffs(peers) - 1) == lane) wcnt[warp][d] = pre + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {  // exclusive prefix across warps per digit
    unsigned run = 0;
    for (int w = 0; w < RS_WARPS; w++) {
      unsigned t = wcnt[w][threadIdx.x];
      wcnt[w][threadIdx.x] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RS_ITEMS; j++) {
    int64_t i = base + j * 32 + lane;
    if (i < n) {
      unsigned d = (unsigned)((k[j] >> shift) & 0xff);
      int64_t pos = boff[d] + wcnt[warp][d] + rank[j];
      keys_out[pos] = k[j];
      vals_out[pos] = vals[i];
    }
  }
}

// Small inputs (n <= RS_SMALL): one 1024-thread block runs every pass in
// shared memory on (key, 16-bit input index) pairs -- per pass a digit
// histogram, its scan, and a stable scatter in rounds of 1024 consecutive
// items (warp ranks from match_any, warps ordered by a per-digit prefix) --
// then gathers the values by index.  Same order as the multi-block sort.
constexpr int RS_SMALL = 8192;
constexpr size_t RS_SMALL_SMEM = (size_t)RS_SMALL * (2 * 8 + 2 * 2) + 32 * RS_BINS * 4 + 2 * RS_BINS * 4;

__global__ void __launch_bounds__(1024) k_radix_small(const unsigned long long *keys, const unsigned *vals,
                                                       unsigned long long *keys_out, unsigned *vals_out, int n,
                                                       int bits) {
  extern __shared__ __align__(16) unsigned char sm[];
  unsigned long long *ka = (unsigned long long *)sm;
  unsigned long long *kb = ka + RS_SMALL;
  unsigned short *ia = (unsigned short *)(kb + RS_SMALL);
  unsigned short *ib = ia + RS_SMALL;
  unsigned *wc = (unsigned *)(ib + RS_SMALL);  // [32][256]
  unsigned *base = wc + 32 * RS_BINS;          // running digit offsets
  unsigned *rtot = base + RS_BINS;             // this round's digit totals
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned lt = lanemask_lt();
  for (int i = tid; i < n; i += 1024) {
    ka[i] = keys[i];
    ia[i] = (unsigned short)i;
  }
  for (int shift = 0; shift < bits; shift += 8) {
    if (tid < RS_BINS) base[tid] = 0;
    __syncthreads();
    for (int i = tid; i < n; i += 1024) atomicAdd(&base[(unsigned)(ka[i] >> shift) & 0xff], 1u);
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the 256 digit counts (8 per lane)
      unsigned v[8], t = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        v[j] = base[lane * 8 + j];
        t += v[j];
      }
      unsigned ex = warp_incl_scan(t) - t;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        base[lane * 8 + j] = ex;
        ex += v[j];
      }
    }
    __syncthreads();
    for (int r0 = 0; r0 < n; r0 += 1024) {
      const int i = r0 + tid;
      for (int q = tid; q < 32 * RS_BINS; q += 1024) wc[q] = 0;
      __syncthreads();
      const unsigned long long k = i < n ? ka[i] : 0ull;
      const unsigned d = i < n ? (unsigned)(k >> shift) & 0xff : 0x100u;
      const unsigned peers = __match_any_sync(FULL, d);
      const unsigned rank = __popc(peers & lt);
      if (d < 0x100u && (__ffs(peers) - 1) == lane) wc[warp * RS_BINS + d] = __popc(peers);
      __syncthreads();
      if (tid < RS_BINS) {  // prefix across warps for digit tid
        unsigned run = 0;
        for (int w = 0; w < 32; w++) {
          const unsigned c = wc[w * RS_BINS + tid];
          wc[w * RS_BINS + tid] = run;
          run += c;
        }
        rtot[tid] = run;
      }
      __syncthreads();
      if (d < 0x100u) {
        const unsigned pos = base[d] + wc[warp * RS_BINS + d] + rank;
        kb[pos] = k;
        ib[pos] = ia[i];
      }
      __syncthreads();
      if (tid < RS_BINS) base[tid] += rtot[tid];
      __syncthreads();
    }
    unsigned long long *tk = ka;
    ka = kb;
    kb = tk;
    unsigned short *ti = ia;
    ia = ib;
    ib = ti;
  }
  for (int i = tid; i < n; i += 1024) {
    keys_out[i] = ka[i];
    vals_out[i] = vals[ia[i]];
  }
}

size_t radix_scratch_bytes(int64_t n) {
  int64_t nt = div_up(n, RS_THREADS * 4);
  return arena_bytes(nt * RS_BINS, 8) + scan_scratch_bytes(nt * RS_BINS);
}

template <int ITEMS>
static int radix_passes(unsigned long long **keys, unsigned **vals, unsigned long long **keys_tmp,
                        unsigned **vals_tmp, int64_t n, int bits, Arena &ar, cudaStream_t s) {
  const int64_t nt = div_up(n, RS_THREADS * ITEMS);
  size_t mark = ar.used;
  long long *hist = ar.take<long long>(nt * RS_BINS);
  size_t mark2 = ar.used;
  for (int shift = 0; shift < bits; shift += 8) {
    DCSR_LAUNCH(k_radix_hist<ITEMS>, (unsigned)nt, RS_THREADS, 0, s, *keys, n, shift, hist, nt);
    ar.used = mark2;
    DCSR_TRY(scan_i64(hist, hist, nt * RS_BINS, nullptr, ar, s));
    DCSR_LAUNCH(k_radix_scatter<ITEMS>, (unsigned)nt, RS_THREADS, 0, s, *keys, *vals, *keys_tmp, *vals_tmp, n,
                shift, hist, nt);
    unsigned long long *tk = *keys;
    *keys = *keys_tmp;
    *keys_tmp = tk;
    unsigned *tv = *vals;
    *vals = *vals_tmp;
    *vals_tmp = tv;
  }
  ar.used = mark;
  return DCSR_OK;
}

int radix_sort_pairs(unsigned long long **keys, unsigned **vals, unsigned long long **keys_tmp,
                     unsigned **vals_tmp, int64_t n, int bits, Arena &ar, cudaStream_t s) {
  if (n <= 1) return DCSR_OK;
  if (n <= RS_SMALL) {
    static bool attr = false;
    if (!attr) {
      DCSR_CUDA(cudaFuncSetAttribute(k_radix_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_SMALL_SMEM));
      attr = true;
    }
    DCSR_LAUNCH(k_radix_small, 1, 1024, RS_SMALL_SMEM, s, *keys, *vals, *keys_tmp, *vals_tmp, (int)n, bits);
    unsigned long long *tk = *keys;
    *keys = *keys_tmp;
    *keys_tmp = tk;
    unsigned *tv = *vals;
    *vals = *vals_tmp;
    *vals_tmp = tv;
    return DCSR_OK;
  }
  if (n <= RS_MID) return radix_passes<4>(keys, vals, keys_tmp, vals_tmp, n, bits, ar, s);
  return radix_passes<16>(keys, vals, keys_tmp, vals_tmp, n, bits, ar, s);
}

// ------------------------------------------------- public segmented ops

// X[I[n]] += run length, one atomic per run (runs found with warp ballots).
__global__ void k_count_sorted(const int32_t *I, int64_t n, int32_t *X) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    int64_t i = base + threadIdx.x;
    int32_t key = i < n ? I[i] : INT32_MIN;
    int32_t prev = __shfl_up_sync(FULL, key, 1);
    const int lane = threadIdx.x & 31;
    if (lane == 0) prev = (i > 0 && i < n) ? I[i - 1] : INT32_MIN;
    bool head = i < n && (key != prev || lane == 0);
    unsigned hm = __ballot_sync(FULL, head);
    unsigned valid = __ballot_sync(FULL, i < n);
    if (head) {
      unsigned later = hm & ~((2u << lane) - 1u);
      int end = later ? (__ffs(later) - 1) : (32 - __clz(valid));
      atomicAdd(&X[key], end - lane);
    }
  }
}

// Reduce-by-key: heads flagged, head positions compacted by scan, then each
// head sums its run left to right (deterministic order).
__global__ void k_rbk_flags(const int32_t *keys, int64_t n, long long *flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}
template <typename V>
__global__ void k_rbk_emit(const int32_t *keys, const V *vals, int64_t n, const long long *pos,
                           int32_t *keys_out, V *vals_out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (i > 0 && keys[i] == keys[i - 1]) return;
  V acc = vals[i];
  for (int64_t j = i + 1; j < n && keys[j] == keys[i]; j++) acc = acc + vals[j];
  keys_out[pos[i]] = keys[i];
  vals_out[pos[i]] = acc;
}

// ------------------------------------------- allocation-free reduce-by-key
//
// Scratch for dcsr_reduce_by_key_noalloc: head positions (one int64 per key)
// and the scan's tile partials, in one static device array.  Every GPU that
// loads the library holds it until exit.  Host code must not pass the
// symbol itself to a kernel (in host code it names a host-side stand-in);
// the device address is looked up once per device.
constexpr size_t NOALLOC_POS_BYTES = (size_t)DCSR_NOALLOC_MAX_KEYS * sizeof(long long);
constexpr size_t NOALLOC_BYTES = NOALLOC_POS_BYTES + 2 * 256 +
                                 ((DCSR_NOALLOC_MAX_KEYS + SCAN_TILE - 1) / SCAN_TILE + 1) * sizeof(long long);
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

static int noalloc_scratch(void **out) {
  static std::mutex mu;
  static void *ptr[128] = {};
  int dev = 0;
  DCSR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return DCSR_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lock(mu);
  if (!ptr[dev]) {
    void *p = nullptr;
    DCSR_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    ptr[dev] = p;
  }
  *out = ptr[dev];
  return DCSR_OK;
}

}  // namespace dcsr

using namespace dcsr;

extern "C" int dcsr_reduce_by_key_noalloc(const int32_t *keys, const void *vals, int64_t n, int32_t dtype,
                                          int32_t *keys_out, void *vals_out, int64_t *n_out, void *stream) {
  if (n < 0 || n > DCSR_NOALLOC_MAX_KEYS || (dtype != DCSR_F32 && dtype != DCSR_F64) || !n_out ||
      (n > 0 && (!keys || !vals || !keys_out || !vals_out)))
    return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    DCSR_CUDA(cudaMemsetAsync(n_out, 0, sizeof(int64_t), s));
    return DCSR_OK;
  }
  void *base = nullptr;
  DCSR_TRY(noalloc_scratch(&base));
  Arena ar;  // a view over the static array: take() only, never reserve()/release()
  ar.base = (char *)base;
  ar.cap = NOALLOC_BYTES;
  ar.used = 0;
  long long *pos = ar.take<long long>(n);  // fully rewritten below before any read
  const unsigned g = (unsigned)div_up(n, 256);
  DCSR_LAUNCH(k_rbk_flags, g, 256, 0, s, keys, n, pos);
  DCSR_TRY(scan_i64(pos, pos, n, (long long *)n_out, ar, s));
  if (dtype == DCSR_F32)
    DCSR_LAUNCH(k_rbk_emit<float>, g, 256, 0, s, keys, (const float *)vals, n, pos, keys_out, (float *)vals_out);
  else
    DCSR_LAUNCH(k_rbk_emit<double>, g, 256, 0, s, keys, (const double *)vals, n, pos, keys_out,
                (double *)vals_out);
  return DCSR_OK;
}

extern "C" int dcsr_count_sorted_indices(const int32_t *I, int64_t n, int32_t *X, void *stream) {
  if (n < 0 || (n > 0 && (!I || !X))) return DCSR_BAD_ARG;
  if (n == 0) return DCSR_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int grid = (int)std::min<int64_t>(div_up(n, 256), (int64_t)sm_count() * 8);
  DCSR_LAUNCH(k_count_sorted, grid, 256, 0, s, I, n, X);
  return DCSR_OK;
}

extern "C" int dcsr_reduce_by_key(const int32_t *keys, const void *vals, int64_t n, int32_t dtype, int32_t *keys_out,
                                  void *vals_out, int64_t *n_out, void *stream) {
  if (n < 0 || (dtype != DCSR_F32 && dtype != DCSR_F64)) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    if (n_out) DCSR_CUDA(cudaMemsetAsync(n_out, 0, sizeof(int64_t), s));
    return DCSR_OK;
  }
  Arena ar;
  DCSR_TRY(ar.reserve(arena_bytes(n, 8) + scan_scratch_bytes(n), s));
  long long *pos = ar.take<long long>(n);
  unsigned g = (unsigned)div_up(n, 256);
  DCSR_LAUNCH(k_rbk_flags, g, 256, 0, s, keys, n, pos);
  DCSR_TRY(scan_i64(pos, pos, n, (long long *)n_out, ar, s));
  if (dtype == DCSR_F32)
    DCSR_LAUNCH(k_rbk_emit<float>, g, 256, 0, s, keys, (const float *)vals, n, pos, keys_out, (float *)vals_out);
  else
    DCSR_LAUNCH(k_rbk_emit<double>, g, 256, 0, s, keys, (const double *)vals, n, pos, keys_out,
                (double *)vals_out);
  ar.release(s);
  return DCSR_OK;
}
