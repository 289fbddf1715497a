// prims.cu -- device-wide primitives: exclusive scan, stable LSD radix sort of
// (key, value) pairs, and the public segmented primitives
// (count_sorted_indices, reduce_by_key).  All hand-written for sm_100a.
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace dcsr {

std::atomic<uint64_t> g_launches{0};

bool debug_sync() {
  static const bool on = [] {
    const char *e = getenv("DCSR_DEBUG_SYNC");
    return e && e[0] == '1';
  }();
  return on;
}

void debug_check(cudaStream_t s, const char *kernel, const char *file, int line) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) fprintf(stderr, "dcsr: kernel %s (%s:%d) failed: %s\n", kernel, file, line, cudaGetErrorString(e));
}

int sm_count() {
  // function-local statics are initialised once, thread-safely (the server
  // launches from several threads)
  static const int n = [] {
    int dev = 0, c = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    return c > 0 ? c : 148;
  }();
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

// ------------------------------------------------- decoupled look-back
//
// Single-pass kernels: every block takes the next tile number from a device
// counter (so all tiles before it are running or finished), publishes its
// tile's aggregate, adds the aggregates of the tiles before it back to the
// nearest published inclusive prefix, and publishes its own inclusive prefix.
// A wait is only ever on an earlier tile, which therefore always finishes;
// every wait still has an iteration limit, after which it counts a fault and
// stops waiting.

__device__ unsigned long long g_spin_faults = 0;
constexpr int SPIN_LIMIT = 1 << 22;
// Wait limit of the look-back kernels (SPIN_LIMIT unless a test lowered it)
// and a test switch that keeps the first tile of every single-pass kernel
// from publishing, so the waits on it run out (dcsr_debug_lookback).
__device__ int g_spin_limit = SPIN_LIMIT;
__device__ int g_lb_stall = 0;
constexpr int LB_W = 8;  // earlier tiles whose flags one radix look-back step loads together

__device__ __forceinline__ unsigned long long ld_vol(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}

// Look-back words are packed: a tag (the epoch's low 30 bits, a 2-bit kind)
// above a 32-bit value, so a word is published with one store and read with
// one load -- no fences, no second load.  A sort's word per (tile, digit)
// holds a count (kind 1: the tile's aggregate, 2: its inclusive prefix); a
// scan's four words per tile hold the halves of its 64-bit aggregate and
// inclusive prefix (kind 1: written).  A word is current when its tag is the
// kernel's; the tag repeats every 2^30 kernels on one area, so the kernel
// whose last block advances the epoch to such a multiple clears the area
// (lb_advance) and a stale word never matches.
constexpr unsigned long long LB_EMASK = (1ull << 30) - 1;
__device__ __forceinline__ unsigned long long lb_pack(unsigned long long e, int kind, unsigned v) {
  return ((e & LB_EMASK) << 34) | ((unsigned long long)kind << 32) | v;
}

// A wait that gave up: count it, mark the area's fault word with this
// kernel's epoch (its other waits then give up early) and report
// DCSR_TIMEOUT in the operation's status word.
__device__ __forceinline__ void lb_give_up(const Lookback &lb, unsigned long long e) {
  atomicAdd(&g_spin_faults, 1ull);
  *(volatile unsigned long long *)lb.fault = (e & LB_EMASK) + 1;
  if (lb.status) atomicCAS(reinterpret_cast<unsigned long long *>(lb.status), 0ull, (unsigned long long)DCSR_TIMEOUT);
}
// True when another wait of this kernel (epoch e) gave up already.
__device__ __forceinline__ bool lb_faulted(const Lookback &lb, unsigned long long e) {
  return ld_vol(lb.fault) == (e & LB_EMASK) + 1;
}

// Thread 0 of every block: the block's tile and the kernel's epoch.
__device__ __forceinline__ void lb_begin(const Lookback &lb, unsigned *tile, unsigned long long *ep) {
  if (threadIdx.x == 0) {
    *tile = atomicAdd(lb.tiles, 1u);
    *ep = ld_vol(lb.epoch);
  }
}

// End of every block (all threads): true in the last block to finish.
__device__ __forceinline__ bool lb_end(const Lookback &lb) {
  __shared__ int last;
  __syncthreads();
  // (no fence: this block's results reach later kernels at the launch boundary)
  if (threadIdx.x == 0) last = atomicAdd(lb.done, 1u) == gridDim.x - 1;
  __syncthreads();
  return last;
}

// The last block (all its threads): reset the counters and advance the
// epoch; at a multiple of 2^30 clear the slots first (packed radix tags).
__device__ __forceinline__ void lb_advance(const Lookback &lb) {
  __shared__ unsigned long long next;
  if (threadIdx.x == 0) next = ld_vol(lb.epoch) + 1;
  __syncthreads();
  if ((next & LB_EMASK) == 0)
    for (unsigned long long i = threadIdx.x; i < lb.slots; i += blockDim.x) lb.flag[i] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    *(volatile unsigned *)lb.tiles = 0;
    *(volatile unsigned *)lb.done = 0;
    __threadfence();
    *(volatile unsigned long long *)lb.epoch = next;
  }
}

long long spin_faults() {
  unsigned long long v = 0;
  if (cudaMemcpyFromSymbol(&v, g_spin_faults, sizeof(v)) != cudaSuccess) return -1;
  return (long long)v;
}

int debug_lookback(int spin_limit, int stall) {
  const int lim = spin_limit > 0 ? spin_limit : SPIN_LIMIT;
  DCSR_CUDA(cudaMemcpyToSymbol(g_spin_limit, &lim, sizeof(int)));
  DCSR_CUDA(cudaMemcpyToSymbol(g_lb_stall, &stall, sizeof(int)));
  DCSR_CUDA(cudaDeviceSynchronize());
  return DCSR_OK;
}

// Scan operands: one array, or two independent arrays of the same length
// scanned by one launch (tiles [0, nt) scan the first, [nt, 2nt) the second).
struct ScanArgs {
  const long long *in[2];
  long long *out[2];
  long long *total[2];
  int64_t n, nt;
};

// Exclusive scan, one pass: tiles of SCAN_TILE values; warp 0 looks back over
// 32 earlier tiles of its array at a time.  In place (in == out) is allowed.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_1p(ScanArgs a, Lookback lb) {
  __shared__ long long tile[SCAN_TILE];
  __shared__ unsigned sh_tile;
  __shared__ unsigned long long sh_ep;
  __shared__ long long sh_prefix;
  lb_begin(lb, &sh_tile, &sh_ep);
  __syncthreads();
  const int64_t t = sh_tile;
  const unsigned long long e = sh_ep;
  if (t >= gridDim.x) {  // a tile counter left non-zero (a bug): report it, touch nothing
    if (threadIdx.x == 0) lb_give_up(lb, e);
    if (lb_end(lb)) lb_advance(lb);
    return;
  }
  const int arr = t >= a.nt ? 1 : 0;
  const int64_t t0 = arr * a.nt;  // this array's first tile
  const long long *__restrict__ in = a.in[arr];
  long long *out = a.out[arr];
  const int64_t n = a.n;
  const int64_t base = (t - t0) * SCAN_TILE;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    const int64_t i = base + j * SCAN_THREADS + threadIdx.x;
    tile[j * SCAN_THREADS + threadIdx.x] = i < n ? in[i] : 0;
  }
  __syncthreads();
  long long loc[SCAN_ITEMS];
  long long sum = 0;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    loc[j] = tile[threadIdx.x * SCAN_ITEMS + j];
    sum += loc[j];
  }
  long long bt;
  long long ex = block_excl_scan(sum, &bt);
  if (threadIdx.x < 32) {
    // look-back: slot words 4t..4t+3 hold the tile's aggregate (low, high
    // half) and inclusive prefix (low, high half), each a packed word written
    // once per epoch, so a reader that sees both halves of one pair current
    // has a consistent value -- no fences
    const int lane = threadIdx.x;
    const unsigned long long tag = e & LB_EMASK;
    unsigned long long *w = lb.flag;
    auto cur = [&](unsigned long long x) { return (x >> 34) == tag && ((x >> 32) & 3) == 1; };
    long long excl = 0;
    if (t == t0) {
      if (lane == 0 && !(g_lb_stall && t == 0)) {
        *(volatile unsigned long long *)(w + 4 * t + 2) = lb_pack(e, 1, (unsigned)bt);
        *(volatile unsigned long long *)(w + 4 * t + 3) = lb_pack(e, 1, (unsigned)((unsigned long long)bt >> 32));
      }
    } else {
      if (lane == 0) {
        *(volatile unsigned long long *)(w + 4 * t + 0) = lb_pack(e, 1, (unsigned)bt);
        *(volatile unsigned long long *)(w + 4 * t + 1) = lb_pack(e, 1, (unsigned)((unsigned long long)bt >> 32));
      }
      int idle = 0;
      for (int64_t j = t - 1;;) {
        const int64_t q = j - lane;  // lane 0: the nearest earlier tile
        bool ready = true, inc = true;
        long long v = 0;
        if (q >= t0) {  // before the array's first tile: an inclusive prefix of 0
          const unsigned long long a0 = ld_vol(w + 4 * q), a1 = ld_vol(w + 4 * q + 1);
          const unsigned long long i0 = ld_vol(w + 4 * q + 2), i1 = ld_vol(w + 4 * q + 3);
          inc = cur(i0) && cur(i1);
          ready = inc || (cur(a0) && cur(a1));
          const unsigned long long lo = inc ? i0 : a0, hi = inc ? i1 : a1;
          v = (long long)(((hi & 0xffffffffull) << 32) | (lo & 0xffffffffull));
        }
        const unsigned rm = __ballot_sync(FULL, ready), im = __ballot_sync(FULL, ready && inc);
        const int first = im ? __ffs(im) - 1 : 32;  // nearest inclusive prefix in this window
        const unsigned need = first >= 31 ? FULL : ((2u << first) - 1u);
        if ((rm & need) == need) {  // everything up to it published
          excl += warp_sum(lane <= first ? v : 0ll);
          if (first < 32) break;
          j -= 32;
          idle = 0;
          continue;
        }
        if (++idle >= g_spin_limit || ((idle & 1023) == 1023 && __any_sync(FULL, lb_faulted(lb, e)))) {
          if (lane == 0) lb_give_up(lb, e);
          break;
        }
        if (idle >= 32) __nanosleep(64);
      }
      if (lane == 0) {
        const unsigned long long p = (unsigned long long)(excl + bt);
        *(volatile unsigned long long *)(w + 4 * t + 2) = lb_pack(e, 1, (unsigned)p);
        *(volatile unsigned long long *)(w + 4 * t + 3) = lb_pack(e, 1, (unsigned)(p >> 32));
      }
    }
    if (lane == 0) sh_prefix = excl;
  }
  __syncthreads();
  ex += sh_prefix;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    tile[threadIdx.x * SCAN_ITEMS + j] = ex;
    ex += loc[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    const int64_t i = base + j * SCAN_THREADS + threadIdx.x;
    if (i < n) out[i] = tile[j * SCAN_THREADS + threadIdx.x];
  }
  if (threadIdx.x == 0 && a.total[arr] && base + SCAN_TILE >= n) *a.total[arr] = sh_prefix + bt;
  if (lb_end(lb)) lb_advance(lb);
}

// Small inputs: one block; coalesced loads into shared memory, each thread
// scans 4 consecutive values, one block scan, coalesced stores.
constexpr int SCAN_SMALL = 1024 * 4;
__global__ void __launch_bounds__(1024) k_scan_small(ScanArgs a) {
  const long long *__restrict__ in = a.in[blockIdx.x];
  long long *out = a.out[blockIdx.x];
  long long *total = a.total[blockIdx.x];
  const int64_t n = a.n;
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
  ScanArgs a{{in, nullptr}, {out, nullptr}, {total, nullptr}, n, div_up(n, SCAN_TILE)};
  if (n <= SCAN_SMALL) {
    DCSR_LAUNCH(k_scan_small, 1, 1024, 0, s, a);
    return DCSR_OK;
  }
  Lookback lb;
  DCSR_TRY(ar.lookback((size_t)(4 * a.nt), s, &lb));  // four look-back words per tile
  DCSR_LAUNCH(k_scan_1p, (unsigned)a.nt, SCAN_THREADS, 0, s, a, lb);
  return DCSR_OK;
}

int scan2_i64(const long long *in0, long long *out0, long long *total0, const long long *in1, long long *out1,
              long long *total1, int64_t n, Arena &ar, cudaStream_t s) {
  if (n <= 0) {
    if (total0) DCSR_CUDA(cudaMemsetAsync(total0, 0, sizeof(long long), s));
    if (total1) DCSR_CUDA(cudaMemsetAsync(total1, 0, sizeof(long long), s));
    return DCSR_OK;
  }
  ScanArgs a{{in0, in1}, {out0, out1}, {total0, total1}, n, div_up(n, SCAN_TILE)};
  if (n <= SCAN_SMALL) {
    DCSR_LAUNCH(k_scan_small, 2, 1024, 0, s, a);
    return DCSR_OK;
  }
  Lookback lb;
  DCSR_TRY(ar.lookback((size_t)(8 * a.nt), s, &lb));
  DCSR_LAUNCH(k_scan_1p, (unsigned)(2 * a.nt), SCAN_THREADS, 0, s, a, lb);
  return DCSR_OK;
}

// ------------------------------------------------------------ radix sort
//
// Stable LSD radix sort, 8-bit digits.  Up to RS_MID = 2^22 keys, one pass
// over the keys per digit plus one histogram pass (a 1M-triple update's sort
// ran 12 % faster this way than with the three-kernel passes below): (1) one kernel counts the digits of every
// pass at once into per-pass histograms; (2) per pass, one scatter kernel:
// each block takes the next tile, ranks its items per warp with match_any
// (ties keep input order), orders its warps by a per-digit prefix, and finds
// the items of each digit in the tiles before it by decoupled look-back (one
// thread per digit, LB_W earlier tiles per step); the digit's global start is
// the exclusive scan of the pass's histogram.  Larger inputs use three
// kernels per pass (tile histograms, the exclusive scan of the digit-major
// histogram table, a scatter with the same ranking and the scanned offsets),
// which bounds the look-back area (one slot per tile and digit) for the
// largest sorts and for sorts above RS_MID inside a stream capture.

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_BINS = 256;
// items per lane: 16 for large inputs (three kernels per pass), 8 up to RS_MID
// items (single-pass scatter)
#ifndef DCSR_RS_MID_LOG2
#define DCSR_RS_MID_LOG2 22
#endif
constexpr int64_t RS_MID = int64_t(1) << DCSR_RS_MID_LOG2;
// Outside a stream capture the single-pass tier also takes sorts of up to
// RS_BIG keys: its look-back area (one slot per tile and digit, 16 MB at
// 2^24 keys) is grown on demand there, and the 16.1M-key sort of an R-MAT
// 2^20 COO load ran 0.8 ms faster than with three kernels per pass.  Inside
// a capture the tier stops at RS_MID, whose area a batch reserves before
// capturing.  Either tier gives the same (stable) order.
constexpr int64_t RS_BIG = int64_t(1) << 25;

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

// Digit histograms of every pass (keys read once), into the look-back
// area's histogram table (zero on entry: the previous sort's last pass left
// it cleared).
__global__ void __launch_bounds__(RS_THREADS) k_radix_hist_all(const unsigned long long *keys, int64_t n,
                                                                int passes, Lookback lb) {
  __shared__ unsigned h[8 * RS_BINS];
  for (int i = threadIdx.x; i < 8 * RS_BINS; i += RS_THREADS) h[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * RS_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RS_THREADS) {
    const unsigned long long k = keys[i];
    for (int p = 0; p < passes; p++) atomicAdd(&h[p * RS_BINS + (unsigned)((k >> (8 * p)) & 0xff)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * RS_BINS; i += RS_THREADS)
    if (h[i]) atomicAdd(lb.hist + i, h[i]);
}

template <int OS_THREADS, int RS_ITEMS, int MIN_BLOCKS>
__global__ void __launch_bounds__(OS_THREADS, MIN_BLOCKS) k_radix_onesweep(const unsigned long long *keys,
                                                                   const unsigned *vals, unsigned long long *keys_out,
                                                                   unsigned *vals_out, int64_t n, int pass,
                                                                   int last_pass, Lookback lb) {
  constexpr int RS_TILE = OS_THREADS * RS_ITEMS, OS_WARPS = OS_THREADS / 32;
  __shared__ unsigned wcnt[OS_WARPS][RS_BINS];
  __shared__ long long boff[RS_BINS];
  __shared__ unsigned sh_tile;
  __shared__ unsigned long long sh_ep;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, d = threadIdx.x;
  const int shift = 8 * pass;
  lb_begin(lb, &sh_tile, &sh_ep);
  for (int i = threadIdx.x; i < OS_WARPS * RS_BINS; i += OS_THREADS) (&wcnt[0][0])[i] = 0;
  // the digit's first position in the output: exclusive scan of the
  // histogram (thread d < RS_BINS owns digit d from here on)
  long long all;
  const long long gbase =
      block_excl_scan((long long)(d < RS_BINS ? __ldcg(lb.hist + pass * RS_BINS + d) : 0u), &all);
  const int64_t t = sh_tile;
  const unsigned long long e = sh_ep;
  if (t >= gridDim.x) {  // a tile counter left non-zero (a bug): report it, touch nothing
    if (threadIdx.x == 0) lb_give_up(lb, e);
    if (lb_end(lb)) lb_advance(lb);
    return;
  }
  const int64_t base = t * RS_TILE + (int64_t)warp * (32 * RS_ITEMS);
  unsigned long long k[RS_ITEMS];
  unsigned rank[RS_ITEMS], val[RS_ITEMS];
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int j = 0; j < RS_ITEMS; j++) {  // keys and values in one round of loads
    const int64_t i = base + j * 32 + lane;
    k[j] = i < n ? keys[i] : ~0ull;
    val[j] = i < n ? vals[i] : 0u;
  }
#pragma unroll
  for (int j = 0; j < RS_ITEMS; j++) {
    const int64_t i = base + j * 32 + lane;
    const unsigned dg = i < n ? (unsigned)((k[j] >> shift) & 0xff) : 0x100u;
    const unsigned peers = __match_any_sync(FULL, dg);
    const unsigned pre = dg < 0x100u ? wcnt[warp][dg] : 0u;
    rank[j] = pre + __popc(peers & lt);
    __syncwarp();
    if (dg < 0x100u && (__ffs(peers) - 1) == lane) wcnt[warp][dg] = pre + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  unsigned run = 0;  // exclusive prefix across warps per digit; run = the tile's count of digit d
  if (d < RS_BINS)
    for (int w = 0; w < OS_WARPS; w++) {
      const unsigned c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
  // items of digit d in the tiles before this one: look back over windows of
  // LB_W earlier tiles (their flags loaded together), consuming published
  // aggregates up to the nearest published inclusive prefix
  long long excl = 0;
  const int64_t slot = t * RS_BINS + d;
  if (d >= RS_BINS) {
    // no digit: nothing to look back for
  } else if (t == 0) {
    if (!g_lb_stall) *(volatile unsigned long long *)(lb.flag + slot) = lb_pack(e, 2, run);
  } else {
    *(volatile unsigned long long *)(lb.flag + slot) = lb_pack(e, 1, run);
    const unsigned long long tag = e & LB_EMASK;
    int64_t q = t - 1;
    int idle = 0;
    bool done = false;
    while (!done) {
      unsigned long long f[LB_W];
#pragma unroll
      for (int j = 0; j < LB_W; j++)
        f[j] = q - j >= 0 ? ld_vol(lb.flag + (q - j) * RS_BINS + d) : lb_pack(e, 2, 0);  // before tile 0: 0
      int used = 0;
#pragma unroll
      for (int j = 0; j < LB_W; j++) {
        // stop at the first tile that has not published in this epoch
        if (done || used < j || (f[j] >> 34) != tag || ((f[j] >> 32) & 3) == 0) continue;
        excl += (long long)(f[j] & 0xffffffffull);
        used = j + 1;
        done = ((f[j] >> 32) & 3) == 2;
      }
      q -= used;
      if (used == 0) {  // the nearest tile has not published yet
        if (++idle >= g_spin_limit || ((idle & 1023) == 1023 && lb_faulted(lb, e))) {
          lb_give_up(lb, e);
          break;
        }
        if (idle >= 32) __nanosleep(64);
      }
    }
    *(volatile unsigned long long *)(lb.flag + slot) = lb_pack(e, 2, (unsigned)(excl + run));
  }
  if (d < RS_BINS) boff[d] = gbase + excl;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RS_ITEMS; j++) {
    const int64_t i = base + j * 32 + lane;
    if (i < n) {
      const unsigned dg = (unsigned)((k[j] >> shift) & 0xff);
      const int64_t pos = boff[dg] + wcnt[warp][dg] + rank[j];
      keys_out[pos] = k[j];
      vals_out[pos] = val[j];
    }
  }
  if (lb_end(lb)) {
    if (last_pass)  // leave the histogram table cleared for the next sort
      for (int i = threadIdx.x; i < 8 * RS_BINS; i += OS_THREADS) lb.hist[i] = 0;
    __syncthreads();
    lb_advance(lb);
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
  if (n <= RS_MID) return 0;
  return arena_bytes(div_up(n, RS_THREADS * 16) * RS_BINS, 8);
}

size_t lookback_slots(int64_t n) {
  // mid-size sorts: one slot per (tile, digit); large sorts: the scan of their
  // histogram table; scans: one slot per tile
  const int64_t sort = n <= RS_MID ? div_up(n, RS_THREADS * 8) * RS_BINS
                                   : div_up(div_up(n, RS_THREADS * 16) * RS_BINS, SCAN_TILE);
  return (size_t)(std::max<int64_t>(sort, 8 * div_up(n, SCAN_TILE)) + 1);  // two-array scans: 4 words x 2 tiles
}

// Large inputs: three kernels per pass (tile histograms, table scan, scatter).
static int radix_passes_table(unsigned long long **keys, unsigned **vals, unsigned long long **keys_tmp,
                              unsigned **vals_tmp, int64_t n, int bits, Arena &ar, cudaStream_t s) {
  constexpr int ITEMS = 16;
  const int64_t nt = div_up(n, RS_THREADS * ITEMS);
  size_t mark = ar.used;
  long long *hist = ar.take<long long>(nt * RS_BINS);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  for (int shift = 0; shift < bits; shift += 8) {
    DCSR_LAUNCH(k_radix_hist<ITEMS>, (unsigned)nt, RS_THREADS, 0, s, *keys, n, shift, hist, nt);
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

// Mid-size inputs: one histogram kernel, then one single-pass scatter per pass.
// Tile shape of the single-pass scatter: OS_T threads x OS_I keys per thread
// (tiles of 4096 and 8192 keys, with 256-1024 threads, ran no faster: the
// pass time is the chain of memory round trips of one tile, not its size).
constexpr int OS_T = 256, OS_I = 8, OS_MB = 2;
static int radix_passes_onesweep(unsigned long long **keys, unsigned **vals, unsigned long long **keys_tmp,
                                 unsigned **vals_tmp, int64_t n, int bits, Arena &ar, cudaStream_t s) {
  constexpr int ITEMS = OS_T * OS_I / RS_THREADS;  // keys per tile / RS_THREADS
  const int passes = (int)div_up(bits, 8);
  if (passes <= 0) return DCSR_OK;
  const int64_t nt = div_up(n, RS_THREADS * ITEMS);
  Lookback lb;
  DCSR_TRY(ar.lookback((size_t)(nt * RS_BINS), s, &lb));
  const int gh = (int)std::min<int64_t>(div_up(n, RS_THREADS * 8), 4 * sm_count());
  DCSR_LAUNCH(k_radix_hist_all, gh, RS_THREADS, 0, s, *keys, n, passes, lb);
  for (int p = 0; p < passes; p++) {
    DCSR_LAUNCH((k_radix_onesweep<OS_T, OS_I, OS_MB>), (unsigned)nt, OS_T, 0, s, *keys, *vals, *keys_tmp, *vals_tmp,
                n, p,
                p == passes - 1 ? 1 : 0, lb);
    unsigned long long *tk = *keys;
    *keys = *keys_tmp;
    *keys_tmp = tk;
    unsigned *tv = *vals;
    *vals = *vals_tmp;
    *vals_tmp = tv;
  }
  return DCSR_OK;
}

int radix_sort_pairs(unsigned long long **keys, unsigned **vals, unsigned long long **keys_tmp,
                     unsigned **vals_tmp, int64_t n, int bits, Arena &ar, cudaStream_t s) {
  if (n <= 1) return DCSR_OK;
  if (n <= RS_SMALL) {
    static const cudaError_t attr =
        cudaFuncSetAttribute(k_radix_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_SMALL_SMEM);
    DCSR_CUDA(attr);
    DCSR_LAUNCH(k_radix_small, 1, 1024, RS_SMALL_SMEM, s, *keys, *vals, *keys_tmp, *vals_tmp, (int)n, bits);
    unsigned long long *tk = *keys;
    *keys = *keys_tmp;
    *keys_tmp = tk;
    unsigned *tv = *vals;
    *vals = *vals_tmp;
    *vals_tmp = tv;
    return DCSR_OK;
  }
  if (n <= RS_MID) return radix_passes_onesweep(keys, vals, keys_tmp, vals_tmp, n, bits, ar, s);
  if (n <= RS_BIG) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    DCSR_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusNone) return radix_passes_onesweep(keys, vals, keys_tmp, vals_tmp, n, bits, ar, s);
  }
  return radix_passes_table(keys, vals, keys_tmp, vals_tmp, n, bits, ar, s);
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

// Reduce-by-key: heads flagged, head positions compacted by scan.  A run is
// summed in pieces of at most RBK_PIECE keys (a piece starts at the run's
// head or at a multiple of RBK_PIECE inside the run), each piece left to
// right by one thread; the thread at the head writes its piece's sum and the
// pieces that continue a run leave theirs in cpart; a second kernel adds a
// run's continuation pieces to its head piece in order.  The order of the
// additions is fixed by the input alone, so results are deterministic, and no
// thread sums more than RBK_PIECE values (a run of 2^20 equal keys is summed
// by 4096 threads, then 4096 partials by one).
constexpr int64_t RBK_PIECE = 256;
__global__ void k_rbk_flags(const int32_t *keys, int64_t n, long long *flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}
template <typename V>
__global__ void k_rbk_emit(const int32_t *keys, const V *vals, int64_t n, const long long *pos,
                           int32_t *keys_out, V *vals_out, V *cpart) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool head = i == 0 || keys[i] != keys[i - 1];
  if (!head && i % RBK_PIECE != 0) return;
  const int64_t end = (i / RBK_PIECE + 1) * RBK_PIECE < n ? (i / RBK_PIECE + 1) * RBK_PIECE : n;
  V acc = vals[i];
  for (int64_t j = i + 1; j < end && keys[j] == keys[i]; j++) acc = acc + vals[j];
  if (head) {
    keys_out[pos[i]] = keys[i];
    vals_out[pos[i]] = acc;
  } else {
    cpart[i / RBK_PIECE] = acc;
  }
}
// One thread per piece boundary b = s * RBK_PIECE (s >= 1): the owner of a
// run that crosses b is the boundary whose previous piece holds the run's
// head; it adds the run's continuation pieces s, s+1, ... to the head piece.
template <typename V>
__global__ void k_rbk_fix(const int32_t *keys, int64_t n, const long long *pos, V *vals_out, const V *cpart) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int64_t b = s * RBK_PIECE;
  if (b >= n || keys[b] != keys[b - 1]) return;       // no run crosses b
  if (pos[b] == pos[b - RBK_PIECE]) return;  // no head in [b - RBK_PIECE, b): an earlier boundary owns the run
  const int64_t out = pos[b] - 1;  // the run's output slot (heads before b, minus one)
  V acc = vals_out[out];
  const int32_t key = keys[b];
  for (int64_t t = s; t * RBK_PIECE < n; t++) {
    if (keys[t * RBK_PIECE] != key) break;  // the run ended before this piece (keys are sorted)
    acc = acc + cpart[t];
  }
  vals_out[out] = acc;
}

template <typename V>
static int rbk_launch(const int32_t *keys, const V *vals, int64_t n, long long *pos, long long *n_out, int32_t *keys_out,
                      V *vals_out, V *cpart, Arena &ar, cudaStream_t s) {
  const unsigned g = (unsigned)div_up(n, 256);
  DCSR_LAUNCH(k_rbk_flags, g, 256, 0, s, keys, n, pos);
  DCSR_TRY(scan_i64(pos, pos, n, n_out, ar, s));
  DCSR_LAUNCH(k_rbk_emit<V>, g, 256, 0, s, keys, vals, n, pos, keys_out, vals_out, cpart);
  const int64_t nb = (n - 1) / RBK_PIECE;  // piece boundaries inside [1, n)
  if (nb > 0) DCSR_LAUNCH(k_rbk_fix<V>, (unsigned)div_up(nb, 256), 256, 0, s, keys, n, pos, vals_out, cpart);
  return DCSR_OK;
}

// ------------------------------------------- allocation-free reduce-by-key
//
// Scratch for dcsr_reduce_by_key_noalloc: head positions (one int64 per key),
// the continuation-piece partials and the scan's look-back area, in one
// static device array (zero at module
// load, as the look-back protocol needs).  Every GPU that loads the library
// holds it until exit.  Host code must not pass the symbol itself to a
// kernel (in host code it names a host-side stand-in); the device address is
// looked up once per device.
constexpr size_t NOALLOC_POS_BYTES = (size_t)DCSR_NOALLOC_MAX_KEYS * sizeof(long long);
constexpr size_t NOALLOC_PART_BYTES = (size_t)(DCSR_NOALLOC_MAX_KEYS / RBK_PIECE + 1) * sizeof(double);
constexpr size_t NOALLOC_LB_SLOTS = 4 * ((DCSR_NOALLOC_MAX_KEYS + SCAN_TILE - 1) / SCAN_TILE) + 4;
constexpr size_t NOALLOC_ARENA_BYTES = NOALLOC_POS_BYTES + 256 + NOALLOC_PART_BYTES + 256;
constexpr size_t NOALLOC_BYTES = NOALLOC_ARENA_BYTES + LB_HEADER + 8 * NOALLOC_LB_SLOTS;
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
  Arena ar;  // a view over the static array: take() and lookback() only, never reserve()/release()
  ar.base = (char *)base;
  ar.cap = NOALLOC_ARENA_BYTES;
  ar.used = 0;
  ar.lb = (unsigned char *)base + NOALLOC_ARENA_BYTES;
  ar.lb_slots = NOALLOC_LB_SLOTS;
  // every word below is written before it is read in each call: positions
  // by the flag kernel, a partial by the piece that owns it
  long long *pos = ar.take<long long>(n);
  double *cpart = ar.take<double>(n / RBK_PIECE + 1);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  if (dtype == DCSR_F32)
    return rbk_launch<float>(keys, (const float *)vals, n, pos, (long long *)n_out, keys_out, (float *)vals_out,
                             (float *)cpart, ar, s);
  return rbk_launch<double>(keys, (const double *)vals, n, pos, (long long *)n_out, keys_out, (double *)vals_out,
                            cpart, ar, s);
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
  DCSR_TRY(ar.reserve(arena_bytes(n, 8) + arena_bytes(n / RBK_PIECE + 1, 8) + scan_scratch_bytes(n), s));
  long long *pos = ar.take<long long>(n);
  double *cpart = ar.take<double>(n / RBK_PIECE + 1);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  const int rc = dtype == DCSR_F32 ? rbk_launch<float>(keys, (const float *)vals, n, pos, (long long *)n_out, keys_out,
                                                       (float *)vals_out, (float *)cpart, ar, s)
                                   : rbk_launch<double>(keys, (const double *)vals, n, pos, (long long *)n_out,
                                                        keys_out, (double *)vals_out, cpart, ar, s);
  ar.release(s);
  return rc;
}
