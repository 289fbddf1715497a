// common.cuh -- shared internals of the DCSR library: the handle, the device
// view of a matrix, layout policy, status words, the scratch arena and warp
// helpers.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/dcsr_b200.h"

namespace dcsr {

constexpr int WARP = 32;
constexpr unsigned FULL = 0xffffffffu;

extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Debugging aid: with DCSR_DEBUG_SYNC=1 in the environment every launch
// outside stream capture is followed by a synchronisation of its stream,
// and a failing kernel is named (file:line) on stderr.
bool debug_sync();
void debug_check(cudaStream_t s, const char *kernel, const char *file, int line);

// The library's device memory (devmem.cu): a block of the regions that
// dcsr_pool_reserve mapped, ordered after its previous user's work on
// another stream, else the driver's stream-ordered allocation.  Every
// buffer the library allocates goes through these two calls.
cudaError_t dev_alloc_raw(void **p, size_t bytes, cudaStream_t s);
cudaError_t dev_free(void *p, cudaStream_t s);
template <typename T>
inline cudaError_t dev_alloc(T **p, size_t bytes, cudaStream_t s) {
  return dev_alloc_raw(reinterpret_cast<void **>(p), bytes, s);
}
// Maps a region so that at least `bytes` of the current device's regions
// are free; region usage of the current device.
int reserve_regions(int64_t bytes, cudaStream_t s);
int region_usage(int64_t *reserved, int64_t *free_bytes, int64_t *fallback);

#define DCSR_CUDA(call)                                                                         \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess) {                                                                    \
      fprintf(stderr, "dcsr: CUDA error %s at %s:%d\n", cudaGetErrorString(_e), __FILE__, __LINE__); \
      return _e == cudaErrorMemoryAllocation ? DCSR_OOM : DCSR_CUDA_ERROR;                      \
    }                                                                                           \
  } while (0)

#define DCSR_TRY(call)             \
  do {                             \
    int _s = (call);               \
    if (_s != DCSR_OK) return _s;  \
  } while (0)

// Launch with the launch counter and an error check.
#define DCSR_LAUNCH(kernel, grid, block, smem, stream, ...)                          \
  do {                                                                               \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                      \
    ::dcsr::count_launch();                                                          \
    DCSR_CUDA(cudaGetLastError());                                                   \
    if (::dcsr::debug_sync()) ::dcsr::debug_check((stream), #kernel, __FILE__, __LINE__); \
  } while (0)

__host__ __device__ inline int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }
__host__ __device__ inline int64_t div_up(int64_t x, int64_t a) { return (x + a - 1) / a; }

// Row capacity for a logical length under the layout policy (integer-only so
// the oracle restates it exactly).
__host__ __device__ inline int64_t policy_cap(const dcsr_opts &o, int64_t len) {
  int64_t c = (len * o.factor_x16 + 15) / 16;
  if (c < o.min_cap) c = o.min_cap;
  if (c < len) c = len;
  return align_up(c, o.align);
}
__host__ __device__ inline int64_t pool_capacity(const dcsr_opts &o, int64_t top) {
  int64_t spare = top * o.spare_x16 / 16;
  if (spare < o.min_spare) spare = o.min_spare;
  return top + spare;
}

// Device status block of a handle (int64 words).
enum StatWord {
  ST_STATUS = 0,   // dcsr_status of the last rejected operation (sticky until read)
  ST_GO = 1,       // 1 when the current update plan was accepted
  ST_NEED = 2,     // pool top the current update requires
  ST_TOUCHED = 3,  // touched rows of the current batch (batch-global word)
  ST_TILES = 4,    // relocation tiles of the current batch (batch-global word)
  ST_TOTAL = 5,    // scratch total (scan results)
  ST_AUX = 6,      // per-update flags (bad index, layer overflow)
  ST_SCRATCH = 7,  // one-off device-side result words
  ST_TOP = 8,      // pool top before the current update
  ST_T0 = 9,       // this matrix's touched-row range [T0, T1) in the batch
  ST_T1 = 10,
  ST_WORDS = 16
};

// Device view of a matrix passed by value to kernels.
template <typename V>
struct Mat {
  int32_t n_rows, n_cols, max_segs, pitch;
  int64_t pool_cap;
  int32_t *row_sizes;
  int32_t *seg;
  int32_t *cols;
  V *vals;
  long long *stat;
  dcsr_opts o;
};

// Device state of the single-pass scan and sort kernels (decoupled look-back):
// an epoch that the last block of every such kernel advances, the dynamic
// tile counter and the finished-block counter that block resets, the radix
// digit histograms (re-zeroed by the sort's last pass), and the look-back
// words, each tagged with the epoch that wrote it (prims.cu).  Zeroed once at
// allocation: a word left by an earlier kernel carries another epoch, so
// nothing is cleared between kernels.
// A wait that reaches its iteration limit gives up: it counts a fault,
// marks the area's fault word with the kernel's epoch (the other waits of
// that kernel then give up early instead of each spinning to the limit) and
// sets the operation's status word (when it has one) to DCSR_TIMEOUT.
struct Lookback {
  unsigned long long *epoch;
  unsigned *tiles, *done;
  unsigned long long *fault;  // epoch tag + 1 of the last kernel whose wait gave up
  unsigned *hist;             // [8][256]
  unsigned long long *flag;   // look-back words
  unsigned long long slots;   // entries of flag
  long long *status;          // the operation's status word, or null
};
constexpr size_t LB_HEADER = 64 + 8 * 256 * 4;

// Stream-ordered scratch arena: one device buffer, bump-allocated per
// operation, grown (stream-ordered free + malloc) when an operation needs more;
// plus the look-back area of the single-pass kernels.
struct Arena {
  char *base = nullptr;
  size_t cap = 0, used = 0;
  unsigned char *lb = nullptr;
  size_t lb_slots = 0;
  // Status word (device) of the operation using the arena: a look-back wait
  // that gives up sets it to DCSR_TIMEOUT.  Set by the operation (null: the
  // fault is only counted, see dcsr_spin_faults).
  long long *status = nullptr;
  // Set when take() could not fit a request (a sizing bug): the caller
  // returns DCSR_OOM instead of launching with the null pointer.
  bool overflow = false;
  // Look-back area with at least `slots` slots (grown, and zeroed, outside
  // stream capture only: a captured graph must find it sized already).
  int lookback(size_t slots, cudaStream_t s, Lookback *out) {
    if (slots > lb_slots || !lb) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      DCSR_CUDA(cudaStreamIsCapturing(s, &cs));
      if (cs != cudaStreamCaptureStatusNone) return DCSR_NOT_SUPPORTED;
      if (lb) DCSR_CUDA(dcsr::dev_free(lb, s));
      lb = nullptr;
      lb_slots = 0;
      const size_t want = slots + slots / 4 + 1024;
      const size_t bytes = LB_HEADER + 8 * want;
      DCSR_CUDA(dcsr::dev_alloc((void **)&lb, bytes, s));
      DCSR_CUDA(cudaMemsetAsync(lb, 0, bytes, s));
      lb_slots = want;
    }
    out->epoch = (unsigned long long *)lb;
    out->tiles = (unsigned *)(lb + 8);
    out->done = (unsigned *)(lb + 12);
    out->fault = (unsigned long long *)(lb + 16);
    out->hist = (unsigned *)(lb + 64);
    out->flag = (unsigned long long *)(lb + LB_HEADER);
    out->slots = lb_slots;
    out->status = status;
    return DCSR_OK;
  }
  int reserve(size_t bytes, cudaStream_t s) {
    used = 0;
    overflow = false;
    if (bytes <= cap) return DCSR_OK;
    if (base) DCSR_CUDA(dcsr::dev_free(base, s));
    base = nullptr;
    cap = 0;
    size_t want = bytes + bytes / 4 + (1 << 20);
    DCSR_CUDA(dcsr::dev_alloc((void **)&base, want, s));
    cap = want;
    return DCSR_OK;
  }
  // Bump allocation from the reserved buffer; nullptr (and overflow set)
  // when the request does not fit -- a sizing bug in the library, which the
  // caller reports as DCSR_OOM before any kernel sees the pointer.
  template <typename T>
  T *take(size_t n) {
    size_t off = align_up((int64_t)used, 256);
    if (off + n * sizeof(T) > cap) {
      fprintf(stderr, "dcsr: scratch arena overflow (%zu > %zu bytes)\n", off + n * sizeof(T), cap);
      overflow = true;
      return nullptr;
    }
    used = off + n * sizeof(T);
    return (T *)(base + off);
  }
  void release(cudaStream_t s) {
    if (base) dcsr::dev_free(base, s);
    if (lb) dcsr::dev_free(lb, s);
    base = nullptr;
    lb = nullptr;
    cap = used = lb_slots = 0;
  }
};

inline size_t arena_bytes(size_t n, size_t elem) { return align_up((int64_t)(n * elem), 256) + 256; }

}  // namespace dcsr

// The opaque handle.
struct dcsr_matrix_s {
  int32_t n_rows = 0, n_cols = 0, dtype = 0, pitch = 0;
  dcsr_opts o{};
  int64_t pool_cap = 0;
  int32_t *row_sizes = nullptr;
  int32_t *seg = nullptr;
  int32_t *cols = nullptr;
  void *vals = nullptr;
  long long *stat = nullptr;
  // Row-pass schedule (handle-local; the reference used a global __constant__
  // bin table): long rows with their chunk offsets, medium rows.
  int32_t *long_rows = nullptr;  // [n_rows + 1]
  long long *long_off = nullptr; // [n_rows + 2] chunk offsets of long rows
  int32_t *long_cnt = nullptr;   // [n_rows + 1] chunk-finisher counters
  int32_t *sched_info = nullptr; // [32]: [0] long rows, [1] chunks, [2] medium rows
  double *part = nullptr;        // chunk partials (reductions)
  int64_t part_cap = 0;
  int2 *chunk_rl = nullptr;      // (row, long-row index) of every chunk
  int64_t chunk_cap = 0;
  // medium-length rows, one descriptor each: (row, length, layer-0 start,
  // layer-0 capacity)
  int4 *med_desc = nullptr;      // [n_rows + 1]
  int4 *chunk_desc = nullptr;    // [chunk_cap] per chunk: its row's (row, length, layer-0 start, capacity)
  // Row-class thresholds of the row passes (rows of at most short_max
  // entries are streamed by row blocks, rows above long_min are chunked).
  int32_t short_max = 64, long_min = 512;
  bool bins_valid = false;
  dcsr::Arena scratch;
  // Pool buffers: buf_cap >= pool_cap entries are allocated.  The buffers a
  // compaction or growth replaced stay as this matrix's spare (within a
  // process-wide byte budget), so the next compaction or growth of the
  // matrix -- a repair's -- takes them instead of allocating; spare_ev orders
  // their reuse after the kernels that last read them.
  int64_t buf_cap = 0;
  int32_t *spare_cols = nullptr;
  void *spare_vals = nullptr;
  int64_t spare_cap = 0;
  cudaEvent_t spare_ev = nullptr;
  int device = 0;

  template <typename V>
  dcsr::Mat<V> view() const {
    dcsr::Mat<V> m;
    std::memset(&m, 0, sizeof(m));  // deterministic padding (descriptor images are compared bytewise)
    m.n_rows = n_rows;
    m.n_cols = n_cols;
    m.max_segs = o.max_segs;
    m.pitch = pitch;
    m.pool_cap = pool_cap;
    m.row_sizes = row_sizes;
    m.seg = seg;
    m.cols = cols;
    m.vals = (V *)vals;
    m.stat = stat;
    m.o = o;
    return m;
  }
  size_t vsize() const { return dtype == DCSR_F64 ? 8 : 4; }
};

namespace dcsr {

// ---------------------------------------------------------- warp helpers

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(FULL, v, o);
    v = w < v ? w : v;
  }
  return v;
}
// Inclusive prefix sum within a warp.
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  int l = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T w = __shfl_up_sync(FULL, v, o);
    if (l >= o) v += w;
  }
  return v;
}

// A row's linked segments.  MAX_SEGS is the compile-time layer limit (the
// reference's MAX_OFFSET = 4); every loop over layers is fully unrolled so
// the arrays stay in registers (dynamic indexing would put them in local
// memory, which measured more traffic than the data itself).
constexpr int MAX_SEGS = 4;
struct Chain {
  int32_t st[MAX_SEGS];
  int32_t cp[MAX_SEGS];
  int ns;
  int64_t total;
  // Physical slot of logical position p (predicated, no early exit: keeps
  // the arrays in registers in every caller).
  __device__ __forceinline__ int64_t phys(int64_t p) const {
    int64_t q = -1;
    bool done = false;
#pragma unroll
    for (int i = 0; i < MAX_SEGS; i++) {
      const bool live = !done && i < ns;
      if (live && p < cp[i]) {
        q = (int64_t)st[i] + p;
        done = true;
      } else if (live) {
        p -= cp[i];
      }
    }
    return q;
  }
  // Link a new last segment (layer ns); reset=true replaces the whole chain.
  __device__ __forceinline__ void append(int32_t s, int32_t c, bool reset) {
    if (reset) {
      ns = 0;
      total = 0;
    }
#pragma unroll
    for (int i = 0; i < MAX_SEGS; i++)
      if (i == ns) {
        st[i] = s;
        cp[i] = c;
      }
    ns++;
    total += c;
  }
};

// The chain of the row owned by lane `owner` (every lane loaded its own row's
// chain; a pass hands it to the lanes that work on that row).
__device__ __forceinline__ Chain shfl_chain(const Chain &own, int owner) {
  Chain c;
#pragma unroll
  for (int l = 0; l < MAX_SEGS; l++) {
    c.st[l] = __shfl_sync(FULL, own.st[l], owner);
    c.cp[l] = __shfl_sync(FULL, own.cp[l], owner);
  }
  c.ns = __shfl_sync(FULL, own.ns, owner);
  c.total = 0;
  return c;
}

// All layer pairs are loaded independently (no dependent load chain), then
// the chain is the leading run of linked layers.
template <typename V>
__device__ __forceinline__ Chain load_chain(const Mat<V> &m, int32_t r) {
  Chain c;
  int2 p[MAX_SEGS];
#pragma unroll
  for (int l = 0; l < MAX_SEGS; l++)
    p[l] = l < m.max_segs ? __ldg(reinterpret_cast<const int2 *>(m.seg + (int64_t)l * m.pitch + 2 * (int64_t)r))
                          : make_int2(-1, -1);
  c.ns = 0;
  c.total = 0;
  bool open = true;
#pragma unroll
  for (int l = 0; l < MAX_SEGS; l++) {
    open = open && p[l].x >= 0;
    c.st[l] = open ? p[l].x : 0;
    c.cp[l] = open ? p[l].y - p[l].x : 0;
    if (open) {
      c.total += p[l].y - p[l].x;
      c.ns = l + 1;
    }
  }
  return c;
}

// The leading layers of row r that hold its first len entries, for passes
// that only read a row: layer 0 is loaded at once (independent of len, so
// its load overlaps the caller's load of the row length); layer l+1 only
// when layers 0..l hold fewer than len entries (most rows need layer 0
// alone, so the other layers' table entries are not read at all).
template <typename V>
__device__ __forceinline__ Chain load_chain_used(const Mat<V> &m, int32_t r, int32_t len) {
  Chain c;
  c.ns = 0;
  int64_t covered = 0;
#pragma unroll
  for (int l = 0; l < MAX_SEGS; l++) {
    c.st[l] = 0;
    c.cp[l] = 0;
    if (l < m.max_segs && c.ns == l && (l == 0 || covered < len)) {
      const int2 p = __ldg(reinterpret_cast<const int2 *>(m.seg + (int64_t)l * m.pitch + 2 * (int64_t)r));
      if (p.x >= 0) {
        c.st[l] = p.x;
        c.cp[l] = p.y - p.x;
        covered += p.y - p.x;
        c.ns = l + 1;
      }
    }
  }
  c.total = covered;
  return c;
}

// Persistent-grid size for a kernel: blocks resident across all SMs.
int persistent_grid(const void *kernel, int block, size_t smem);
int sm_count();

// -------------------------------------------------------------- primitives
// (scan.cu / radix.cu)

// Exclusive scan of int64 values; out may alias in; *total (device) = sum.
int scan_i64(const long long *in, long long *out, int64_t n, long long *total, Arena &ar, cudaStream_t s);
// Two independent exclusive scans of arrays of length n in one launch.
int scan2_i64(const long long *in0, long long *out0, long long *total0, const long long *in1, long long *out1,
              long long *total1, int64_t n, Arena &ar, cudaStream_t s);
size_t scan_scratch_bytes(int64_t n);

// Stable LSD radix sort of (uint64 key, uint32 value) pairs on bits [0, bits).
// Sorted output lands in (*keys, *vals) -- the pointers are swapped with the
// tmp buffers as passes ping-pong.
int radix_sort_pairs(unsigned long long **keys, unsigned **vals, unsigned long long **keys_tmp,
                     unsigned **vals_tmp, int64_t n, int bits, Arena &ar, cudaStream_t s);
size_t radix_scratch_bytes(int64_t n);
// Look-back slots that a scan or a sort of n items needs (Arena::lookback).
size_t lookback_slots(int64_t n);
// Spin waits of the single-pass kernels that ran out of iterations (a bug
// indicator: each wait has an owner that is running or finished).
long long spin_faults();
// Test hook: wait limit of the look-back kernels (<= 0: the default) and a
// switch that keeps the first tile of each single-pass kernel from
// publishing.  Synchronises the device.
int debug_lookback(int spin_limit, int stall);

inline int bits_for(int64_t n) {  // bits to represent values in [0, n)
  int b = 1;
  while (b < 62 && (int64_t(1) << b) < n) b++;
  return b;
}

}  // namespace dcsr
