// rowstream.cu -- row-parallel passes over one DCSR matrix or a set of them:
// SpMV (1..8 RHS), row reductions, DCSR -> CSR/COO export, compaction copy.
//
// Rows are split into three classes by the schedule (rebuilt lazily after
// any change of row lengths), each with its own launch so each has its own
// register budget and its units carry bounded work:
//   short  (<= short_max entries)  a warp takes 32 consecutive rows.  With
//          one value per entry (SpMV k=1, row reductions, the copy pass) it
//          streams each segment layer's entries across its lanes, U windows
//          of 32 entries at a time with every window's loads issued first; a
//          lane's row is found by a binary search over the lanes' row
//          offsets and sums use a segmented scan whose segment test is one
//          compare with the start of the lane's row in the window -- uneven
//          rows cost nothing extra.
//          With k >= 2 values per entry (where the scan's k shuffles per
//          step would dominate) the warp splits into groups of G lanes, G in
//          {1..16} from the block's mean row length; a group walks one row
//          with four loads in flight per lane and reduces over its lanes with
//          log2(G) shuffles.
//   medium (<= long_min)          one warp per row, lanes strided, U loads in
//          flight per lane, one warp reduction per row.
//   long                          CHUNK-entry chunks, one CTA per chunk,
//          STEP entries in flight per CTA step (128-bit loads when aligned);
//          multi-chunk rows combine their partials in chunk order (the CTA
//          that finishes the last chunk sums them).
// A row's result depends only on the row (its length picks its class, the
// block's lengths pick G), never on which launch or batch it runs in.
// Products accumulate in FP64 per lane (fused multiply-add); the k=1
// stream's per-window partials use the matrix type (FP32 partials of at
// most 32 products, then FP64); every rounding step is an explicit
// round-to-nearest intrinsic.
//
// Reference: spmv_dcsr_bin* include/spmv.inl:364-622 (seven bin kernels on
// seven streams, rows read with stale Prow_sizes), CompactIndices
// include/sparse_update.inl:916-1007, DCSRtoCSROffsets :1101-1116.
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "internal.cuh"

namespace dcsr {

constexpr int RS_THREADS_ = 256;
constexpr int RS_WARPS = RS_THREADS_ / 32;
// Long-row entries per chunk unit: one warp's unit in the k = 1 pass
// (k_rows1), one CTA's in the k >= 2 and copy passes.  Small enough that a
// power-law matrix's hottest rows spread over many warps; multi-chunk rows
// combine their partials in chunk order.
#ifndef DCSR_CHUNK
#define DCSR_CHUNK 2048
#endif
constexpr int CHUNK = DCSR_CHUNK;
// Windows of 32 entries a warp has in flight per step, and blocks per SM the
// k = 1 pass is compiled for.
#ifndef DCSR_K1_UN
#define DCSR_K1_UN 4
#endif
// The same for the k = 1 row reductions (sum, max, min, count), which hold
// no columns: twice the SpMV's (149 against 156 us for the row sums of the
// R-MAT 2^20 stream matrix; 16 spills).
#ifndef DCSR_K1_UN_RED
#define DCSR_K1_UN_RED 8
#endif
#ifndef DCSR_K1_MINB
#define DCSR_K1_MINB 3
#endif
#ifndef DCSR_K1B_MINB
#define DCSR_K1B_MINB 4
#endif
// Windows of 32 entries whose loads a short-row block has in flight.
#ifndef DCSR_K1B_U
#define DCSR_K1B_U 4
#endif
// Blocks per SM the copy pass (export, compaction) is compiled for.
#ifndef DCSR_COPY_MINB
#define DCSR_COPY_MINB 3
#endif
// Entries a thread copies per unit and pass (FP64: half).
#ifndef DCSR_COPY_EPT
#define DCSR_COPY_EPT 8
#endif
constexpr int STEP = 4096;    // entries a CTA has in flight per step
enum { P_BLOCKS = 0, P_CHUNKS = 1, P_MED = 2 };

// ------------------------------------------------------------- sources
// A row pass runs over one matrix (RowOne, descriptor passed by value) or a
// set of matrices laid end to end in one row space (RowMany, descriptors in
// device memory, per-class unit prefixes computed on the device).

// split: warps sharing one 32-row block of short rows in the k >= 2 pass
// (each takes every split-th group pass), so a small matrix's few blocks
// still fill the GPU; 1 for everything else.
template <typename V>
struct RowOne {
  RowItem<V> it;
  int split = 1;
  // unit counter and finished-warp counter of the k = 1 passes (the handle's
  // schedule words 8, 9 for the streamed units, 10, 11 for the short-row
  // blocks: zeroed by the schedule rebuild, reset by the last warp of every
  // pass)
  __device__ __forceinline__ unsigned *ctr(int which) const {
    return reinterpret_cast<unsigned *>(it.info + 8 + 2 * which);
  }
  __device__ __forceinline__ int n_items() const { return 1; }
  __device__ __forceinline__ const RowItem<V> &item(int) const { return it; }
  __device__ __forceinline__ int find_row(int64_t) const { return 0; }
  __device__ __forceinline__ int64_t units(int part) const {
    if (part == P_CHUNKS) return it.info[1];
    if (part == P_MED) return div_up(it.info[2], RS_WARPS);
    return div_up(div_up(it.m.n_rows, 32) * split, RS_WARPS);
  }
  __device__ __forceinline__ int locate(int, int64_t u, int64_t &lu) const {
    lu = u;
    return 0;
  }
};

template <typename V>
struct RowMany {
  const RowItem<V> *its;
  int count;
  const long long *pref;  // [3][count+1] unit prefixes per class (short blocks counted split times),
                          // then two words: the unit and finished-warp counters of the
                          // k = 1 passes (streamed units, short-row blocks)
  int split = 1;
  __device__ __forceinline__ unsigned *ctr(int which) const {
    return reinterpret_cast<unsigned *>(const_cast<long long *>(pref + 3 * (count + 1) + which));
  }
  __device__ __forceinline__ int n_items() const { return count; }
  __device__ __forceinline__ const RowItem<V> &item(int i) const { return its[i]; }
  __device__ __forceinline__ int find_row(int64_t g) const {  // matrix holding global row g
    int lo = 0, hi = count;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (its[mid].row0 <= g) lo = mid;
      else hi = mid;
    }
    return lo;
  }
  __device__ __forceinline__ int64_t units(int part) const { return pref[part * (count + 1) + count]; }
  __device__ __forceinline__ int locate(int part, int64_t u, int64_t &lu) const {
    const long long *p = pref + part * (count + 1);
    int lo = 0, hi = count;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (p[mid] <= u) lo = mid;
      else hi = mid;
    }
    lu = u - p[lo];
    return lo;
  }
};

// ---------------------------------------------------------------- schedule
// Per row: lflag = (is_long << 32) | chunks, mflag = is_medium; two scans
// give every long row its index and first chunk and every medium row its
// slot, per matrix (differences of the scans at the matrix's first row).

__device__ __forceinline__ void sched_flags_row(int32_t L, int32_t smax, int32_t lmin, long long &lf,
                                                long long &mf) {
  lf = L > lmin ? ((1ll << 32) | (long long)((L + CHUNK - 1) / CHUNK)) : 0;
  mf = (L > smax && L <= lmin) ? 1 : 0;
}

template <typename V, typename Src>
__global__ void k_sched_flags(Src src, int64_t R, long long *lflag, long long *mflag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g <= R; g += stride) {
    long long lf = 0, mf = 0;
    if (g < R) {
      const RowItem<V> &it = src.item(src.find_row(g));
      sched_flags_row(it.m.row_sizes[g - it.row0], it.short_max, it.long_min, lf, mf);
    }
    lflag[g] = lf;
    mflag[g] = mf;
  }
}

template <typename V, typename Src>
__global__ void k_sched_emit(Src src, int64_t R, const long long *lscan, const long long *mscan) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < R; g += stride) {
    const RowItem<V> &it = src.item(src.find_row(g));
    const int64_t r = g - it.row0;
    const int32_t L = it.m.row_sizes[r];
    if (L > it.short_max) {
      // unit descriptors of the k = 1 pass: (row, length, pool slot of the
      // unit's first entry when the unit lies in layer 0 else -1, chunk number)
      const int2 s0 = *reinterpret_cast<const int2 *>(it.m.seg + 2 * r);  // layer 0
      const int32_t cap0 = s0.y - s0.x;
      if (L > it.long_min) {
        const long long s = lscan[g] - lscan[it.row0];
        const int32_t li = (int32_t)(s >> 32);
        const long long c0 = s & 0xffffffff, nc = (L + CHUNK - 1) / CHUNK;
        const_cast<int32_t *>(it.long_rows)[li] = (int32_t)r;
        const_cast<long long *>(it.long_off)[li] = c0;
        it.long_cnt[li] = 0;
        for (long long c = c0; c < c0 + nc; c++) {
          const int32_t k = (int32_t)(c - c0);
          const int32_t e = (k + 1) * CHUNK < L ? (k + 1) * CHUNK : L;
          const_cast<int2 *>(it.chunk_rl)[c] = make_int2((int32_t)r, li);
          const_cast<int4 *>(it.chunk_desc)[c] = make_int4((int32_t)r, L, e <= cap0 ? s0.x + k * CHUNK : -1, k);
        }
      } else {
        const_cast<int4 *>(it.med_desc)[mscan[g] - mscan[it.row0]] =
            make_int4((int32_t)r, L, L <= cap0 ? s0.x : -1, 0);
      }
    }
  }
}

// Per matrix (one warp each): class counts and the long-row offset sentinel.
template <typename V, typename Src>
__global__ void k_sched_info(Src src, const long long *lscan, const long long *mscan) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = w; i < src.n_items(); i += nw) {
    const RowItem<V> &it = src.item(i);
    const int64_t a = it.row0, b = it.row0 + it.m.n_rows;
    const long long ls = lscan[b] - lscan[a];
    const int32_t n_long = (int32_t)(ls >> 32), n_chunks = (int32_t)(ls & 0xffffffff);
    if (lane == 0) {
      it.info[0] = n_long;
      it.info[1] = n_chunks;
      it.info[2] = (int32_t)(mscan[b] - mscan[a]);
      for (int q = 8; q < 12; q++) it.info[q] = 0;  // k = 1 pass counters
      const_cast<long long *>(it.long_off)[n_long] = n_chunks;
    }
  }
}

static int64_t max_chunks(dcsr_handle h) { return h->pool_cap / CHUNK + h->pool_cap / h->long_min + 2; }

int ensure_part(dcsr_handle h, int K, cudaStream_t s) {
  if (max_chunks(h) > h->chunk_cap) {
    if (h->chunk_rl) DCSR_CUDA(dcsr::dev_free(h->chunk_rl, s));
    if (h->chunk_desc) DCSR_CUDA(dcsr::dev_free(h->chunk_desc, s));
    h->chunk_rl = nullptr;
    h->chunk_desc = nullptr;
    DCSR_CUDA(dcsr::dev_alloc((void **)&h->chunk_rl, sizeof(int2) * max_chunks(h), s));
    DCSR_CUDA(dcsr::dev_alloc((void **)&h->chunk_desc, sizeof(int4) * max_chunks(h), s));
    h->chunk_cap = max_chunks(h);
    h->bins_valid = false;  // the chunk table is gone
  }
  const int64_t need = max_chunks(h) * K;
  if (need <= h->part_cap) return DCSR_OK;
  if (h->part) DCSR_CUDA(dcsr::dev_free(h->part, s));
  h->part = nullptr;
  DCSR_CUDA(dcsr::dev_alloc((void **)&h->part, sizeof(double) * need, s));
  h->part_cap = need;
  return DCSR_OK;
}

template <typename V>
RowItem<V> row_item(dcsr_handle h, const void *x, void *y, int64_t ldx, int64_t ldy, double alpha, double beta) {
  RowItem<V> it;
  std::memset(&it, 0, sizeof(it));  // padding too: batch descriptor images are compared bytewise
  it.m = h->view<V>();
  it.long_rows = h->long_rows;
  it.long_off = h->long_off;
  it.chunk_rl = h->chunk_rl;
  it.med_desc = h->med_desc;
  it.chunk_desc = h->chunk_desc;
  it.info = h->sched_info;
  it.long_cnt = h->long_cnt;
  it.part = h->part;
  it.x = (const V *)x;
  it.y = (V *)y;
  it.ldx = ldx;
  it.ldy = ldy;
  it.alpha = alpha;
  it.beta = beta;
  it.row0 = 0;
  it.short_max = h->short_max;
  it.long_min = h->long_min;
  it.skip = nullptr;
  it.k = 1;
  it.vec = 0;
  return it;
}
template RowItem<float> row_item<float>(dcsr_handle, const void *, void *, int64_t, int64_t, double, double);
template RowItem<double> row_item<double>(dcsr_handle, const void *, void *, int64_t, int64_t, double, double);

static int grid_for(int64_t n, int block) {
  int64_t g = div_up(n, block);
  int64_t cap = (int64_t)sm_count() * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

size_t schedule_scratch_bytes(int64_t R) { return 2 * arena_bytes(R + 2, 8) + scan_scratch_bytes(R + 1); }

// Needs schedule_scratch_bytes(R) free in the arena (reserved by the caller).
template <typename V, typename Src>
static int schedule_src(const Src &src, int count, int64_t R, Arena &ar, cudaStream_t s) {
  long long *lf = ar.take<long long>(R + 2), *mf = ar.take<long long>(R + 2);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  const int g = grid_for(R + 1, 256);
  DCSR_LAUNCH((k_sched_flags<V, Src>), g, 256, 0, s, src, R, lf, mf);
  DCSR_TRY(scan2_i64(lf, lf, nullptr, mf, mf, nullptr, R + 1, ar, s));
  DCSR_LAUNCH((k_sched_emit<V, Src>), g, 256, 0, s, src, R, lf, mf);
  DCSR_LAUNCH((k_sched_info<V, Src>), grid_for((int64_t)count * 32, 256), 256, 0, s, src, lf, mf);
  return DCSR_OK;
}

int schedule_many(const void *items_dev, int dtype, int count, int64_t R, Arena &ar, cudaStream_t s) {
  if (count == 0) return DCSR_OK;
  if (dtype == DCSR_F32)
    return schedule_src<float>(RowMany<float>{(const RowItem<float> *)items_dev, count, nullptr}, count, R, ar, s);
  return schedule_src<double>(RowMany<double>{(const RowItem<double> *)items_dev, count, nullptr}, count, R, ar, s);
}

template <typename V>
static int build_schedule_t(dcsr_handle h, cudaStream_t s, Arena &ar) {
  DCSR_TRY(ensure_part(h, 1, s));
  DCSR_TRY(ar.reserve(schedule_scratch_bytes(h->n_rows), s));
  RowOne<V> src{row_item<V>(h, nullptr, nullptr, 0, 0, 0.0, 0.0)};
  DCSR_TRY(schedule_src<V>(src, 1, h->n_rows, ar, s));
  h->bins_valid = true;
  return DCSR_OK;
}

int build_schedule(dcsr_handle h, cudaStream_t s, Arena *ar) {
  Arena &a = ar ? *ar : h->scratch;
  a.status = h->stat + ST_STATUS;
  if (h->dtype == DCSR_F32) return build_schedule_t<float>(h, s, a);
  return build_schedule_t<double>(h, s, a);
}

// Exclusive prefix over the matrices of each class's unit count (one block
// of 1024 threads, 1024 matrices per round).
template <typename V>
__device__ __forceinline__ void unit_prefix_block(const RowItem<V> *its, int count, long long *pref, int split) {
  __shared__ long long wsum[3][32];
  __shared__ long long carry[3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x < 3) carry[threadIdx.x] = 0;
  __syncthreads();
  for (int b = 0; b < count; b += 1024) {
    const int i = b + threadIdx.x;
    long long u[3] = {0, 0, 0}, inc[3];
    if (i < count) {
      u[P_BLOCKS] = div_up(div_up(its[i].m.n_rows, 32) * split, RS_WARPS);
      u[P_CHUNKS] = its[i].info[1];
      u[P_MED] = div_up(its[i].info[2], RS_WARPS);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      inc[c] = warp_incl_scan(u[c]);
      if (lane == 31) wsum[c][w] = inc[c];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
      for (int c = 0; c < 3; c++) wsum[c][lane] = warp_incl_scan(wsum[c][lane]);
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (i < count) pref[c * (count + 1) + i] = carry[c] + (w ? wsum[c][w - 1] : 0) + inc[c] - u[c];
    __syncthreads();
    if (threadIdx.x < 3) carry[threadIdx.x] += wsum[threadIdx.x][31];
    __syncthreads();
  }
  if (threadIdx.x < 3) pref[threadIdx.x * (count + 1) + count] = carry[threadIdx.x];
  if (threadIdx.x < 2) pref[3 * (count + 1) + threadIdx.x] = 0;  // the k = 1 passes' counters
}

template <typename V>
__global__ void __launch_bounds__(1024) k_unit_prefix(const RowItem<V> *its, int count, long long *pref, int split) {
  unit_prefix_block(its, count, pref, split);
}

// Several SpMV groups' prefixes in one launch, one block per group.
template <typename V>
struct PrefixJobs {
  const RowItem<V> *its[MAX_PREFIX_JOBS];
  int count[MAX_PREFIX_JOBS];
  long long *pref[MAX_PREFIX_JOBS];
  int split[MAX_PREFIX_JOBS];
};

template <typename V>
__global__ void __launch_bounds__(1024) k_unit_prefix_many(PrefixJobs<V> jobs) {
  unit_prefix_block(jobs.its[blockIdx.x], jobs.count[blockIdx.x], jobs.pref[blockIdx.x], jobs.split[blockIdx.x]);
}

// ------------------------------------------------------------- helpers

struct RowBlock {
  int32_t row;  // row id within its matrix (or -1)
  int32_t len;  // logical length
  bool stream;  // streamed by the block (non-empty and short)
};

template <typename V>
__device__ __forceinline__ RowBlock load_block(const Mat<V> &m, int64_t r0, int lane, int32_t smax) {
  RowBlock b;
  const int64_t r = r0 + lane;
  b.row = r < m.n_rows ? (int32_t)r : -1;
  b.len = b.row >= 0 ? __ldg(m.row_sizes + r) : 0;
  b.stream = b.len > 0 && b.len <= smax;
  return b;
}

// Entries of the lane's row in segment layer l (coalesced pair loads across
// the block); cum accumulates the capacity of layers < l.
template <typename V>
__device__ __forceinline__ void next_layer(const Mat<V> &m, const RowBlock &b, int l, int64_t &cum, int32_t &len_l,
                                           int32_t &st_l) {
  len_l = 0;
  st_l = 0;
  if (b.stream && cum < b.len) {
    const int2 sg = __ldg(reinterpret_cast<const int2 *>(m.seg + (int64_t)l * m.pitch + 2 * (int64_t)b.row));
    if (sg.x >= 0) {
      const int64_t cap = sg.y - sg.x;
      len_l = (int32_t)(b.len - cum < cap ? b.len - cum : cap);
      st_l = sg.x;
      cum += cap;
    } else {
      cum = b.len;
    }
  }
}

// The lane whose row holds block position p: the last lane whose row starts
// at or before p (excl, the rows' exclusive offsets, never decreases across
// the lanes; an empty row shares its offset with the next row, so the last
// lane found is the non-empty one), by a binary search over the lanes.
__device__ __forceinline__ int owner_lane(int32_t excl, int32_t p) {
  int lo = 0;
#pragma unroll
  for (int st = 16; st > 0; st >>= 1) {
    const int c = lo + st;  // <= 31
    if (__shfl_sync(FULL, excl, c) <= p) lo = c;
  }
  return lo;
}

// Lanes per row for a block of 32 short rows: the largest power of two
// G <= mean length / 4 (1..16), so a lane has about four or more entries of
// its row in flight and a block takes G passes of 32/G rows.
__device__ __forceinline__ int group_width(int32_t total) {
  const int32_t mean = total >> 5;
  return mean < 8 ? 1 : mean < 16 ? 2 : mean < 32 ? 4 : mean < 64 ? 8 : 16;
}

// Visit the logical entries [0, len) of a row: lane j of a G-lane group takes
// entries j, j+G, ...; f(st, p0, take, before) handles the UN entries
// p0 + i*G (< take) of the layer starting at pool slot st, whose first entry
// is logical position `before`.
template <int UN, typename F>
__device__ __forceinline__ void for_row_entries(const Chain &ch, int32_t len, int j, int G, F &&f) {
  int32_t before = 0;
#pragma unroll
  for (int l = 0; l < MAX_SEGS; l++) {
    if (l < ch.ns && before < len) {
      const int32_t take = ch.cp[l] < len - before ? ch.cp[l] : len - before;
      const int64_t st = ch.st[l];
      for (int32_t p0 = j; p0 < take; p0 += UN * G) f(st, p0, take, before);
      before += ch.cp[l];
    }
  }
}

// VEC: the rows of x are packed (ldx == K) and aligned to the largest power
// of two (<= 32) dividing the row size, so a row is read with vector loads.
template <typename T, typename V, int K, bool VEC>
__device__ __forceinline__ void load_xk(const V *__restrict__ x, int64_t c, int64_t ldx, T (&xv)[K]) {
  if constexpr (VEC && sizeof(V) == 4 && K == 8) {  // two 128-bit loads (measured faster than one 256-bit load)
    const float4 t = __ldg(reinterpret_cast<const float4 *>(x + c * 8));
    const float4 u = __ldg(reinterpret_cast<const float4 *>(x + c * 8) + 1);
    xv[0] = t.x; xv[1] = t.y; xv[2] = t.z; xv[3] = t.w;
    xv[4] = u.x; xv[5] = u.y; xv[6] = u.z; xv[7] = u.w;
  } else if constexpr (VEC && sizeof(V) == 4 && K == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(x + c * 4));
    xv[0] = t.x; xv[1] = t.y; xv[2] = t.z; xv[3] = t.w;
  } else if constexpr (VEC && sizeof(V) == 4 && K == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2 *>(x + c * 2));
    xv[0] = t.x; xv[1] = t.y;
  } else if constexpr (VEC && sizeof(V) == 8 && K % 2 == 0) {
#pragma unroll
    for (int k = 0; k < K; k += 2) {
      const double2 t = __ldg(reinterpret_cast<const double2 *>(x + c * K + k));
      xv[k] = (T)t.x; xv[k + 1] = (T)t.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) xv[k] = (T)__ldg(x + c * ldx + k);
  }
}

enum { OP_SPMV = 0, OP_SUM = 1, OP_MAX = 2, OP_MIN = 3, OP_COUNT = 4 };

template <typename T, int OP>
__device__ __forceinline__ T op_init() {
  return OP == OP_MAX ? (T)-INFINITY : OP == OP_MIN ? (T)INFINITY : (T)0;
}
// Every rounding step is an explicit round-to-nearest intrinsic: the
// compiler may not contract a product into a later sum (it could choose
// differently in different instantiations, and the batched and per-call
// passes must agree bit for bit).
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

template <typename T, int OP>
__device__ __forceinline__ T op_comb(T a, T b) {
  if (OP == OP_MAX) return a > b ? a : b;
  if (OP == OP_MIN) return a < b ? a : b;
  return add_rn(a, b);
}

// acc (op) a*x for one entry with value a and column c (FP64 accumulators)
template <typename V, int K, int OP, bool VEC>
__device__ __forceinline__ void accum_entry(double a, int32_t c, const V *x, int64_t ldx, double (&acc)[K]) {
  if constexpr (OP == OP_SPMV) {
    double xv[K];
    load_xk<double, V, K, VEC>(x, c, ldx, xv);
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = __fma_rn(a, xv[k], acc[k]);
  } else {
    acc[0] = op_comb<double, OP>(acc[0], OP == OP_COUNT ? 1.0 : a);
  }
}

// K < 0: the number of right-hand sides is a runtime value kr <= -K (one
// launch serves matrices with different k); accumulators are sized for -K.
template <int K>
struct KArr {
  static constexpr int N = K < 0 ? -K : K;
};

// acc (op) a*x for one entry, k from the template (K > 0) or the item (K < 0).
template <typename V, int K, int OP, bool VEC>
__device__ __forceinline__ void accum_k(double a, int32_t c, const V *x, int64_t ldx, int kr, bool vec,
                                        double (&acc)[KArr<K>::N]) {
  constexpr int N = KArr<K>::N;
  if constexpr (K > 0) {
    accum_entry<V, K, OP, VEC>(a, c, x, ldx, acc);
  } else if constexpr (OP == OP_SPMV) {
    const V *xr = x + (int64_t)c * ldx;
    double xv[N];
    if (vec && kr == N && N % (16 / (int)sizeof(V)) == 0) {  // whole 16-byte vectors
#pragma unroll
      for (int q = 0; q < N; q += 16 / (int)sizeof(V)) {
        if constexpr (sizeof(V) == 4) {
          const float4 t = __ldg(reinterpret_cast<const float4 *>(xr) + q / 4);
          xv[q] = t.x; xv[q + 1] = t.y; xv[q + 2] = t.z; xv[q + 3] = t.w;
        } else {
          const double2 t = __ldg(reinterpret_cast<const double2 *>(xr) + q / 2);
          xv[q] = t.x; xv[q + 1] = t.y;
        }
      }
    } else if (vec) {  // even kr: pairs
#pragma unroll
      for (int q = 0; q < N; q += 2)
        if (q < kr) {
          if constexpr (sizeof(V) == 4) {
            const float2 t = __ldg(reinterpret_cast<const float2 *>(xr) + q / 2);
            xv[q] = t.x; xv[q + 1] = t.y;
          } else {
            const double2 t = __ldg(reinterpret_cast<const double2 *>(xr) + q / 2);
            xv[q] = t.x; xv[q + 1] = t.y;
          }
        }
    } else {
#pragma unroll
      for (int q = 0; q < N; q++)
        if (q < kr) xv[q] = __ldg(xr + q);
    }
#pragma unroll
    for (int q = 0; q < N; q++)
      if (q < kr) acc[q] = __fma_rn(a, xv[q], acc[q]);
  } else {
    acc[0] = op_comb<double, OP>(acc[0], OP == OP_COUNT ? 1.0 : a);
  }
}

template <typename V, int K, int OP>
__device__ __forceinline__ void write_y(V *y, int64_t ldy, int32_t row, const double (&acc)[KArr<K>::N],
                                        double alpha, double beta, int32_t len, int kr) {
#pragma unroll
  for (int k = 0; k < KArr<K>::N; k++) {
    if (K < 0 && k >= kr) break;
    double v = acc[k];
    if ((OP == OP_MAX || OP == OP_MIN) && len == 0) v = 0.0;
    if (OP == OP_SPMV) {
      v = mul_rn(v, alpha);
      if (beta != 0.0) v = __fma_rn(beta, (double)y[(int64_t)row * ldy + k], v);
    }
    y[(int64_t)row * ldy + k] = (V)v;
  }
}

// ------------------------------------------------- k = 1 short-row block
// One warp, one block of 32 consecutive rows: one value per entry (SpMV
// k = 1, row reductions), the block's entries streamed across the lanes in
// windows of 32, U windows' loads in flight (windows past the block's end
// skipped); a lane's row comes from a binary search over the lanes' row
// offsets, sums use a segmented warp scan.
// d0: the lane's row, its length and its layer-0 segment (start, capacity),
// loaded ahead by the caller (row -1 past the matrix's end).
template <typename V, int OP, bool XU>
__device__ __forceinline__ void short_block_k1(const RowItem<V> &it, int4 d0, int lane) {
  using P = typename std::conditional<sizeof(V) == 4, float, double>::type;  // window partials
  constexpr int U = DCSR_K1B_U;
  const Mat<V> &m = it.m;
  const V *__restrict__ x = it.x;
  RowBlock rb;
  rb.row = d0.x;
  rb.len = d0.y;
  rb.stream = rb.len > 0 && rb.len <= it.short_max;
  double acc = op_init<double, OP>();
  int64_t cum = 0;  // capacity of this lane's row in the layers before l
  for (int l = 0; l < m.max_segs; l++) {
    int32_t len_l = 0, st_l = 0;
    if (l == 0) {
      if (rb.stream) {  // the layer-0 segment came with the descriptor
        len_l = rb.len < d0.w ? rb.len : d0.w;
        st_l = d0.z;
        cum = d0.w;
      }
    } else {
      next_layer(m, rb, l, cum, len_l, st_l);
    }
    if (!__any_sync(FULL, len_l > 0)) break;
    const int32_t incl = warp_incl_scan(len_l);  // block-local (<= 32 * short_max)
    const int32_t excl = incl - len_l;
    const int32_t E = __shfl_sync(FULL, incl, 31);
    for (int32_t base = 0; base < E; base += 32 * U) {
      int32_t q[U];
      int32_t rs[U];  // the window lane where the lane's row starts (0: it runs in from before)
      bool ok[U];
      // windows past the block's end (warp-uniform) are skipped whole
#pragma unroll
      for (int i = 0; i < U; i++) {
        const int32_t w0 = base + 32 * i, p = w0 + lane;
        q[i] = rs[i] = 0;
        ok[i] = false;
        if (w0 >= E) continue;
        const int j = owner_lane(excl, p);
        const int32_t ej = __shfl_sync(FULL, excl, j);
        const int32_t sj = __shfl_sync(FULL, st_l, j);
        ok[i] = p < E;
        rs[i] = ej > w0 ? ej - w0 : 0;
        q[i] = sj + (ok[i] ? p - ej : 0);
      }
      V a[U];
      int32_t col[U];
#pragma unroll
      for (int i = 0; i < U; i++) {
        a[i] = V(0);
        col[i] = 0;
        if (base + 32 * i >= E) continue;
        a[i] = __ldcs(m.vals + q[i]);
        col[i] = OP == OP_SPMV ? __ldcs(m.cols + q[i]) : 0;
      }
      // every window's x gathers issued before the first scan (lanes past
      // the block's end loaded a valid entry: their columns are valid)
      V xv[U];
#pragma unroll
      for (int i = 0; i < U; i++)
        xv[i] = OP != OP_SPMV || base + 32 * i >= E ? V(0)
                : XU                                ? __ldg(x + col[i])
                                                    : __ldg(x + (int64_t)col[i] * it.ldx);
#pragma unroll
      for (int i = 0; i < U; i++) {
        if (base + 32 * i >= E) continue;
        P c = op_init<P, OP>();
        if (ok[i]) {
          if constexpr (OP == OP_SPMV) c = mul_rn((P)a[i], (P)xv[i]);
          else c = OP == OP_COUNT ? (P)1 : (P)a[i];
        }
        // segmented inclusive scan: lanes p-d and p share a row when p-d is
        // at or past the start of p's row in this window
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const P co = __shfl_up_sync(FULL, c, d);
          if (lane - d >= rs[i]) c = op_comb<P, OP>(c, co);
        }
        // lane j collects the tail of its row's run in this window
        const int32_t w0 = base + 32 * i;
        const bool hit = len_l > 0 && excl < w0 + 32 && incl > w0;
        const int tail = (incl < w0 + 32 ? incl : w0 + 32) - 1 - w0;
        const P got = __shfl_sync(FULL, c, hit ? tail : 0);
        if (hit) acc = op_comb<double, OP>(acc, (double)got);
      }
    }
  }
  if (rb.row >= 0 && rb.len <= it.short_max) {
    const double accs[1] = {acc};
    write_y<V, 1, OP>(it.y, it.ldy, rb.row, accs, it.alpha, it.beta, rb.len, 1);
  }
}

// --------------------------------------------------------- reduction pass

// Blocks per SM the row pass is compiled for: the runtime-k families hold up
// to 8 FP64 accumulators and 8 x values per entry in flight, which left them
// at 2-3 blocks (16-24 warps) per SM, too few to hide the gather latency.
// Three blocks for k families 8 and 4 and four for family 2 (a few spilled
// registers) ran the batched SpMV pass of 512 matrices 9% faster than the
// unconstrained build (7.6 vs 8.4 ms).
template <int K>
struct RowsMinBlocks {
  static constexpr int N = K == -8 ? 3 : K == -4 ? 3 : K == -2 ? 4 : 1;
};

template <typename V, int K, int OP, bool VEC, int PART, typename Src>
__global__ void __launch_bounds__(RS_THREADS_, RowsMinBlocks<K>::N) k_rows_reduce(Src src) {
  constexpr int KA = KArr<K>::N;
  __shared__ double red[RS_WARPS][KA];
  __shared__ int last_flag;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t units = src.units(PART);
  for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
    int64_t lu;
    const RowItem<V> &it = src.item(src.locate(PART, u, lu));
    if (it.skip && *it.skip) continue;  // a batch matrix whose update was rejected: y untouched
    const Mat<V> &m = it.m;
    const V *__restrict__ x = it.x;
    const int64_t ldx = it.ldx;
    const int kr = K < 0 ? it.k : K;
    const bool vec = K < 0 ? it.vec != 0 : VEC;
    if constexpr (PART == P_CHUNKS) {
      // ---- one chunk of a long row, whole CTA (the chunk's row comes with
      // it; its chunk number and the long-row tables only for multi-chunk rows)
      const int2 rl = it.chunk_rl[lu];
      const int32_t row = rl.x;
      const int64_t li = rl.y;
      const int64_t L = m.row_sizes[row];
      const int64_t nch = (L + CHUNK - 1) / CHUNK;
      const int64_t chunk = nch == 1 ? 0 : lu - it.long_off[li];
      const Chain ch = load_chain(m, row);
      const int64_t c0 = chunk * CHUNK, c1 = c0 + CHUNK < L ? c0 + CHUNK : L;
      double acc[KA];
#pragma unroll
      for (int k = 0; k < KA; k++) acc[k] = op_init<double, OP>();
      const bool fast = ch.cp[0] >= c1;  // chunk inside layer 0
      if (K > 0 && fast && sizeof(V) == 4 && ((ch.st[0] + c0) & 3) == 0) {
        constexpr int G = STEP / 4 / RS_THREADS_;
        for (int64_t s0 = c0; s0 < c1; s0 += STEP) {
          const int64_t s1 = s0 + STEP < c1 ? s0 + STEP : c1;
          const int64_t base = ch.st[0] + s0;
          const int nv = (int)((s1 - s0) >> 2);
          float4 a4[G];
          int4 c4[G] = {};
#pragma unroll
          for (int g = 0; g < G; g++) {
            const int v = threadIdx.x + g * RS_THREADS_;
            if (v < nv) {
              a4[g] = __ldcs(reinterpret_cast<const float4 *>(m.vals + base) + v);
              if (OP == OP_SPMV) c4[g] = __ldcs(reinterpret_cast<const int4 *>(m.cols + base) + v);
            }
          }
#pragma unroll
          for (int g = 0; g < G; g++) {
            if (threadIdx.x + g * RS_THREADS_ < nv) {
              accum_k<V, K, OP, VEC>(a4[g].x, c4[g].x, x, ldx, kr, vec, acc);
              accum_k<V, K, OP, VEC>(a4[g].y, c4[g].y, x, ldx, kr, vec, acc);
              accum_k<V, K, OP, VEC>(a4[g].z, c4[g].z, x, ldx, kr, vec, acc);
              accum_k<V, K, OP, VEC>(a4[g].w, c4[g].w, x, ldx, kr, vec, acc);
            }
          }
          for (int64_t p = s0 + ((int64_t)nv << 2) + threadIdx.x; p < s1; p += RS_THREADS_)
            accum_k<V, K, OP, VEC>((double)__ldcs(m.vals + ch.st[0] + p),
                                       OP == OP_SPMV ? __ldcs(m.cols + ch.st[0] + p) : 0, x, ldx, kr, vec, acc);
        }
      } else {
        for (int64_t p = c0 + threadIdx.x; p < c1; p += RS_THREADS_) {
          const int64_t q = fast ? (int64_t)ch.st[0] + p : ch.phys(p);
          accum_k<V, K, OP, VEC>((double)__ldcs(m.vals + q), OP == OP_SPMV ? __ldcs(m.cols + q) : 0, x, ldx, kr, vec,
                                     acc);
        }
      }
#pragma unroll
      for (int k = 0; k < KA; k++) {
        if (K < 0 && k >= kr) break;
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = op_comb<double, OP>(v, __shfl_xor_sync(FULL, v, o));
        if (lane == 0) red[w][k] = v;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double t[KA];
#pragma unroll
        for (int k = 0; k < KA; k++) {
        if (K < 0 && k >= kr) break;
          t[k] = red[0][k];
          for (int q = 1; q < RS_WARPS; q++) t[k] = op_comb<double, OP>(t[k], red[q][k]);
        }
        if (nch == 1) {  // the whole row in one unit: no partials
          write_y<V, K, OP>(it.y, it.ldy, row, t, it.alpha, it.beta, (int32_t)L, kr);
          last_flag = 0;
        } else {
#pragma unroll
          for (int k = 0; k < KA; k++) it.part[(it.long_off[li] + chunk) * KA + k] = t[k];
          __threadfence();
          last_flag = atomicAdd(&it.long_cnt[li], 1) == nch - 1;
        }
      }
      __syncthreads();
      if (last_flag && threadIdx.x == 0) {
        __threadfence();
        double out[KA];
#pragma unroll
        for (int k = 0; k < KA; k++) out[k] = op_init<double, OP>();
        for (int64_t q = 0; q < nch; q++)
#pragma unroll
          for (int k = 0; k < KA; k++)
            out[k] = op_comb<double, OP>(out[k], __ldcg(it.part + (it.long_off[li] + q) * KA + k));
        write_y<V, K, OP>(it.y, it.ldy, row, out, it.alpha, it.beta, (int32_t)L, kr);
        it.long_cnt[li] = 0;
      }
      __syncthreads();
    } else if constexpr (PART == P_MED) {
      // ---- one medium row per warp, UN loads in flight per lane
      const int64_t mi = lu * RS_WARPS + w;
      if (mi >= it.info[2]) continue;
      const int32_t row = it.med_desc[mi].x;
      const int64_t L = m.row_sizes[row];
      const Chain ch = load_chain(m, row);
      double acc[KA];
#pragma unroll
      for (int k = 0; k < KA; k++) acc[k] = op_init<double, OP>();
      constexpr int UN = KArr<K>::N <= 2 ? 8 : 4;
      int64_t before = 0;
#pragma unroll
      for (int l = 0; l < MAX_SEGS; l++) {
        if (l < ch.ns && before < L) {
          const int64_t take = (int64_t)ch.cp[l] < L - before ? (int64_t)ch.cp[l] : L - before;
          const int64_t st = ch.st[l];
          for (int64_t b0 = 0; b0 < take; b0 += 32 * UN) {
            V a[UN];
            int32_t col[UN];
#pragma unroll
            for (int i = 0; i < UN; i++) {
              const int64_t p = b0 + 32 * i + lane;
              const int64_t q = st + (p < take ? p : 0);
              a[i] = __ldcs(m.vals + q);
              col[i] = OP == OP_SPMV ? __ldcs(m.cols + q) : 0;
            }
#pragma unroll
            for (int i = 0; i < UN; i++)
              if (b0 + 32 * i + lane < take) accum_k<V, K, OP, VEC>((double)a[i], col[i], x, ldx, kr, vec, acc);
          }
          before += ch.cp[l];
        }
      }
#pragma unroll
      for (int k = 0; k < KA; k++) {
        if (K < 0 && k >= kr) break;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[k] = op_comb<double, OP>(acc[k], __shfl_xor_sync(FULL, acc[k], o));
      }
      if (lane == 0) write_y<V, K, OP>(it.y, it.ldy, row, acc, it.alpha, it.beta, (int32_t)L, kr);
    } else {
      // ---- short rows: a warp takes 32 consecutive rows
      const int S = K == 1 ? 1 : src.split;  // warps per 32-row block (k >= 2 pass only)
      const int64_t wu = lu * RS_WARPS + w;
      const int64_t blk = wu / S;
      const int sub = (int)(wu - blk * S);
      if (blk * 32 >= m.n_rows) continue;
      if constexpr (K == 1) {
        const int64_t r = blk * 32 + lane;
        int4 d0 = make_int4(-1, 0, 0, 0);
        if (r < m.n_rows) {
          const int2 s0 = __ldg(reinterpret_cast<const int2 *>(m.seg + 2 * r));
          d0 = make_int4((int32_t)r, __ldg(m.row_sizes + r), s0.x, s0.y - s0.x);
        }
        short_block_k1<V, OP, false>(it, d0, lane);
      } else {
        // K values per entry: G lanes per row
        const RowBlock rb = load_block(m, blk * 32, lane, it.short_max);
        const Chain own = load_chain_used(m, rb.row >= 0 ? rb.row : 0, rb.stream ? rb.len : 0);
        const int G = group_width(warp_sum(rb.stream ? rb.len : 0));
        const int per = 32 / G, j = lane & (G - 1), g = lane / G;
        for (int pass = sub; pass < G; pass += S) {
          const int owner = pass * per + g;
          const int32_t row = __shfl_sync(FULL, rb.row, owner);
          const int32_t len = __shfl_sync(FULL, rb.len, owner);
          const Chain ch = shfl_chain(own, owner);
          double acc[KA];
#pragma unroll
          for (int k = 0; k < KA; k++) acc[k] = op_init<double, OP>();
          if (row >= 0 && len > 0 && len <= it.short_max) {
            constexpr int UN = KArr<K>::N <= 2 ? 8 : 4;  // entries in flight per lane
            for_row_entries<UN>(ch, len, j, G, [&](int64_t st, int32_t p0, int32_t take, int32_t) {
              V a[UN];
              int32_t col[UN];
#pragma unroll
              for (int i = 0; i < UN; i++) {
                const int32_t p = p0 + i * G;
                const int64_t q = st + (p < take ? p : 0);
                a[i] = __ldcs(m.vals + q);
                col[i] = OP == OP_SPMV ? __ldcs(m.cols + q) : 0;
              }
#pragma unroll
              for (int i = 0; i < UN; i++)
                if (p0 + i * G < take) accum_k<V, K, OP, VEC>((double)a[i], col[i], x, ldx, kr, vec, acc);
            });
          }
#pragma unroll
          for (int k = 0; k < KA; k++) {
            if (K < 0 && k >= kr) break;
            for (int o = G >> 1; o > 0; o >>= 1) acc[k] = op_comb<double, OP>(acc[k], __shfl_xor_sync(FULL, acc[k], o));
          }
          if (j == 0 && row >= 0 && len <= it.short_max) write_y<V, K, OP>(it.y, it.ldy, row, acc, it.alpha, it.beta, len, kr);
        }
      }
    }
  }
}

// ---------------------------------------------------- k = 1 single pass
// SpMV with one right-hand side and the row reductions: every class in one
// launch of warp units, taken from a device counter (longest first: long-row
// chunks, then medium rows, then 32-row short blocks), so no class waits for
// another's tail and a warp's next unit number is fetched while it works on
// the current one.  A chunk or medium row is streamed lane-consecutively
// (UN windows of 32 entries in flight per warp), the products of one window
// step summed in the matrix type in a fixed order and the step sums
// accumulated in FP64; a row of several chunks combines their partials in
// chunk order (the warp that finishes its last chunk does it).  The pass is
// bound by the x gathers (random 4-byte reads of x, one L1 line each).

// Entries [c0, c1) of a row (chain ch) streamed across the warp; returns the
// lane's partial.


// Entries [c0, c1) of a row whose range lies in one segment starting at pool
// slot st: two sets of UN windows, the loads of the next set in flight while
// the current set's x values are gathered and summed.  Returns the lane's
// partial.
template <typename V, int OP>
__device__ __forceinline__ double stream_seg(const RowItem<V> &it, int64_t st, int64_t c0, int64_t c1, int lane) {
  using P = typename std::conditional<sizeof(V) == 4, float, double>::type;
  constexpr int UN = sizeof(V) == 8 && DCSR_K1_UN > 1 ? DCSR_K1_UN / 2 : DCSR_K1_UN;  // FP64: half the windows
  const V *__restrict__ vals = it.m.vals + st;
  const int32_t *__restrict__ cols = it.m.cols + st;
  const V *__restrict__ x = it.x;
  V a[UN], an[UN];
  int32_t col[UN], coln[UN];
#pragma unroll
  for (int i = 0; i < UN; i++) {
    const int64_t p = c0 + 32 * i + lane, q = p < c1 ? p : c0;
    a[i] = __ldcs(vals + q);
    col[i] = OP == OP_SPMV ? __ldcs(cols + q) : 0;
  }
  double acc = op_init<double, OP>();
  for (int64_t b0 = c0; b0 < c1; b0 += 32 * UN) {
    const int64_t nb = b0 + 32 * UN;
    if (nb < c1) {
#pragma unroll
      for (int i = 0; i < UN; i++) {
        const int64_t p = nb + 32 * i + lane, q = p < c1 ? p : c0;
        an[i] = __ldcs(vals + q);
        coln[i] = OP == OP_SPMV ? __ldcs(cols + q) : 0;
      }
    }
    P w = op_init<P, OP>();
#pragma unroll
    for (int i = 0; i < UN; i++) {
      if (b0 + 32 * i + lane < c1) {
        P t;
        if constexpr (OP == OP_SPMV) t = mul_rn((P)a[i], (P)__ldg(x + (int64_t)col[i] * it.ldx));
        else t = OP == OP_COUNT ? (P)1 : (P)a[i];
        w = op_comb<P, OP>(w, t);
      }
    }
    acc = op_comb<double, OP>(acc, (double)w);
#pragma unroll
    for (int i = 0; i < UN; i++) {
      a[i] = an[i];
      col[i] = coln[i];
    }
  }
  return acc;
}

// The same over a range that crosses segments (a chained row): UN windows
// per step, each entry's slot found through the chain.  Same summation
// order as the single-segment stream.  Not inlined (chained units are rare;
// their registers stay out of the streaming loop); takes plain pointers.
template <typename V, int OP>
__device__ __forceinline__ double stream_chain(const V *vals, const int32_t *cols, const V *x, int64_t ldx, Chain ch,
                                            int64_t c0, int64_t c1, int lane) {
  using P = typename std::conditional<sizeof(V) == 4, float, double>::type;
  constexpr int UN = sizeof(V) == 8 && DCSR_K1_UN > 1 ? DCSR_K1_UN / 2 : DCSR_K1_UN;
  const int64_t first = ch.phys(c0);
  double acc = op_init<double, OP>();
  for (int64_t b0 = c0; b0 < c1; b0 += 32 * UN) {
    V a[UN];
    int32_t col[UN];
#pragma unroll
    for (int i = 0; i < UN; i++) {
      const int64_t p = b0 + 32 * i + lane;
      const int64_t q = p < c1 ? ch.phys(p) : first;
      a[i] = __ldcs(vals + q);
      col[i] = OP == OP_SPMV ? __ldcs(cols + q) : 0;
    }
    P w = op_init<P, OP>();
#pragma unroll
    for (int i = 0; i < UN; i++) {
      if (b0 + 32 * i + lane < c1) {
        P t;
        if constexpr (OP == OP_SPMV) t = mul_rn((P)a[i], (P)__ldg(x + (int64_t)col[i] * ldx));
        else t = OP == OP_COUNT ? (P)1 : (P)a[i];
        w = op_comb<P, OP>(w, t);
      }
    }
    acc = op_comb<double, OP>(acc, (double)w);
  }
  return acc;
}

template <int OP>
__device__ __forceinline__ double warp_comb(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = op_comb<double, OP>(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// A unit of the k = 1 pass, decoded, with its descriptor loaded.  A long-row
// chunk or a medium row is a "streamed" unit: every lane holds (row, row
// length, pool slot of the unit's first entry or -1 when the unit crosses a
// segment boundary, chunk number within the row).  A block of short rows
// holds, in each lane, that lane's row: (row or -1, length, layer-0 start,
// layer-0 capacity).
enum { U1_CHUNK = 0, U1_MED = 1, U1_BLOCK = 2, U1_NONE = 3 };
struct Unit1 {
  int32_t u;   // unit number (>= total: past the end)
  int32_t lu;  // chunk index within the matrix's chunk table (chunks)
  int kind;
  int item;    // matrix of the unit
  int4 d;
};

template <typename V, typename Src>
__device__ __forceinline__ Unit1 unit1_load(const Src &src, int64_t u, int64_t NC, int64_t NM, int64_t total,
                                            int lane) {
  Unit1 x;
  x.u = (int32_t)(u < total ? u : total);
  x.kind = U1_NONE;
  x.item = 0;
  x.lu = 0;
  x.d = make_int4(-1, 0, -1, 0);
  if (u >= total) return x;
  int64_t lu;
  if (u < NC) {
    x.item = src.locate(P_CHUNKS, u, lu);
    const RowItem<V> &it = src.item(x.item);
    if (it.skip && *it.skip) return x;
    x.kind = U1_CHUNK;
    x.lu = (int32_t)lu;
    x.d = it.chunk_desc[lu];
  } else if (u < NC + NM) {
    x.item = src.locate(P_MED, (u - NC) / RS_WARPS, lu);
    const RowItem<V> &it = src.item(x.item);
    const int64_t mi = lu * RS_WARPS + (u - NC) % RS_WARPS;
    if ((it.skip && *it.skip) || mi >= it.info[2]) return x;
    x.kind = U1_MED;
    x.d = it.med_desc[mi];
  } else {
    const int64_t bu = u - NC - NM;
    x.item = src.locate(P_BLOCKS, bu / RS_WARPS, lu);
    const RowItem<V> &it = src.item(x.item);
    const int64_t blk = lu * RS_WARPS + bu % RS_WARPS;
    if ((it.skip && *it.skip) || blk * 32 >= it.m.n_rows) return x;
    x.kind = U1_BLOCK;
    const int64_t r = blk * 32 + lane;
    if (r < it.m.n_rows) {
      const int2 s0 = __ldg(reinterpret_cast<const int2 *>(it.m.seg + 2 * r));
      x.d = make_int4((int32_t)r, __ldg(it.m.row_sizes + r), s0.x, s0.y - s0.x);
    }
  }
  return x;
}

__device__ __forceinline__ bool streamed(const Unit1 &x) { return x.kind == U1_CHUNK || x.kind == U1_MED; }
// The entry range [c0, c1) of a streamed unit within its row.
__device__ __forceinline__ void unit_range(const Unit1 &x, int64_t &c0, int64_t &c1) {
  if (x.kind == U1_CHUNK) {
    c0 = (int64_t)x.d.w * CHUNK;
    c1 = c0 + CHUNK < x.d.y ? c0 + CHUNK : x.d.y;
  } else {
    c0 = 0;
    c1 = x.d.y;
  }
}

// Loads of one step (UN windows of 32 entries) of a streamed unit lying in
// one segment (first pool slot d.z), entries [o, o + 32*UN) of the unit.
template <typename V, int UN, int OP>
__device__ __forceinline__ void load_step(const Mat<V> &m, int32_t base, int32_t n, int32_t o, int lane, V (&a)[UN],
                                          int32_t (&col)[UN]) {
#pragma unroll
  for (int i = 0; i < UN; i++) {
    const int32_t p = o + 32 * i + lane, q = base + (p < n ? p : 0);  // pool slots are below 2^31
    a[i] = __ldcs(m.vals + q);
    col[i] = OP == OP_SPMV ? __ldcs(m.cols + q) : 0;
  }
}

// The end of a streamed unit: its total (t, in every lane) is the row's
// result, or one chunk's partial; the warp that adds the row's last chunk
// combines the partials in chunk order.
template <typename V, int OP>
__device__ __forceinline__ void finish_unit(const RowItem<V> &it, const Unit1 &x, double t, int lane) {
  const int32_t row = x.d.x, L = x.d.y;
  const int64_t nch = x.kind == U1_CHUNK ? (L + CHUNK - 1) / CHUNK : 1;
  if (nch == 1) {
    if (lane == 0) {
      const double o[1] = {t};
      write_y<V, 1, OP>(it.y, it.ldy, row, o, it.alpha, it.beta, L, 1);
    }
    return;
  }
  const int64_t p0 = x.lu - x.d.w;  // the row's first chunk (chunks of a row are consecutive)
  int last = 0;
  if (lane == 0) {
    const int32_t li = it.chunk_rl[x.lu].y;
    it.part[x.lu] = t;
    __threadfence();
    last = atomicAdd(&it.long_cnt[li], 1) == nch - 1;
    if (last) it.long_cnt[li] = 0;
  }
  if (__shfl_sync(FULL, last, 0)) {
    // every chunk's partial is published: lanes take partials lane,
    // lane+32, ... in order, then a fixed xor tree
    __threadfence();
    double v = op_init<double, OP>();
    for (int64_t q = lane; q < nch; q += 32) v = op_comb<double, OP>(v, __ldcg(it.part + p0 + q));
    v = warp_comb<OP>(v);
    if (lane == 0) {
      const double o[1] = {v};
      write_y<V, 1, OP>(it.y, it.ldy, row, o, it.alpha, it.beta, L, 1);
    }
  }
}

// The streamed units (long-row chunks, then medium rows) of a k = 1 pass.
template <typename V, int OP, typename Src, bool XU>
__global__ void __launch_bounds__(RS_THREADS_, DCSR_K1_MINB) k_rows1(Src src) {
  using P = typename std::conditional<sizeof(V) == 4, float, double>::type;
  constexpr int UNO = OP == OP_SPMV ? DCSR_K1_UN : DCSR_K1_UN_RED;
  constexpr int UN = sizeof(V) == 8 && UNO > 1 ? UNO / 2 : UNO;
  constexpr int W = 32 * UN;  // entries of one step
  const int lane = threadIdx.x & 31;
  const int64_t NC = src.units(P_CHUNKS), NM = src.units(P_MED) * RS_WARPS;
  const int64_t total = NC + NM;
  unsigned *ctr = src.ctr(0);
  // A unit number is taken by lane 0 with an atomic and broadcast only when
  // it is needed, one unit later: the atomic's round trip overlaps a unit.
  unsigned pend = 0;
  auto fetch_issue = [&]() {
    if (lane == 0) pend = atomicAdd(ctr, 1u);
  };
  auto fetch_take = [&]() -> int64_t { return (int64_t)__shfl_sync(FULL, pend, 0); };
  // Units in flight per warp: cur (streamed step by step), nx (its
  // descriptor loaded or in flight) and the number of the one after.  Two
  // register buffers take turns: the loads of the next step go into one
  // while the current step's x values are gathered from the other (no copy
  // between them, so nothing waits for a load before its data is used), and
  // the next step may be the next unit's first -- the stream does not stop at
  // unit ends.
  fetch_issue();
  Unit1 cur = unit1_load<V>(src, fetch_take(), NC, NM, total, lane);
  fetch_issue();
  Unit1 nx = unit1_load<V>(src, fetch_take(), NC, NM, total, lane);
  fetch_issue();
  V a0[UN], a1[UN];
  int32_t k0[UN], k1[UN];
  int64_t c0 = 0, c1 = 0;  // cur's range
  int32_t o = 0;           // the current step's offset in it
  if (streamed(cur)) {
    unit_range(cur, c0, c1);
    if (cur.d.z >= 0) load_step<V, UN, OP>(src.item(cur.item).m, cur.d.z, (int32_t)(c1 - c0), 0, lane, a0, k0);
  }
  double acc = op_init<double, OP>();
  // One step: consume (ca, cc), loading the following step into (na, nc).
  auto step = [&](V(&ca)[UN], int32_t(&cc)[UN], V(&na)[UN], int32_t(&nc)[UN]) {
    bool advance = true;
    if (streamed(cur)) {
      const RowItem<V> &it = src.item(cur.item);
      if (cur.d.z < 0) {
        // a unit across segment boundaries (a chained row): streamed on its own
        const double t = warp_comb<OP>(
            stream_chain<V, OP>(it.m.vals, it.m.cols, it.x, it.ldx, load_chain(it.m, cur.d.x), c0, c1, lane));
        finish_unit<V, OP>(it, cur, t, lane);
        if (streamed(nx) && nx.d.z >= 0) {  // the next unit's first step, into the buffer consumed next
          int64_t d0, d1;
          unit_range(nx, d0, d1);
          load_step<V, UN, OP>(src.item(nx.item).m, nx.d.z, (int32_t)(d1 - d0), 0, lane, na, nc);
        }
      } else {
        const int32_t n = (int32_t)(c1 - c0);
        const bool last = o + W >= n;
        if (!last) {
          load_step<V, UN, OP>(it.m, cur.d.z, n, o + W, lane, na, nc);
        } else if (streamed(nx) && nx.d.z >= 0) {
          int64_t d0, d1;
          unit_range(nx, d0, d1);
          load_step<V, UN, OP>(src.item(nx.item).m, nx.d.z, (int32_t)(d1 - d0), 0, lane, na, nc);
        }
        // every x gather of the step issued before the first is used (lanes
        // past the unit's end loaded its first entry: their columns are valid)
        V xv[UN];
#pragma unroll
        for (int i = 0; i < UN; i++)
          xv[i] = OP != OP_SPMV ? V(0) : XU ? __ldg(it.x + cc[i]) : __ldg(it.x + (int64_t)cc[i] * it.ldx);
        P w = op_init<P, OP>();
#pragma unroll
        for (int i = 0; i < UN; i++) {
          if (o + 32 * i + lane < n) {
            P t;
            if constexpr (OP == OP_SPMV) t = mul_rn((P)ca[i], (P)xv[i]);
            else t = OP == OP_COUNT ? (P)1 : (P)ca[i];
            w = op_comb<P, OP>(w, t);
          }
        }
        acc = op_comb<double, OP>(acc, (double)w);
        if (last) {
          finish_unit<V, OP>(it, cur, warp_comb<OP>(acc), lane);
          acc = op_init<double, OP>();
        } else {
          o += W;
          advance = false;
        }
      }
    } else if (streamed(nx) && nx.d.z >= 0) {  // a skipped unit: the next one's first step
      int64_t d0, d1;
      unit_range(nx, d0, d1);
      load_step<V, UN, OP>(src.item(nx.item).m, nx.d.z, (int32_t)(d1 - d0), 0, lane, na, nc);
    }
    if (advance) {
      cur = nx;
      nx = unit1_load<V>(src, fetch_take(), NC, NM, total, lane);
      fetch_issue();
      o = 0;
      if (streamed(cur)) unit_range(cur, c0, c1);
    }
  };
  while (cur.u < total) {
    step(a0, k0, a1, k1);
    if (cur.u >= total) break;
    step(a1, k1, a0, k0);
  }
  // the last warp to finish resets the counters for the next pass (the
  // atomic still pending in lane 0 belongs to nobody: every number past
  // the end is discarded)
  if (lane == 0 && atomicAdd(ctr + 1, 1u) == gridDim.x * RS_WARPS - 1) {
    ctr[0] = 0;
    ctr[1] = 0;
  }
}

// The short-row blocks of a k = 1 pass: a warp per block of 32 rows, the
// next block's descriptors (each lane's row length and layer-0 segment)
// loaded while the current block runs.
template <typename V, int OP, typename Src, bool XU>
__global__ void __launch_bounds__(RS_THREADS_, DCSR_K1B_MINB) k_rows1_blocks(Src src) {
  const int lane = threadIdx.x & 31;
  const int64_t NB = src.units(P_BLOCKS) * RS_WARPS;
  unsigned *ctr = src.ctr(1);
  unsigned pend = 0;  // lane 0's atomic, broadcast one block later
  auto fetch_issue = [&]() {
    if (lane == 0) pend = atomicAdd(ctr, 1u);
  };
  auto fetch_take = [&]() -> int64_t { return (int64_t)__shfl_sync(FULL, pend, 0); };
  // units numbered after the streamed ones (NC + NM): unit1_load decodes them as blocks
  const int64_t base = src.units(P_CHUNKS) + src.units(P_MED) * RS_WARPS, total = base + NB;
  fetch_issue();
  Unit1 cur = unit1_load<V>(src, base + fetch_take(), base, 0, total, lane);
  fetch_issue();
  while (cur.u < total) {
    const Unit1 nx = unit1_load<V>(src, base + fetch_take(), base, 0, total, lane);
    fetch_issue();
    if (cur.kind == U1_BLOCK) short_block_k1<V, OP, XU>(src.item(cur.item), cur.d, lane);
    cur = nx;
  }
  if (lane == 0 && atomicAdd(ctr + 1, 1u) == gridDim.x * RS_WARPS - 1) {
    ctr[0] = 0;
    ctr[1] = 0;
  }
}

// -------------------------------------------------------------- copy pass
// Copies each row's logical entries to dst_off[r] in (out_cols, out_vals),
// optionally writing COO row ids and an int32 row pointer (one matrix).

template <typename V, int PART>
__global__ void __launch_bounds__(RS_THREADS_, DCSR_COPY_MINB) k_rows_copy(RowItem<V> it, const long long *__restrict__ dst_off,
                                                           int32_t *__restrict__ out_cols, V *__restrict__ out_vals,
                                                           int32_t *__restrict__ out_rows,
                                                           int32_t *__restrict__ out_rowptr, int64_t limit) {
  constexpr int U = 4;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const Mat<V> &m = it.m;
  RowOne<V> src{it};
  const int64_t units = src.units(PART);
  if (PART == P_BLOCKS && out_rowptr && blockIdx.x == 0 && threadIdx.x == 0)
    out_rowptr[m.n_rows] = (int32_t)dst_off[m.n_rows];
  if constexpr (PART == P_CHUNKS || PART == P_MED) {
    // Long-row chunks (a CTA each) or medium rows (a warp each), two per
    // step (unit u and the one a grid stride later): both units' descriptor
    // chains (unit -> row -> length, segments, destination) and then all
    // their entries are in flight together -- one unit alone left the warps
    // waiting on its chain for a fraction of the data.
    static_assert(CHUNK % RS_THREADS_ == 0, "whole chunks per thread");
    constexpr bool CH = PART == P_CHUNKS;
    constexpr int NTHR = CH ? RS_THREADS_ : 32;
    // a thread's entries per unit and pass: chunks DCSR_COPY_EPT, medium rows
    // (shorter, a warp each) half that, FP64 half again (8 / 4 measured
    // 217 us for the R-MAT 2^20 stream matrix's export, 8 / 8 with spills
    // 267 us, 4 / 4 219 us; one unit per step 244 us)
    constexpr int EMAX = (CH ? DCSR_COPY_EPT : DCSR_COPY_EPT / 2) / (sizeof(V) == 8 ? 2 : 1);
    constexpr int EPT = CH && CHUNK / RS_THREADS_ < EMAX ? CHUNK / RS_THREADS_ : EMAX;
    const int tid = CH ? threadIdx.x : lane;
    // unit numbers: chunks per CTA, medium rows per warp
    const int64_t n_units = CH ? units : it.info[2];
    const int64_t first = CH ? blockIdx.x : (int64_t)blockIdx.x * RS_WARPS + w;
    const int64_t stride = CH ? gridDim.x : (int64_t)gridDim.x * RS_WARPS;
    for (int64_t u = first; u < n_units; u += 2 * stride) {
      int32_t row[2];
      int64_t c0[2], c1[2], d[2];
      Chain ch[2];
      bool fast[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t uu = u + h * stride;
        row[h] = -1;
        c0[h] = c1[h] = d[h] = 0;
        fast[h] = true;
        ch[h].ns = 0;
        if (uu < n_units) {
          int64_t L;
          if (CH) {
            const int2 rl = it.chunk_rl[uu];
            row[h] = rl.x;
            L = m.row_sizes[rl.x];
            const int64_t chunk = L <= CHUNK ? 0 : uu - it.long_off[rl.y];
            c0[h] = chunk * CHUNK;
            c1[h] = c0[h] + CHUNK < L ? c0[h] + CHUNK : L;
          } else {
            row[h] = it.med_desc[uu].x;
            L = m.row_sizes[row[h]];
            c1[h] = L;
          }
          ch[h] = load_chain(m, row[h]);
          d[h] = dst_off[row[h]];
          fast[h] = ch[h].cp[0] >= c1[h];
          if (out_rowptr && c0[h] == 0 && tid == 0) out_rowptr[row[h]] = (int32_t)d[h];
        }
      }
      const int64_t span = CH ? CHUNK : (c1[0] > c1[1] ? c1[0] : c1[1]);  // medium rows start at 0
      for (int64_t s0 = 0; s0 < span; s0 += (int64_t)EPT * NTHR) {
        int32_t cv[2 * EPT];
        V vv[2 * EPT];
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
          for (int g = 0; g < EPT; g++) {
            const int64_t p = c0[h] + s0 + tid + (int64_t)g * NTHR;
            if (p < c1[h]) {
              const int64_t q = fast[h] ? (int64_t)ch[h].st[0] + p : ch[h].phys(p);
              cv[h * EPT + g] = __ldcs(m.cols + q);
              vv[h * EPT + g] = __ldcs(m.vals + q);
            }
          }
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
          for (int g = 0; g < EPT; g++) {
            const int64_t p = c0[h] + s0 + tid + (int64_t)g * NTHR;
            if (p < c1[h] && d[h] + p < limit) {
              out_cols[d[h] + p] = cv[h * EPT + g];
              out_vals[d[h] + p] = vv[h * EPT + g];
              if (out_rows) out_rows[d[h] + p] = row[h];
            }
          }
      }
    }
  } else {
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {  // a block of 32 short rows per warp
      const int64_t blk = u * RS_WARPS + w;
      if (blk * 32 >= m.n_rows) continue;
      const int64_t r0 = blk * 32;
      const RowBlock rb = load_block(m, r0, lane, it.short_max);
      const int64_t dme = rb.row >= 0 ? dst_off[rb.row] : 0;
      if (out_rowptr && rb.row >= 0 && rb.len <= it.short_max) out_rowptr[rb.row] = (int32_t)dme;
      int64_t cum = 0;
      for (int l = 0; l < m.max_segs; l++) {
        const int64_t dl = dme + cum;  // destination of this layer's part
        int32_t len_l, st_l;
        next_layer(m, rb, l, cum, len_l, st_l);
        if (!__any_sync(FULL, len_l > 0)) break;
        const int32_t incl = warp_incl_scan(len_l);
        const int32_t excl = incl - len_l;
        const int32_t E = __shfl_sync(FULL, incl, 31);
        for (int32_t base = 0; base < E; base += 32 * U) {
          int64_t q[U], dst[U];
          int jw[U];
#pragma unroll
          for (int i = 0; i < U; i++) {
            const int32_t w0 = base + 32 * i;
            const int j = owner_lane(excl, w0 + lane);
            const int32_t ej = __shfl_sync(FULL, excl, j);
            const int32_t sj = __shfl_sync(FULL, st_l, j);
            const int64_t dj = __shfl_sync(FULL, dl, j);
            const bool ok = w0 + lane < E;
            const int32_t off = ok ? w0 + lane - ej : 0;
            jw[i] = ok ? j : -1;
            q[i] = (int64_t)sj + off;
            dst[i] = dj + off;
          }
          int32_t cv[U];
          V vv[U];
#pragma unroll
          for (int i = 0; i < U; i++) {
            cv[i] = __ldcs(m.cols + q[i]);
            vv[i] = __ldcs(m.vals + q[i]);
          }
#pragma unroll
          for (int i = 0; i < U; i++) {
            if (jw[i] >= 0 && dst[i] < limit) {
              out_cols[dst[i]] = cv[i];
              out_vals[dst[i]] = vv[i];
              if (out_rows) out_rows[dst[i]] = (int32_t)(r0 + jw[i]);
            }
          }
        }
      }
    }
  }
}

static int grid_of(const void *k) { return persistent_grid(k, RS_THREADS_, 0); }

template <typename V, int K, int OP, bool VEC, typename Src>
static int launch_reduce_src(const Src &src, cudaStream_t s) {
  if constexpr (K == 1) {  // one value per entry: streamed units, then short-row blocks
    // VEC (k = 1): x has unit stride, gathered without the stride multiply
    constexpr bool XU = VEC && OP == OP_SPMV;
    static const int g = grid_of((const void *)k_rows1<V, OP, Src, XU>);
    static const int gb = grid_of((const void *)k_rows1_blocks<V, OP, Src, XU>);
    DCSR_LAUNCH((k_rows1<V, OP, Src, XU>), g, RS_THREADS_, 0, s, src);
    DCSR_LAUNCH((k_rows1_blocks<V, OP, Src, XU>), gb, RS_THREADS_, 0, s, src);
    return DCSR_OK;
  } else {
    static const int g0 = grid_of((const void *)k_rows_reduce<V, K, OP, VEC, P_BLOCKS, Src>);
    static const int g1 = grid_of((const void *)k_rows_reduce<V, K, OP, VEC, P_CHUNKS, Src>);
    static const int g2 = grid_of((const void *)k_rows_reduce<V, K, OP, VEC, P_MED, Src>);
    DCSR_LAUNCH((k_rows_reduce<V, K, OP, VEC, P_CHUNKS, Src>), g1, RS_THREADS_, 0, s, src);
    DCSR_LAUNCH((k_rows_reduce<V, K, OP, VEC, P_MED, Src>), g2, RS_THREADS_, 0, s, src);
    DCSR_LAUNCH((k_rows_reduce<V, K, OP, VEC, P_BLOCKS, Src>), g0, RS_THREADS_, 0, s, src);
    return DCSR_OK;
  }
}

// Warps per 32-row block of short rows for the k >= 2 pass: doubled (up to
// 8) while the blocks times the split stay under 12 warps per SM, so a
// matrix of a few thousand rows is not left to a few dozen warps, each
// walking 32 rows' groups one after another.
int short_split(int64_t blocks, int k) {
  if (k == 1) return 1;
  int S = 1;
  while (S < 8 && blocks * S * 2 <= (int64_t)sm_count() * 12) S *= 2;
  return S;
}

template <typename V, int K, int OP, bool VEC>
static int launch_reduce(dcsr_handle h, const V *x, int64_t ldx, V *y, int64_t ldy, double alpha, double beta,
                         cudaStream_t s) {
  RowOne<V> src{row_item<V>(h, x, y, ldx, ldy, alpha, beta)};
  src.split = OP == OP_SPMV ? short_split(div_up(h->n_rows, 32), K) : 1;
  return launch_reduce_src<V, K, OP, VEC>(src, s);
}

template <typename V, int K>
static int spmv_k(dcsr_handle h, const V *x, int64_t ldx, V *y, int64_t ldy, double alpha, double beta,
                  cudaStream_t s) {
  const size_t rb = K * sizeof(V), al = (rb & (0 - rb)) >= 32 ? 32 : (rb & (0 - rb));  // row alignment
  // k >= 2: packed, aligned rows of x (vector loads); k = 1: x of unit stride
  const bool vec = K == 1 ? ldx == 1 : (K % 2 == 0) && ldx == K && ((uintptr_t)x % al) == 0;
  if (vec) return launch_reduce<V, K, OP_SPMV, true>(h, x, ldx, y, ldy, alpha, beta, s);
  return launch_reduce<V, K, OP_SPMV, false>(h, x, ldx, y, ldy, alpha, beta, s);
}

template <typename V>
static int spmv_dispatch(dcsr_handle h, const V *x, int32_t k, int64_t ldx, V *y, int64_t ldy, double alpha,
                         double beta, cudaStream_t s) {
  if (k == 1 && h->n_rows <= K1_GROUP_ROWS) {  // the runtime-k pass with the item's k = 1
    RowOne<V> src{row_item<V>(h, x, y, ldx, ldy, alpha, beta)};
    src.split = short_split(div_up(h->n_rows, 32), 2);
    return launch_reduce_src<V, -2, OP_SPMV, false>(src, s);
  }
  switch (k) {
    case 1: return spmv_k<V, 1>(h, x, ldx, y, ldy, alpha, beta, s);
    case 2: return spmv_k<V, 2>(h, x, ldx, y, ldy, alpha, beta, s);
    case 3: return spmv_k<V, 3>(h, x, ldx, y, ldy, alpha, beta, s);
    case 4: return spmv_k<V, 4>(h, x, ldx, y, ldy, alpha, beta, s);
    case 5: return spmv_k<V, 5>(h, x, ldx, y, ldy, alpha, beta, s);
    case 6: return spmv_k<V, 6>(h, x, ldx, y, ldy, alpha, beta, s);
    case 7: return spmv_k<V, 7>(h, x, ldx, y, ldy, alpha, beta, s);
    case 8: return spmv_k<V, 8>(h, x, ldx, y, ldy, alpha, beta, s);
  }
  return DCSR_BAD_ARG;
}

template <typename V>
static int reduce_dispatch(dcsr_handle h, int32_t op, V *y, cudaStream_t s) {
  switch (op) {
    case DCSR_REDUCE_SUM: return launch_reduce<V, 1, OP_SUM, false>(h, nullptr, 0, y, 1, 1.0, 0.0, s);
    case DCSR_REDUCE_MAX: return launch_reduce<V, 1, OP_MAX, false>(h, nullptr, 0, y, 1, 1.0, 0.0, s);
    case DCSR_REDUCE_MIN: return launch_reduce<V, 1, OP_MIN, false>(h, nullptr, 0, y, 1, 1.0, 0.0, s);
    case DCSR_REDUCE_COUNT: return launch_reduce<V, 1, OP_COUNT, false>(h, nullptr, 0, y, 1, 1.0, 0.0, s);
  }
  return DCSR_BAD_ARG;
}

// Batched SpMV over a set of matrices of one k family: kf = 1 (k = 1,
// streamed short rows), 2, 4 or 8 (each item's k <= kf, read by the kernel).
template <typename V>
static int spmv_many_t(const RowItem<V> *its, int count, int kf, long long *pref, bool prefixed, int split,
                       cudaStream_t s) {
  if (kf == 1) split = 1;
  if (!prefixed) DCSR_LAUNCH(k_unit_prefix<V>, 1, 1024, 0, s, its, count, pref, split);
  RowMany<V> src{its, count, pref, split};
  switch (kf) {
    case 1: return launch_reduce_src<V, 1, OP_SPMV, false>(src, s);
    case 2: return launch_reduce_src<V, -2, OP_SPMV, false>(src, s);
    case 4: return launch_reduce_src<V, -4, OP_SPMV, false>(src, s);
    case 8: return launch_reduce_src<V, -8, OP_SPMV, false>(src, s);
  }
  return DCSR_BAD_ARG;
}

int spmv_many(const void *items_dev, int dtype, int count, int k, long long *pref, cudaStream_t s, bool prefixed,
              int split) {
  if (count == 0) return DCSR_OK;
  if (dtype == DCSR_F32)
    return spmv_many_t<float>((const RowItem<float> *)items_dev, count, k, pref, prefixed, split, s);
  return spmv_many_t<double>((const RowItem<double> *)items_dev, count, k, pref, prefixed, split, s);
}

template <typename V>
static int unit_prefix_many_t(const void *const *items, const int *counts, long long *const *prefs,
                              const int *splits, int n, cudaStream_t s) {
  PrefixJobs<V> jobs;
  std::memset(&jobs, 0, sizeof(jobs));
  for (int i = 0; i < n; i++) {
    jobs.its[i] = (const RowItem<V> *)items[i];
    jobs.count[i] = counts[i];
    jobs.pref[i] = prefs[i];
    jobs.split[i] = splits[i];
  }
  DCSR_LAUNCH(k_unit_prefix_many<V>, n, 1024, 0, s, jobs);
  return DCSR_OK;
}

int unit_prefix_many(const void *const *items, const int *counts, long long *const *prefs, const int *splits, int n,
                     int dtype, cudaStream_t s) {
  if (n < 1) return DCSR_OK;
  if (n > MAX_PREFIX_JOBS) return DCSR_BAD_ARG;
  if (dtype == DCSR_F32) return unit_prefix_many_t<float>(items, counts, prefs, splits, n, s);
  return unit_prefix_many_t<double>(items, counts, prefs, splits, n, s);
}

template <typename V>
static int launch_copy(dcsr_handle h, const long long *dst_off, int32_t *out_cols, V *out_vals, int32_t *out_rows,
                       int32_t *out_rowptr, int64_t limit, cudaStream_t s) {
  static const int g0 = grid_of((const void *)k_rows_copy<V, P_BLOCKS>);
  static const int g1 = grid_of((const void *)k_rows_copy<V, P_CHUNKS>);
  static const int g2 = grid_of((const void *)k_rows_copy<V, P_MED>);
  const RowItem<V> it = row_item<V>(h, nullptr, nullptr, 0, 0, 0.0, 0.0);
  DCSR_LAUNCH((k_rows_copy<V, P_CHUNKS>), g1, RS_THREADS_, 0, s, it, dst_off, out_cols, out_vals, out_rows, out_rowptr,
              limit);
  DCSR_LAUNCH((k_rows_copy<V, P_MED>), g2, RS_THREADS_, 0, s, it, dst_off, out_cols, out_vals, out_rows, out_rowptr,
              limit);
  DCSR_LAUNCH((k_rows_copy<V, P_BLOCKS>), g0, RS_THREADS_, 0, s, it, dst_off, out_cols, out_vals, out_rows,
              out_rowptr, limit);
  return DCSR_OK;
}

int copy_rows(dcsr_handle h, const long long *dst_off, int32_t *out_cols, void *out_vals, int32_t *out_rows,
              int32_t *out_rowptr, cudaStream_t s, int64_t limit) {
  if (!h->bins_valid) DCSR_TRY(build_schedule(h, s));
  if (h->dtype == DCSR_F32)
    return launch_copy<float>(h, dst_off, out_cols, (float *)out_vals, out_rows, out_rowptr, limit, s);
  return launch_copy<double>(h, dst_off, out_cols, (double *)out_vals, out_rows, out_rowptr, limit, s);
}

}  // namespace dcsr

using namespace dcsr;

namespace dcsr {
int spmv_call(dcsr_handle h, const void *x, int32_t k, int64_t ldx, void *y, int64_t ldy, double alpha, double beta,
              cudaStream_t s, Arena *ar) {
  if (h->n_rows == 0) return DCSR_OK;
  DCSR_TRY(ensure_part(h, k == 1 && h->n_rows <= K1_GROUP_ROWS ? 2 : k, s));  // partials of the k <= 2 pass
  if (!h->bins_valid) DCSR_TRY(build_schedule(h, s, ar));
  if (h->dtype == DCSR_F32)
    return spmv_dispatch<float>(h, (const float *)x, k, ldx, (float *)y, ldy, alpha, beta, s);
  return spmv_dispatch<double>(h, (const double *)x, k, ldx, (double *)y, ldy, alpha, beta, s);
}
}  // namespace dcsr

extern "C" int dcsr_spmv(dcsr_handle h, const void *x, int32_t k, int64_t ldx, void *y, int64_t ldy, double alpha,
                         double beta, void *stream) {
  if (!h || k < 1 || k > 8 || ldx < k || ldy < k || (h->n_rows > 0 && !y) || (h->n_cols > 0 && !x))
    return DCSR_BAD_ARG;
  return spmv_call(h, x, k, ldx, y, ldy, alpha, beta, (cudaStream_t)stream);
}

extern "C" int dcsr_row_reduce(dcsr_handle h, int32_t op, void *y, void *stream) {
  if (!h || (h->n_rows > 0 && !y) || op < 0 || op > 3) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (h->n_rows == 0) return DCSR_OK;
  DCSR_TRY(ensure_part(h, 1, s));
  if (!h->bins_valid) DCSR_TRY(build_schedule(h, s));
  if (h->dtype == DCSR_F32) return reduce_dispatch<float>(h, op, (float *)y, s);
  return reduce_dispatch<double>(h, op, (double *)y, s);
}
