// rowstream.cu -- row-parallel passes over a DCSR matrix: SpMV (1..8 RHS),
// row reductions, DCSR -> CSR/COO export and the compaction copy.
//
// Work decomposition (one persistent launch per pass):
//   long rows   (length > LONG_ROW) are cut into CHUNK-entry chunks, one CTA
//               per chunk (128-bit loads when the segment is 16-byte aligned);
//               reductions combine chunk partials in chunk order (the CTA that
//               finishes a row's last chunk sums them), so results do not
//               depend on scheduling.
//   other rows  a warp takes 32 consecutive rows and streams their layer-0
//               entries across its lanes (row found by a shuffle search over
//               the lanes' prefix sums), so consecutive rows' contiguous pool
//               ranges are read coalesced; reductions use a segmented warp
//               scan; entries in further chained segments are done row by row
//               by the whole warp.
// Long-row chunks come first in the unit order so they start early.
//
// The schedule (long-row list + chunk offsets) is rebuilt lazily after any
// change of row lengths.  Reference: spmv_dcsr_bin* include/spmv.inl:364-622
// (seven bin kernels on seven streams, rows read with stale Prow_sizes),
// CompactIndices include/sparse_update.inl:916-1007, DCSRtoCSROffsets :1101.
#include "internal.cuh"

namespace dcsr {

constexpr int RS_THREADS_ = 256;
constexpr int LONG_ROW = 512;
constexpr int CHUNK = 4096;

// ---------------------------------------------------------------- schedule

// packed[r] = (is_long << 32) | chunks  (r < n), packed[n] = 0
__global__ void k_sched_flags(const int32_t *row_sizes, int32_t n, long long *packed) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += stride) {
    long long v = 0;
    if (r < n) {
      const int32_t L = row_sizes[r];
      if (L > LONG_ROW) v = (1ll << 32) | (long long)((L + CHUNK - 1) / CHUNK);
    }
    packed[r] = v;
  }
}
__global__ void k_sched_emit(const int32_t *row_sizes, int32_t n, const long long *scanned, int32_t *long_rows,
                             long long *long_off, int32_t *info) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += stride) {
    const long long s = scanned[r];
    if (r == n) {
      info[0] = (int32_t)(s >> 32);          // long rows
      info[1] = (int32_t)(s & 0xffffffff);   // chunks
      long_off[s >> 32] = s & 0xffffffff;
      continue;
    }
    if (row_sizes[r] > LONG_ROW) {
      long_rows[s >> 32] = (int32_t)r;
      long_off[s >> 32] = s & 0xffffffff;
    }
  }
}

int build_schedule(dcsr_handle h, cudaStream_t s) {
  const int32_t n = h->n_rows;
  Arena &ar = h->scratch;
  DCSR_TRY(ar.reserve(arena_bytes(n + 2, 8) + scan_scratch_bytes(n + 1), s));
  long long *packed = ar.take<long long>(n + 2);
  const int g = (int)std::min<int64_t>(div_up(n + 1, 256), (int64_t)sm_count() * 16);
  DCSR_LAUNCH(k_sched_flags, g, 256, 0, s, h->row_sizes, n, packed);
  DCSR_TRY(scan_i64(packed, packed, n + 1, nullptr, ar, s));
  DCSR_LAUNCH(k_sched_emit, g, 256, 0, s, h->row_sizes, n, packed, h->long_rows, h->long_off, h->sched_info);
  // finisher counters start at zero; finishers reset their own counter
  DCSR_CUDA(cudaMemsetAsync(h->long_cnt, 0, sizeof(int32_t) * (n + 1), s));
  h->bins_valid = true;
  return DCSR_OK;
}

// ------------------------------------------------------------- helpers

// Row containing stream position e: largest lane j with excl_j <= e.
__device__ __forceinline__ int find_row(int64_t e, int64_t excl) {
  int j = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    const int cand = j + step;
    const int64_t v = __shfl_sync(FULL, excl, cand & 31);
    if (cand < 32 && v <= e) j = cand;
  }
  return j;
}

// Per-lane row of the warp's row block [r0, r0+32).
struct RowBlock {
  int32_t row;   // global row id (or -1)
  int32_t len;   // logical length
  bool stream;   // streamed by the block (non-empty and not long)
};

template <typename V>
__device__ __forceinline__ RowBlock load_block(const Mat<V> &m, int64_t r0, int lane) {
  RowBlock b;
  const int64_t r = r0 + lane;
  b.row = r < m.n_rows ? (int32_t)r : -1;
  b.len = b.row >= 0 ? __ldg(m.row_sizes + r) : 0;
  b.stream = b.len > 0 && b.len <= LONG_ROW;
  return b;
}

// Entries of the lane's row that live in segment layer l (coalesced pair
// loads across the block); cum accumulates the capacity of layers < l.
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

template <typename V, int K, bool VEC>
__device__ __forceinline__ void load_xk(const V *__restrict__ x, int64_t c, int64_t ldx, double (&xv)[K]) {
  if constexpr (VEC && sizeof(V) == 4 && K == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(x + c * 4));
    xv[0] = t.x; xv[1] = t.y; xv[2] = t.z; xv[3] = t.w;
  } else if constexpr (VEC && sizeof(V) == 4 && K == 8) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(x + c * 8));
    const float4 u = __ldg(reinterpret_cast<const float4 *>(x + c * 8) + 1);
    xv[0] = t.x; xv[1] = t.y; xv[2] = t.z; xv[3] = t.w;
    xv[4] = u.x; xv[5] = u.y; xv[6] = u.z; xv[7] = u.w;
  } else if constexpr (VEC && sizeof(V) == 4 && K == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2 *>(x + c * 2));
    xv[0] = t.x; xv[1] = t.y;
  } else if constexpr (VEC && sizeof(V) == 8 && K % 2 == 0) {
#pragma unroll
    for (int k = 0; k < K; k += 2) {
      const double2 t = __ldg(reinterpret_cast<const double2 *>(x + c * K + k));
      xv[k] = t.x; xv[k + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) xv[k] = (double)__ldg(x + c * ldx + k);
  }
}

enum { OP_SPMV = 0, OP_SUM = 1, OP_MAX = 2, OP_MIN = 3, OP_COUNT = 4 };

template <int OP>
__device__ __forceinline__ double op_init() {
  return OP == OP_MAX ? -INFINITY : OP == OP_MIN ? INFINITY : 0.0;
}
template <int OP>
__device__ __forceinline__ double op_comb(double a, double b) {
  if (OP == OP_MAX) return a > b ? a : b;
  if (OP == OP_MIN) return a < b ? a : b;
  return a + b;
}

// Contribution of one entry to the K accumulators.
template <typename V, int K, int OP, bool VEC>
__device__ __forceinline__ void contrib(const Mat<V> &m, int64_t q, const V *x, int64_t ldx, double (&c)[K]) {
  const double a = (double)__ldcs(m.vals + q);
  if constexpr (OP == OP_SPMV) {
    const int32_t col = __ldcs(m.cols + q);
    double xv[K];
    load_xk<V, K, VEC>(x, col, ldx, xv);
#pragma unroll
    for (int k = 0; k < K; k++) c[k] = a * xv[k];
  } else {
    c[0] = OP == OP_COUNT ? 1.0 : a;
  }
}

template <typename V, int K, int OP>
__device__ __forceinline__ void write_y(V *y, int64_t ldy, int32_t row, const double (&acc)[K], double alpha,
                                        double beta, int32_t len) {
#pragma unroll
  for (int k = 0; k < K; k++) {
    double v = acc[k];
    if ((OP == OP_MAX || OP == OP_MIN) && len == 0) v = 0.0;
    if (OP == OP_SPMV) {
      v *= alpha;
      if (beta != 0.0) v += beta * (double)y[(int64_t)row * ldy + k];
    }
    y[(int64_t)row * ldy + k] = (V)v;
  }
}

// --------------------------------------------------------- reduction pass

template <typename V, int K, int OP, bool VEC>
__global__ void __launch_bounds__(RS_THREADS_) k_rows_reduce(Mat<V> m, const int32_t *__restrict__ long_rows,
                                                             const long long *__restrict__ long_off,
                                                             const int32_t *__restrict__ info, int32_t *long_cnt,
                                                             double *part, const V *__restrict__ x, int64_t ldx,
                                                             V *__restrict__ y, int64_t ldy, double alpha,
                                                             double beta) {
  __shared__ double red[RS_THREADS_ / 32][K];
  __shared__ int last_flag;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int32_t n_long = info[0];
  const int64_t n_chunks = info[1];
  const int64_t n_blocks = div_up(m.n_rows, 32);
  const int64_t units = n_chunks + div_up(n_blocks, RS_THREADS_ / 32);
  for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
    if (u < n_chunks) {
      // ---- one chunk of a long row, whole CTA
      int64_t lo = 0, hi = n_long;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (long_off[mid] <= u) lo = mid + 1;
        else hi = mid;
      }
      const int64_t li = lo - 1;
      const int32_t row = long_rows[li];
      const int64_t chunk = u - long_off[li];
      const int64_t nch = long_off[li + 1] - long_off[li];
      const int64_t L = m.row_sizes[row];
      const Chain ch = load_chain(m, row);
      const int64_t c0 = chunk * CHUNK, c1 = c0 + CHUNK < L ? c0 + CHUNK : L;
      double acc[K];
#pragma unroll
      for (int k = 0; k < K; k++) acc[k] = op_init<OP>();
      const bool fast = ch.cp[0] >= c1;  // chunk inside layer 0
      if (fast && ((ch.st[0] + c0) & 3) == 0 && sizeof(V) == 4) {
        const int64_t base = ch.st[0] + c0;
        const int64_t nv = (c1 - c0) >> 2;
        for (int64_t v = threadIdx.x; v < nv; v += RS_THREADS_) {
          const float4 a4 = __ldcs(reinterpret_cast<const float4 *>(m.vals + base) + v);
          const float av[4] = {a4.x, a4.y, a4.z, a4.w};
          if constexpr (OP == OP_SPMV) {
            const int4 c4 = __ldcs(reinterpret_cast<const int4 *>(m.cols + base) + v);
            const int32_t cv[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int e = 0; e < 4; e++) {
              double xv[K];
              load_xk<V, K, VEC>(x, cv[e], ldx, xv);
#pragma unroll
              for (int k = 0; k < K; k++) acc[k] = fma((double)av[e], xv[k], acc[k]);
            }
          } else {
#pragma unroll
            for (int e = 0; e < 4; e++) acc[0] = op_comb<OP>(acc[0], OP == OP_COUNT ? 1.0 : (double)av[e]);
          }
        }
        for (int64_t p = c0 + (nv << 2) + threadIdx.x; p < c1; p += RS_THREADS_) {
          double c[K];
          contrib<V, K, OP, VEC>(m, ch.st[0] + p, x, ldx, c);
#pragma unroll
          for (int k = 0; k < K; k++) acc[k] = op_comb<OP>(acc[k], c[k]);
        }
      } else {
        for (int64_t p = c0 + threadIdx.x; p < c1; p += RS_THREADS_) {
          double c[K];
          contrib<V, K, OP, VEC>(m, fast ? ch.st[0] + p : ch.phys(p), x, ldx, c);
#pragma unroll
          for (int k = 0; k < K; k++) acc[k] = op_comb<OP>(acc[k], c[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = op_comb<OP>(v, __shfl_xor_sync(FULL, v, o));
        if (lane == 0) red[w][k] = v;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double t[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
          t[k] = red[0][k];
          for (int q = 1; q < RS_THREADS_ / 32; q++) t[k] = op_comb<OP>(t[k], red[q][k]);
          part[(long_off[li] + chunk) * K + k] = t[k];
        }
        __threadfence();
        const int done = atomicAdd(&long_cnt[li], 1);
        last_flag = done == nch - 1;
      }
      __syncthreads();
      if (last_flag && threadIdx.x == 0) {
        __threadfence();
        double out[K];
#pragma unroll
        for (int k = 0; k < K; k++) out[k] = op_init<OP>();
        for (int64_t q = 0; q < nch; q++)
#pragma unroll
          for (int k = 0; k < K; k++) out[k] = op_comb<OP>(out[k], __ldcg(part + (long_off[li] + q) * K + k));
        write_y<V, K, OP>(y, ldy, row, out, alpha, beta, (int32_t)L);
        long_cnt[li] = 0;
      }
      __syncthreads();
      continue;
    }
    // ---- row blocks: one warp per 32 consecutive rows
    const int64_t blk = (u - n_chunks) * (RS_THREADS_ / 32) + w;
    if (blk >= n_blocks) continue;
    const int64_t r0 = blk * 32;
    const RowBlock rb = load_block(m, r0, lane);
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = op_init<OP>();
    int64_t cum = 0;  // capacity of this lane's row in the layers before l
    for (int l = 0; l < m.max_segs; l++) {
      int32_t len_l, st_l;
      next_layer(m, rb, l, cum, len_l, st_l);
      if (!__any_sync(FULL, len_l > 0)) break;
      const int64_t incl = warp_incl_scan((int64_t)len_l);
      const int64_t excl = incl - len_l;
      const int64_t E = __shfl_sync(FULL, incl, 31);
      for (int64_t base = 0; base < E; base += 32) {
        const int64_t e = base + lane;
        const int j = find_row(e < E ? e : E - 1, excl);
        const int64_t ej = __shfl_sync(FULL, excl, j);
        const int32_t sj = __shfl_sync(FULL, st_l, j);
        double c[K];
        if (e < E) {
          contrib<V, K, OP, VEC>(m, (int64_t)sj + (e - ej), x, ldx, c);
        } else {
#pragma unroll
          for (int k = 0; k < K; k++) c[k] = op_init<OP>();
        }
        // segmented inclusive scan by row j (rows are non-decreasing over lanes)
        const int jj = e < E ? j : 32;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int jo = __shfl_up_sync(FULL, jj, d);
#pragma unroll
          for (int k = 0; k < K; k++) {
            const double co = __shfl_up_sync(FULL, c[k], d);
            if (lane >= d && jo == jj) c[k] = op_comb<OP>(c[k], co);
          }
        }
        // lane j collects the tail of its row's run in this 32-entry window
        const bool hit = len_l > 0 && excl < base + 32 && incl > base;
        const int tail = (int)((incl < base + 32 ? incl : base + 32) - 1 - base);
#pragma unroll
        for (int k = 0; k < K; k++) {
          const double got = __shfl_sync(FULL, c[k], hit ? tail : 0);
          if (hit) acc[k] = op_comb<OP>(acc[k], got);
        }
      }
    }
    if (rb.row >= 0 && rb.len <= LONG_ROW) write_y<V, K, OP>(y, ldy, rb.row, acc, alpha, beta, rb.len);
  }
}

// -------------------------------------------------------------- copy pass
// Copies each row's logical entries to dst_off[r] in (out_cols, out_vals),
// optionally writing COO row ids and an int32 row pointer.

template <typename V>
__global__ void __launch_bounds__(RS_THREADS_) k_rows_copy(Mat<V> m, const int32_t *__restrict__ long_rows,
                                                           const long long *__restrict__ long_off,
                                                           const int32_t *__restrict__ info,
                                                           const long long *__restrict__ dst_off,
                                                           int32_t *__restrict__ out_cols, V *__restrict__ out_vals,
                                                           int32_t *__restrict__ out_rows,
                                                           int32_t *__restrict__ out_rowptr) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int32_t n_long = info[0];
  const int64_t n_chunks = info[1];
  const int64_t n_blocks = div_up(m.n_rows, 32);
  const int64_t units = n_chunks + div_up(n_blocks, RS_THREADS_ / 32);
  if (out_rowptr && blockIdx.x == 0 && threadIdx.x == 0) out_rowptr[m.n_rows] = (int32_t)dst_off[m.n_rows];
  for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
    if (u < n_chunks) {
      int64_t lo = 0, hi = n_long;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (long_off[mid] <= u) lo = mid + 1;
        else hi = mid;
      }
      const int64_t li = lo - 1;
      const int32_t row = long_rows[li];
      const int64_t chunk = u - long_off[li];
      const int64_t L = m.row_sizes[row];
      const Chain ch = load_chain(m, row);
      const int64_t c0 = chunk * CHUNK, c1 = c0 + CHUNK < L ? c0 + CHUNK : L;
      const int64_t d = dst_off[row];
      if (out_rowptr && chunk == 0 && threadIdx.x == 0) out_rowptr[row] = (int32_t)d;
      const bool fast = ch.cp[0] >= c1;
      for (int64_t p = c0 + threadIdx.x; p < c1; p += RS_THREADS_) {
        const int64_t q = fast ? (int64_t)ch.st[0] + p : ch.phys(p);
        out_cols[d + p] = __ldcs(m.cols + q);
        out_vals[d + p] = __ldcs(m.vals + q);
        if (out_rows) out_rows[d + p] = row;
      }
      continue;
    }
    const int64_t blk = (u - n_chunks) * (RS_THREADS_ / 32) + w;
    if (blk >= n_blocks) continue;
    const int64_t r0 = blk * 32;
    const RowBlock rb = load_block(m, r0, lane);
    const int64_t dme = rb.row >= 0 ? dst_off[rb.row] : 0;
    if (out_rowptr && rb.row >= 0) out_rowptr[rb.row] = (int32_t)dme;
    int64_t cum = 0;
    for (int l = 0; l < m.max_segs; l++) {
      const int64_t dl = dme + cum;  // destination of this layer's part
      int32_t len_l, st_l;
      next_layer(m, rb, l, cum, len_l, st_l);
      if (!__any_sync(FULL, len_l > 0)) break;
      const int64_t incl = warp_incl_scan((int64_t)len_l);
      const int64_t excl = incl - len_l;
      const int64_t E = __shfl_sync(FULL, incl, 31);
      for (int64_t base = 0; base < E; base += 32) {
        const int64_t e = base + lane;
        const int j = find_row(e < E ? e : E - 1, excl);
        const int64_t ej = __shfl_sync(FULL, excl, j);
        const int32_t sj = __shfl_sync(FULL, st_l, j);
        const int64_t dj = __shfl_sync(FULL, dl, j);
        if (e < E) {
          const int64_t q = (int64_t)sj + (e - ej);
          out_cols[dj + (e - ej)] = __ldcs(m.cols + q);
          out_vals[dj + (e - ej)] = __ldcs(m.vals + q);
          if (out_rows) out_rows[dj + (e - ej)] = (int32_t)(r0 + j);
        }
      }
    }
  }
}

static int grid_of(const void *k) {
  return persistent_grid(k, RS_THREADS_, 0);
}

template <typename V, int K, int OP, bool VEC>
static int launch_reduce(dcsr_handle h, const V *x, int64_t ldx, V *y, int64_t ldy, double alpha, double beta,
                         cudaStream_t s) {
  static int grid = 0;
  if (!grid) grid = grid_of((const void *)k_rows_reduce<V, K, OP, VEC>);
  DCSR_TRY(ensure_part(h, K, s));
  DCSR_LAUNCH((k_rows_reduce<V, K, OP, VEC>), grid, RS_THREADS_, 0, s, h->view<V>(), h->long_rows, h->long_off,
              h->sched_info, h->long_cnt, h->part, x, ldx, y, ldy, alpha, beta);
  return DCSR_OK;
}

int ensure_part(dcsr_handle h, int K, cudaStream_t s) {
  // chunks <= nnz / CHUNK + long rows <= pool / CHUNK + n_rows
  const int64_t need = (h->pool_cap / CHUNK + h->pool_cap / LONG_ROW + 2) * K;
  if (need <= h->part_cap) return DCSR_OK;
  if (h->part) DCSR_CUDA(cudaFreeAsync(h->part, s));
  h->part = nullptr;
  DCSR_CUDA(cudaMallocAsync((void **)&h->part, sizeof(double) * need, s));
  h->part_cap = need;
  return DCSR_OK;
}

template <typename V, int K>
static int spmv_k(dcsr_handle h, const V *x, int64_t ldx, V *y, int64_t ldy, double alpha, double beta,
                  cudaStream_t s) {
  const size_t al = K * sizeof(V) >= 16 ? 16 : K * sizeof(V);
  const bool vec = K > 1 && (K % 2 == 0) && ldx == K && ((uintptr_t)x % al) == 0;
  if (vec) return launch_reduce<V, K, OP_SPMV, true>(h, x, ldx, y, ldy, alpha, beta, s);
  return launch_reduce<V, K, OP_SPMV, false>(h, x, ldx, y, ldy, alpha, beta, s);
}

template <typename V>
static int spmv_dispatch(dcsr_handle h, const V *x, int32_t k, int64_t ldx, V *y, int64_t ldy, double alpha,
                         double beta, cudaStream_t s) {
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

int copy_rows(dcsr_handle h, const long long *dst_off, int32_t *out_cols, void *out_vals, int32_t *out_rows,
              int32_t *out_rowptr, cudaStream_t s) {
  if (!h->bins_valid) DCSR_TRY(build_schedule(h, s));
  static int gf = 0, gd = 0;
  if (h->dtype == DCSR_F32) {
    if (!gf) gf = grid_of((const void *)k_rows_copy<float>);
    DCSR_LAUNCH(k_rows_copy<float>, gf, RS_THREADS_, 0, s, h->view<float>(), h->long_rows, h->long_off,
                h->sched_info, dst_off, out_cols, (float *)out_vals, out_rows, out_rowptr);
  } else {
    if (!gd) gd = grid_of((const void *)k_rows_copy<double>);
    DCSR_LAUNCH(k_rows_copy<double>, gd, RS_THREADS_, 0, s, h->view<double>(), h->long_rows, h->long_off,
                h->sched_info, dst_off, out_cols, (double *)out_vals, out_rows, out_rowptr);
  }
  return DCSR_OK;
}

}  // namespace dcsr

using namespace dcsr;

extern "C" int dcsr_spmv(dcsr_handle h, const void *x, int32_t k, int64_t ldx, void *y, int64_t ldy, double alpha,
                         double beta, void *stream) {
  if (!h || k < 1 || k > 8 || ldx < k || ldy < k || (h->n_rows > 0 && !y) || (h->n_cols > 0 && !x))
    return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (h->n_rows == 0) return DCSR_OK;
  if (!h->bins_valid) DCSR_TRY(build_schedule(h, s));
  if (h->dtype == DCSR_F32)
    return spmv_dispatch<float>(h, (const float *)x, k, ldx, (float *)y, ldy, alpha, beta, s);
  return spmv_dispatch<double>(h, (const double *)x, k, ldx, (double *)y, ldy, alpha, beta, s);
}

extern "C" int dcsr_row_reduce(dcsr_handle h, int32_t op, void *y, void *stream) {
  if (!h || (h->n_rows > 0 && !y) || op < 0 || op > 3) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (h->n_rows == 0) return DCSR_OK;
  if (!h->bins_valid) DCSR_TRY(build_schedule(h, s));
  if (h->dtype == DCSR_F32) return reduce_dispatch<float>(h, op, (float *)y, s);
  return reduce_dispatch<double>(h, op, (double *)y, s);
}
