// matrix.cu -- DCSR handle lifecycle, CSR/COO/HYB -> DCSR loading, DCSR ->
// CSR/COO export, compaction (defragmentation), pool growth, SpMV row bins,
// the synchronous update repair policy and the status API.
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.cuh"

namespace dcsr {

enum { AUX_BAD_INDEX = 1, AUX_NONCANON = 4, AUX_BAD_ROWPTR = 8 };

// ------------------------------------------------------------- kernels

// caps[r] = policy_cap(len_r) with len_r from an int64 row pointer, caps[n] = 0.
__global__ void k_caps_from_rp(const long long *rp, int32_t n, dcsr_opts o, long long *caps) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += stride)
    caps[r] = r < n ? policy_cap(o, rp[r + 1] - rp[r]) : 0;
}
__global__ void k_caps_from_sizes(const int32_t *row_sizes, int32_t n, dcsr_opts o, long long *caps) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += stride)
    caps[r] = r < n ? policy_cap(o, row_sizes[r]) : 0;
}

// Layer 0 = (off, off+cap), other layers cleared; row_sizes from lens (rp
// diff) when rp != nullptr; pool top = offs[n].
__global__ void k_layout(int32_t *seg, int32_t *row_sizes, int32_t n, int32_t pitch, int max_segs,
                         const long long *offs, const long long *rp) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += stride) {
    if (r == n) {
      row_sizes[n] = (int32_t)offs[n];
      continue;
    }
    *reinterpret_cast<int2 *>(seg + 2 * r) = make_int2((int32_t)offs[r], (int32_t)offs[r + 1]);
    for (int l = 1; l < max_segs; l++) *reinterpret_cast<int2 *>(seg + (int64_t)l * pitch + 2 * r) = make_int2(-1, -1);
    if (rp) row_sizes[r] = (int32_t)(rp[r + 1] - rp[r]);
  }
}

// Copy CSR rows into their new layer-0 segments (warp per row, grid-stride).
// CSR rows into their pool segments: a warp per row, four windows of 32
// entries in flight.  A row longer than COPY_LONG entries is cut into pieces
// of COPY_LONG entries, listed here as (row, piece) and copied a CTA per
// piece by k_copy_csr_pieces: one warp would copy a power-law graph's
// hottest rows alone, and the whole load would wait for it.
constexpr int COPY_LONG = 4096;
template <typename V>
__global__ void k_copy_csr(int32_t n, const long long *__restrict__ offs, const long long *__restrict__ rp,
                           const int32_t *__restrict__ cols, const V *__restrict__ vals, int32_t *__restrict__ pcols,
                           V *__restrict__ pvals, unsigned long long *pieces, int32_t *piece_count) {
  constexpr int U = 4;
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
    const int64_t s = rp[r], L = rp[r + 1] - s, d = offs[r];
    if (L > COPY_LONG) {
      const int np = (int)((L + COPY_LONG - 1) / COPY_LONG);
      int base = 0;
      if (lane == 0) base = atomicAdd(piece_count, np);
      base = __shfl_sync(FULL, base, 0);
      for (int q = lane; q < np; q += 32) pieces[base + q] = ((unsigned long long)(uint32_t)r << 32) | (uint32_t)q;
      continue;
    }
    for (int64_t j0 = 0; j0 < L; j0 += 32 * U) {
      int32_t c[U];
      V v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t j = j0 + 32 * u + lane;
        if (j < L) {
          c[u] = __ldcs(cols + s + j);
          v[u] = __ldcs(vals + s + j);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t j = j0 + 32 * u + lane;
        if (j < L) {
          pcols[d + j] = c[u];
          pvals[d + j] = v[u];
        }
      }
    }
  }
}

// The listed pieces of long rows, a CTA per piece.
template <typename V>
__global__ void k_copy_csr_pieces(const unsigned long long *pieces, const int32_t *piece_count,
                                  const long long *__restrict__ offs, const long long *__restrict__ rp,
                                  const int32_t *__restrict__ cols, const V *__restrict__ vals,
                                  int32_t *__restrict__ pcols, V *__restrict__ pvals) {
  constexpr int U = 4;
  const int32_t cnt = *piece_count;
  const int nt = blockDim.x;
  for (int64_t b = blockIdx.x; b < cnt; b += gridDim.x) {
    const unsigned long long pc = pieces[b];
    const int32_t r = (int32_t)(pc >> 32);
    const int64_t q = (int64_t)(uint32_t)pc;
    const int64_t s = rp[r], L = rp[r + 1] - s, d = offs[r];
    const int64_t j1 = (q + 1) * COPY_LONG < L ? (q + 1) * COPY_LONG : L;
    for (int64_t jb = q * COPY_LONG + threadIdx.x; jb < j1; jb += (int64_t)U * nt) {
      int32_t c[U];
      V v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t j = jb + (int64_t)u * nt;
        if (j < j1) {
          c[u] = __ldcs(cols + s + j);
          v[u] = __ldcs(vals + s + j);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t j = jb + (int64_t)u * nt;
        if (j < j1) {
          pcols[d + j] = c[u];
          pvals[d + j] = v[u];
        }
      }
    }
  }
}

// CSR input check: row pointer monotone, columns in range, rows strictly
// ascending (canonical); converts row_ptr to int64.
__global__ void k_csr_check(const int32_t *row_ptr, const int32_t *cols, int32_t n, int32_t n_cols, long long *rp64,
                            long long *stat) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long flags = 0;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
    const int32_t s = row_ptr[r], e = row_ptr[r + 1];
    if (lane == 0) {
      rp64[r] = s;
      if (r == n - 1) rp64[n] = e;
      if (e < s || (r == 0 && s != 0)) flags |= AUX_BAD_ROWPTR;
    }
    if (e < s) continue;
    for (int32_t j = s + lane; j < e; j += 32) {
      const int32_t c = cols[j];
      if (c < 0 || c >= n_cols) flags |= AUX_BAD_INDEX;
      if (j > s && cols[j - 1] >= c) flags |= AUX_NONCANON;
    }
  }
  flags = __reduce_or_sync(FULL, (unsigned)flags);
  if (lane == 0 && flags) atomicOr((unsigned long long *)&stat[ST_AUX], flags);
}

__global__ void k_expand_rows(const long long *rp, int32_t n, int32_t *rows) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw)
    for (int64_t j = rp[r] + lane; j < rp[r + 1]; j += 32) rows[j] = (int32_t)r;
}

__global__ void k_lens(const int32_t *row_sizes, int32_t n, long long *out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += stride)
    out[r] = r < n ? row_sizes[r] : 0;
}

__global__ void k_sum_lens(const int32_t *row_sizes, int32_t n, long long *out) {
  long long s = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) s += row_sizes[r];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd((unsigned long long *)out, (unsigned long long)s);
}

// HYB -> COO: valid ELL slots (column-major, -1 padding) in (row, slot)
// order, then the COO overflow in its given order.
__global__ void k_ell_flags(const int32_t *ell_cols, int32_t n, int32_t width, int64_t pitch, long long *flag) {
  const int64_t total = (int64_t)n * width;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const int64_t r = i / width, j = i % width;
    flag[i] = ell_cols[j * pitch + r] >= 0 ? 1 : 0;
  }
}
template <typename V>
__global__ void k_ell_emit(const int32_t *ell_cols, const V *ell_vals, int32_t n, int32_t width, int64_t pitch,
                           const long long *pos, int32_t *rows, int32_t *cols, V *vals) {
  const int64_t total = (int64_t)n * width;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const int64_t r = i / width, j = i % width;
    const int32_t c = ell_cols[j * pitch + r];
    if (c < 0) continue;
    rows[pos[i]] = (int32_t)r;
    cols[pos[i]] = c;
    vals[pos[i]] = ell_vals[j * pitch + r];
  }
}

static int grid_for(int64_t n, int block) {
  int64_t g = div_up(n, block);
  int64_t cap = (int64_t)sm_count() * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

// ------------------------------------------------------------ host side

// Spare pool buffers kept by all matrices together (bytes), and the budget.
static std::atomic<int64_t> g_spare_bytes{0};
constexpr int64_t SPARE_BUDGET = 8ll << 30;

static int64_t pool_bytes(dcsr_handle h, int64_t cap) { return cap * (int64_t)(sizeof(int32_t) + h->vsize()); }

static void drop_spare(dcsr_handle h, cudaStream_t s) {
  if (!h->spare_cols) return;
  dcsr::dev_free(h->spare_cols, s);
  dcsr::dev_free(h->spare_vals, s);
  g_spare_bytes -= pool_bytes(h, h->spare_cap);
  h->spare_cols = nullptr;
  h->spare_vals = nullptr;
  h->spare_cap = 0;
}

// New pool buffers of at least cap entries (*got: their capacity): the
// matrix's spare when it is large enough, else a stream-ordered allocation.
static int alloc_pool(dcsr_handle h, int64_t cap, int32_t **cols, void **vals, int64_t *got, cudaStream_t s) {
  if (cap < 1) cap = 1;
  if (h->spare_cols && h->spare_cap >= cap) {
    DCSR_CUDA(cudaStreamWaitEvent(s, h->spare_ev, 0));
    *cols = h->spare_cols;
    *vals = h->spare_vals;
    *got = h->spare_cap;
    g_spare_bytes -= pool_bytes(h, h->spare_cap);
    h->spare_cols = nullptr;
    h->spare_vals = nullptr;
    h->spare_cap = 0;
    return DCSR_OK;
  }
  DCSR_CUDA(dcsr::dev_alloc((void **)cols, cap * sizeof(int32_t), s));
  DCSR_CUDA(dcsr::dev_alloc(vals, cap * h->vsize(), s));
  *got = cap;
  return DCSR_OK;
}

// Retire the current pool buffers (after the kernels enqueued on s that read
// them): kept as the spare when the budget allows, else freed.
static void free_pool(dcsr_handle h, cudaStream_t s) {
  if (h->cols) {
    const int64_t b = pool_bytes(h, h->buf_cap);
    if (h->spare_cols && h->spare_cap < h->buf_cap) drop_spare(h, s);
    if (!h->spare_cols && g_spare_bytes + b <= SPARE_BUDGET &&
        (h->spare_ev || cudaEventCreateWithFlags(&h->spare_ev, cudaEventDisableTiming) == cudaSuccess) &&
        cudaEventRecord(h->spare_ev, s) == cudaSuccess) {
      h->spare_cols = h->cols;
      h->spare_vals = h->vals;
      h->spare_cap = h->buf_cap;
      g_spare_bytes += b;
    } else {
      dcsr::dev_free(h->cols, s);
      dcsr::dev_free(h->vals, s);
    }
  }
  h->cols = nullptr;
  h->vals = nullptr;
  h->buf_cap = 0;
}

static int clear_status(dcsr_handle h, cudaStream_t s);

size_t load_scratch_bytes(dcsr_handle h) {
  return arena_bytes(h->n_rows + 2, 8) + arena_bytes(1, 8) + scan_scratch_bytes(h->n_rows + 1);
}

int load_from_csr64(dcsr_handle h, const long long *rp, const int32_t *cols, const void *vals, cudaStream_t s) {
  Arena &ar = h->scratch;  // caller reserved load_scratch_bytes() beyond its own use
  const int32_t n = h->n_rows;
  long long *caps = ar.take<long long>(n + 2);
  int32_t *piece_count = ar.take<int32_t>(1);  // pieces of long rows listed by k_copy_csr
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  DCSR_CUDA(cudaMemsetAsync(piece_count, 0, sizeof(int32_t), s));
  DCSR_LAUNCH(k_caps_from_rp, grid_for(n + 1, 256), 256, 0, s, rp, n, h->o, caps);
  DCSR_TRY(scan_i64(caps, caps, n + 1, h->stat + ST_TOTAL, ar, s));
  long long host[ST_WORDS];
  DCSR_CUDA(cudaMemcpyAsync(host, h->stat, sizeof(host), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  if (host[ST_STATUS] == DCSR_TIMEOUT) {  // a look-back wait of the sort or scan gave up
    DCSR_TRY(clear_status(h, s));
    return DCSR_TIMEOUT;
  }
  if (host[ST_AUX] & AUX_BAD_INDEX) {
    DCSR_CUDA(cudaMemsetAsync(h->stat + ST_AUX, 0, sizeof(long long), s));
    return DCSR_BAD_INDEX;
  }
  const int64_t top = host[ST_TOTAL];
  if (top > 0x7fffffffLL) return DCSR_OOM;
  int64_t cap = pool_capacity(h->o, top);
  if (cap > 0x7fffffffLL) cap = 0x7fffffffLL;
  int32_t *nc;
  void *nv;
  int64_t got;
  DCSR_TRY(alloc_pool(h, cap, &nc, &nv, &got, s));
  free_pool(h, s);
  h->cols = nc;
  h->vals = nv;
  h->buf_cap = got;
  h->pool_cap = cap;
  DCSR_LAUNCH(k_layout, grid_for(n + 1, 256), 256, 0, s, h->seg, h->row_sizes, n, h->pitch, h->o.max_segs, caps, rp);
  // pieces of rows longer than COPY_LONG: at most 2 * top / COPY_LONG
  unsigned long long *pieces = nullptr;
  DCSR_CUDA(dcsr::dev_alloc(&pieces, sizeof(unsigned long long) * (size_t)(2 * top / COPY_LONG + 1), s));
  const unsigned gp = (unsigned)(8 * sm_count());  // the pieces' grid
  if (h->dtype == DCSR_F32) {
    DCSR_LAUNCH(k_copy_csr<float>, grid_for((int64_t)n * 32, 256), 256, 0, s, n, caps, rp, cols, (const float *)vals,
                h->cols, (float *)h->vals, pieces, piece_count);
    DCSR_LAUNCH(k_copy_csr_pieces<float>, gp, 256, 0, s, pieces, piece_count, caps, rp, cols, (const float *)vals,
                h->cols, (float *)h->vals);
  } else {
    DCSR_LAUNCH(k_copy_csr<double>, grid_for((int64_t)n * 32, 256), 256, 0, s, n, caps, rp, cols,
                (const double *)vals, h->cols, (double *)h->vals, pieces, piece_count);
    DCSR_LAUNCH(k_copy_csr_pieces<double>, gp, 256, 0, s, pieces, piece_count, caps, rp, cols, (const double *)vals,
                h->cols, (double *)h->vals);
  }
  DCSR_CUDA(dcsr::dev_free(pieces, s));
  h->bins_valid = false;
  // A load is a one-off: a resident matrix keeps no load-sized scratch (the
  // stream-ordered pool keeps the memory for the next allocation).
  h->scratch.release(s);
  return DCSR_OK;
}

// Rows staged elsewhere (row r: lens[r] entries at src_off[r] in scols /
// svals, int64 offsets) become the matrix's content with the layout policy's
// capacities -- the CSR load without its host round trip before the copy:
// the pool is allocated at cap_bound entries (the caller's upper bound of
// pool_capacity(top)), the rows are placed, and one synchronisation reads
// the pool top to set the pool capacity.
template <typename V>
__global__ void k_place_rows(int32_t n, const long long *__restrict__ offs, const long long *__restrict__ src_off,
                             const long long *__restrict__ lens, const int32_t *__restrict__ scols,
                             const V *__restrict__ svals, int32_t *__restrict__ pcols, V *__restrict__ pvals) {
  constexpr int U = 4;  // windows of 32 entries whose loads are in flight together
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
    const int64_t s0 = src_off[r], L = lens[r], d = offs[r];
    for (int64_t j0 = 0; j0 < L; j0 += 32 * U) {
      int32_t c[U];
      V v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t j = j0 + 32 * u + lane;
        if (j < L) {
          c[u] = __ldcs(scols + s0 + j);
          v[u] = __ldcs(svals + s0 + j);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t j = j0 + 32 * u + lane;
        if (j < L) {
          pcols[d + j] = c[u];
          pvals[d + j] = v[u];
        }
      }
    }
  }
}
__global__ void k_caps_from_lens(const long long *lens, int32_t n, dcsr_opts o, long long *caps) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += stride)
    caps[r] = r < n ? policy_cap(o, lens[r]) : 0;
}
__global__ void k_sizes_from_lens(const long long *lens, int32_t n, int32_t *row_sizes) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) row_sizes[r] = (int32_t)lens[r];
}

int load_from_rows(dcsr_handle h, const long long *src_off, const long long *lens, const int32_t *scols,
                   const void *svals, int64_t cap_bound, cudaStream_t s) {
  const int32_t n = h->n_rows;
  Arena &ar = h->scratch;
  ar.status = h->stat + ST_STATUS;
  DCSR_TRY(ar.reserve(arena_bytes(n + 2, 8) + scan_scratch_bytes(n + 1), s));
  long long *caps = ar.take<long long>(n + 2);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  if (cap_bound > 0x7fffffffLL) return DCSR_OOM;
  DCSR_LAUNCH(k_caps_from_lens, grid_for(n + 1, 256), 256, 0, s, lens, n, h->o, caps);
  DCSR_TRY(scan_i64(caps, caps, n + 1, h->stat + ST_TOTAL, ar, s));
  int32_t *nc;
  void *nv;
  int64_t got;
  DCSR_TRY(alloc_pool(h, cap_bound, &nc, &nv, &got, s));
  free_pool(h, s);
  h->cols = nc;
  h->vals = nv;
  h->buf_cap = got;
  DCSR_LAUNCH(k_layout, grid_for(n + 1, 256), 256, 0, s, h->seg, h->row_sizes, n, h->pitch, h->o.max_segs, caps,
              (const long long *)nullptr);
  if (n > 0) DCSR_LAUNCH(k_sizes_from_lens, grid_for(n, 256), 256, 0, s, lens, n, h->row_sizes);
  if (n > 0) {
    if (h->dtype == DCSR_F32)
      DCSR_LAUNCH(k_place_rows<float>, grid_for((int64_t)n * 32, 256), 256, 0, s, n, caps, src_off, lens, scols,
                  (const float *)svals, h->cols, (float *)h->vals);
    else
      DCSR_LAUNCH(k_place_rows<double>, grid_for((int64_t)n * 32, 256), 256, 0, s, n, caps, src_off, lens, scols,
                  (const double *)svals, h->cols, (double *)h->vals);
  }
  long long host[ST_WORDS];
  DCSR_CUDA(cudaMemcpyAsync(host, h->stat, sizeof(host), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  h->bins_valid = false;
  h->scratch.release(s);
  if (host[ST_STATUS] == DCSR_TIMEOUT) {
    DCSR_TRY(clear_status(h, s));
    return DCSR_TIMEOUT;
  }
  int64_t cap = pool_capacity(h->o, host[ST_TOTAL]);
  if (cap > 0x7fffffffLL) cap = 0x7fffffffLL;
  if (cap > got) return DCSR_OOM;  // the caller's bound was not one (a bug)
  h->pool_cap = cap;
  return DCSR_OK;
}

int reserve(dcsr_handle h, int64_t cap, cudaStream_t s) {
  if (cap <= h->pool_cap && h->vals) return DCSR_OK;
  if (cap > 0x7fffffffLL) return DCSR_OOM;
  if (h->vals && cap <= h->buf_cap) {  // the buffers (a spare taken earlier) are large enough already
    h->pool_cap = cap;
    return DCSR_OK;
  }
  int32_t *nc;
  void *nv;
  int64_t got;
  DCSR_TRY(alloc_pool(h, cap, &nc, &nv, &got, s));
  if (h->vals && h->pool_cap > 0) {
    DCSR_CUDA(cudaMemcpyAsync(nc, h->cols, h->pool_cap * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    DCSR_CUDA(cudaMemcpyAsync(nv, h->vals, h->pool_cap * h->vsize(), cudaMemcpyDeviceToDevice, s));
  }
  free_pool(h, s);
  h->cols = nc;
  h->vals = nv;
  h->buf_cap = got;
  h->pool_cap = cap;
  return DCSR_OK;
}

// Allocations the reserved regions cannot hold use stream-ordered
// allocation; keep freed blocks in the device's default pool instead of
// returning them at every sync, so a compaction's fresh pool does not re-map
// memory each time (once per device).
void keep_pool_memory() {
  static std::mutex mu;
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    cudaMemPool_t mp;
    if (cudaDeviceGetDefaultMemPool(&mp, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    configured[dev] = true;
  }
}

// The library's own non-blocking stream on the current device (created once
// per device): matrix creation allocates and initialises on it and waits for
// it alone.
int lifecycle_stream(cudaStream_t *out) {
  static std::mutex mu;
  static cudaStream_t streams[64] = {};
  int dev = 0;
  DCSR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return DCSR_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lock(mu);
  if (!streams[dev]) DCSR_CUDA(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking));
  *out = streams[dev];
  return DCSR_OK;
}

int compact(dcsr_handle h, cudaStream_t s) {
  const int32_t n = h->n_rows;
  Arena &ar = h->scratch;
  ar.status = h->stat + ST_STATUS;
  if (!h->bins_valid) DCSR_TRY(build_schedule(h, s));  // before taking arena memory
  DCSR_TRY(ar.reserve(arena_bytes(n + 2, 8) + scan_scratch_bytes(n + 1), s));
  long long *caps = ar.take<long long>(n + 2);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  DCSR_LAUNCH(k_caps_from_sizes, grid_for(n + 1, 256), 256, 0, s, h->row_sizes, n, h->o, caps);
  DCSR_TRY(scan_i64(caps, caps, n + 1, h->stat + ST_TOTAL, ar, s));
  long long host[ST_WORDS];
  DCSR_CUDA(cudaMemcpyAsync(host, h->stat, sizeof(host), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  if (host[ST_STATUS] == DCSR_TIMEOUT) return DCSR_TIMEOUT;  // the scan's look-back gave up (status kept)
  const long long top = host[ST_TOTAL];
  if (top > 0x7fffffffLL) return DCSR_OOM;
  int64_t cap = pool_capacity(h->o, top);
  if (cap < h->pool_cap) cap = h->pool_cap;
  if (cap > 0x7fffffffLL) cap = 0x7fffffffLL;
  int32_t *nc;
  void *nv;
  int64_t got;
  DCSR_TRY(alloc_pool(h, cap, &nc, &nv, &got, s));
  DCSR_TRY(copy_rows(h, caps, nc, nv, nullptr, nullptr, s));
  DCSR_LAUNCH(k_layout, grid_for(n + 1, 256), 256, 0, s, h->seg, h->row_sizes, n, h->pitch, h->o.max_segs, caps,
              (const long long *)nullptr);
  free_pool(h, s);
  h->cols = nc;
  h->vals = nv;
  h->buf_cap = got;
  h->pool_cap = cap;
  // the schedule's row descriptors hold segment starts, which moved
  h->bins_valid = false;
  // the scratch (sized by this matrix's earlier updates) stays for the
  // update a repair runs next: re-allocating it there stalled repairs
  return DCSR_OK;
}

static int read_stat(dcsr_handle h, cudaStream_t s, long long *host) {
  DCSR_CUDA(cudaMemcpyAsync(host, h->stat, sizeof(long long) * ST_WORDS, cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  return DCSR_OK;
}
static int clear_status(dcsr_handle h, cudaStream_t s) {
  DCSR_CUDA(cudaMemsetAsync(h->stat + ST_STATUS, 0, sizeof(long long), s));
  return DCSR_OK;
}

}  // namespace dcsr

using namespace dcsr;

// ------------------------------------------------------------------ C ABI

extern "C" {

void dcsr_default_opts(dcsr_opts *o, int32_t mode) {
  if (!o) return;
  o->max_segs = 4;
  o->mode = mode;
  o->alpha = 4;
  o->spare_x16 = 16;
  o->min_spare = 4096;
  o->reloc_min = 2048;
  if (mode == DCSR_APPEND) {
    o->factor_x16 = 16;
    o->min_cap = 0;
    o->align = 1;
  } else {
    o->factor_x16 = 32;
    o->min_cap = 4;
    o->align = 4;
  }
}

int dcsr_create(dcsr_handle *out, int32_t n_rows, int32_t n_cols, int32_t dtype, const dcsr_opts *opts) {
  if (!out || n_rows < 0 || n_cols < 0 || (dtype != DCSR_F32 && dtype != DCSR_F64)) return DCSR_BAD_ARG;
  dcsr_opts o;
  if (opts) o = *opts;
  else dcsr_default_opts(&o, DCSR_MERGE);
  if (o.max_segs < 1 || o.max_segs > MAX_SEGS || o.factor_x16 < 16 || o.align < 1 || (o.align & (o.align - 1)) ||
      o.min_cap < 0 || o.alpha < 0 || o.spare_x16 < 0 || o.min_spare < 0 || (o.mode != DCSR_MERGE && o.mode != DCSR_APPEND))
    return DCSR_BAD_ARG;
  keep_pool_memory();
  cudaStream_t ls = nullptr;
  DCSR_TRY(lifecycle_stream(&ls));
  dcsr_matrix_s *h = new dcsr_matrix_s;
  h->n_rows = n_rows;
  h->n_cols = n_cols;
  h->dtype = dtype;
  h->o = o;
  h->pitch = (int32_t)align_up(2 * (int64_t)n_rows, 32);
  cudaGetDevice(&h->device);
  const size_t nseg = (size_t)h->pitch * o.max_segs;
  // Stream-ordered allocation and initialisation on the library's own
  // non-blocking stream, then a wait for that stream only: creating a matrix
  // does not stall work on other streams.
  int st = DCSR_OK;
  if (dcsr::dev_alloc((void **)&h->row_sizes, sizeof(int32_t) * (n_rows + 1), ls) != cudaSuccess ||
      dcsr::dev_alloc((void **)&h->seg, sizeof(int32_t) * (nseg ? nseg : 1), ls) != cudaSuccess ||
      dcsr::dev_alloc((void **)&h->stat, sizeof(long long) * ST_WORDS, ls) != cudaSuccess ||
      dcsr::dev_alloc((void **)&h->long_rows, sizeof(int32_t) * (n_rows + 1), ls) != cudaSuccess ||
      dcsr::dev_alloc((void **)&h->long_off, sizeof(long long) * (n_rows + 2), ls) != cudaSuccess ||
      dcsr::dev_alloc((void **)&h->long_cnt, sizeof(int32_t) * (n_rows + 1), ls) != cudaSuccess ||
      dcsr::dev_alloc((void **)&h->med_desc, sizeof(int4) * (n_rows + 1), ls) != cudaSuccess ||
      dcsr::dev_alloc((void **)&h->sched_info, sizeof(int32_t) * 32, ls) != cudaSuccess)
    st = DCSR_OOM;
  if (st == DCSR_OK) {
    h->scratch.status = h->stat + ST_STATUS;  // look-back timeouts of this matrix's operations
    if (cudaMemsetAsync(h->row_sizes, 0, sizeof(int32_t) * (n_rows + 1), ls) != cudaSuccess ||
        cudaMemsetAsync(h->seg, 0xff, sizeof(int32_t) * (nseg ? nseg : 1), ls) != cudaSuccess ||
        cudaMemsetAsync(h->stat, 0, sizeof(long long) * ST_WORDS, ls) != cudaSuccess ||
        cudaMemsetAsync(h->sched_info, 0, sizeof(int32_t) * 32, ls) != cudaSuccess ||
        cudaMemsetAsync(h->long_cnt, 0, sizeof(int32_t) * (n_rows + 1), ls) != cudaSuccess)
      st = DCSR_CUDA_ERROR;
    if (st == DCSR_OK) st = reserve(h, pool_capacity(o, 0), ls);
    if (cudaStreamSynchronize(ls) != cudaSuccess && st == DCSR_OK) st = DCSR_CUDA_ERROR;
  }
  if (st != DCSR_OK) {
    dcsr_destroy(h);
    return st;
  }
  *out = h;
  return DCSR_OK;
}

int dcsr_destroy(dcsr_handle h) {
  if (!h) return DCSR_BAD_ARG;
  // Stream-ordered frees on the legacy default stream, which follows the work
  // already queued on blocking streams; the host does not wait.  Work on
  // non-blocking streams that uses the matrix must be complete (or ordered
  // before the legacy stream) first.
  cudaStream_t s0 = 0;
  h->scratch.release(s0);
  drop_spare(h, s0);
  void *bufs[] = {h->cols, h->vals, h->row_sizes, h->seg, h->stat, h->long_rows, h->long_off,
                  h->long_cnt, h->med_desc, h->sched_info, h->part, h->chunk_rl, h->chunk_desc};
  for (void *p : bufs)
    if (p) dcsr::dev_free(p, s0);
  if (h->spare_ev) cudaEventDestroy(h->spare_ev);
  delete h;
  return DCSR_OK;
}

int dcsr_info(dcsr_handle h, dcsr_info_t *info) {
  if (!h || !info) return DCSR_BAD_ARG;
  info->n_rows = h->n_rows;
  info->n_cols = h->n_cols;
  info->dtype = h->dtype;
  info->pitch = h->pitch;
  info->pool_cap = h->pool_cap;
  info->row_sizes = h->row_sizes;
  info->seg = h->seg;
  info->cols = h->cols;
  info->vals = h->vals;
  info->opts = h->o;
  return DCSR_OK;
}

int dcsr_get_layout(dcsr_handle h, int32_t *row_sizes, int32_t *seg, void *stream) {
  if (!h) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (row_sizes)
    DCSR_CUDA(cudaMemcpyAsync(row_sizes, h->row_sizes, sizeof(int32_t) * (h->n_rows + 1), cudaMemcpyDefault, s));
  if (seg)
    DCSR_CUDA(cudaMemcpyAsync(seg, h->seg, sizeof(int32_t) * (size_t)h->pitch * h->o.max_segs, cudaMemcpyDefault, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  return DCSR_OK;
}

int dcsr_from_csr(dcsr_handle h, const int32_t *row_ptr, const int32_t *cols, const void *vals, int64_t nnz,
                  void *stream) {
  if (!h || !row_ptr || (nnz > 0 && (!cols || !vals)) || nnz < 0 || nnz > 0x7fffffffLL) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int32_t n = h->n_rows;
  Arena &ar = h->scratch;
  DCSR_TRY(ar.reserve(arena_bytes(n + 2, 8) + load_scratch_bytes(h), s));
  long long *rp = ar.take<long long>(n + 2);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  DCSR_CUDA(cudaMemsetAsync(h->stat + ST_AUX, 0, sizeof(long long), s));
  if (n > 0) DCSR_LAUNCH(k_csr_check, grid_for((int64_t)n * 32, 256), 256, 0, s, row_ptr, cols, n, h->n_cols, rp, h->stat);
  else DCSR_CUDA(cudaMemsetAsync(rp, 0, sizeof(long long), s));
  long long host[ST_WORDS], total = 0;
  DCSR_CUDA(cudaMemcpyAsync(&total, rp + n, sizeof(total), cudaMemcpyDeviceToHost, s));
  DCSR_TRY(read_stat(h, s, host));
  const long long aux = host[ST_AUX];
  if (total != nnz) {
    DCSR_CUDA(cudaMemsetAsync(h->stat + ST_AUX, 0, sizeof(long long), s));
    return DCSR_BAD_ARG;
  }
  DCSR_CUDA(cudaMemsetAsync(h->stat + ST_AUX, 0, sizeof(long long), s));
  if (aux & AUX_BAD_ROWPTR) return DCSR_BAD_ARG;
  if (aux & AUX_BAD_INDEX) return DCSR_BAD_INDEX;
  if ((aux & AUX_NONCANON) && h->o.mode == DCSR_MERGE) {
    // canonicalise through the COO path (sort by (row,col), sum duplicates)
    DCSR_TRY(ar.reserve(arena_bytes(n + 2, 8) + arena_bytes(nnz + 1, 4) + coo_to_csr_scratch(h, nnz) +
                            load_scratch_bytes(h), s));
    long long *rp2 = ar.take<long long>(n + 2);
    int32_t *rows = ar.take<int32_t>(nnz + 1);
    if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
    DCSR_LAUNCH(k_csr_check, grid_for((int64_t)n * 32, 256), 256, 0, s, row_ptr, cols, n, h->n_cols, rp2, h->stat);
    DCSR_LAUNCH(k_expand_rows, grid_for((int64_t)n * 32, 256), 256, 0, s, rp2, n, rows);
    DCSR_CUDA(cudaMemsetAsync(h->stat + ST_AUX, 0, sizeof(long long), s));
    long long *crp;
    int32_t *cc;
    void *cv;
    DCSR_TRY(coo_to_csr64(h, rows, cols, vals, nnz, true, ar, &crp, &cc, &cv, nullptr, s));
    return load_from_csr64(h, crp, cc, cv, s);
  }
  return load_from_csr64(h, rp, cols, vals, s);
}

int dcsr_from_coo(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                  void *stream) {
  if (!h || nnz < 0 || nnz > 0x7fffffffLL || (nnz > 0 && (!rows || !cols || !vals))) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  Arena &ar = h->scratch;
  DCSR_TRY(ar.reserve(coo_to_csr_scratch(h, nnz) + load_scratch_bytes(h), s));
  DCSR_CUDA(cudaMemsetAsync(h->stat + ST_AUX, 0, sizeof(long long), s));
  long long *rp;
  int32_t *cc;
  void *cv;
  DCSR_TRY(coo_to_csr64(h, rows, cols, vals, nnz, h->o.mode == DCSR_MERGE, ar, &rp, &cc, &cv, nullptr, s));
  return load_from_csr64(h, rp, cc, cv, s);
}

int dcsr_from_hyb(dcsr_handle h, const int32_t *ell_cols, const void *ell_vals, int32_t ell_width, int64_t ell_pitch,
                  const int32_t *coo_rows, const int32_t *coo_cols, const void *coo_vals, int64_t coo_nnz,
                  void *stream) {
  if (!h || ell_width < 0 || coo_nnz < 0 || (ell_width > 0 && (!ell_cols || !ell_vals || ell_pitch < h->n_rows)))
    return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t slots = (int64_t)h->n_rows * ell_width;
  const int64_t T = slots + coo_nnz;
  if (T > 0x7fffffffLL) return DCSR_BAD_ARG;
  // stage 1: ELL -> COO triples (separate scratch so the COO path can reserve its own)
  int32_t *rows = nullptr, *cols = nullptr;
  void *vals = nullptr;
  long long *flag = nullptr;
  DCSR_CUDA(dcsr::dev_alloc((void **)&rows, sizeof(int32_t) * (T + 1), s));
  DCSR_CUDA(dcsr::dev_alloc((void **)&cols, sizeof(int32_t) * (T + 1), s));
  DCSR_CUDA(dcsr::dev_alloc(&vals, h->vsize() * (T + 1), s));
  DCSR_CUDA(dcsr::dev_alloc((void **)&flag, sizeof(long long) * (slots + 1), s));
  Arena tmp;
  tmp.status = h->stat + ST_STATUS;
  DCSR_TRY(tmp.reserve(scan_scratch_bytes(slots + 1), s));
  long long nell = 0;
  if (slots > 0) {
    DCSR_LAUNCH(k_ell_flags, grid_for(slots, 256), 256, 0, s, ell_cols, h->n_rows, ell_width, ell_pitch, flag);
    DCSR_TRY(scan_i64(flag, flag, slots, h->stat + ST_TOTAL, tmp, s));
    if (h->dtype == DCSR_F32)
      DCSR_LAUNCH(k_ell_emit<float>, grid_for(slots, 256), 256, 0, s, ell_cols, (const float *)ell_vals, h->n_rows,
                  ell_width, ell_pitch, flag, rows, cols, (float *)vals);
    else
      DCSR_LAUNCH(k_ell_emit<double>, grid_for(slots, 256), 256, 0, s, ell_cols, (const double *)ell_vals, h->n_rows,
                  ell_width, ell_pitch, flag, rows, cols, (double *)vals);
    DCSR_CUDA(cudaMemcpyAsync(&nell, h->stat + ST_TOTAL, sizeof(nell), cudaMemcpyDeviceToHost, s));
    DCSR_CUDA(cudaStreamSynchronize(s));
  }
  if (coo_nnz > 0) {
    DCSR_CUDA(cudaMemcpyAsync(rows + nell, coo_rows, sizeof(int32_t) * coo_nnz, cudaMemcpyDeviceToDevice, s));
    DCSR_CUDA(cudaMemcpyAsync(cols + nell, coo_cols, sizeof(int32_t) * coo_nnz, cudaMemcpyDeviceToDevice, s));
    DCSR_CUDA(cudaMemcpyAsync((char *)vals + nell * h->vsize(), coo_vals, h->vsize() * coo_nnz,
                              cudaMemcpyDeviceToDevice, s));
  }
  int st = dcsr_from_coo(h, rows, cols, vals, nell + coo_nnz, stream);
  tmp.release(s);
  dcsr::dev_free(rows, s);
  dcsr::dev_free(cols, s);
  dcsr::dev_free(vals, s);
  dcsr::dev_free(flag, s);
  return st;
}

int dcsr_nnz(dcsr_handle h, int64_t *nnz, void *stream) {
  if (!h || !nnz) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  DCSR_CUDA(cudaMemsetAsync(h->stat + ST_AUX + 1, 0, sizeof(long long), s));
  if (h->n_rows > 0)
    DCSR_LAUNCH(k_sum_lens, grid_for(h->n_rows, 256), 256, 0, s, h->row_sizes, h->n_rows, h->stat + ST_AUX + 1);
  long long v = 0;
  DCSR_CUDA(cudaMemcpyAsync(&v, h->stat + ST_AUX + 1, sizeof(v), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  *nnz = v;
  return DCSR_OK;
}

static int export_impl(dcsr_handle h, int32_t *row_ptr, int32_t *rows, int32_t *cols, void *vals, cudaStream_t s,
                       int64_t limit = INT64_MAX, Arena *arp = nullptr) {
  const int32_t n = h->n_rows;
  Arena &ar = arp ? *arp : h->scratch;
  ar.status = h->stat + ST_STATUS;
  if (!h->bins_valid) DCSR_TRY(build_schedule(h, s, arp));  // before taking arena memory
  DCSR_TRY(ar.reserve(arena_bytes(n + 2, 8) + scan_scratch_bytes(n + 1), s));
  long long *rp = ar.take<long long>(n + 2);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  DCSR_LAUNCH(k_lens, grid_for(n + 1, 256), 256, 0, s, h->row_sizes, n, rp);
  DCSR_TRY(scan_i64(rp, rp, n + 1, nullptr, ar, s));
  return copy_rows(h, rp, cols, vals, rows, row_ptr, s, limit);
}


int dcsr_to_csr(dcsr_handle h, int32_t *row_ptr, int32_t *cols, void *vals, void *stream) {
  if (!h || !row_ptr) return DCSR_BAD_ARG;
  return export_impl(h, row_ptr, nullptr, cols, vals, (cudaStream_t)stream);
}

int dcsr_to_coo(dcsr_handle h, int32_t *rows, int32_t *cols, void *vals, void *stream) {
  if (!h) return DCSR_BAD_ARG;
  return export_impl(h, nullptr, rows, cols, vals, (cudaStream_t)stream);
}

int dcsr_update(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz, void *stream) {
  if (!h || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals))) return DCSR_BAD_ARG;
  return update_async(h, rows, cols, vals, nnz, (cudaStream_t)stream);
}

int dcsr_update_sync(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                     void *stream) {
  if (!h || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals))) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  long long host[ST_WORDS];
  DCSR_TRY(clear_status(h, s));
  DCSR_TRY(update_async(h, rows, cols, vals, nnz, s));
  DCSR_TRY(read_stat(h, s, host));
  int st = (int)host[ST_STATUS];
  if (st == DCSR_POOL_EXHAUSTED || st == DCSR_LAYER_OVERFLOW) {
    DCSR_TRY(clear_status(h, s));
    DCSR_TRY(compact(h, s));
    DCSR_TRY(update_async(h, rows, cols, vals, nnz, s));
    DCSR_TRY(read_stat(h, s, host));
    st = (int)host[ST_STATUS];
    if (st == DCSR_POOL_EXHAUSTED) {
      DCSR_TRY(clear_status(h, s));
      DCSR_TRY(reserve(h, pool_capacity(h->o, host[ST_NEED]), s));
      DCSR_TRY(update_async(h, rows, cols, vals, nnz, s));
      DCSR_TRY(read_stat(h, s, host));
      st = (int)host[ST_STATUS];
    }
  }
  DCSR_TRY(clear_status(h, s));
  return st;
}

int dcsr_get_status(dcsr_handle h, void *stream, int32_t *status) {
  if (!h || !status) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  long long host[ST_WORDS];
  DCSR_TRY(read_stat(h, s, host));
  *status = (int32_t)host[ST_STATUS];
  return clear_status(h, s);
}

int dcsr_compact(dcsr_handle h, void *stream) {
  if (!h) return DCSR_BAD_ARG;
  return compact(h, (cudaStream_t)stream);
}

int dcsr_reserve(dcsr_handle h, int64_t pool_cap, void *stream) {
  if (!h || pool_cap < 0) return DCSR_BAD_ARG;
  return reserve(h, pool_cap, (cudaStream_t)stream);
}

// ---------------------------------------------------------------- snapshot
// Binary image of a matrix's layout: a fixed header, then row_sizes[n+1],
// seg[max_segs*pitch], cols[top] and vals[top] (top = row_sizes[n], the
// pool's bump pointer; slots beyond it hold nothing).  Little-endian, as the
// host writes it.
namespace {
struct SnapHeader {
  char magic[8];  // "DCSRSNP1"
  int32_t version, n_rows, n_cols, dtype;
  dcsr_opts opts;
  int32_t pitch;
  int64_t pool_cap, top;
  int64_t reserved[4];
};
constexpr char SNAP_MAGIC[8] = {'D', 'C', 'S', 'R', 'S', 'N', 'P', '1'};

int64_t snap_bytes(dcsr_handle h, int64_t top) {
  return (int64_t)sizeof(SnapHeader) + 4 * ((int64_t)h->n_rows + 1) + 4 * (int64_t)h->pitch * h->o.max_segs +
         (4 + (int64_t)h->vsize()) * top;
}
int read_top(dcsr_handle h, cudaStream_t s, int64_t *top) {
  int32_t t = 0;
  DCSR_CUDA(cudaMemcpyAsync(&t, h->row_sizes + h->n_rows, sizeof(t), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  *top = t;
  return DCSR_OK;
}
}  // namespace

int dcsr_snapshot_bytes(dcsr_handle h, int64_t *bytes, void *stream) {
  if (!h || !bytes) return DCSR_BAD_ARG;
  int64_t top;
  DCSR_TRY(read_top(h, (cudaStream_t)stream, &top));
  *bytes = snap_bytes(h, top);
  return DCSR_OK;
}

int dcsr_snapshot(dcsr_handle h, void *host_buf, int64_t buf_bytes, void *stream) {
  if (!h || !host_buf) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int64_t top;
  DCSR_TRY(read_top(h, s, &top));
  if (buf_bytes < snap_bytes(h, top)) return DCSR_BAD_ARG;
  SnapHeader hd;
  std::memset(&hd, 0, sizeof(hd));
  std::memcpy(hd.magic, SNAP_MAGIC, 8);
  hd.version = 1;
  hd.n_rows = h->n_rows;
  hd.n_cols = h->n_cols;
  hd.dtype = h->dtype;
  hd.opts = h->o;
  hd.pitch = h->pitch;
  hd.pool_cap = h->pool_cap;
  hd.top = top;
  char *p = (char *)host_buf;
  std::memcpy(p, &hd, sizeof(hd));
  p += sizeof(hd);
  const size_t rs = 4 * ((size_t)h->n_rows + 1), sg = 4 * (size_t)h->pitch * h->o.max_segs;
  DCSR_CUDA(cudaMemcpyAsync(p, h->row_sizes, rs, cudaMemcpyDeviceToHost, s));
  p += rs;
  DCSR_CUDA(cudaMemcpyAsync(p, h->seg, sg, cudaMemcpyDeviceToHost, s));
  p += sg;
  if (top > 0) {
    DCSR_CUDA(cudaMemcpyAsync(p, h->cols, 4 * (size_t)top, cudaMemcpyDeviceToHost, s));
    p += 4 * (size_t)top;
    DCSR_CUDA(cudaMemcpyAsync(p, h->vals, h->vsize() * (size_t)top, cudaMemcpyDeviceToHost, s));
  }
  DCSR_CUDA(cudaStreamSynchronize(s));
  return DCSR_OK;
}

int dcsr_snapshot_header(const void *host_buf, int64_t buf_bytes, int32_t *n_rows, int32_t *n_cols, int32_t *dtype,
                         dcsr_opts *opts) {
  if (!host_buf || buf_bytes < (int64_t)sizeof(SnapHeader)) return DCSR_BAD_ARG;
  SnapHeader hd;
  std::memcpy(&hd, host_buf, sizeof(hd));
  if (std::memcmp(hd.magic, SNAP_MAGIC, 8) != 0 || hd.version != 1) return DCSR_BAD_ARG;
  if (n_rows) *n_rows = hd.n_rows;
  if (n_cols) *n_cols = hd.n_cols;
  if (dtype) *dtype = hd.dtype;
  if (opts) *opts = hd.opts;
  return DCSR_OK;
}

int dcsr_restore(dcsr_handle h, const void *host_buf, int64_t buf_bytes, void *stream) {
  if (!h || !host_buf || buf_bytes < (int64_t)sizeof(SnapHeader)) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  SnapHeader hd;
  std::memcpy(&hd, host_buf, sizeof(hd));
  if (std::memcmp(hd.magic, SNAP_MAGIC, 8) != 0 || hd.version != 1 || hd.n_rows != h->n_rows ||
      hd.n_cols != h->n_cols || hd.dtype != h->dtype || hd.opts.max_segs != h->o.max_segs || hd.pitch != h->pitch ||
      hd.top < 0 || hd.pool_cap < hd.top || hd.pool_cap > 0x7fffffffLL)
    return DCSR_BAD_ARG;
  h->o = hd.opts;  // the layout policy the image was built under
  if (buf_bytes < snap_bytes(h, hd.top)) return DCSR_BAD_ARG;
  const char *p = (const char *)host_buf + sizeof(hd);
  const size_t rs = 4 * ((size_t)h->n_rows + 1), sg = 4 * (size_t)h->pitch * h->o.max_segs;
  int32_t *nc;
  void *nv;
  int64_t got;
  DCSR_TRY(alloc_pool(h, hd.pool_cap, &nc, &nv, &got, s));
  free_pool(h, s);
  h->cols = nc;
  h->vals = nv;
  h->buf_cap = got;
  h->pool_cap = hd.pool_cap;
  DCSR_CUDA(cudaMemcpyAsync(h->row_sizes, p, rs, cudaMemcpyHostToDevice, s));
  p += rs;
  DCSR_CUDA(cudaMemcpyAsync(h->seg, p, sg, cudaMemcpyHostToDevice, s));
  p += sg;
  if (hd.top > 0) {
    DCSR_CUDA(cudaMemcpyAsync(h->cols, p, 4 * (size_t)hd.top, cudaMemcpyHostToDevice, s));
    p += 4 * (size_t)hd.top;
    DCSR_CUDA(cudaMemcpyAsync(h->vals, p, h->vsize() * (size_t)hd.top, cudaMemcpyHostToDevice, s));
  }
  h->bins_valid = false;
  DCSR_CUDA(cudaStreamSynchronize(s));  // the host buffer may be released on return
  return DCSR_OK;
}

int dcsr_bin_rows(dcsr_handle h, void *stream) {
  if (!h) return DCSR_BAD_ARG;
  return build_schedule(h, (cudaStream_t)stream);
}

int dcsr_set_row_classes(dcsr_handle h, int32_t short_max, int32_t long_min) {
  if (!h || short_max < 1 || short_max > 256 || long_min < short_max || long_min < 256 || long_min > (1 << 20))
    return DCSR_BAD_ARG;
  if (h->short_max != short_max || h->long_min != long_min) {
    h->short_max = short_max;
    h->long_min = long_min;
    h->bins_valid = false;  // rows change class: rebuild the schedule before the next pass
  }
  return DCSR_OK;
}

int dcsr_get_row_classes(dcsr_handle h, int32_t *short_max, int32_t *long_min) {
  if (!h || !short_max || !long_min) return DCSR_BAD_ARG;
  *short_max = h->short_max;
  *long_min = h->long_min;
  return DCSR_OK;
}

const char *dcsr_status_string(int st) {
  switch (st) {
    case DCSR_OK: return "OK";
    case DCSR_POOL_EXHAUSTED: return "POOL_EXHAUSTED";
    case DCSR_LAYER_OVERFLOW: return "LAYER_OVERFLOW";
    case DCSR_BAD_INDEX: return "BAD_INDEX";
    case DCSR_OOM: return "OOM";
    case DCSR_BAD_ARG: return "BAD_ARG";
    case DCSR_TIMEOUT: return "TIMEOUT";
    case DCSR_CUDA_ERROR: return "CUDA_ERROR";
    case DCSR_NOT_SUPPORTED: return "NOT_SUPPORTED";
    default: return "UNKNOWN";
  }
}

uint64_t dcsr_launch_count(void) { return g_launches.load(); }

int dcsr_pool_reserve(int64_t bytes, void *stream) {
  if (bytes < 0) return DCSR_BAD_ARG;
  if (bytes == 0) return DCSR_OK;
  keep_pool_memory();
  return dcsr::reserve_regions(bytes, (cudaStream_t)stream);
}

int dcsr_pool_usage(int64_t *reserved, int64_t *free_bytes, int64_t *fallback_allocs) {
  return dcsr::region_usage(reserved, free_bytes, fallback_allocs);
}

int dcsr_debug_lookback(int32_t spin_limit, int32_t stall_first_tile) {
  return dcsr::debug_lookback(spin_limit, stall_first_tile ? 1 : 0);
}

int dcsr_spin_faults(int64_t *count) {
  if (!count) return DCSR_BAD_ARG;
  const long long v = dcsr::spin_faults();
  if (v < 0) return DCSR_CUDA_ERROR;
  *count = v;
  return DCSR_OK;
}
const char *dcsr_version(void) { return "dcsr_b200 0.1 (sm_100a)"; }

}  // extern "C"

namespace dcsr {
int export_csr(dcsr_handle h, int32_t *row_ptr, int32_t *cols, void *vals, int64_t limit, cudaStream_t s,
               Arena *ar) {
  return export_impl(h, row_ptr, nullptr, cols, vals, s, limit, ar);
}
}  // namespace dcsr
