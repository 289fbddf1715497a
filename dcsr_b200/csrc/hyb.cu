// hyb.cu -- DCSR -> HYB conversion and the HYB SpMV.
//
// HYB (cusp's hyb_matrix, the reference's hyb_matrix wrapper of
// include/dcsr_matrix.h:149-172): an ELL part of `width` slots per row,
// stored column-major (slot k of row r at k*pitch + r), unused slots holding
// column -1 and value 0, plus a COO part holding each row's entries beyond
// its first `width`.  Canonical order here: a row's entries in its DCSR order
// (ascending columns in MERGE mode), the first `width` in the ELL slots, the
// rest in the COO part in row order (the reference fills the COO part with
// atomics and sorts it by row, include/load.h:61-106,174-205, which leaves
// the order within a row to the atomics).  The HYB SpMV sums a row's ELL
// slots in slot order, then its COO entries in order (reference spmv_hyb,
// include/spmv.inl:105-156, which scans the whole COO part for every row;
// here a row with a full ELL part finds its COO range by binary search).
#include "internal.cuh"

namespace dcsr {

namespace {

int grid_for(int64_t n, int block) {
  int64_t g = div_up(n, block);
  int64_t cap = (int64_t)sm_count() * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

template <typename V>
__global__ void k_hyb_overflow(Mat<V> m, int32_t width, long long *ov) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= m.n_rows; r += (int64_t)gridDim.x * blockDim.x)
    ov[r] = r < m.n_rows && m.row_sizes[r] > width ? m.row_sizes[r] - width : 0;
}

// One thread per row: its first `width` entries into the ELL slots (padding
// the rest of them), the others to its COO range at ov[r].
template <typename V>
__global__ void k_hyb_emit(Mat<V> m, int32_t width, int64_t pitch, const long long *ov, int32_t *ell_cols,
                           V *ell_vals, int32_t *coo_rows, int32_t *coo_cols, V *coo_vals) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m.n_rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t L = m.row_sizes[r];
    const Chain ch = load_chain(m, (int32_t)r);
    const int64_t o = ov[r];
    for (int32_t j = 0; j < L; j++) {
      const int64_t q = ch.phys(j);
      const int32_t c = m.cols[q];
      const V v = m.vals[q];
      if (j < width) {
        ell_cols[(int64_t)j * pitch + r] = c;
        ell_vals[(int64_t)j * pitch + r] = v;
      } else {
        coo_rows[o + j - width] = (int32_t)r;
        coo_cols[o + j - width] = c;
        coo_vals[o + j - width] = v;
      }
    }
    for (int32_t j = L; j < width; j++) {
      ell_cols[(int64_t)j * pitch + r] = -1;
      ell_vals[(int64_t)j * pitch + r] = V(0);
    }
  }
}

// y = alpha * A x + beta * y for a HYB matrix; one thread per row (the ELL
// slots of consecutive rows are consecutive: coalesced).  Products summed in
// FP64 in slot order, then the row's COO entries in order.
template <typename V>
__global__ void k_hyb_spmv(int32_t n_rows, int32_t width, int64_t pitch, const int32_t *__restrict__ ell_cols,
                           const V *__restrict__ ell_vals, int64_t coo_nnz, const int32_t *__restrict__ coo_rows,
                           const int32_t *__restrict__ coo_cols, const V *__restrict__ coo_vals,
                           const V *__restrict__ x, V *y, double alpha, double beta) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    int32_t last = -1;
    for (int32_t k = 0; k < width; k++) {
      const int32_t c = __ldg(ell_cols + (int64_t)k * pitch + r);
      last = c;
      if (c < 0) break;
      acc = __fma_rn((double)__ldg(ell_vals + (int64_t)k * pitch + r), (double)__ldg(x + c), acc);
    }
    if ((width == 0 || last >= 0) && coo_nnz > 0) {  // a full ELL part: the row may continue in the COO part
      int64_t lo = 0, hi = coo_nnz;  // first COO entry of row r
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(coo_rows + mid) < r) lo = mid + 1;
        else hi = mid;
      }
      for (int64_t q = lo; q < coo_nnz && __ldg(coo_rows + q) == r; q++)
        acc = __fma_rn((double)__ldg(coo_vals + q), (double)__ldg(x + __ldg(coo_cols + q)), acc);
    }
    double v = acc * alpha;
    if (beta != 0.0) v = __fma_rn(beta, (double)y[r], v);
    y[r] = (V)v;
  }
}

// ---- HYB update (the reference's UpdateMatrix(hyb), include/load.h:327-373,
// kernel UpdateMatrix_hyb, include/sparse_update.inl:321-366): triples in
// row order (a stable sort by row), each to its row's next free ELL slot or,
// the ELL part full, to the COO part, which stays sorted by row with a row's
// earlier COO entries first.

// Sort keys (row) and triple numbers; flags[0] |= 1 for an index out of range.
__global__ void k_hu_keys(const int32_t *rows, const int32_t *cols, int64_t T, int32_t n_rows, int32_t n_cols,
                          unsigned long long *key, unsigned *idx, long long *flags) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = rows[i], c = cols[i];
    const bool ok = r >= 0 && r < n_rows && c >= 0 && c < n_cols;
    if (!ok) atomicOr((unsigned long long *)flags, 1ull);
    key[i] = ok ? (unsigned long long)r : 0ull;
    idx[i] = (unsigned)i;
  }
}

// Per sorted triple: its rank j among its row's triples and the row's ELL
// fill f (the filled slots are a prefix: a binary search for the first
// column -1); ELL slot f + j while it is below the width, else a COO entry
// (ov = 1, scanned into positions in row order).
__global__ void k_hu_plan(const unsigned long long *key, int64_t T, int32_t width, int64_t pitch,
                          const int32_t *ell_cols, int32_t *slot, long long *ov) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= T; i += (int64_t)gridDim.x * blockDim.x) {
    if (i == T) {
      ov[T] = 0;
      continue;
    }
    const unsigned long long r = key[i];
    int64_t lo = 0, hi = i;  // first triple of row r
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (key[mid] < r) lo = mid + 1;
      else hi = mid;
    }
    const int64_t j = i - lo;
    int32_t a = 0, b = width;  // first free ELL slot of row r
    while (a < b) {
      const int32_t mid = (a + b) >> 1;
      if (ell_cols[(int64_t)mid * pitch + (int64_t)r] >= 0) a = mid + 1;
      else b = mid;
    }
    const bool ell = (int64_t)a + j < (int64_t)width;
    slot[i] = ell ? (int32_t)(a + j) : -1;
    ov[i] = ell ? 0 : 1;
  }
}

// ELL slots written in place; new COO entries gathered in row order.
template <typename V>
__global__ void k_hu_emit(const unsigned long long *key, const unsigned *idx, int64_t T, const int32_t *slot,
                          const long long *ov, int64_t pitch, const int32_t *cols, const V *vals, int32_t *ell_cols,
                          V *ell_vals, int32_t *nr, int32_t *nc, V *nv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = (int64_t)key[i];
    const unsigned t = idx[i];
    const int32_t k = slot[i];
    if (k >= 0) {
      ell_cols[(int64_t)k * pitch + r] = cols[t];
      ell_vals[(int64_t)k * pitch + r] = vals[t];
    } else {
      const int64_t p = ov[i];
      nr[p] = (int32_t)r;
      nc[p] = cols[t];
      nv[p] = vals[t];
    }
  }
}

// Count of sorted rows[0, n) below r (strict) or at most r.
__device__ __forceinline__ int64_t rows_before(const int32_t *rows, int64_t n, int32_t r, bool inclusive) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    const int32_t v = rows[mid];
    if (v < r || (inclusive && v == r)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// The merged COO part: old entry a at a + (new rows below its row), new
// entry b at b + (old rows at or below its row) -- a stable merge by row.
template <typename V>
__global__ void k_hu_merge(const int32_t *orow, const int32_t *ocol, const V *oval, int64_t m, const int32_t *nr,
                           const int32_t *nc, const V *nv, int64_t q, int32_t *coo_rows, int32_t *coo_cols,
                           V *coo_vals) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m + q; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < m) {
      const int32_t r = orow[i];
      const int64_t p = i + rows_before(nr, q, r, false);
      coo_rows[p] = r;
      coo_cols[p] = ocol[i];
      coo_vals[p] = oval[i];
    } else {
      const int64_t b = i - m;
      const int32_t r = nr[b];
      const int64_t p = b + rows_before(orow, m, r, true);
      coo_rows[p] = r;
      coo_cols[p] = nc[b];
      coo_vals[p] = nv[b];
    }
  }
}

template <typename V>
int hyb_update_body(int32_t n_rows, int32_t n_cols, int32_t width, int64_t pitch, int32_t *ell_cols, V *ell_vals,
                    int32_t *coo_rows, int32_t *coo_cols, V *coo_vals, int64_t coo_cap, int64_t *coo_nnz,
                    const int32_t *rows, const int32_t *cols, const V *vals, int64_t T, Arena &ar, cudaStream_t s) {
  const int64_t m = *coo_nnz;
  const size_t bytes = arena_bytes(4, 8) + 2 * arena_bytes(T, 8) + 2 * arena_bytes(T, 4) + arena_bytes(T, 4) +
                       arena_bytes(T + 1, 8) + 2 * arena_bytes(T, 4) + arena_bytes(T, sizeof(V)) +
                       2 * arena_bytes(m, 4) + arena_bytes(m, sizeof(V)) + radix_scratch_bytes(T) +
                       scan_scratch_bytes(T + 1);
  DCSR_TRY(ar.reserve(bytes, s));
  long long *st = ar.take<long long>(4);  // [0] look-back status, [1] bad-index flag, [2] new COO entries
  ar.status = st;
  unsigned long long *k0 = ar.take<unsigned long long>(T), *k1 = ar.take<unsigned long long>(T);
  unsigned *i0 = ar.take<unsigned>(T), *i1 = ar.take<unsigned>(T);
  int32_t *slot = ar.take<int32_t>(T);
  long long *ov = ar.take<long long>(T + 1);
  int32_t *nr = ar.take<int32_t>(T), *nc = ar.take<int32_t>(T);
  V *nv = ar.take<V>(T);
  int32_t *orow = ar.take<int32_t>(m), *ocol = ar.take<int32_t>(m);
  V *oval = ar.take<V>(m);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  DCSR_CUDA(cudaMemsetAsync(st, 0, 4 * sizeof(long long), s));
  DCSR_LAUNCH(k_hu_keys, grid_for(T, 256), 256, 0, s, rows, cols, T, n_rows, n_cols, k0, i0, st + 1);
  if (T > 1) DCSR_TRY(radix_sort_pairs(&k0, &i0, &k1, &i1, T, bits_for(n_rows), ar, s));
  DCSR_LAUNCH(k_hu_plan, grid_for(T + 1, 256), 256, 0, s, k0, T, width, pitch, ell_cols, slot, ov);
  DCSR_TRY(scan_i64(ov, ov, T + 1, st + 2, ar, s));
  // the one read: validity and the new COO count (the capacity check comes before any write)
  long long host[3];
  DCSR_CUDA(cudaMemcpyAsync(host, st, sizeof(host), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  if (host[0] == DCSR_TIMEOUT) return DCSR_TIMEOUT;
  if (host[1]) return DCSR_BAD_INDEX;
  const int64_t q = host[2];
  if (m + q > coo_cap) return DCSR_POOL_EXHAUSTED;
  if (q > 0 && (!coo_rows || !coo_cols || !coo_vals)) return DCSR_BAD_ARG;
  DCSR_LAUNCH(k_hu_emit<V>, grid_for(T, 256), 256, 0, s, k0, i0, T, slot, ov, pitch, cols, vals, ell_cols, ell_vals,
              nr, nc, nv);
  if (q > 0) {
    if (m > 0) {
      DCSR_CUDA(cudaMemcpyAsync(orow, coo_rows, 4 * m, cudaMemcpyDeviceToDevice, s));
      DCSR_CUDA(cudaMemcpyAsync(ocol, coo_cols, 4 * m, cudaMemcpyDeviceToDevice, s));
      DCSR_CUDA(cudaMemcpyAsync(oval, coo_vals, sizeof(V) * m, cudaMemcpyDeviceToDevice, s));
    }
    DCSR_LAUNCH(k_hu_merge<V>, grid_for(m + q, 256), 256, 0, s, orow, ocol, oval, m, nr, nc, nv, q, coo_rows, coo_cols,
                coo_vals);
  }
  *coo_nnz = m + q;
  return DCSR_OK;
}

template <typename V>
int hyb_update_t(int32_t n_rows, int32_t n_cols, int32_t width, int64_t pitch, int32_t *ell_cols, V *ell_vals,
                 int32_t *coo_rows, int32_t *coo_cols, V *coo_vals, int64_t coo_cap, int64_t *coo_nnz,
                 const int32_t *rows, const int32_t *cols, const V *vals, int64_t T, cudaStream_t s) {
  Arena ar;  // scratch of this call, released (stream-ordered) on every path
  const int rc = hyb_update_body<V>(n_rows, n_cols, width, pitch, ell_cols, ell_vals, coo_rows, coo_cols, coo_vals,
                                    coo_cap, coo_nnz, rows, cols, vals, T, ar, s);
  ar.release(s);
  return rc;
}

int overflow_scan(dcsr_handle h, int32_t width, cudaStream_t s, long long **ov, int64_t *total) {
  Arena &ar = h->scratch;
  ar.status = h->stat + ST_STATUS;
  DCSR_TRY(ar.reserve(arena_bytes(h->n_rows + 2, 8) + scan_scratch_bytes(h->n_rows + 1), s));
  *ov = ar.take<long long>(h->n_rows + 2);
  if (ar.overflow) return DCSR_OOM;  // scratch sizing bug: no kernel sees a null pointer
  if (h->dtype == DCSR_F32)
    DCSR_LAUNCH(k_hyb_overflow<float>, grid_for(h->n_rows + 1, 256), 256, 0, s, h->view<float>(), width, *ov);
  else
    DCSR_LAUNCH(k_hyb_overflow<double>, grid_for(h->n_rows + 1, 256), 256, 0, s, h->view<double>(), width, *ov);
  DCSR_TRY(scan_i64(*ov, *ov, h->n_rows + 1, h->stat + ST_TOTAL, ar, s));
  long long host[ST_WORDS];
  DCSR_CUDA(cudaMemcpyAsync(host, h->stat, sizeof(host), cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  if (host[ST_STATUS] == DCSR_TIMEOUT) return DCSR_TIMEOUT;
  *total = host[ST_TOTAL];
  return DCSR_OK;
}

}  // namespace
}  // namespace dcsr

using namespace dcsr;

extern "C" int dcsr_hyb_overflow(dcsr_handle h, int32_t ell_width, int64_t *coo_nnz, void *stream) {
  if (!h || ell_width < 0 || !coo_nnz) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  long long *ov;
  int64_t total = 0;
  DCSR_TRY(overflow_scan(h, ell_width, s, &ov, &total));
  *coo_nnz = total;
  return DCSR_OK;
}

extern "C" int dcsr_to_hyb(dcsr_handle h, int32_t ell_width, int64_t ell_pitch, int32_t *ell_cols, void *ell_vals,
                           int32_t *coo_rows, int32_t *coo_cols, void *coo_vals, int64_t coo_cap, int64_t *coo_nnz,
                           void *stream) {
  if (!h || ell_width < 0 || ell_pitch < h->n_rows || !coo_nnz || (ell_width > 0 && (!ell_cols || !ell_vals)))
    return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  long long *ov;
  int64_t total = 0;
  DCSR_TRY(overflow_scan(h, ell_width, s, &ov, &total));
  *coo_nnz = total;
  if (total > coo_cap || (total > 0 && (!coo_rows || !coo_cols || !coo_vals))) return DCSR_BAD_ARG;
  if (h->n_rows == 0) return DCSR_OK;
  const int g = grid_for(h->n_rows, 128);
  if (h->dtype == DCSR_F32)
    DCSR_LAUNCH(k_hyb_emit<float>, g, 128, 0, s, h->view<float>(), ell_width, ell_pitch, ov, ell_cols,
                (float *)ell_vals, coo_rows, coo_cols, (float *)coo_vals);
  else
    DCSR_LAUNCH(k_hyb_emit<double>, g, 128, 0, s, h->view<double>(), ell_width, ell_pitch, ov, ell_cols,
                (double *)ell_vals, coo_rows, coo_cols, (double *)coo_vals);
  return DCSR_OK;
}

extern "C" int dcsr_hyb_spmv(int32_t n_rows, int32_t dtype, int32_t ell_width, int64_t ell_pitch,
                             const int32_t *ell_cols, const void *ell_vals, int64_t coo_nnz, const int32_t *coo_rows,
                             const int32_t *coo_cols, const void *coo_vals, const void *x, void *y, double alpha,
                             double beta, void *stream) {
  if (n_rows < 0 || ell_width < 0 || ell_pitch < n_rows || coo_nnz < 0 || (dtype != DCSR_F32 && dtype != DCSR_F64) ||
      (ell_width > 0 && (!ell_cols || !ell_vals)) || (coo_nnz > 0 && (!coo_rows || !coo_cols || !coo_vals)) ||
      (n_rows > 0 && (!x || !y)))
    return DCSR_BAD_ARG;
  if (n_rows == 0) return DCSR_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int g = grid_for(n_rows, 256);
  if (dtype == DCSR_F32)
    DCSR_LAUNCH(k_hyb_spmv<float>, g, 256, 0, s, n_rows, ell_width, ell_pitch, ell_cols, (const float *)ell_vals,
                coo_nnz, coo_rows, coo_cols, (const float *)coo_vals, (const float *)x, (float *)y, alpha, beta);
  else
    DCSR_LAUNCH(k_hyb_spmv<double>, g, 256, 0, s, n_rows, ell_width, ell_pitch, ell_cols, (const double *)ell_vals,
                coo_nnz, coo_rows, coo_cols, (const double *)coo_vals, (const double *)x, (double *)y, alpha, beta);
  return DCSR_OK;
}

extern "C" int dcsr_hyb_update(int32_t n_rows, int32_t n_cols, int32_t dtype, int32_t ell_width, int64_t ell_pitch,
                               int32_t *ell_cols, void *ell_vals, int32_t *coo_rows, int32_t *coo_cols,
                               void *coo_vals, int64_t coo_cap, int64_t *coo_nnz, const int32_t *rows,
                               const int32_t *cols, const void *vals, int64_t nnz, void *stream) {
  if (n_rows < 0 || n_cols < 0 || ell_width < 0 || ell_pitch < n_rows || (dtype != DCSR_F32 && dtype != DCSR_F64) ||
      !coo_nnz || *coo_nnz < 0 || *coo_nnz > coo_cap || nnz < 0 || (ell_width > 0 && (!ell_cols || !ell_vals)) ||
      (*coo_nnz > 0 && (!coo_rows || !coo_cols || !coo_vals)) || (nnz > 0 && (!rows || !cols || !vals)))
    return DCSR_BAD_ARG;
  if (nnz == 0) return DCSR_OK;
  if (n_rows == 0 || n_cols == 0) return DCSR_BAD_INDEX;  // no triple can be in range
  if (nnz > 0xffffffffLL) return DCSR_NOT_SUPPORTED;  // triple numbers are 32-bit
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == DCSR_F32)
    return hyb_update_t<float>(n_rows, n_cols, ell_width, ell_pitch, ell_cols, (float *)ell_vals, coo_rows, coo_cols,
                               (float *)coo_vals, coo_cap, coo_nnz, rows, cols, (const float *)vals, nnz, s);
  return hyb_update_t<double>(n_rows, n_cols, ell_width, ell_pitch, ell_cols, (double *)ell_vals, coo_rows, coo_cols,
                              (double *)coo_vals, coo_cap, coo_nnz, rows, cols, (const double *)vals, nnz, s);
}
