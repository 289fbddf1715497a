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
