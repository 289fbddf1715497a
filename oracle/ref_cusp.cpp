// ref_cusp.cpp -- C-ABI harness around the reference's own cusp host path.
//
// TEST INFRASTRUCTURE ONLY (oracle pinning and the CPU baseline).  Compiled by
// oracle/Makefile against the reference tree (vendored cusp 0.5.1 / thrust
// 1.8.1 headers) into oracle/_ref/: once on the sequential host system
// (bit-reproducible left-to-right sums, used to pin the oracle) and
// once with the OpenMP device system (the multi-core CPU baseline).
//
// The functions call the reference's stock cusp operators unchanged:
//   cusp::multiply(csr, x, y)        cusp/system/detail/sequential/multiply/csr_spmv.h:41-73
//   cusp::add(coo, coo, coo)         cusp/system/detail/generic/elementwise.inl:75-231
//   cusp::multiply(csr, csr, csr)    cusp/system/detail/sequential/multiply/csr_spgemm.h:38-182
//   cusp::sort_by_row(r, c, v)       cusp/detail/sort.inl:38-67 (stable)
//   cusp::krylov::cg(A, x, b, mon)   cusp/krylov/detail/cg.inl (the reference's included solver)
// which are the CSR comparison / update operations the reference's drivers
// time (src/Fill_Test.inl:236-264, src/SPMM_Test.inl:142).
#include <cusp/coo_matrix.h>
#include <cusp/csr_matrix.h>
#include <cusp/elementwise.h>
#include <cusp/krylov/cg.h>
#include <cusp/monitor.h>
#include <cusp/multiply.h>
#include <cusp/sort.h>

#include <cstdint>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <cstring>
#include <vector>

// REF_SEQ: every operator runs on the sequential host system (cpp); else on
// the OpenMP device system.  Both builds define THRUST_DEVICE_SYSTEM_OMP.
#ifdef REF_SEQ
typedef cusp::host_memory DM;
#else
typedef cusp::device_memory DM;
#endif
typedef cusp::host_memory HM;

namespace {

struct Result {
  int64_t nnz = 0;
  int32_t n_rows = 0;
  std::vector<int32_t> rows, cols;  // rows: COO rows or CSR row_ptr
  std::vector<double> vals;
};

template <typename V>
cusp::csr_matrix<int, V, HM> host_csr(int32_t n, int32_t m, const int32_t *rp, const int32_t *ci,
                                       const double *vv) {
  int64_t nnz = rp[n];
  cusp::csr_matrix<int, V, HM> A(n, m, nnz);
  for (int32_t i = 0; i <= n; i++) A.row_offsets[i] = rp[i];
  for (int64_t j = 0; j < nnz; j++) {
    A.column_indices[j] = ci[j];
    A.values[j] = (V)vv[j];
  }
  return A;
}

template <typename V>
void spmv_impl(int32_t n, int32_t m, const int32_t *rp, const int32_t *ci, const double *vv,
               const double *x, double *y) {
  cusp::csr_matrix<int, V, DM> A = host_csr<V>(n, m, rp, ci, vv);
  cusp::array1d<V, HM> xh(m), yh(n, 0);
  for (int32_t i = 0; i < m; i++) xh[i] = (V)x[i];
  cusp::array1d<V, DM> xd = xh, yd = yh;
  cusp::multiply(A, xd, yd);
  yh = yd;
  for (int32_t i = 0; i < n; i++) y[i] = (double)yh[i];
}

template <typename V>
Result *add_impl(int32_t n, int32_t m, const int32_t *rp, const int32_t *ci, const double *vv,
                 const int32_t *br, const int32_t *bc, const double *bv, int64_t bn) {
  cusp::csr_matrix<int, V, HM> Ah = host_csr<V>(n, m, rp, ci, vv);
  cusp::coo_matrix<int, V, HM> Bh(n, m, bn);
  for (int64_t j = 0; j < bn; j++) {
    Bh.row_indices[j] = br[j];
    Bh.column_indices[j] = bc[j];
    Bh.values[j] = (V)bv[j];
  }
  cusp::coo_matrix<int, V, DM> A = Ah, B = Bh, C;
  cusp::add(A, B, C);
  cusp::coo_matrix<int, V, HM> Ch = C;
  Result *r = new Result;
  r->nnz = Ch.num_entries;
  r->n_rows = n;
  r->rows.assign(Ch.row_indices.begin(), Ch.row_indices.end());
  r->cols.assign(Ch.column_indices.begin(), Ch.column_indices.end());
  r->vals.resize(r->nnz);
  for (int64_t j = 0; j < r->nnz; j++) r->vals[j] = (double)Ch.values[j];
  return r;
}

template <typename V>
Result *spgemm_impl(int32_t n, int32_t k, int32_t m, const int32_t *arp, const int32_t *aci,
                    const double *av, const int32_t *brp, const int32_t *bci, const double *bv) {
  cusp::csr_matrix<int, V, DM> A = host_csr<V>(n, k, arp, aci, av);
  cusp::csr_matrix<int, V, DM> B = host_csr<V>(k, m, brp, bci, bv);
  cusp::csr_matrix<int, V, DM> C;
  cusp::multiply(A, B, C);
  cusp::csr_matrix<int, V, HM> Ch = C;
  Result *r = new Result;
  r->nnz = Ch.num_entries;
  r->n_rows = n;
  r->rows.assign(Ch.row_offsets.begin(), Ch.row_offsets.end());
  r->cols.assign(Ch.column_indices.begin(), Ch.column_indices.end());
  r->vals.resize(r->nnz);
  for (int64_t j = 0; j < r->nnz; j++) r->vals[j] = (double)Ch.values[j];
  return r;
}

template <typename V>
void sort_by_row_impl(int32_t *rows, int32_t *cols, double *vals, int64_t n) {
  cusp::array1d<int, HM> r(rows, rows + n), c(cols, cols + n);
  cusp::array1d<V, HM> v(n);
  for (int64_t j = 0; j < n; j++) v[j] = (V)vals[j];
  cusp::array1d<int, DM> rd = r, cd = c;
  cusp::array1d<V, DM> vd = v;
  cusp::sort_by_row(rd, cd, vd);
  r = rd;
  c = cd;
  v = vd;
  for (int64_t j = 0; j < n; j++) {
    rows[j] = r[j];
    cols[j] = c[j];
    vals[j] = (double)v[j];
  }
}

// A resident CSR matrix for the timed update-stream baseline: one step is
// the reference's CSR update (cusp::add, src/Fill_Test.inl:243-245) followed
// by SpMV, row-sum (SpMV with x = 1) and the CSR copy-out.
template <typename V>
struct Stream {
  cusp::csr_matrix<int, V, DM> A;
  cusp::array1d<V, DM> x, ones, y, rs;
};

// Unpreconditioned CG with cusp's monitor (stop when ||r|| <= abs + rel*||b||
// or after max_iter iterations); x holds the initial guess on entry.
template <typename V>
void cg_impl(int32_t n, const int32_t *rp, const int32_t *ci, const double *vv, const double *b, double *x,
             int32_t max_iter, double rel, double abs_tol, int32_t *iters, double *resid) {
  cusp::csr_matrix<int, V, DM> A = host_csr<V>(n, n, rp, ci, vv);
  cusp::array1d<V, HM> bh(n), xh(n);
  for (int32_t i = 0; i < n; i++) {
    bh[i] = (V)b[i];
    xh[i] = (V)x[i];
  }
  cusp::array1d<V, DM> bd = bh, xd = xh;
  cusp::monitor<V> mon(bd, (size_t)max_iter, (V)rel, (V)abs_tol);
  cusp::krylov::cg(A, xd, bd, mon);
  xh = xd;
  for (int32_t i = 0; i < n; i++) x[i] = (double)xh[i];
  *iters = (int32_t)mon.iteration_count();
  *resid = (double)mon.residual_norm();
}

}  // namespace

extern "C" {

void ref_cg(int32_t dtype, int32_t n, const int32_t *rp, const int32_t *ci, const double *vv, const double *b,
            double *x, int32_t max_iter, double rel, double abs_tol, int32_t *iters, double *resid) {
  if (dtype == 0) cg_impl<float>(n, rp, ci, vv, b, x, max_iter, rel, abs_tol, iters, resid);
  else cg_impl<double>(n, rp, ci, vv, b, x, max_iter, rel, abs_tol, iters, resid);
}

int ref_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void ref_spmv(int32_t dtype, int32_t n, int32_t m, const int32_t *rp, const int32_t *ci, const double *vv,
              const double *x, double *y) {
  if (dtype == 0) spmv_impl<float>(n, m, rp, ci, vv, x, y);
  else spmv_impl<double>(n, m, rp, ci, vv, x, y);
}

void *ref_add(int32_t dtype, int32_t n, int32_t m, const int32_t *rp, const int32_t *ci, const double *vv,
              const int32_t *br, const int32_t *bc, const double *bv, int64_t bn) {
  if (dtype == 0) return add_impl<float>(n, m, rp, ci, vv, br, bc, bv, bn);
  return add_impl<double>(n, m, rp, ci, vv, br, bc, bv, bn);
}

void *ref_spgemm(int32_t dtype, int32_t n, int32_t k, int32_t m, const int32_t *arp, const int32_t *aci,
                 const double *av, const int32_t *brp, const int32_t *bci, const double *bv) {
  if (dtype == 0) return spgemm_impl<float>(n, k, m, arp, aci, av, brp, bci, bv);
  return spgemm_impl<double>(n, k, m, arp, aci, av, brp, bci, bv);
}

void ref_sort_by_row(int32_t dtype, int32_t *rows, int32_t *cols, double *vals, int64_t n) {
  if (dtype == 0) sort_by_row_impl<float>(rows, cols, vals, n);
  else sort_by_row_impl<double>(rows, cols, vals, n);
}

int64_t ref_result_nnz(void *h) { return ((Result *)h)->nnz; }
int64_t ref_result_rows_len(void *h) { return (int64_t)((Result *)h)->rows.size(); }
void ref_result_get(void *h, int32_t *rows, int32_t *cols, double *vals) {
  Result *r = (Result *)h;
  if (rows) std::memcpy(rows, r->rows.data(), r->rows.size() * sizeof(int32_t));
  if (cols) std::memcpy(cols, r->cols.data(), r->cols.size() * sizeof(int32_t));
  if (vals) std::memcpy(vals, r->vals.data(), r->vals.size() * sizeof(double));
}
void ref_result_free(void *h) { delete (Result *)h; }

// Update-stream baseline (FP32, the update-stream workload's value type).
void *ref_stream_create(int32_t n, int32_t m, const int32_t *rp, const int32_t *ci, const double *vv,
                        const double *x) {
  Stream<float> *s = new Stream<float>;
  s->A = host_csr<float>(n, m, rp, ci, vv);
  cusp::array1d<float, HM> xh(m);
  for (int32_t i = 0; i < m; i++) xh[i] = (float)x[i];
  s->x = xh;
  s->ones = cusp::array1d<float, DM>(m, 1.0f);
  s->y = cusp::array1d<float, DM>(n, 0.0f);
  s->rs = cusp::array1d<float, DM>(n, 0.0f);
  return s;
}

// One round: merge the batch (cusp::add, duplicates summed, zeros dropped),
// then y = A x, row sums, and a CSR copy of the result.  Returns new nnz.
int64_t ref_stream_step(void *h, const int32_t *br, const int32_t *bc, const double *bv, int64_t bn,
                        double *y, double *rowsum) {
  Stream<float> *s = (Stream<float> *)h;
  int32_t n = (int32_t)s->A.num_rows, m = (int32_t)s->A.num_cols;
  cusp::coo_matrix<int, float, HM> Bh(n, m, bn);
  for (int64_t j = 0; j < bn; j++) {
    Bh.row_indices[j] = br[j];
    Bh.column_indices[j] = bc[j];
    Bh.values[j] = (float)bv[j];
  }
  cusp::coo_matrix<int, float, DM> B = Bh, Acoo = s->A, C;
  cusp::add(Acoo, B, C);
  s->A = C;
  cusp::multiply(s->A, s->x, s->y);
  cusp::multiply(s->A, s->ones, s->rs);
  cusp::csr_matrix<int, float, DM> exported = s->A;
  if (y) {
    cusp::array1d<float, HM> yh = s->y, rh = s->rs;
    for (int32_t i = 0; i < n; i++) {
      y[i] = yh[i];
      if (rowsum) rowsum[i] = rh[i];
    }
  }
  return (int64_t)exported.num_entries;
}

void ref_stream_free(void *h) { delete (Stream<float> *)h; }

// Resident FP32 CSR matrices for the served-workload baseline: each request
// is one stock cusp operation on one matrix -- an update is cusp::add of the
// batch (src/Fill_Test.inl:243-245), an SpMV is one cusp::multiply per
// right-hand side (cusp's CSR SpMV takes one vector), an export is a copy of
// the CSR arrays out of the matrix.
void *ref_res_create(int32_t n, int32_t m, const int32_t *rp, const int32_t *ci, const float *vv) {
  Stream<float> *s = new Stream<float>;
  int64_t nnz = rp[n];
  cusp::csr_matrix<int, float, HM> A(n, m, nnz);
  for (int32_t i = 0; i <= n; i++) A.row_offsets[i] = rp[i];
  for (int64_t j = 0; j < nnz; j++) {
    A.column_indices[j] = ci[j];
    A.values[j] = vv[j];
  }
  s->A = A;
  s->x = cusp::array1d<float, DM>(m, 0.0f);
  s->y = cusp::array1d<float, DM>(n, 0.0f);
  return s;
}

int64_t ref_res_update(void *h, const int32_t *br, const int32_t *bc, const float *bv, int64_t bn) {
  Stream<float> *s = (Stream<float> *)h;
  int32_t n = (int32_t)s->A.num_rows, m = (int32_t)s->A.num_cols;
  cusp::coo_matrix<int, float, HM> Bh(n, m, bn);
  for (int64_t j = 0; j < bn; j++) {
    Bh.row_indices[j] = br[j];
    Bh.column_indices[j] = bc[j];
    Bh.values[j] = bv[j];
  }
  cusp::coo_matrix<int, float, DM> B = Bh, Acoo = s->A, C;
  cusp::add(Acoo, B, C);
  s->A = C;
  return (int64_t)s->A.num_entries;
}

// y[:, j] = A x[:, j] for j < k; x is [m x k], y is [n x k] row-major.
void ref_res_spmv(void *h, const float *x, int32_t k, float *y) {
  Stream<float> *s = (Stream<float> *)h;
  int32_t n = (int32_t)s->A.num_rows, m = (int32_t)s->A.num_cols;
  cusp::array1d<float, HM> xh(m), yh(n);
  for (int32_t j = 0; j < k; j++) {
    for (int32_t i = 0; i < m; i++) xh[i] = x[(int64_t)i * k + j];
    s->x = xh;
    cusp::multiply(s->A, s->x, s->y);
    yh = s->y;
    for (int32_t i = 0; i < n; i++) y[(int64_t)i * k + j] = yh[i];
  }
}

int64_t ref_res_export(void *h, int32_t *rp, int32_t *ci, float *vv) {
  Stream<float> *s = (Stream<float> *)h;
  cusp::csr_matrix<int, float, HM> Ch = s->A;
  const int64_t nnz = (int64_t)Ch.num_entries;
  if (rp)
    for (size_t i = 0; i < Ch.row_offsets.size(); i++) rp[i] = Ch.row_offsets[i];
  if (ci)
    for (int64_t j = 0; j < nnz; j++) {
      ci[j] = Ch.column_indices[j];
      vv[j] = Ch.values[j];
    }
  return nnz;
}

void ref_res_free(void *h) { delete (Stream<float> *)h; }

}  // extern "C"
