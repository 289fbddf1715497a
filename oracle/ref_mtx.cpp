// ref_mtx.cpp -- TEST INFRASTRUCTURE: a C entry point around the reference's
// own Matrix Market reader, ReadMatrixFile (reference
// include/load_matrix.h:48-119), compiled from the reference tree where it
// lies (oracle/Makefile builds oracle/_ref/libref_mtx.so).  Used only by the
// tests that pin dcsr_b200/mmio.py's reference-value mode.
//
// load_matrix.h also declares the reference's GPU loaders and timing
// wrappers; they are templates over the reference's DCSR/HYB types, so the
// types and the `device` functions they call are only declared here (never
// instantiated).
#include <cuda_runtime_api.h>
#include <omp.h>

#include <cusp/array1d.h>
#include <cusp/coo_matrix.h>
#include <cusp/csr_matrix.h>
#include <cusp/gallery/poisson.h>
#include <cusp/hyb_matrix.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "include/sparse.h"

template <typename I, typename V, typename M, size_t B> class dcsr_matrix;
template <typename I, typename V, typename M, size_t B> class dcsr_matrix_B;
template <typename I, typename V, typename M> class hyb_matrix;
namespace device {
template <class... A> void LoadMatrix(A &&...);
template <class... A> void BinRows(A &&...);
}  // namespace device

#include "include/matrix_info.h"
#include "include/load_matrix.h"

// Reads `path` with ReadMatrixFile<int, double> (1-based indices); copies at
// most `cap` entries (file order) into r, c, v.  Returns the entry count, or
// 0 when the file cannot be opened.
extern "C" int ref_read_mtx(const char *path, int *n_rows, int *n_cols, long cap, int *r, int *c, double *v) {
  std::vector<std::vector<std::pair<int, double> > > mat;
  CuspVectorInt_h rv, cv;
  cusp::array1d<double, cusp::host_memory> vv;
  int nr = 0, nc = 0;
  const int nnz = ReadMatrixFile<int, double>(std::string(path), mat, rv, cv, vv, nr, nc);
  *n_rows = nr;
  *n_cols = nc;
  for (long i = 0; i < nnz && i < cap; i++) {
    r[i] = rv[i];
    c[i] = cv[i];
    v[i] = vv[i];
  }
  return nnz;
}
