// fill_test.cpp -- C++ driver through the reference-style `device::` API
// (include/dcsr_b200.hpp), shaped like the reference's Fill_Test
// (src/Fill_Test.inl): load a matrix, bin + compact, repeated SpMV, then an
// update loop with periodic compaction and SpMV, and a CSR export.  It checks
// the results against a host computation and prints "FILL_TEST OK".
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <random>
#include <vector>

#include "dcsr_b200.hpp"

#define CK(x)                                                                   \
  do {                                                                          \
    cudaError_t e = (x);                                                        \
    if (e != cudaSuccess) {                                                     \
      fprintf(stderr, "CUDA %s at %d\n", cudaGetErrorString(e), __LINE__);     \
      return 2;                                                                 \
    }                                                                           \
  } while (0)

template <typename T>
static T *to_dev(const std::vector<T> &h) {
  T *d = nullptr;
  cudaMalloc((void **)&d, sizeof(T) * std::max<size_t>(h.size(), 1));
  cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  return d;
}

int main() {
  const int n = 20000, m = 20000;
  std::mt19937 gen(42);
  std::uniform_int_distribution<int> col(0, m - 1), row(0, n - 1);
  std::uniform_real_distribution<float> val(-1.f, 1.f);
  std::map<std::pair<int, int>, double> host;  // reference content (merge semantics)
  std::vector<int> r, c;
  std::vector<float> v;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < 8; j++) {
      int cc = col(gen);
      float vv = val(gen);
      r.push_back(i);
      c.push_back(cc);
      v.push_back(vv);
      auto key = std::make_pair(i, cc);
      auto it = host.find(key);
      if (it == host.end()) host[key] = vv;
      else it->second = (double)(float)((float)it->second + vv);
    }
  try {
    dcsr::dcsr_matrix<float> A(n, m, DCSR_MERGE);
    device::Initialize_Matrix(A);
    int *dr = to_dev(r), *dc = to_dev(c);
    float *dv = to_dev(v);
    device::LoadMatrix(A, dr, dc, dv, (int64_t)r.size());
    device::BinRows(A);
    device::SortMatrixRow(A);
    std::vector<float> x(m);
    for (auto &e : x) e = val(gen);
    float *dx = to_dev(x), *dy = nullptr;
    CK(cudaMalloc((void **)&dy, sizeof(float) * n));
    for (int it = 0; it < 10; it++) device::spmv(A, dx, dy);
    // update loop: 20 slices, compaction every 5 (src/Fill_Test.inl:296-325)
    for (int s = 0; s < 20; s++) {
      std::vector<int> ur, uc;
      std::vector<float> uv;
      for (int t = 0; t < 2000; t++) {
        int rr = row(gen), cc = col(gen);
        float vv = val(gen);
        ur.push_back(rr);
        uc.push_back(cc);
        uv.push_back(vv);
        auto key = std::make_pair(rr, cc);
        auto it = host.find(key);
        if (it == host.end()) host[key] = vv;
        else it->second = (double)(float)((float)it->second + vv);
      }
      int *a = to_dev(ur), *b = to_dev(uc);
      float *w = to_dev(uv);
      int st = device::UpdateMatrix(A, a, b, w, (int64_t)ur.size());
      if (st != DCSR_OK) {
        fprintf(stderr, "update status %d\n", st);
        return 1;
      }
      if (s > 0 && s % 5 == 0) device::SortMatrixRow(A);
      device::spmv(A, dx, dy);
      cudaFree(a);
      cudaFree(b);
      cudaFree(w);
    }
    CK(cudaDeviceSynchronize());
    // export and compare with the host map (sorted by (row, col))
    const int64_t nnz = A.num_entries();
    if (nnz != (int64_t)host.size()) {
      fprintf(stderr, "nnz %lld != %zu\n", (long long)nnz, host.size());
      return 1;
    }
    int *rp_d, *c_d;
    float *v_d;
    CK(cudaMalloc((void **)&rp_d, sizeof(int) * (n + 1)));
    CK(cudaMalloc((void **)&c_d, sizeof(int) * nnz));
    CK(cudaMalloc((void **)&v_d, sizeof(float) * nnz));
    device::ExportCSR(A, rp_d, c_d, v_d);
    std::vector<int> rp(n + 1), cc(nnz);
    std::vector<float> vv(nnz);
    CK(cudaMemcpy(rp.data(), rp_d, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cc.data(), c_d, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(vv.data(), v_d, sizeof(float) * nnz, cudaMemcpyDeviceToHost));
    int64_t p = 0;
    for (int i = 0; i < n; i++)
      for (int j = rp[i]; j < rp[i + 1]; j++, p++) {
        auto it = host.find(std::make_pair(i, cc[j]));
        if (it == host.end() || (float)it->second != vv[j]) {
          fprintf(stderr, "mismatch at row %d col %d\n", i, cc[j]);
          return 1;
        }
      }
    // SpMV against the host map in double
    std::vector<double> yref(n, 0.0), bound(n, 0.0);
    for (auto &kv : host) {
      yref[kv.first.first] += kv.second * x[kv.first.second];
      bound[kv.first.first] += std::fabs(kv.second * x[kv.first.second]);
    }
    std::vector<float> y(n);
    device::spmv(A, dx, dy);
    CK(cudaMemcpy(y.data(), dy, sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++)
      if (std::fabs(y[i] - yref[i]) > 1e-6 * bound[i] + 1e-30) {
        fprintf(stderr, "spmv mismatch row %d\n", i);
        return 1;
      }
    cudaFree(dr);
    cudaFree(dc);
    cudaFree(dv);
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(rp_d);
    cudaFree(c_d);
    cudaFree(v_d);
  } catch (const dcsr::error &e) {
    fprintf(stderr, "dcsr error: %s\n", e.what());
    return 1;
  }
  printf("FILL_TEST OK\n");
  return 0;
}
