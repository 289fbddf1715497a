// spmv.cu -- DCSR SpMV with 1..8 right-hand sides and row reductions.
//
// One persistent launch covers every row: rows are grouped by length class
// (handle-local bins, see matrix.cu) into work units, a unit being 256/W rows
// for a W-lane sub-warp class (W = 1..32) or one row for the >= 512 class
// (whole CTA).  Units of the long-row class come first so they do not form a
// tail.  Each row follows its segment chain with its current logical length
// (the reference read stale Prow_sizes, include/spmv.inl:390,467,555).
// Products accumulate in FP64 for both value types (one rounding at the end).
//
// Reference: device::spmv(dcsr,...) include/spmv.h:121-248 with the seven
// binned kernels spmv_dcsr_bin_scalar / spmv_dcsr_bin<2..32> /
// spmv_dcsr_bin_large include/spmv.inl:364-622, launched there as seven
// kernels on seven streams with a process-global __constant__ bin table.
#include <algorithm>

#include "internal.cuh"

namespace dcsr {

enum { OP_SPMV = 0, OP_SUM = 1, OP_MAX = 2, OP_MIN = 3, OP_COUNT = 4 };
constexpr int SPMV_THREADS = 256;

template <typename V, int K, bool VEC>
__device__ __forceinline__ void load_x(const V *__restrict__ x, int64_t c, int64_t ldx, double (&xv)[K]) {
  if constexpr (VEC && sizeof(V) == 4 && K == 4) {
    float4 t = __ldg(reinterpret_cast<const float4 *>(x + c * K));
    xv[0] = t.x; xv[1] = t.y; xv[2] = t.z; xv[3] = t.w;
  } else if constexpr (VEC && sizeof(V) == 4 && K == 8) {
    float4 t = __ldg(reinterpret_cast<const float4 *>(x + c * K));
    float4 u = __ldg(reinterpret_cast<const float4 *>(x + c * K) + 1);
    xv[0] = t.x; xv[1] = t.y; xv[2] = t.z; xv[3] = t.w;
    xv[4] = u.x; xv[5] = u.y; xv[6] = u.z; xv[7] = u.w;
  } else if constexpr (VEC && sizeof(V) == 4 && K == 2) {
    float2 t = __ldg(reinterpret_cast<const float2 *>(x + c * K));
    xv[0] = t.x; xv[1] = t.y;
  } else if constexpr (VEC && sizeof(V) == 8 && K >= 2) {
#pragma unroll
    for (int k = 0; k < K; k += 2) {
      double2 t = __ldg(reinterpret_cast<const double2 *>(x + c * K + k));
      xv[k] = t.x; xv[k + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; k++) xv[k] = (double)__ldg(x + c * ldx + k);
  }
}

template <int OP>
__device__ __forceinline__ double acc_init() {
  if (OP == OP_MAX) return -INFINITY;
  if (OP == OP_MIN) return INFINITY;
  return 0.0;
}
template <int OP>
__device__ __forceinline__ double acc_comb(double a, double b) {
  if (OP == OP_MAX) return a > b ? a : b;
  if (OP == OP_MIN) return a < b ? a : b;
  return a + b;
}

// Accumulate one row's entries handled by lane `sub` of a group of W lanes.
template <typename V, int K, int OP, bool VEC>
__device__ __forceinline__ void row_accumulate(const Mat<V> &m, int32_t row, int sub, int W, const V *x, int64_t ldx,
                                               double (&acc)[K]) {
  const int64_t L = m.row_sizes[row];
  if (OP == OP_COUNT) {
    if (sub == 0) acc[0] = (double)L;
    return;
  }
  int64_t p = 0;
#pragma unroll 1
  for (int l = 0; l < m.max_segs && p < L; l++) {
    const int2 sg = __ldg(reinterpret_cast<const int2 *>(m.seg + (int64_t)l * m.pitch + 2 * (int64_t)row));
    const int64_t take = (int64_t)(sg.y - sg.x) < L - p ? (int64_t)(sg.y - sg.x) : L - p;
    const int32_t *__restrict__ cc = m.cols + sg.x;
    const V *__restrict__ vv = m.vals + sg.x;
#pragma unroll 4
    for (int64_t j = sub; j < take; j += W) {
      const double a = (double)__ldcs(vv + j);
      if (OP == OP_SPMV) {
        const int32_t c = __ldcs(cc + j);
        double xv[K];
        load_x<V, K, VEC>(x, c, ldx, xv);
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = fma(a, xv[k], acc[k]);
      } else {
        acc[0] = acc_comb<OP>(acc[0], a);
      }
    }
    p += take;
  }
}

template <typename V, int K, int OP>
__device__ __forceinline__ void write_row(V *y, int64_t ldy, int32_t row, const double (&acc)[K], double alpha,
                                          double beta, bool empty) {
#pragma unroll
  for (int k = 0; k < K; k++) {
    double v = acc[k];
    if ((OP == OP_MAX || OP == OP_MIN) && empty) v = 0.0;
    if (OP == OP_SPMV) {
      v *= alpha;
      if (beta != 0.0) v += beta * (double)y[(int64_t)row * ldy + k];
    }
    y[(int64_t)row * ldy + k] = (V)v;
  }
}

template <typename V, int K, int OP, bool VEC>
__global__ void __launch_bounds__(SPMV_THREADS) k_spmv(Mat<V> m, const int32_t *__restrict__ perm,
                                                       const int32_t *__restrict__ info, const V *__restrict__ x,
                                                       int64_t ldx, V *__restrict__ y, int64_t ldy, double alpha,
                                                       double beta) {
  __shared__ int32_t si[16];
  __shared__ double red[SPMV_THREADS / 32][K];
  if (threadIdx.x < 16) si[threadIdx.x] = info[threadIdx.x];
  __syncthreads();
  const int units = si[15];
  for (int u = blockIdx.x; u < units; u += gridDim.x) {
    int s = 0;
    while (s < 6 && si[8 + s + 1] <= u) s++;
    const int cls = 6 - s;
    const int local = u - si[8 + s];
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = acc_init<OP>();
    if (cls == 6) {
      const int32_t row = perm[si[6] + local];
      row_accumulate<V, K, OP, VEC>(m, row, threadIdx.x, SPMV_THREADS, x, ldx, acc);
#pragma unroll
      for (int k = 0; k < K; k++) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = acc_comb<OP>(v, __shfl_xor_sync(FULL, v, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = v;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double out[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
          out[k] = red[0][k];
          for (int w = 1; w < SPMV_THREADS / 32; w++) out[k] = acc_comb<OP>(out[k], red[w][k]);
        }
        if (OP == OP_COUNT) out[0] = (double)m.row_sizes[row];
        write_row<V, K, OP>(y, ldy, row, out, alpha, beta, m.row_sizes[row] == 0);
      }
      __syncthreads();
    } else {
      const int W = 1 << cls;
      const int sub = threadIdx.x & (W - 1);
      const int idx = local * (SPMV_THREADS >> cls) + (threadIdx.x >> cls);
      const int cnt = si[cls + 1] - si[cls];
      int32_t row = -1;
      if (idx < cnt) {
        row = perm[si[cls] + idx];
        row_accumulate<V, K, OP, VEC>(m, row, sub, W, x, ldx, acc);
      }
#pragma unroll
      for (int k = 0; k < K; k++)
        for (int o = W >> 1; o > 0; o >>= 1) acc[k] = acc_comb<OP>(acc[k], __shfl_xor_sync(FULL, acc[k], o, W));
      if (row >= 0 && sub == 0) write_row<V, K, OP>(y, ldy, row, acc, alpha, beta, m.row_sizes[row] == 0);
    }
  }
}

template <typename V, int K, int OP, bool VEC>
static int launch_spmv(dcsr_handle h, const V *x, int64_t ldx, V *y, int64_t ldy, double alpha, double beta,
                       cudaStream_t s) {
  static int grid = 0;
  if (!grid) grid = persistent_grid((const void *)k_spmv<V, K, OP, VEC>, SPMV_THREADS, 0);
  DCSR_LAUNCH((k_spmv<V, K, OP, VEC>), grid, SPMV_THREADS, 0, s, h->view<V>(), h->bin_perm, h->bin_info, x, ldx, y,
              ldy, alpha, beta);
  return DCSR_OK;
}

template <typename V, int K>
static int spmv_k(dcsr_handle h, const V *x, int64_t ldx, V *y, int64_t ldy, double alpha, double beta,
                  cudaStream_t s) {
  const bool vec = K > 1 && ldx == K && ((uintptr_t)x % (K * sizeof(V) >= 16 ? 16 : K * sizeof(V))) == 0;
  if (vec) return launch_spmv<V, K, OP_SPMV, true>(h, x, ldx, y, ldy, alpha, beta, s);
  return launch_spmv<V, K, OP_SPMV, false>(h, x, ldx, y, ldy, alpha, beta, s);
}

template <typename V>
static int spmv_dispatch(dcsr_handle h, const V *x, int32_t k, int64_t ldx, V *y, int64_t ldy, double alpha,
                         double beta, cudaStream_t s) {
  switch (k) {
    case 1: return spmv_k<V, 1>(h, x, ldx, y, ldy, alpha, beta, s);
    case 2: return spmv_k<V, 2>(h, x, ldx, y, ldy, alpha, beta, s);
    case 3: return launch_spmv<V, 3, OP_SPMV, false>(h, x, ldx, y, ldy, alpha, beta, s);
    case 4: return spmv_k<V, 4>(h, x, ldx, y, ldy, alpha, beta, s);
    case 5: return launch_spmv<V, 5, OP_SPMV, false>(h, x, ldx, y, ldy, alpha, beta, s);
    case 6: return launch_spmv<V, 6, OP_SPMV, false>(h, x, ldx, y, ldy, alpha, beta, s);
    case 7: return launch_spmv<V, 7, OP_SPMV, false>(h, x, ldx, y, ldy, alpha, beta, s);
    case 8: return spmv_k<V, 8>(h, x, ldx, y, ldy, alpha, beta, s);
  }
  return DCSR_BAD_ARG;
}

template <typename V>
static int reduce_dispatch(dcsr_handle h, int32_t op, V *y, cudaStream_t s) {
  switch (op) {
    case DCSR_REDUCE_SUM: return launch_spmv<V, 1, OP_SUM, false>(h, nullptr, 0, y, 1, 1.0, 0.0, s);
    case DCSR_REDUCE_MAX: return launch_spmv<V, 1, OP_MAX, false>(h, nullptr, 0, y, 1, 1.0, 0.0, s);
    case DCSR_REDUCE_MIN: return launch_spmv<V, 1, OP_MIN, false>(h, nullptr, 0, y, 1, 1.0, 0.0, s);
    case DCSR_REDUCE_COUNT: return launch_spmv<V, 1, OP_COUNT, false>(h, nullptr, 0, y, 1, 1.0, 0.0, s);
  }
  return DCSR_BAD_ARG;
}

}  // namespace dcsr

using namespace dcsr;

extern "C" int dcsr_spmv(dcsr_handle h, const void *x, int32_t k, int64_t ldx, void *y, int64_t ldy, double alpha,
                         double beta, void *stream) {
  if (!h || k < 1 || k > 8 || ldx < k || ldy < k || (h->n_rows > 0 && !y) || (h->n_cols > 0 && !x))
    return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (h->n_rows == 0) return DCSR_OK;
  if (!h->bins_valid) DCSR_TRY(bin_rows(h, s));
  if (h->dtype == DCSR_F32)
    return spmv_dispatch<float>(h, (const float *)x, k, ldx, (float *)y, ldy, alpha, beta, s);
  return spmv_dispatch<double>(h, (const double *)x, k, ldx, (double *)y, ldy, alpha, beta, s);
}

extern "C" int dcsr_row_reduce(dcsr_handle h, int32_t op, void *y, void *stream) {
  if (!h || (h->n_rows > 0 && !y) || op < 0 || op > 3) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (h->n_rows == 0) return DCSR_OK;
  if (!h->bins_valid) DCSR_TRY(bin_rows(h, s));
  if (h->dtype == DCSR_F32) return reduce_dispatch<float>(h, op, (float *)y, s);
  return reduce_dispatch<double>(h, op, (double *)y, s);
}
