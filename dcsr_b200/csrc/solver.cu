// solver.cu -- conjugate gradient over the DCSR SpMV: the solver consumer of
// the reference tree.  The reference ships cusp's CG (cusp/krylov/cg.h,
// cusp/krylov/detail/cg.inl) with cusp's monitor as its stop rule
// (cusp/detail/monitor.inl: finished() when ||r||_2 <= abs_tol +
// rel_tol*||b||_2 or after iteration_limit iterations, tested before every
// iteration).  This is the same unpreconditioned iteration with every step
// on the device: y = A p (the library's SpMV), alpha = rz / <y, p>,
// x += alpha p, r -= alpha y, rz' = <r, r>, beta = rz' / rz, p = r + beta p.
// The scalars live in device memory; the host enqueues iterations in chunks
// and reads the stop flag between chunks, so a solve synchronises about
// log2(iterations) + iterations/16 times.  Dot products are block partials
// summed in block order by the last block to finish (a fixed grid per
// length), so a solve is deterministic.
#include <cmath>

#include "internal.cuh"

namespace dcsr {

namespace {

constexpr int CG_THREADS = 256;
constexpr int CG_MAX_BLOCKS = 512;

struct CgState {
  double rz;     // <r, r> of the current residual
  double alpha, beta;
  double rnorm;  // ||r||_2
  double tol;    // abs_tol + rel_tol * ||b||_2
  int32_t done;  // the stop rule held before the next iteration
  int32_t iters;
  int32_t max_iter;
  unsigned cnt;  // finished blocks of the current reduction
  double part[2][CG_MAX_BLOCKS];
};

// Block sum in a fixed order (warp xor trees, then warp sums in order).
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[CG_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < CG_THREADS / 32; w++) t += ws[w];
  __syncthreads();
  return t;  // valid in thread 0
}

// Publish this block's partials; true (in thread 0) for the last block, which
// then holds every block's partial in st->part.
__device__ __forceinline__ bool publish(CgState *st, double a, double b) {
  __shared__ int last;
  if (threadIdx.x == 0) {
    st->part[0][blockIdx.x] = a;
    st->part[1][blockIdx.x] = b;
    __threadfence();
    last = atomicAdd(&st->cnt, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  return last;
}

__device__ __forceinline__ double sum_parts(const CgState *st, int which) {
  double t = 0.0;
  for (unsigned b = 0; b < gridDim.x; b++) t += __ldcg(&st->part[which][b]);
  return t;
}

// r = b - y, p = r; rz = <r, r>, tol from ||b||.
template <typename V>
__global__ void __launch_bounds__(CG_THREADS) k_cg_init(const V *b, const V *y, V *r, V *p, int64_t n, CgState *st,
                                                        double rel, double abs_tol, int32_t max_iter) {
  double rr = 0.0, bb = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * CG_THREADS) {
    const V ri = b[i] - y[i];
    r[i] = ri;
    p[i] = ri;
    rr = __fma_rn((double)ri, (double)ri, rr);
    bb = __fma_rn((double)b[i], (double)b[i], bb);
  }
  rr = block_sum(rr);
  bb = block_sum(bb);
  if (publish(st, rr, bb) && threadIdx.x == 0) {
    __threadfence();
    st->rz = sum_parts(st, 0);
    st->rnorm = sqrt(st->rz);
    st->tol = abs_tol + rel * sqrt(sum_parts(st, 1));
    st->iters = 0;
    st->max_iter = max_iter;
    st->done = (st->rnorm <= st->tol || max_iter <= 0) ? 1 : 0;
    st->cnt = 0;
  }
}

// alpha = rz / <y, p>
template <typename V>
__global__ void __launch_bounds__(CG_THREADS) k_cg_alpha(const V *y, const V *p, int64_t n, CgState *st) {
  if (st->done) return;
  double yp = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * CG_THREADS)
    yp = __fma_rn((double)y[i], (double)p[i], yp);
  yp = block_sum(yp);
  if (publish(st, yp, 0.0) && threadIdx.x == 0) {
    __threadfence();
    st->alpha = st->rz / sum_parts(st, 0);
    st->cnt = 0;
  }
}

// x += alpha p, r -= alpha y; rz' = <r, r>, beta, the stop rule.
template <typename V>
__global__ void __launch_bounds__(CG_THREADS) k_cg_step(V *x, V *r, const V *p, const V *y, int64_t n, CgState *st) {
  if (st->done) return;
  const V alpha = (V)st->alpha;
  double rr = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * CG_THREADS) {
    x[i] = x[i] + alpha * p[i];
    const V ri = r[i] - alpha * y[i];
    r[i] = ri;
    rr = __fma_rn((double)ri, (double)ri, rr);
  }
  rr = block_sum(rr);
  if (publish(st, rr, 0.0) && threadIdx.x == 0) {
    __threadfence();
    const double rz = sum_parts(st, 0);
    st->beta = rz / st->rz;
    st->rz = rz;
    st->rnorm = sqrt(rz);
    st->iters += 1;
    st->done = (st->rnorm <= st->tol || st->iters >= st->max_iter) ? 1 : 0;
    st->cnt = 0;
  }
}

// p = r + beta p (after the last iteration p is not used again).
template <typename V>
__global__ void __launch_bounds__(CG_THREADS) k_cg_dir(V *p, const V *r, int64_t n, const CgState *st) {
  if (st->done) return;
  const V beta = (V)st->beta;
  for (int64_t i = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * CG_THREADS)
    p[i] = r[i] + beta * p[i];
}

template <typename V>
int cg_t(dcsr_handle h, const V *b, V *x, int32_t max_iter, double rel, double abs_tol, int32_t *iters,
         double *resid, cudaStream_t s) {
  const int64_t n = h->n_rows;
  const int grid = (int)std::min<int64_t>(std::max<int64_t>(div_up(n, CG_THREADS * 8), 1), CG_MAX_BLOCKS);
  V *work = nullptr;
  CgState *st = nullptr;
  DCSR_CUDA(dcsr::dev_alloc((void **)&work, sizeof(V) * 3 * (size_t)(n > 0 ? n : 1), s));
  DCSR_CUDA(dcsr::dev_alloc((void **)&st, sizeof(CgState), s));
  V *r = work, *p = work + n, *y = work + 2 * n;
  int rc = DCSR_OK;
  auto run = [&]() -> int {
    DCSR_CUDA(cudaMemsetAsync(st, 0, sizeof(CgState), s));
    DCSR_TRY(spmv_call(h, x, 1, 1, y, 1, 1.0, 0.0, s));  // y = A x0 (builds the schedule if needed)
    DCSR_LAUNCH(k_cg_init<V>, grid, CG_THREADS, 0, s, b, y, r, p, n, st, rel, abs_tol, max_iter);
    int32_t host[2] = {0, 0};  // done, iters
    int chunk = 1;
    for (int guard = 0; guard < max_iter + 2; guard += chunk) {
      DCSR_CUDA(cudaMemcpyAsync(host, &st->done, sizeof(host), cudaMemcpyDeviceToHost, s));
      DCSR_CUDA(cudaStreamSynchronize(s));
      if (host[0]) break;
      for (int j = 0; j < chunk; j++) {
        DCSR_TRY(spmv_call(h, p, 1, 1, y, 1, 1.0, 0.0, s));
        DCSR_LAUNCH(k_cg_alpha<V>, grid, CG_THREADS, 0, s, y, p, n, st);
        DCSR_LAUNCH(k_cg_step<V>, grid, CG_THREADS, 0, s, x, r, p, y, n, st);
        DCSR_LAUNCH(k_cg_dir<V>, grid, CG_THREADS, 0, s, p, r, n, st);
      }
      chunk = chunk < 16 ? chunk * 2 : 16;
    }
    double rn = 0.0;
    DCSR_CUDA(cudaMemcpyAsync(host, &st->done, sizeof(host), cudaMemcpyDeviceToHost, s));
    DCSR_CUDA(cudaMemcpyAsync(&rn, &st->rnorm, sizeof(rn), cudaMemcpyDeviceToHost, s));
    DCSR_CUDA(cudaStreamSynchronize(s));
    if (iters) *iters = host[1];
    if (resid) *resid = rn;
    return DCSR_OK;
  };
  rc = run();
  dcsr::dev_free(work, s);
  dcsr::dev_free(st, s);
  return rc;
}

}  // namespace
}  // namespace dcsr

using namespace dcsr;

extern "C" int dcsr_cg(dcsr_handle A, const void *b, void *x, int32_t max_iter, double rel_tol, double abs_tol,
                       int32_t *iters, double *resid, void *stream) {
  if (!A || A->n_rows != A->n_cols || (A->n_rows > 0 && (!b || !x)) || max_iter < 0 || rel_tol < 0 || abs_tol < 0)
    return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (A->dtype == DCSR_F32)
    return cg_t<float>(A, (const float *)b, (float *)x, max_iter, rel_tol, abs_tol, iters, resid, s);
  return cg_t<double>(A, (const double *)b, (double *)x, max_iter, rel_tol, abs_tol, iters, resid, s);
}
