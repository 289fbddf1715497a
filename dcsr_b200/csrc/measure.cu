// measure.cu -- a measurement aid for the SpMV roofline: the memory access
// pattern of a k = 1 SpMV without its row bookkeeping.  For n entries given
// as plain arrays (a matrix's CSR export), every entry's column and value are
// read (coalesced, 8 entries in flight per thread) and x is gathered at the
// column; products are summed per block into out[block].  Its time is what
// the SpMV's data movement costs at best on this matrix: the same bytes
// from HBM and the same random 4-byte reads of x, but no row boundaries.
#include <algorithm>

#include "internal.cuh"

namespace dcsr {
namespace {

template <int U>
__global__ void __launch_bounds__(256) k_gather_floor(const int32_t *__restrict__ cols, const float *__restrict__ vals,
                                                      int64_t n, const float *__restrict__ x, float *out) {
  float s = 0.f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x * U;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x * U + threadIdx.x; b < n; b += stride) {
    int32_t c[U];
    float a[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int64_t i = b + (int64_t)u * blockDim.x;
      c[u] = i < n ? __ldcs(cols + i) : 0;
      a[u] = i < n ? __ldcs(vals + i) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < U; u++) s = fmaf(a[u], __ldg(x + c[u]), s);
  }
  s = warp_sum(s);
  __shared__ float ws[8];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < 8; w++) t += ws[w];
    out[blockIdx.x] = t;
  }
}

}  // namespace
}  // namespace dcsr

using namespace dcsr;

extern "C" int dcsr_measure_gather(const int32_t *cols, const float *vals, int64_t n, const float *x, float *out,
                                   int32_t out_len, void *stream) {
  if (n < 0 || (n > 0 && (!cols || !vals || !x)) || !out || out_len < 1) return DCSR_BAD_ARG;
  const int g = (int)std::min<int64_t>(out_len, (int64_t)sm_count() * 8);
  DCSR_LAUNCH(k_gather_floor<8>, g, 256, 0, (cudaStream_t)stream, cols, vals, n, x, out);
  return DCSR_OK;
}
