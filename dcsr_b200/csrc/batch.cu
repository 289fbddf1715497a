// batch.cu -- the batched form: many matrices, each with an update batch and
// an SpMV, run as one merged update (one key sort, one plan, one apply over
// the union of their triples), one schedule rebuild over all their rows and
// one SpMV pass per distinct RHS count -- about thirty kernels for the whole
// set, whatever its size, optionally replayed as one CUDA graph.
//
// Kernels read the matrices through device-resident descriptor arrays
// (BatchItem / RowItem).  A captured graph therefore stays valid when a
// matrix's buffers move (repair, per-call compaction or growth): before every
// run the host rebuilds the descriptors from the handles and re-uploads them,
// to the same device addresses, only when they changed.
//
// The reference has no batched form: it runs one UpdateMatrix
// (include/load.h:258-325) and one spmv (include/spmv.h:121-248) per matrix.
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.cuh"

namespace dcsr {

template <typename V>
__global__ void k_batch_gate(const BatchItem<V> *its, int count, int32_t *skip) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    skip[i] = its[i].m.stat[ST_GO] == 0;
}

template <typename V>
__global__ void k_batch_status(const BatchItem<V> *its, int count, int32_t *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    long long *st = its[i].m.stat;
    out[i] = (int32_t)st[ST_STATUS];
    st[ST_STATUS] = 0;
  }
}

}  // namespace dcsr

using namespace dcsr;

struct dcsr_batch_s {
  int count = 0, dtype = 0, mode = 0, device = 0;
  std::vector<dcsr_batch_item> items;
  int64_t T = 0, R = 0;
  int rb = 1, cb = 1;
  struct Group {
    int k = 1;
    bool vec = false;
    std::vector<int> idx;  // matrices of this group, in item order
    size_t off = 0;        // descriptor offset in the image
    long long *pref = nullptr;
  };
  std::vector<Group> groups;
  // one device image: BatchItem[count] | RowItem[count] (row space) | groups
  size_t off_row = 0, img_bytes = 0;
  unsigned char *img_dev = nullptr;
  unsigned char *img_host = nullptr;  // pinned: last uploaded image
  std::vector<unsigned char> img_new;
  int32_t *skip = nullptr;
  int32_t *status_dev = nullptr;
  long long *gstat = nullptr;
  Arena ar;
  size_t ar_need = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_kernels = 0;  // kernel nodes of the captured graph
};

namespace {

size_t desc_size(int dtype, bool row) {
  if (dtype == DCSR_F32) return row ? sizeof(RowItem<float>) : sizeof(BatchItem<float>);
  return row ? sizeof(RowItem<double>) : sizeof(BatchItem<double>);
}

template <typename V>
void fill_image(dcsr_batch b, unsigned char *img) {
  BatchItem<V> *up = (BatchItem<V> *)img;
  RowItem<V> *rows = (RowItem<V> *)(img + b->off_row);
  long long toff = 0, row0 = 0;
  for (int i = 0; i < b->count; i++) {
    const dcsr_batch_item &it = b->items[i];
    dcsr_handle h = it.matrix;
    BatchItem<V> u;
    std::memset(&u, 0, sizeof(u));
    u.m = h->view<V>();
    u.rows = it.rows;
    u.cols = it.cols;
    u.vals = (const V *)it.vals;
    u.toff = toff;
    u.T = it.nnz;
    up[i] = u;
    toff += it.nnz;
    RowItem<V> r = row_item<V>(h, nullptr, nullptr, 0, 0, 0.0, 0.0);
    r.row0 = row0;
    row0 += h->n_rows;
    rows[i] = r;
  }
  for (auto &g : b->groups) {
    RowItem<V> *gi = (RowItem<V> *)(img + g.off);
    for (size_t j = 0; j < g.idx.size(); j++) {
      const int i = g.idx[j];
      const dcsr_batch_item &it = b->items[i];
      RowItem<V> r = row_item<V>(it.matrix, it.x, it.y, it.ldx, it.ldy, it.alpha, it.beta);
      r.skip = b->skip + i;
      gi[j] = r;
    }
  }
}

// Rebuild the descriptor image from the handles; upload it when it changed
// (and make sure every handle's schedule buffers fit its pool first).
int refresh(dcsr_batch b, cudaStream_t s) {
  for (auto &g : b->groups)
    for (int i : g.idx) DCSR_TRY(ensure_part(b->items[i].matrix, g.k, s));
  for (int i = 0; i < b->count; i++) DCSR_TRY(ensure_part(b->items[i].matrix, 1, s));
  b->img_new.assign(b->img_bytes, 0);
  if (b->dtype == DCSR_F32) fill_image<float>(b, b->img_new.data());
  else fill_image<double>(b, b->img_new.data());
  if (std::memcmp(b->img_new.data(), b->img_host, b->img_bytes) != 0) {
    // the previous upload (if any) has completed: every upload is followed by a sync
    std::memcpy(b->img_host, b->img_new.data(), b->img_bytes);
    DCSR_CUDA(cudaMemcpyAsync(b->img_dev, b->img_host, b->img_bytes, cudaMemcpyHostToDevice, s));
    DCSR_CUDA(cudaStreamSynchronize(s));
  }
  return DCSR_OK;
}

// The batch's device work (capturable: no allocation, no host sync).
int enqueue(dcsr_batch b, cudaStream_t s) {
  const bool merge = b->mode == DCSR_MERGE;
  if (b->T > 0) {
    DCSR_TRY(update_many(b->img_dev, b->dtype, b->count, b->T, merge, b->rb, b->cb, b->gstat, b->ar, s));
    const int g = (b->count + 255) / 256;
    if (b->dtype == DCSR_F32)
      DCSR_LAUNCH(k_batch_gate<float>, g, 256, 0, s, (const BatchItem<float> *)b->img_dev, b->count, b->skip);
    else
      DCSR_LAUNCH(k_batch_gate<double>, g, 256, 0, s, (const BatchItem<double> *)b->img_dev, b->count, b->skip);
  } else {
    DCSR_CUDA(cudaMemsetAsync(b->skip, 0, sizeof(int32_t) * b->count, s));
  }
  DCSR_TRY(b->ar.reserve(schedule_scratch_bytes(b->R), s));
  DCSR_TRY(schedule_many(b->img_dev + b->off_row, b->dtype, b->count, b->R, b->ar, s));
  for (auto &g : b->groups)
    DCSR_TRY(spmv_many(b->img_dev + g.off, b->dtype, (int)g.idx.size(), g.k, g.vec, g.pref, s));
  return DCSR_OK;
}

void mark_scheduled(dcsr_batch b) {
  for (auto &it : b->items) it.matrix->bins_valid = true;
}

void release(dcsr_batch b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto &g : b->groups)
    if (g.pref) cudaFree(g.pref);
  if (b->img_dev) cudaFree(b->img_dev);
  if (b->img_host) cudaFreeHost(b->img_host);
  if (b->skip) cudaFree(b->skip);
  if (b->status_dev) cudaFree(b->status_dev);
  if (b->gstat) cudaFree(b->gstat);
  b->ar.release(nullptr);
  delete b;
}

}  // namespace

extern "C" {

int dcsr_batch_create(dcsr_batch *out, const dcsr_batch_item *items, int32_t count, void *stream) {
  if (!out || count < 1 || !items) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int dtype = items[0].matrix ? items[0].matrix->dtype : -1;
  const int mode = items[0].matrix ? items[0].matrix->o.mode : -1;
  int32_t max_rows = 1, max_cols = 1;
  int64_t T = 0, R = 0;
  std::vector<dcsr_handle> seen;
  for (int i = 0; i < count; i++) {
    const dcsr_batch_item &it = items[i];
    dcsr_handle h = it.matrix;
    if (!h || h->dtype != dtype || h->o.mode != mode || it.nnz < 0 || (it.nnz > 0 && (!it.rows || !it.cols || !it.vals)))
      return DCSR_BAD_ARG;
    if (it.x && (it.k < 1 || it.k > 8 || it.ldx < it.k || it.ldy < it.k || (h->n_rows > 0 && !it.y)))
      return DCSR_BAD_ARG;
    seen.push_back(h);
    T += it.nnz;
    R += h->n_rows;
    max_rows = h->n_rows > max_rows ? h->n_rows : max_rows;
    max_cols = h->n_cols > max_cols ? h->n_cols : max_cols;
  }
  std::sort(seen.begin(), seen.end());
  if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) return DCSR_BAD_ARG;  // a matrix twice
  if (T > 0x7fffffffLL) return DCSR_NOT_SUPPORTED;

  dcsr_batch b = new dcsr_batch_s;
  b->count = count;
  b->dtype = dtype;
  b->mode = mode;
  b->items.assign(items, items + count);
  b->T = T;
  b->R = R;
  b->rb = bits_for((int64_t)max_rows);
  b->cb = bits_for((int64_t)max_cols);
  cudaGetDevice(&b->device);
  // SpMV groups by (k, vectorisable x)
  for (int i = 0; i < count; i++) {
    const dcsr_batch_item &it = items[i];
    if (!it.x || it.matrix->n_rows == 0) continue;
    const size_t vs = it.matrix->vsize();
    const size_t al = it.k * vs >= 16 ? 16 : it.k * vs;
    const bool vec = it.k > 1 && it.k % 2 == 0 && it.ldx == it.k && ((uintptr_t)it.x % al) == 0;
    int gi = -1;
    for (size_t q = 0; q < b->groups.size(); q++)
      if (b->groups[q].k == it.k && b->groups[q].vec == vec) gi = (int)q;
    if (gi < 0) {
      b->groups.emplace_back();
      gi = (int)b->groups.size() - 1;
      b->groups[gi].k = it.k;
      b->groups[gi].vec = vec;
    }
    b->groups[gi].idx.push_back(i);
  }
  size_t off = align_up((int64_t)(count * desc_size(dtype, false)), 256);
  b->off_row = off;
  off = align_up((int64_t)(off + count * desc_size(dtype, true)), 256);
  for (auto &g : b->groups) {
    g.off = off;
    off = align_up((int64_t)(off + g.idx.size() * desc_size(dtype, true)), 256);
  }
  b->img_bytes = off;
  int st = DCSR_OK;
  if (cudaMalloc((void **)&b->img_dev, b->img_bytes) != cudaSuccess ||
      cudaMallocHost((void **)&b->img_host, b->img_bytes) != cudaSuccess ||
      cudaMalloc((void **)&b->skip, sizeof(int32_t) * count) != cudaSuccess ||
      cudaMalloc((void **)&b->status_dev, sizeof(int32_t) * count) != cudaSuccess ||
      cudaMalloc((void **)&b->gstat, sizeof(long long) * ST_WORDS) != cudaSuccess)
    st = DCSR_OOM;
  for (auto &g : b->groups)
    if (st == DCSR_OK && cudaMalloc((void **)&g.pref, sizeof(long long) * 3 * (g.idx.size() + 1)) != cudaSuccess)
      st = DCSR_OOM;
  // scratch for the largest phase, reserved now so runs (and captures) never allocate
  const size_t upd = T > 0 ? update_scratch_bytes(T, dtype == DCSR_F64 ? 8 : 4) : 0;
  const size_t sch = schedule_scratch_bytes(R);
  b->ar_need = upd > sch ? upd : sch;
  if (st == DCSR_OK) st = b->ar.reserve(b->ar_need, s);
  if (st == DCSR_OK) {
    std::memset(b->img_host, 0, b->img_bytes);
    if (cudaMemsetAsync(b->img_dev, 0, b->img_bytes, s) != cudaSuccess ||
        cudaMemsetAsync(b->gstat, 0, sizeof(long long) * ST_WORDS, s) != cudaSuccess)
      st = DCSR_CUDA_ERROR;
  }
  if (st == DCSR_OK) st = refresh(b, s);
  if (st != DCSR_OK) {
    cudaStreamSynchronize(s);
    release(b);
    return st;
  }
  *out = b;
  return DCSR_OK;
}

int dcsr_batch_run(dcsr_batch b, void *stream) {
  if (!b) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  DCSR_TRY(refresh(b, s));
  DCSR_TRY(enqueue(b, s));
  mark_scheduled(b);
  return DCSR_OK;
}

int dcsr_batch_capture(dcsr_batch b, void *stream) {
  if (!b || !stream) return DCSR_BAD_ARG;  // the legacy default stream cannot be captured
  cudaStream_t s = (cudaStream_t)stream;
  DCSR_TRY(refresh(b, s));
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  DCSR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const int st = enqueue(b, s);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  if (st != DCSR_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  DCSR_CUDA(e);
  b->graph = g;
  DCSR_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  size_t n = 0;
  DCSR_CUDA(cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  DCSR_CUDA(cudaGraphGetNodes(g, nodes.data(), &n));
  b->graph_kernels = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    DCSR_CUDA(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) b->graph_kernels++;
  }
  return DCSR_OK;
}

int dcsr_batch_launch(dcsr_batch b, void *stream) {
  if (!b || !b->exec) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  DCSR_TRY(refresh(b, s));
  DCSR_CUDA(cudaGraphLaunch(b->exec, s));
  count_launch(b->graph_kernels);
  mark_scheduled(b);
  return DCSR_OK;
}

int dcsr_batch_status(dcsr_batch b, int32_t *statuses, void *stream) {
  if (!b || !statuses) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int g = (b->count + 255) / 256;
  if (b->dtype == DCSR_F32)
    DCSR_LAUNCH(k_batch_status<float>, g, 256, 0, s, (const BatchItem<float> *)b->img_dev, b->count, b->status_dev);
  else
    DCSR_LAUNCH(k_batch_status<double>, g, 256, 0, s, (const BatchItem<double> *)b->img_dev, b->count, b->status_dev);
  DCSR_CUDA(cudaMemcpyAsync(statuses, b->status_dev, sizeof(int32_t) * b->count, cudaMemcpyDeviceToHost, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  return DCSR_OK;
}

int dcsr_batch_repair(dcsr_batch b, const int32_t *statuses, int32_t *repaired, void *stream) {
  if (!b || !statuses) return DCSR_BAD_ARG;
  int n = 0;
  for (int i = 0; i < b->count; i++) {
    if (statuses[i] == DCSR_OK) continue;
    const dcsr_batch_item &it = b->items[i];
    int st = statuses[i];
    if (st == DCSR_POOL_EXHAUSTED || st == DCSR_LAYER_OVERFLOW)
      st = dcsr_update_sync(it.matrix, it.rows, it.cols, it.vals, it.nnz, stream);
    // the batch skipped this matrix's SpMV: run it on the repaired (or, for
    // an unrepairable update, unchanged) matrix, as the per-call path would
    if (it.x) DCSR_TRY(dcsr_spmv(it.matrix, it.x, it.k, it.ldx, it.y, it.ldy, it.alpha, it.beta, stream));
    if (st == DCSR_OK) n++;
  }
  if (repaired) *repaired = n;
  return DCSR_OK;
}

int dcsr_batch_destroy(dcsr_batch b) {
  if (!b) return DCSR_BAD_ARG;
  cudaDeviceSynchronize();
  release(b);
  return DCSR_OK;
}

}  // extern "C"
