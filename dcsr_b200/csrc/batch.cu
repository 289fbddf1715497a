// batch.cu -- the batched form: many matrices, each with an update batch and
// an SpMV, run as one merged update (one key sort, one plan, one apply over
// the union of their triples), one schedule rebuild over all their rows and
// one SpMV pass per distinct RHS count -- about fifty kernels for the whole
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

// (status, pool top needed) per updated matrix; a look-back timeout of the
// batch's merged sort or scans (the batch-global status word) is reported
// for every matrix that has no status of its own.
template <typename V>
__global__ void k_batch_status2(const BatchItem<V> *its, int count, const long long *gstat, long long *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    long long *st = its[i].m.stat;
    out[2 * i] = st[ST_STATUS] ? st[ST_STATUS] : gstat[ST_STATUS];
    out[2 * i + 1] = st[ST_NEED];
    st[ST_STATUS] = 0;
  }
}

namespace {

size_t desc_size(int dtype, bool row) {
  if (dtype == DCSR_F32) return row ? sizeof(RowItem<float>) : sizeof(BatchItem<float>);
  return row ? sizeof(RowItem<double>) : sizeof(BatchItem<double>);
}

template <typename V>
void fill_image(const BatchCore &b, unsigned char *img) {
  BatchItem<V> *up = (BatchItem<V> *)img;
  RowItem<V> *rows = (RowItem<V> *)(img + b.off_row);
  long long toff = 0, row0 = 0;
  for (size_t j = 0; j < b.upd.size(); j++) {
    const dcsr_batch_item &it = b.items[b.upd[j]];
    dcsr_handle h = it.matrix;
    BatchItem<V> u;
    std::memset(&u, 0, sizeof(u));
    u.m = h->view<V>();
    u.rows = it.rows;
    u.cols = it.cols;
    u.vals = (const V *)it.vals;
    u.toff = toff;
    u.T = it.nnz;
    up[j] = u;
    toff += it.nnz;
  }
  for (size_t q = 0; q < b.sched.size(); q++) {
    dcsr_handle h = b.items[b.sched[q]].matrix;
    RowItem<V> r = row_item<V>(h, nullptr, nullptr, 0, 0, 0.0, 0.0);
    r.row0 = row0;
    row0 += h->n_rows;
    rows[q] = r;
  }
  for (auto &g : b.groups) {
    RowItem<V> *gi = (RowItem<V> *)(img + g.off);
    for (size_t j = 0; j < g.idx.size(); j++) {
      const int i = g.idx[j];
      const dcsr_batch_item &it = b.items[i];
      RowItem<V> r = row_item<V>(it.matrix, it.x, it.y, it.ldx, it.ldy, it.alpha, it.beta);
      r.skip = b.upd_of[i] >= 0 ? b.skip + b.upd_of[i] : nullptr;  // only an update can be rejected
      r.k = it.k;
      // x rows as 8/16/32-byte vectors: even k, packed rows, base aligned to
      // the largest power of two (<= 32) dividing the row size
      const size_t rb = it.k * sizeof(V), al = (rb & (0 - rb)) >= 32 ? 32 : (rb & (0 - rb));
      r.vec = it.k > 1 && it.k % 2 == 0 && it.ldx == it.k && ((uintptr_t)it.x % al) == 0;
      gi[j] = r;
    }
  }
}

template <typename T>
int grow_dev(T **p, size_t n, size_t &cap, cudaStream_t s) {
  if (n <= cap && *p) return DCSR_OK;
  if (*p) DCSR_CUDA(dcsr::dev_free(*p, s));
  *p = nullptr;
  cap = 0;
  DCSR_CUDA(dcsr::dev_alloc((void **)p, sizeof(T) * (n ? n : 1), s));
  cap = n;
  return DCSR_OK;
}

}  // namespace

int BatchCore::plan(const dcsr_batch_item *its, int n, cudaStream_t s, bool all_schedules) {
  if (n < 1 || !its || !its[0].matrix) return DCSR_BAD_ARG;
  const int dt = its[0].matrix->dtype, md = its[0].matrix->o.mode;
  int64_t t = 0, r = 0;
  std::vector<dcsr_handle> seen;
  seen.reserve(n);
  for (int i = 0; i < n; i++) {
    const dcsr_batch_item &it = its[i];
    dcsr_handle h = it.matrix;
    if (!h || h->dtype != dt || h->o.mode != md || it.nnz < 0 || (it.nnz > 0 && (!it.rows || !it.cols || !it.vals)))
      return DCSR_BAD_ARG;
    if (it.x && (it.k < 1 || it.k > 8 || it.ldx < it.k || it.ldy < it.k || (h->n_rows > 0 && !it.y)))
      return DCSR_BAD_ARG;
    seen.push_back(h);
    t += it.nnz;
    r += h->n_rows;
  }
  std::sort(seen.begin(), seen.end());
  if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) return DCSR_BAD_ARG;  // a matrix twice
  if (t > 0x7fffffffLL) return DCSR_NOT_SUPPORTED;
  count = n;
  dtype = dt;
  mode = md;
  items.assign(its, its + n);
  T = t;
  // the update pipeline runs over the matrices with triples only; its key
  // widths come from those matrices
  upd.clear();
  upd_of.assign(n, -1);
  int32_t upd_rows = 1, upd_cols = 1;
  for (int i = 0; i < n; i++)
    if (its[i].nnz > 0) {
      upd_of[i] = (int)upd.size();
      upd.push_back(i);
      upd_rows = its[i].matrix->n_rows > upd_rows ? its[i].matrix->n_rows : upd_rows;
      upd_cols = its[i].matrix->n_cols > upd_cols ? its[i].matrix->n_cols : upd_cols;
    }
  rb = bits_for((int64_t)upd_rows);
  cb = bits_for((int64_t)upd_cols);
  // SpMV groups by k family: 1, 2, 4 (k = 3, 4) and 8 (k = 5..8); the kernel
  // reads each item's k, so a run has at most four SpMV passes whatever the
  // mix of k
  groups.clear();
  for (int i = 0; i < n; i++) {
    const dcsr_batch_item &it = its[i];
    if (!it.x || it.matrix->n_rows == 0) continue;
    // k families 1 (large matrices), 2 (k <= 2; k = 1 of small matrices), 4, 8
    const int gk = it.k == 1 ? (it.matrix->n_rows <= K1_GROUP_ROWS ? 2 : 1) : it.k <= 2 ? 2 : it.k <= 4 ? 4 : 8;
    int gi = -1;
    for (size_t q = 0; q < groups.size(); q++)
      if (groups[q].k == gk) gi = (int)q;
    if (gi < 0) {
      groups.emplace_back();
      gi = (int)groups.size() - 1;
      groups[gi].k = gk;
    }
    groups[gi].idx.push_back(i);
  }
  // schedules to rebuild: every matrix, or the updated ones and those whose
  // schedule is stale (after sizing their schedule buffers, which can
  // invalidate a schedule); the SpMVs of the others may run beside the update
  DCSR_TRY(ensure_buffers(s));
  sched.clear();
  R = 0;
  std::vector<char> in_sched(n, 0);
  for (int i = 0; i < n; i++)
    if (all_schedules || its[i].nnz > 0 || !its[i].matrix->bins_valid) {
      sched.push_back(i);
      in_sched[i] = 1;
      R += its[i].matrix->n_rows;
    }
  {
    std::vector<Group> split;
    for (auto &g : groups) {
      Group main_g, side_g;
      main_g.k = side_g.k = g.k;
      side_g.side = true;
      for (int i : g.idx) (in_sched[i] ? main_g : side_g).idx.push_back(i);
      if (!main_g.idx.empty()) split.push_back(main_g);
      if (!side_g.idx.empty()) split.push_back(side_g);
    }
    groups.swap(split);
  }
  size_t off = align_up((int64_t)(upd.size() * desc_size(dtype, false)), 256);
  off_row = off;
  off = align_up((int64_t)(off + sched.size() * desc_size(dtype, true)), 256);
  size_t poff = 0;
  for (auto &g : groups) {
    g.off = off;
    off = align_up((int64_t)(off + g.idx.size() * desc_size(dtype, true)), 256);
    g.pref_off = poff;
    poff += 3 * (g.idx.size() + 1) + 2;  // unit prefixes + the k = 1 passes' counter words
    int64_t blocks = 0;
    for (int i : g.idx) blocks += div_up(its[i].matrix->n_rows, 32);
    g.split = split_force > 0 && g.k >= 2 ? split_force : short_split(blocks, g.k);
  }
  img_bytes = off;
  if (img_bytes > img_cap) {
    if (up_ev) DCSR_CUDA(cudaEventSynchronize(up_ev));  // the last upload has left the pinned image
    if (img_host) DCSR_CUDA(cudaFreeHost(img_host));
    img_host = nullptr;
    DCSR_TRY(grow_dev(&img_dev, img_bytes, img_cap, s));
    DCSR_CUDA(cudaMallocHost((void **)&img_host, img_bytes));
    std::memset(img_host, 0, img_bytes);
  }
  size_t cc = cnt_cap;
  DCSR_TRY(grow_dev(&skip, n, cc, s));
  cc = 2 * (size_t)cnt_cap;
  DCSR_TRY(grow_dev(&status_dev, 2 * (size_t)n, cc, s));
  cnt_cap = n > cnt_cap ? n : cnt_cap;
  DCSR_TRY(grow_dev(&pref, poff, pref_cap, s));
  if (!gstat) {
    DCSR_CUDA(dcsr::dev_alloc((void **)&gstat, sizeof(long long) * ST_WORDS, s));
    DCSR_CUDA(cudaMemsetAsync(gstat, 0, sizeof(long long) * ST_WORDS, s));
  }
  return DCSR_OK;
}

int BatchCore::reserve_items(int n, int dt, cudaStream_t s) {
  // BatchItem + schedule RowItem + SpMV RowItem per item, 256-byte section
  // padding for the (at most 10: updates, schedules, 4 k families x main and
  // side) sections
  const size_t bytes = align_up((int64_t)(n * (desc_size(dt, false) + 2 * desc_size(dt, true)) + 10 * 256), 256);
  if (bytes > img_cap) {
    if (up_ev) DCSR_CUDA(cudaEventSynchronize(up_ev));  // the last upload has left the pinned image
    if (img_host) DCSR_CUDA(cudaFreeHost(img_host));
    img_host = nullptr;
    DCSR_TRY(grow_dev(&img_dev, bytes, img_cap, s));
    DCSR_CUDA(cudaMallocHost((void **)&img_host, bytes));
    std::memset(img_host, 0, bytes);
  }
  size_t cc = cnt_cap;
  DCSR_TRY(grow_dev(&skip, n, cc, s));
  cc = 2 * (size_t)cnt_cap;
  DCSR_TRY(grow_dev(&status_dev, 2 * (size_t)n, cc, s));
  cnt_cap = n > cnt_cap ? n : cnt_cap;
  DCSR_TRY(grow_dev(&pref, 3 * (size_t)(n + 8) + 16, pref_cap, s));
  return DCSR_OK;
}

int BatchCore::ensure_buffers(cudaStream_t s) {
  for (auto &g : groups)
    for (int i : g.idx) DCSR_TRY(ensure_part(items[i].matrix, g.k, s));
  for (int i = 0; i < count; i++) DCSR_TRY(ensure_part(items[i].matrix, 1, s));
  return DCSR_OK;
}

int BatchCore::upload(cudaStream_t s, bool sync, bool force) {
  img_new.assign(img_bytes, 0);
  if (dtype == DCSR_F32) fill_image<float>(*this, img_new.data());
  else fill_image<double>(*this, img_new.data());
  if (force || std::memcmp(img_new.data(), img_host, img_bytes) != 0) {
    std::memcpy(img_host, img_new.data(), img_bytes);
    DCSR_CUDA(cudaMemcpyAsync(img_dev, img_host, img_bytes, cudaMemcpyHostToDevice, s));
    if (!up_ev) DCSR_CUDA(cudaEventCreateWithFlags(&up_ev, cudaEventDisableTiming));
    DCSR_CUDA(cudaEventRecord(up_ev, s));
    if (sync) DCSR_CUDA(cudaStreamSynchronize(s));
  }
  return DCSR_OK;
}

int BatchCore::reserve_scratch(cudaStream_t s) {
  const size_t upd = T > 0 ? update_scratch_bytes(T, dtype == DCSR_F64 ? 8 : 4) : 0;
  const size_t sch = schedule_scratch_bytes(R);
  DCSR_TRY(ar.reserve(upd > sch ? upd : sch, s));
  // look-back area for the update's sort and scans and the schedule's scans
  // (sized here, outside any stream capture)
  Lookback lb;
  return ar.lookback(lookback_slots((T > R ? T : R) + 2), s, &lb);
}

int BatchCore::enqueue(cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join) {
  const bool merge = mode == DCSR_MERGE;
  ar.status = gstat + ST_STATUS;  // look-back timeouts of the run's sorts and scans
  bool beside = false;
  for (auto &g : groups) beside |= g.side;
  beside = beside && s2 && fork && join;
  // unit prefixes of a set of groups, one launch (a group's prefixes read
  // its matrices' schedules: side groups' are valid now, the others' after
  // the schedule rebuild below)
  auto prefixes = [&](bool side) -> int {
    const void *its[MAX_PREFIX_JOBS];
    int cnt[MAX_PREFIX_JOBS], spl[MAX_PREFIX_JOBS];
    long long *pr[MAX_PREFIX_JOBS];
    int n = 0;
    for (auto &g : groups)
      if ((g.side && beside) == side && n < MAX_PREFIX_JOBS) {
        its[n] = img_dev + g.off;
        cnt[n] = (int)g.idx.size();
        pr[n] = pref + g.pref_off;
        spl[n] = g.split;
        n++;
      }
    return unit_prefix_many(its, cnt, pr, spl, n, dtype, s);
  };
  if (beside) {  // SpMVs of untouched matrices with valid schedules, on s2 beside the update
    DCSR_TRY(prefixes(true));
    DCSR_CUDA(cudaEventRecord(fork, s));
    DCSR_CUDA(cudaStreamWaitEvent(s2, fork, 0));
    for (auto &g : groups)
      if (g.side)
        DCSR_TRY(spmv_many(img_dev + g.off, dtype, (int)g.idx.size(), g.k, pref + g.pref_off, s2, true, g.split));
    DCSR_CUDA(cudaEventRecord(join, s2));
  }
  const int nu = (int)upd.size();
  if (T > 0 && nu > 0) {
    DCSR_TRY(update_many(img_dev, dtype, nu, T, merge, rb, cb, gstat, ar, s));
    const int g = (nu + 255) / 256;
    if (dtype == DCSR_F32)
      DCSR_LAUNCH(k_batch_gate<float>, g, 256, 0, s, (const BatchItem<float> *)img_dev, nu, skip);
    else
      DCSR_LAUNCH(k_batch_gate<double>, g, 256, 0, s, (const BatchItem<double> *)img_dev, nu, skip);
  }
  if (!sched.empty()) {
    DCSR_TRY(ar.reserve(schedule_scratch_bytes(R), s));
    DCSR_TRY(schedule_many(img_dev + off_row, dtype, (int)sched.size(), R, ar, s));
  }
  DCSR_TRY(prefixes(false));
  for (auto &g : groups)
    if (!g.side || !beside)
      DCSR_TRY(spmv_many(img_dev + g.off, dtype, (int)g.idx.size(), g.k, pref + g.pref_off, s, true, g.split));
  if (beside) DCSR_CUDA(cudaStreamWaitEvent(s, join, 0));
  return DCSR_OK;
}

int BatchCore::status_async(long long *host, cudaStream_t s) {
  const int nu = (int)upd.size();
  if (nu == 0) return DCSR_OK;
  const int g = (nu + 255) / 256;
  if (dtype == DCSR_F32)
    DCSR_LAUNCH(k_batch_status2<float>, g, 256, 0, s, (const BatchItem<float> *)img_dev, nu, gstat, status_dev);
  else
    DCSR_LAUNCH(k_batch_status2<double>, g, 256, 0, s, (const BatchItem<double> *)img_dev, nu, gstat, status_dev);
  DCSR_CUDA(cudaMemsetAsync(gstat + ST_STATUS, 0, sizeof(long long), s));
  DCSR_CUDA(cudaMemcpyAsync(host, status_dev, sizeof(long long) * 2 * nu, cudaMemcpyDeviceToHost, s));
  return DCSR_OK;
}

void BatchCore::mark_scheduled() {
  for (auto &it : items) it.matrix->bins_valid = true;
}

void BatchCore::release() {
  // Device buffers: stream-ordered frees on the legacy default stream (after
  // the work queued on blocking streams; the host does not wait).  The pinned
  // image: once its last upload has been copied.
  if (img_dev) dcsr::dev_free(img_dev, 0);
  if (skip) dcsr::dev_free(skip, 0);
  if (status_dev) dcsr::dev_free(status_dev, 0);
  if (pref) dcsr::dev_free(pref, 0);
  if (gstat) dcsr::dev_free(gstat, 0);
  ar.release(0);
  if (up_ev) {
    cudaEventSynchronize(up_ev);
    cudaEventDestroy(up_ev);
    up_ev = nullptr;
  }
  if (img_host) cudaFreeHost(img_host);
  img_dev = img_host = nullptr;
  skip = nullptr;
  status_dev = pref = gstat = nullptr;
}

}  // namespace dcsr

using namespace dcsr;

struct dcsr_batch_s {
  BatchCore core;
  long long *status_host = nullptr;  // pinned [2*count]
  bool status_read = false;          // status_host holds the last status read (for dcsr_batch_grow)
  std::vector<long long> last_need;  // per item: pool top needed at the previous grow check (-1: none)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_kernels = 0;  // kernel nodes of the captured graph
};

namespace {

void release(dcsr_batch b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->status_host) cudaFreeHost(b->status_host);
  b->core.release();
  delete b;
}

}  // namespace

extern "C" {

int dcsr_batch_create(dcsr_batch *out, const dcsr_batch_item *items, int32_t count, void *stream) {
  if (!out || count < 1 || !items) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  dcsr_batch b = new dcsr_batch_s;
  int st = b->core.plan(items, count, s, true);
  // scratch for the largest phase, reserved now so runs (and captures) never allocate
  if (st == DCSR_OK) st = b->core.reserve_scratch(s);
  if (st == DCSR_OK && cudaMallocHost((void **)&b->status_host, sizeof(long long) * 2 * count) != cudaSuccess)
    st = DCSR_OOM;
  if (st == DCSR_OK) st = b->core.upload(s, true, true);
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
  DCSR_TRY(b->core.ensure_buffers(s));
  DCSR_TRY(b->core.upload(s, true));
  DCSR_TRY(b->core.reserve_scratch(s));
  DCSR_TRY(b->core.enqueue(s));
  b->core.mark_scheduled();
  return DCSR_OK;
}

int dcsr_batch_capture(dcsr_batch b, void *stream) {
  if (!b || !stream) return DCSR_BAD_ARG;  // the legacy default stream cannot be captured
  cudaStream_t s = (cudaStream_t)stream;
  DCSR_TRY(b->core.ensure_buffers(s));
  DCSR_TRY(b->core.upload(s, true));
  DCSR_TRY(b->core.reserve_scratch(s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  DCSR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const int st = b->core.enqueue(s);
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
  DCSR_TRY(b->core.ensure_buffers(s));
  DCSR_TRY(b->core.upload(s, true));
  DCSR_CUDA(cudaGraphLaunch(b->exec, s));
  count_launch(b->graph_kernels);
  b->core.mark_scheduled();
  return DCSR_OK;
}

int dcsr_batch_status(dcsr_batch b, int32_t *statuses, void *stream) {
  if (!b || !statuses) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  DCSR_TRY(b->core.status_async(b->status_host, s));
  DCSR_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < b->core.count; i++) {
    const int j = b->core.upd_of[i];
    statuses[i] = j >= 0 ? (int32_t)b->status_host[2 * j] : DCSR_OK;
  }
  b->status_read = true;
  return DCSR_OK;
}

int dcsr_batch_grow(dcsr_batch b, int32_t *grown, void *stream) {
  if (!b) return DCSR_BAD_ARG;
  int n = 0;
  if (b->status_read) {  // the words of the last status read: (status, pool top needed) per update
    b->last_need.resize(b->core.count, -1);
    for (int i = 0; i < b->core.count; i++) {
      const int j = b->core.upd_of[i];
      if (j < 0) continue;
      dcsr_handle h = b->core.items[i].matrix;
      if (b->status_host[2 * j] != DCSR_OK) {
        // rejected (and repaired per call): its pool top moved outside the
        // batch; room for twice its triples beyond the repaired pool
        b->last_need[i] = -1;
        const long long T = b->core.items[i].nnz;
        if (T > 0) {
          DCSR_TRY(reserve(h, grow_target(h, h->pool_cap + 2 * T), (cudaStream_t)stream));
          n++;
        }
        continue;
      }
      const long long need = b->status_host[2 * j + 1];
      // grown when less room is left than the larger of an eighth of the
      // pool and two more runs growing it as much as the last one did (or
      // adding all of the item's triples: its next update has as many), then
      // to room for four such runs, so a growing matrix is grown every few
      // runs rather than every run (each growth allocates and copies a pool)
      const long long prev = b->last_need[i];
      const long long step = prev >= 0 && need > prev ? need - prev : 0;
      b->last_need[i] = need;
      const long long T = b->core.items[i].nnz;  // at most T new entries next run, before relocations
      const long long run = step > T ? step : T;
      const long long room = h->pool_cap / 8 > 2 * run ? h->pool_cap / 8 : 2 * run;
      if (h->pool_cap - need < room) {
        DCSR_TRY(reserve(h, grow_target(h, need + 2 * room), (cudaStream_t)stream));  // keeps the pool top
        n++;
      }
    }
    b->status_read = false;
  }
  if (grown) *grown = n;
  return DCSR_OK;
}

int dcsr_batch_repair(dcsr_batch b, const int32_t *statuses, int32_t *repaired, void *stream) {
  if (!b || !statuses) return DCSR_BAD_ARG;
  int n = 0;
  for (int i = 0; i < b->core.count; i++) {
    if (statuses[i] == DCSR_OK) continue;
    const dcsr_batch_item &it = b->core.items[i];
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

int dcsr_batch_autotune(dcsr_batch b, void *stream, int32_t *short_max, int32_t *long_min, float *best_us) {
  if (!b) return DCSR_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  BatchCore &c = b->core;
  // the batch's SpMV items without their updates, into scratch outputs
  std::vector<dcsr_batch_item> items;
  size_t ybytes = 0;
  for (const auto &it : c.items)
    if (it.x && it.matrix->n_rows > 0) ybytes += align_up((int64_t)(it.matrix->vsize() * it.k * it.matrix->n_rows), 256);
  unsigned char *yscratch = nullptr;
  if (ybytes) DCSR_CUDA(dcsr::dev_alloc((void **)&yscratch, ybytes, s));
  size_t off = 0;
  for (const auto &it : c.items) {
    if (!it.x || it.matrix->n_rows == 0) continue;
    dcsr_batch_item t = it;
    t.rows = t.cols = nullptr;
    t.vals = nullptr;
    t.nnz = 0;
    t.y = yscratch + off;
    t.ldy = t.k;
    t.beta = 0.0;
    off += align_up((int64_t)(it.matrix->vsize() * it.k * it.matrix->n_rows), 256);
    items.push_back(t);
  }
  int32_t best_s = c.items[0].matrix->short_max, best_l = c.items[0].matrix->long_min;
  int best_split = 0;
  float best = -1.0f;
  int st = DCSR_OK;
  if (!items.empty()) {
    BatchCore tmp;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // three timed runs (after one warm-up) of the SpMV pass under one setting
    auto measure = [&](int32_t sm, int32_t lm, int split, float &sum) -> int {
      for (auto &it : items) dcsr_set_row_classes(it.matrix, sm, lm);
      tmp.split_force = split;
      DCSR_TRY(tmp.plan(items.data(), (int)items.size(), s, true));
      DCSR_TRY(tmp.upload(s, true));
      DCSR_TRY(tmp.reserve_scratch(s));
      DCSR_TRY(tmp.enqueue(s));
      sum = 0.0f;
      for (int rep = 0; rep < 3; rep++) {
        cudaEventRecord(e0, s);
        DCSR_TRY(tmp.enqueue(s));
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        sum += ms;
      }
      return DCSR_OK;
    };
    // row-class thresholds under the automatic split, then the split of the
    // k >= 2 groups' short-row blocks under the best thresholds (the split
    // changes which warp takes a row's lane group, never a row's result)
    const int32_t shorts[] = {32, 64, 128};
    const int32_t longs[] = {512, 1024, 4096, 16384};
    for (int32_t sm : shorts) {
      for (int32_t lm : longs) {
        float sum = 0.0f;
        if ((st = measure(sm, lm, 0, sum)) != DCSR_OK) break;
        if (best < 0.0f || sum < best) {
          best = sum;
          best_s = sm;
          best_l = lm;
        }
      }
      if (st != DCSR_OK) break;
    }
    bool has_k2 = false;
    for (const auto &g : tmp.groups) has_k2 |= g.k >= 2;
    for (int split = 1; st == DCSR_OK && has_k2 && split <= 8; split *= 2) {
      float sum = 0.0f;
      if ((st = measure(best_s, best_l, split, sum)) != DCSR_OK) break;
      if (sum < best) {
        best = sum;
        best_split = split;
      }
    }
    cudaStreamSynchronize(s);
    tmp.release();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  c.split_force = best_split;
  for (auto &g : c.groups) {
    if (g.k < 2) continue;
    int64_t blocks = 0;
    for (int i : g.idx) blocks += div_up(c.items[i].matrix->n_rows, 32);
    g.split = best_split > 0 ? best_split : short_split(blocks, g.k);
  }
  for (auto &it : c.items) dcsr_set_row_classes(it.matrix, best_s, best_l);
  if (yscratch) dcsr::dev_free(yscratch, s);
  DCSR_CUDA(cudaStreamSynchronize(s));
  if (st != DCSR_OK) return st;
  if (short_max) *short_max = best_s;
  if (long_min) *long_min = best_l;
  if (best_us) *best_us = best < 0.0f ? 0.0f : 1e3f * best / 3.0f;
  return DCSR_OK;
}

int dcsr_batch_short_split(dcsr_batch b, int32_t *split) {
  if (!b || !split) return DCSR_BAD_ARG;
  *split = b->core.split_force;
  return DCSR_OK;
}

int dcsr_batch_destroy(dcsr_batch b) {
  if (!b) return DCSR_BAD_ARG;
  release(b);
  return DCSR_OK;
}

}  // extern "C"
