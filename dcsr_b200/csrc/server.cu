// server.cu -- the serving form: a request loop over resident matrices with
// admission by device memory and continuous batching through BatchCore.
//
// Worker threads (opts.workers, default 2) own the device side; worker w owns
// the slots w, w + workers, ...  Each turn a worker
//   1. retires every in-flight batch whose completion event has fired:
//      repairs rejected updates (compact / grow / retry, then the skipped
//      SpMV), grows pools that are nearly full, frees the batch's staging,
//      releases its matrices and memory, publishes the results;
//   2. if a slot is free, forms a batch from the queue in arrival order:
//      a request joins unless its matrix is in flight or already blocked in
//      this batch, or it would break the per-matrix order (within a batch a
//      matrix takes at most an update, then an SpMV, or an export alone);
//      admission stops at the first request whose device bytes exceed what
//      is left of the budget;
//   3. launches it on the slot's stream: host -> device copies of the
//      requests' inputs, the merged update + grouped SpMV of BatchCore, the
//      exports, device -> host copies of the results, a completion event.
// Up to `depth` batches are in flight on different streams, so copies and
// kernels of consecutive batches overlap on the device, and the host work of
// forming and launching batches (tens of microseconds of launch calls each)
// runs on several threads.  Batch formation is serialised by the server lock
// and marks the batch's matrices busy and its bytes in use before the lock is
// released, so two workers never take requests of one matrix out of order.
// Results do not depend on how requests were batched: each matrix sees the
// same sequence of operations, and every kernel's result for a matrix is
// independent of the other matrices in its launch.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>

#include "internal.cuh"

namespace dcsr {
namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  dcsr_request r;
  uint64_t ticket = 0;
  Clock::time_point t_submit, t_launch;
  int64_t cost = 0;
  size_t off[3] = {0, 0, 0};  // staging offsets: update rows/cols/vals | spmv x/y | export rp/cols/vals
  int item = -1;              // batch item of its matrix (update / SpMV), export number (export)
  bool direct = false;        // export written straight into the caller's device buffers
  int32_t status = DCSR_OK;
  int64_t nnz = 0;
};

struct Slot {
  cudaStream_t s = nullptr;
  cudaEvent_t done = nullptr;
  // second stream: SpMVs of matrices the batch does not update run on it
  // beside the update pipeline, forked from and joined back into s
  cudaStream_t s2 = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  bool single = false;  // the batch ran as one per-call operator
  BatchCore core;
  bool busy = false;
  std::vector<Req> reqs;
  std::vector<int> mats;
  std::vector<dcsr_batch_item> items;
  std::vector<int> item_upd, item_spmv;  // request index per item (-1: none)
  unsigned char *stage = nullptr;
  long long *status_host = nullptr;
  int status_cap = 0;
  int32_t *nnz_host = nullptr;  // pinned: entry count of each export
  int nnz_cap = 0;
  int64_t cost = 0;
  bool statuses = false;
  int phase = 0;  // 1: batch in flight; 2: exports' entries being copied out
  // tracing (DCSR_SERVER_TRACE): events around the batch's device work
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  Clock::time_point h_start, h_launched, h_retire;
  int repairs = 0, grows = 0;
};

struct TraceRow {
  int n, upd, spmv, exp, repairs, grows;
  long long triples;
  double host_us, gpu_us, turnaround_us, retire_us;
};

}  // namespace
}  // namespace dcsr

using namespace dcsr;

struct dcsr_server_s {
  std::vector<dcsr_handle> mats;
  std::vector<char> busy;
  std::vector<uint32_t> stamp;  // per matrix: batch-formation generation
  std::vector<int> state;       // per matrix in the forming batch: 0 none, 1 update, 2 spmv, 3 export, -1 blocked
  uint32_t gen = 0;
  dcsr_server_opts o{};
  int64_t budget = 0, in_use = 0;
  std::mutex mu;
  std::condition_variable cv_submit, cv_done;
  std::deque<Req> queue;
  std::unordered_map<uint64_t, dcsr_result> done;
  uint64_t next_ticket = 1;
  std::vector<Slot> slots;
  std::vector<std::thread> workers;
  bool stop = false;
  int64_t completed = 0, batches = 0;
  int device = 0;
  int fatal = DCSR_OK;
  cudaMemPool_t pool = nullptr;     // the device's default pool (pre-grown at create)
  uint64_t pool_reserved0 = 0;      // its reserved bytes before: trimmed back to them at destroy
  std::string trace_path;  // DCSR_SERVER_TRACE: per-batch timings written at destroy
  std::vector<TraceRow> trace;
};

namespace {

size_t vs_of(dcsr_handle h) { return h->vsize(); }
size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

int64_t req_cost(dcsr_handle h, const dcsr_request &r) {
  const int64_t vs = (int64_t)vs_of(h), n = h->n_rows, m = h->n_cols;
  switch (r.kind) {
    case DCSR_REQ_UPDATE: return r.nnz * (8 + vs) + (int64_t)update_scratch_bytes(r.nnz, vs) + 16 * n + 4096;
    case DCSR_REQ_SPMV: return (int64_t)r.k * vs * (m + n) + 16 * n + 4096;
    default: return 4 * (n + 1) + h->pool_cap * (4 + vs) + 8 * (n + 2) + 4096;
  }
}

int check_req(dcsr_server s, const dcsr_request &r) {
  if (r.matrix < 0 || r.matrix >= (int)s->mats.size()) return DCSR_BAD_ARG;
  dcsr_handle h = s->mats[r.matrix];
  switch (r.kind) {
    case DCSR_REQ_UPDATE: return r.nnz < 0 || (r.nnz > 0 && (!r.rows || !r.cols || !r.vals)) ? DCSR_BAD_ARG : DCSR_OK;
    case DCSR_REQ_SPMV:
      return r.k < 1 || r.k > 8 || (h->n_cols > 0 && !r.x) || (h->n_rows > 0 && !r.y) ? DCSR_BAD_ARG : DCSR_OK;
    case DCSR_REQ_EXPORT: return !r.row_ptr || r.cap < 0 || (r.cap > 0 && (!r.out_cols || !r.out_vals)) ? DCSR_BAD_ARG
                                                                                                         : DCSR_OK;
  }
  return DCSR_BAD_ARG;
}

void publish(dcsr_server s, std::vector<Req> &reqs, int batch_size) {
  const auto now = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto &q : reqs) {
    dcsr_result res;
    res.status = q.status;
    res.batch_size = batch_size;
    res.nnz = q.nnz;
    res.queue_us = std::chrono::duration<double, std::micro>(q.t_launch - q.t_submit).count();
    res.latency_us = std::chrono::duration<double, std::micro>(now - q.t_submit).count();
    s->done[q.ticket] = res;
    s->completed++;
  }
  s->cv_done.notify_all();
}

// Form a batch from the queue (caller holds the lock).  Requests are taken
// in arrival order; the scan stops when the batch is full, at the first
// request that does not fit the memory budget, or after a bounded number of
// skipped requests; skipped ones go back to the front in their order.
void form(dcsr_server s, std::vector<Req> &take) {
  const int maxb = s->o.plain ? 1 : s->o.max_batch;
  const size_t max_skip = 4 * (size_t)maxb + 1024;
  s->gen++;
  int64_t room = s->budget - s->in_use;
  std::vector<Req> skipped;
  while (!s->queue.empty() && (int)take.size() < maxb && skipped.size() < max_skip) {
    Req q = std::move(s->queue.front());
    s->queue.pop_front();
    const int m = q.r.matrix;
    if (s->stamp[m] != s->gen) {
      s->stamp[m] = s->gen;
      s->state[m] = s->busy[m] ? -1 : 0;
    }
    const int kind = q.r.kind == DCSR_REQ_UPDATE ? 1 : q.r.kind == DCSR_REQ_SPMV ? 2 : 3;
    int &st = s->state[m];
    // order within a batch: update < SpMV; an export only alone
    const bool fits_order = st >= 0 && kind > st && !(kind == 3 && st != 0) && !(st == 3);
    if (!fits_order) {
      st = -1;  // every later request of this matrix waits too
      skipped.push_back(std::move(q));
      continue;
    }
    if (q.cost > room) {
      if (take.empty() && s->in_use == 0 && q.cost > s->budget) {
        q.status = DCSR_OOM;  // can never be admitted: fail it rather than block the queue
        q.t_launch = Clock::now();
        std::vector<Req> one(1, q);
        s->mu.unlock();
        publish(s, one, 0);
        s->mu.lock();
        continue;
      }
      skipped.push_back(std::move(q));  // FIFO admission: later requests wait for memory too
      break;
    }
    st = kind;
    room -= q.cost;
    take.push_back(std::move(q));
  }
  for (auto it = skipped.rbegin(); it != skipped.rend(); ++it) s->queue.push_front(std::move(*it));
  // the batch owns its matrices and bytes from here (still under the lock)
  if (!take.empty()) {
    for (auto &q : take) {
      s->in_use += q.cost;
      s->busy[q.r.matrix] = 1;
    }
    s->batches++;
  }
}

int launch(dcsr_server s, Slot &sl, std::vector<Req> &take) {
  cudaStream_t st = sl.s;
  const auto now = Clock::now();
  sl.h_start = now;
  if (sl.t0) DCSR_CUDA(cudaEventRecord(sl.t0, st));
  sl.reqs.swap(take);
  sl.mats.clear();
  sl.items.clear();
  sl.item_upd.clear();
  sl.item_spmv.clear();
  sl.cost = 0;
  sl.statuses = false;
  // staging layout: host inputs of updates and SpMVs, every export's output
  // (exports are staged even to device buffers: the entry count is only
  // known on the device, so the caller's buffer is filled by a bounded copy)
  size_t bytes = 0;
  int n_exp = 0;
  std::unordered_map<int, int> item_of;
  for (size_t i = 0; i < sl.reqs.size(); i++) {
    Req &q = sl.reqs[i];
    q.t_launch = now;
    sl.cost += q.cost;
    dcsr_handle h = s->mats[q.r.matrix];
    const size_t vs = vs_of(h);
    if (q.r.kind == DCSR_REQ_UPDATE && !q.r.on_device) {
      q.off[0] = bytes;
      bytes = al256(bytes + 4 * q.r.nnz);
      q.off[1] = bytes;
      bytes = al256(bytes + 4 * q.r.nnz);
      q.off[2] = bytes;
      bytes = al256(bytes + vs * q.r.nnz);
    } else if (q.r.kind == DCSR_REQ_SPMV && !q.r.on_device) {
      q.off[0] = bytes;
      bytes = al256(bytes + vs * q.r.k * h->n_cols);
      q.off[1] = bytes;
      bytes = al256(bytes + vs * q.r.k * h->n_rows);
    } else if (q.r.kind == DCSR_REQ_EXPORT) {
      // device buffers take the export directly (bounded by cap on the device)
      q.direct = q.r.on_device;
      if (!q.direct) {
        q.off[0] = bytes;
        bytes = al256(bytes + 4 * ((size_t)h->n_rows + 1));
        q.off[1] = bytes;
        bytes = al256(bytes + 4 * (size_t)h->pool_cap);
        q.off[2] = bytes;
        bytes = al256(bytes + vs * (size_t)h->pool_cap);
      }
      q.item = n_exp++;
    }
    if (!item_of.count(q.r.matrix)) sl.mats.push_back(q.r.matrix);
    if (q.r.kind != DCSR_REQ_EXPORT) {
      auto it = item_of.find(q.r.matrix);
      if (it == item_of.end()) {
        dcsr_batch_item bi;
        std::memset(&bi, 0, sizeof(bi));
        bi.matrix = h;
        item_of[q.r.matrix] = (int)sl.items.size();
        sl.items.push_back(bi);
        sl.item_upd.push_back(-1);
        sl.item_spmv.push_back(-1);
        it = item_of.find(q.r.matrix);
      }
      q.item = it->second;
      (q.r.kind == DCSR_REQ_UPDATE ? sl.item_upd : sl.item_spmv)[q.item] = (int)i;
    } else {
      item_of.emplace(q.r.matrix, -1);
    }
  }
  sl.busy = true;  // the slot owns its requests, matrices and memory (marked by form)
  if (n_exp > sl.nnz_cap) {
    if (sl.nnz_host) DCSR_CUDA(cudaFreeHost(sl.nnz_host));
    sl.nnz_host = nullptr;
    DCSR_CUDA(cudaMallocHost((void **)&sl.nnz_host, sizeof(int32_t) * n_exp));
    sl.nnz_cap = n_exp;
  }
  sl.stage = nullptr;
  if (bytes) DCSR_CUDA(dcsr::dev_alloc((void **)&sl.stage, bytes, st));
  // inputs host -> device; batch items over the staged (or the caller's device) buffers
  for (auto &q : sl.reqs) {
    dcsr_handle h = s->mats[q.r.matrix];
    const size_t vs = vs_of(h);
    unsigned char *b = sl.stage;
    if (q.r.kind == DCSR_REQ_UPDATE && q.r.nnz > 0) {
      dcsr_batch_item &bi = sl.items[q.item];
      if (q.r.on_device) {
        bi.rows = q.r.rows;
        bi.cols = q.r.cols;
        bi.vals = q.r.vals;
      } else {
        DCSR_CUDA(cudaMemcpyAsync(b + q.off[0], q.r.rows, 4 * q.r.nnz, cudaMemcpyHostToDevice, st));
        DCSR_CUDA(cudaMemcpyAsync(b + q.off[1], q.r.cols, 4 * q.r.nnz, cudaMemcpyHostToDevice, st));
        DCSR_CUDA(cudaMemcpyAsync(b + q.off[2], q.r.vals, vs * q.r.nnz, cudaMemcpyHostToDevice, st));
        bi.rows = (const int32_t *)(b + q.off[0]);
        bi.cols = (const int32_t *)(b + q.off[1]);
        bi.vals = b + q.off[2];
      }
      bi.nnz = q.r.nnz;
    } else if (q.r.kind == DCSR_REQ_SPMV) {
      dcsr_batch_item &bi = sl.items[q.item];
      if (q.r.on_device) {
        bi.x = q.r.x;
        bi.y = q.r.y;
      } else {
        DCSR_CUDA(cudaMemcpyAsync(b + q.off[0], q.r.x, vs * q.r.k * h->n_cols, cudaMemcpyHostToDevice, st));
        if (q.r.beta != 0.0)
          DCSR_CUDA(cudaMemcpyAsync(b + q.off[1], q.r.y, vs * q.r.k * h->n_rows, cudaMemcpyHostToDevice, st));
        bi.x = b + q.off[0];
        bi.y = b + q.off[1];
      }
      bi.k = q.r.k;
      bi.ldx = bi.ldy = q.r.k;
      bi.alpha = q.r.alpha;
      bi.beta = q.r.beta;
    }
  }
  if (s->o.plain) {
    // the per-call path: one request, its operator, synchronously
    Req &q = sl.reqs[0];
    dcsr_handle h = s->mats[q.r.matrix];
    if (q.r.kind == DCSR_REQ_UPDATE) {
      const dcsr_batch_item &bi = sl.items[q.item];
      q.status = dcsr_update_sync(h, bi.rows, bi.cols, bi.vals, q.r.nnz, st);
    } else if (q.r.kind == DCSR_REQ_SPMV) {
      const dcsr_batch_item &bi = sl.items[q.item];
      DCSR_TRY(dcsr_spmv(h, bi.x, q.r.k, q.r.k, bi.y, q.r.k, q.r.alpha, q.r.beta, st));
    }
  } else if (sl.reqs.size() == 1 && sl.items.size() == 1) {
    // a lone update or SpMV (low load): its per-call operator, asynchronously --
    // the same result as in a batch with fewer launches
    sl.single = true;
    Req &q = sl.reqs[0];
    dcsr_handle h = s->mats[q.r.matrix];
    const dcsr_batch_item &bi = sl.items[0];
    if (q.r.kind == DCSR_REQ_UPDATE) {
      DCSR_TRY(update_async(h, bi.rows, bi.cols, bi.vals, bi.nnz, st, &sl.core.ar));
      if (sl.status_cap < 1) {
        DCSR_CUDA(cudaMallocHost((void **)&sl.status_host, sizeof(long long) * 2));
        sl.status_cap = 1;
      }
      // (status, needed pool top) as the batch status kernel reports them
      DCSR_CUDA(cudaMemcpyAsync(sl.status_host, h->stat + ST_STATUS, sizeof(long long), cudaMemcpyDeviceToHost, st));
      DCSR_CUDA(cudaMemcpyAsync(sl.status_host + 1, h->stat + ST_NEED, sizeof(long long), cudaMemcpyDeviceToHost, st));
      DCSR_CUDA(cudaMemsetAsync(h->stat + ST_STATUS, 0, sizeof(long long), st));
      sl.statuses = true;
    } else {
      DCSR_TRY(spmv_call(h, bi.x, bi.k, bi.ldx, (void *)bi.y, bi.ldy, bi.alpha, bi.beta, st, &sl.core.ar));
    }
  } else if (!sl.items.empty()) {
    DCSR_TRY(sl.core.plan(sl.items.data(), (int)sl.items.size(), st, false));
    DCSR_TRY(sl.core.upload(st, false, true));
    DCSR_TRY(sl.core.reserve_scratch(st));
    sl.single = false;
    DCSR_TRY(sl.core.enqueue(st, sl.s2, sl.fork, sl.join));
    bool any_upd = false;
    for (int v : sl.item_upd) any_upd |= v >= 0;
    if (any_upd) {
      if (sl.status_cap < (int)sl.items.size()) {
        if (sl.status_host) DCSR_CUDA(cudaFreeHost(sl.status_host));
        sl.status_host = nullptr;
        DCSR_CUDA(cudaMallocHost((void **)&sl.status_host, sizeof(long long) * 2 * sl.items.size()));
        sl.status_cap = (int)sl.items.size();
      }
      DCSR_TRY(sl.core.status_async(sl.status_host, st));
      sl.statuses = true;
    }
    sl.core.mark_scheduled();
  }
  // exports, then results to the caller
  for (auto &q : sl.reqs) {
    dcsr_handle h = s->mats[q.r.matrix];
    const size_t vs = vs_of(h);
    unsigned char *b = sl.stage;
    if (q.r.kind == DCSR_REQ_SPMV && !q.r.on_device) {
      DCSR_CUDA(cudaMemcpyAsync(q.r.y, b + q.off[1], vs * q.r.k * h->n_rows, cudaMemcpyDeviceToHost, st));
    } else if (q.r.kind == DCSR_REQ_EXPORT) {
      int32_t *rp = q.direct ? q.r.row_ptr : (int32_t *)(b + q.off[0]);
      int32_t *oc = q.direct ? q.r.out_cols : (int32_t *)(b + q.off[1]);
      void *ov = q.direct ? q.r.out_vals : b + q.off[2];
      DCSR_TRY(export_csr(h, rp, oc, ov, q.direct ? q.r.cap : INT64_MAX, st, &sl.core.ar));
      DCSR_CUDA(cudaMemcpyAsync(sl.nnz_host + q.item, rp + h->n_rows, 4, cudaMemcpyDeviceToHost, st));
      // a staged export's row pointer now; its entries once their count is known
      if (!q.direct)
        DCSR_CUDA(cudaMemcpyAsync(q.r.row_ptr, rp, 4 * ((size_t)h->n_rows + 1), cudaMemcpyDefault, st));
    }
  }
  if (sl.t1) DCSR_CUDA(cudaEventRecord(sl.t1, st));
  DCSR_CUDA(cudaEventRecord(sl.done, st));
  sl.h_launched = Clock::now();
  sl.phase = 1;
  return DCSR_OK;
}

// Release a finished batch and publish its results.
int finish(dcsr_server s, Slot &sl) {
  if (sl.t0) {
    TraceRow t{(int)sl.reqs.size(), 0, 0, 0, sl.repairs, sl.grows, 0, 0.0, 0.0, 0.0, 0.0};
    t.retire_us = std::chrono::duration<double, std::micro>(Clock::now() - sl.h_retire).count();
    for (auto &q : sl.reqs) {
      if (q.r.kind == DCSR_REQ_UPDATE) {
        t.upd++;
        t.triples += q.r.nnz;
      } else if (q.r.kind == DCSR_REQ_SPMV) {
        t.spmv++;
      } else {
        t.exp++;
      }
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, sl.t0, sl.t1);
    t.gpu_us = 1e3 * ms;
    t.host_us = std::chrono::duration<double, std::micro>(sl.h_launched - sl.h_start).count();
    t.turnaround_us = std::chrono::duration<double, std::micro>(Clock::now() - sl.h_start).count();
    std::lock_guard<std::mutex> lk(s->mu);
    s->trace.push_back(t);
  }
  if (sl.stage) DCSR_CUDA(dcsr::dev_free(sl.stage, sl.s));
  sl.stage = nullptr;
  sl.busy = false;
  sl.phase = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->in_use -= sl.cost;
    for (int m : sl.mats) s->busy[m] = 0;
  }
  publish(s, sl.reqs, (int)sl.reqs.size());
  sl.reqs.clear();
  return DCSR_OK;
}

// The batch's event fired.  Phase 1: repairs, pool pre-growth, export sizes;
// staged exports then copy exactly their entries out (phase 2) before the
// batch finishes.
int retire(dcsr_server s, Slot &sl) {
  cudaStream_t st = sl.s;
  if (sl.phase == 2) return finish(s, sl);
  sl.h_retire = Clock::now();
  sl.repairs = sl.grows = 0;
  if (sl.statuses) {
    for (size_t i = 0; i < sl.items.size(); i++) {
      const int ui = sl.item_upd[i];
      if (ui < 0) continue;
      Req &q = sl.reqs[ui];
      dcsr_handle h = s->mats[q.r.matrix];
      // the status words of updated matrices, in the order of the batch's updates
      const int j = sl.single ? 0 : sl.core.upd_of[i];
      int status = (int)sl.status_host[2 * j];
      const long long need = sl.status_host[2 * j + 1];
      if (status != DCSR_OK) {
        sl.repairs++;
        if (status == DCSR_POOL_EXHAUSTED || status == DCSR_LAYER_OVERFLOW)
          status = dcsr_update_sync(h, sl.items[i].rows, sl.items[i].cols, sl.items[i].vals, sl.items[i].nnz, st);
        const int si = sl.item_spmv[i];
        if (si >= 0) {  // its SpMV was skipped in the batch
          // (the skipped pass left the staged y as it was copied in)
          Req &p = sl.reqs[si];
          const size_t vs = vs_of(h);
          DCSR_TRY(dcsr_spmv(h, sl.items[i].x, p.r.k, p.r.k, sl.items[i].y, p.r.k, p.r.alpha, p.r.beta, st));
          if (!p.r.on_device)
            DCSR_CUDA(cudaMemcpyAsync(p.r.y, sl.items[i].y, vs * p.r.k * h->n_rows, cudaMemcpyDeviceToHost, st));
        }
        DCSR_CUDA(cudaStreamSynchronize(st));
      } else if (h->pool_cap - need < h->pool_cap / 8) {
        // nearly full: grow ahead of the next update (stream-ordered, no sync)
        sl.grows++;
        DCSR_TRY(reserve(h, grow_target(h, need), st));
      }
      q.status = status;
    }
  }
  bool copies = false;
  for (auto &q : sl.reqs) {
    if (q.r.kind != DCSR_REQ_EXPORT) continue;
    q.nnz = sl.nnz_host[q.item];
    if (q.nnz > q.r.cap) q.status = DCSR_BAD_ARG;
    const int64_t n_copy = q.nnz < q.r.cap ? q.nnz : q.r.cap;
    if (!q.direct && n_copy > 0) {
      const size_t vs = vs_of(s->mats[q.r.matrix]);
      DCSR_CUDA(cudaMemcpyAsync(q.r.out_cols, sl.stage + q.off[1], 4 * n_copy, cudaMemcpyDefault, st));
      DCSR_CUDA(cudaMemcpyAsync(q.r.out_vals, sl.stage + q.off[2], vs * n_copy, cudaMemcpyDefault, st));
      copies = true;
    }
  }
  // staged exports' copies, and pools grown ahead (a new pool filled by a
  // copy on this stream), must complete before the batch finishes: finish
  // releases the matrices, and the next batch using one may run on another
  // stream
  if (copies || sl.grows > 0) {
    DCSR_CUDA(cudaEventRecord(sl.done, st));
    sl.phase = 2;
    return DCSR_OK;
  }
  return finish(s, sl);
}

// A batch that could not be launched or retired: its requests fail with
// `status`.  A CUDA error is sticky (the context may be unusable): every
// later request fails with it too.
void fail_slot(dcsr_server s, Slot &sl, int status) {
  for (auto &q : sl.reqs) q.status = status;
  sl.phase = 0;
  if (sl.busy) {
    if (sl.stage) dcsr::dev_free(sl.stage, sl.s);
    sl.stage = nullptr;
    std::lock_guard<std::mutex> lk(s->mu);
    s->in_use -= sl.cost;
    for (int m : sl.mats) s->busy[m] = 0;
  }
  sl.busy = false;
  if (status == DCSR_CUDA_ERROR) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->fatal = status;
  }
  publish(s, sl.reqs, (int)sl.reqs.size());
  sl.reqs.clear();
}

void worker_main(dcsr_server s, int w, int W) {
  cudaSetDevice(s->device);
  std::vector<Slot *> mine;
  for (size_t i = w; i < s->slots.size(); i += W) mine.push_back(&s->slots[i]);
  for (;;) {
    bool progressed = false;
    for (Slot *slp : mine) {
      Slot &sl = *slp;
      if (!sl.busy) continue;
      const cudaError_t e = cudaEventQuery(sl.done);
      if (e == cudaErrorNotReady) continue;
      const int st = e == cudaSuccess ? retire(s, sl) : DCSR_CUDA_ERROR;
      if (st != DCSR_OK) fail_slot(s, sl, st);
      progressed = true;
    }
    Slot *free_slot = nullptr;
    for (Slot *slp : mine)
      if (!slp->busy) {
        free_slot = slp;
        break;
      }
    if (free_slot) {
      std::vector<Req> take;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->fatal != DCSR_OK) {  // a CUDA error: fail everything queued
          std::vector<Req> all(s->queue.begin(), s->queue.end());
          s->queue.clear();
          for (auto &q : all) {
            q.status = s->fatal;
            q.t_launch = Clock::now();
          }
          s->mu.unlock();
          publish(s, all, 0);
          s->mu.lock();
        } else {
          form(s, take);
        }
      }
      if (!take.empty()) {
        const int st = launch(s, *free_slot, take);
        if (st != DCSR_OK) {
          if (free_slot->reqs.empty()) free_slot->reqs.swap(take);
          fail_slot(s, *free_slot, st);
        }
        progressed = true;
      }
    }
    if (!progressed) {
      std::unique_lock<std::mutex> lk(s->mu);
      bool inflight = false;
      for (Slot *slp : mine) inflight |= slp->busy;
      if (s->stop && s->queue.empty() && !inflight) break;
      if (!inflight) {
        s->cv_submit.wait_for(lk, std::chrono::milliseconds(2));
      } else {
        lk.unlock();
        std::this_thread::yield();
      }
    }
  }
}

}  // namespace

extern "C" {

void dcsr_server_default_opts(dcsr_server_opts *o) {
  if (!o) return;
  o->max_batch = 256;
  o->depth = 8;
  o->mem_budget = 0;
  o->mem_reserve = 1ll << 30;
  o->plain = 0;
  o->workers = 2;
}

int dcsr_server_create(dcsr_server *out, const dcsr_handle *matrices, int32_t count, const dcsr_server_opts *opts) {
  if (!out || !matrices || count < 1) return DCSR_BAD_ARG;
  dcsr_server_opts o;
  dcsr_server_default_opts(&o);
  if (opts) o = *opts;
  if (o.max_batch < 1 || o.depth < 1 || o.depth > 16 || o.mem_budget < 0 || o.mem_reserve < 0 || o.workers < 1 ||
      o.workers > 8)
    return DCSR_BAD_ARG;
  for (int i = 0; i < count; i++)
    if (!matrices[i]) return DCSR_BAD_ARG;
  dcsr_server s = new dcsr_server_s;
  s->o = o;
  s->mats.assign(matrices, matrices + count);
  s->busy.assign(count, 0);
  s->stamp.assign(count, 0);
  s->state.assign(count, 0);
  cudaGetDevice(&s->device);
  if (o.mem_budget > 0) {
    s->budget = o.mem_budget;
  } else {
    size_t fr = 0, tot = 0;
    DCSR_CUDA(cudaMemGetInfo(&fr, &tot));
    s->budget = (int64_t)fr - o.mem_reserve;
    if (s->budget < (64ll << 20)) s->budget = 64ll << 20;
  }
  const int depth = o.plain ? 1 : o.depth;
  s->slots.resize(depth);
  const char *tp = std::getenv("DCSR_SERVER_TRACE");
  if (tp && *tp) s->trace_path = tp;
  for (auto &sl : s->slots) {
    if (cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&sl.s2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.join, cudaEventDisableTiming) != cudaSuccess) {
      delete s;
      return DCSR_CUDA_ERROR;
    }
    if (!s->trace_path.empty() &&
        (cudaEventCreate(&sl.t0) != cudaSuccess || cudaEventCreate(&sl.t1) != cudaSuccess)) {
      delete s;
      return DCSR_CUDA_ERROR;
    }
    // every per-batch buffer sized for a full batch now: the loop then never
    // allocates pinned memory (whose release synchronises the device)
    const int n = o.plain ? 1 : o.max_batch;
    if (sl.core.reserve_items(n, s->mats[0]->dtype, sl.s) != DCSR_OK ||
        cudaMallocHost((void **)&sl.status_host, sizeof(long long) * 2 * n) != cudaSuccess ||
        cudaMallocHost((void **)&sl.nnz_host, sizeof(int32_t) * n) != cudaSuccess) {
      delete s;
      return DCSR_OOM;
    }
    sl.status_cap = n;
    sl.nnz_cap = n;
    cudaStreamSynchronize(sl.s);
  }
  // Pre-grow the stream-ordered pool the per-batch staging and scratch come
  // from (freed blocks stay in it), so the loop's allocations map no memory:
  // a quarter of the budget covers the staging of `depth` full batches of
  // host-buffer requests (a few GB each at max_batch 256).  Mapping new memory
  // in the loop costs milliseconds to hundreds of milliseconds per call.
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&s->pool, dev) == cudaSuccess)
      cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemCurrent, &s->pool_reserved0);
    const int64_t warm = std::min<int64_t>(std::max<int64_t>(s->budget / 4, 64ll << 20), 32ll << 30);
    void *p = nullptr;
    if (cudaMallocAsync(&p, (size_t)warm, s->slots[0].s) == cudaSuccess) cudaFreeAsync(p, s->slots[0].s);
    cudaStreamSynchronize(s->slots[0].s);
  }
  const int nw = o.plain ? 1 : std::min(o.workers, depth);
  for (int w = 0; w < nw; w++) s->workers.emplace_back(worker_main, s, w, nw);
  *out = s;
  return DCSR_OK;
}

int dcsr_server_submit(dcsr_server s, const dcsr_request *req, uint64_t *ticket) {
  if (!s || !req || !ticket) return DCSR_BAD_ARG;
  DCSR_TRY(check_req(s, *req));
  Req q;
  q.r = *req;
  q.t_submit = Clock::now();
  q.cost = req_cost(s->mats[req->matrix], *req);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return DCSR_BAD_ARG;
    q.ticket = s->next_ticket++;
    *ticket = q.ticket;
    s->queue.push_back(std::move(q));
  }
  s->cv_submit.notify_all();  // every worker: any of them may have a free slot
  return DCSR_OK;
}

int dcsr_server_wait(dcsr_server s, uint64_t ticket, int64_t timeout_us, dcsr_result *out) {
  if (!s || !out) return DCSR_BAD_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (ticket == 0 || ticket >= s->next_ticket) return DCSR_BAD_ARG;
  auto ready = [&] { return s->done.count(ticket) > 0; };
  if (timeout_us < 0) s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready)) return DCSR_TIMEOUT;
  *out = s->done[ticket];
  s->done.erase(ticket);
  return DCSR_OK;
}

int dcsr_server_stats(dcsr_server s, int64_t *completed, int64_t *batches, int64_t *mem_in_use) {
  if (!s) return DCSR_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (completed) *completed = s->completed;
  if (batches) *batches = s->batches;
  if (mem_in_use) *mem_in_use = s->in_use;
  return DCSR_OK;
}

int dcsr_server_destroy(dcsr_server s) {
  if (!s) return DCSR_BAD_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_submit.notify_all();
  for (auto &t : s->workers)
    if (t.joinable()) t.join();
  if (!s->trace_path.empty()) {
    if (FILE *f = std::fopen(s->trace_path.c_str(), "w")) {
      std::fprintf(f, "requests,updates,spmvs,exports,repairs,grows,triples,host_launch_us,gpu_us,turnaround_us,"
                      "retire_us\n");
      for (auto &t : s->trace)
        std::fprintf(f, "%d,%d,%d,%d,%d,%d,%lld,%.1f,%.1f,%.1f,%.1f\n", t.n, t.upd, t.spmv, t.exp, t.repairs, t.grows,
                     t.triples, t.host_us, t.gpu_us, t.turnaround_us, t.retire_us);
      std::fclose(f);
    }
  }
  for (auto &sl : s->slots) {
    if (sl.s) cudaStreamSynchronize(sl.s);
    if (sl.t0) cudaEventDestroy(sl.t0);
    if (sl.t1) cudaEventDestroy(sl.t1);
    sl.core.release();
    if (sl.status_host) cudaFreeHost(sl.status_host);
    if (sl.nnz_host) cudaFreeHost(sl.nnz_host);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.fork) cudaEventDestroy(sl.fork);
    if (sl.join) cudaEventDestroy(sl.join);
    if (sl.s2) cudaStreamDestroy(sl.s2);
    if (sl.s) cudaStreamDestroy(sl.s);
  }
  // hand back the unused memory the pre-growth and the loop left in the pool
  if (s->pool) cudaMemPoolTrimTo(s->pool, (size_t)s->pool_reserved0);
  delete s;
  return DCSR_OK;
}

int dcsr_server_replay(dcsr_server s, const dcsr_request *requests, const double *arrival_us, int64_t count,
                       dcsr_result *results, double *wall_us) {
  if (!s || (count > 0 && (!requests || !arrival_us || !results))) return DCSR_BAD_ARG;
  std::vector<uint64_t> tickets(count);
  std::vector<double> late(count);
  const auto t0 = Clock::now();
  for (int64_t i = 0; i < count; i++) {
    const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(
                              arrival_us[i]));
    for (auto now = Clock::now(); now < due; now = Clock::now()) {
      if (due - now > std::chrono::microseconds(200)) std::this_thread::sleep_for(due - now - std::chrono::microseconds(100));
    }
    late[i] = std::chrono::duration<double, std::micro>(Clock::now() - due).count();
    DCSR_TRY(dcsr_server_submit(s, &requests[i], &tickets[i]));
  }
  double last = 0;
  for (int64_t i = 0; i < count; i++) {
    DCSR_TRY(dcsr_server_wait(s, tickets[i], -1, &results[i]));
    results[i].queue_us += late[i];
    results[i].latency_us += late[i];
    const double done = arrival_us[i] + results[i].latency_us;
    last = done > last ? done : last;
  }
  if (wall_us) *wall_us = last;
  return DCSR_OK;
}

}  // extern "C"
