// internal.cuh -- cross-file internal API of the DCSR library.
#pragma once
#include <vector>

#include "common.cuh"

namespace dcsr {

// Lay out a matrix from a CSR whose row_ptr is int64 on the device (rows
// already canonical for the handle's mode): policy capacities, fresh pool,
// content copy.  Synchronises once (pool size).
int load_from_csr64(dcsr_handle h, const long long *rp, const int32_t *cols, const void *vals, cudaStream_t s);
size_t load_scratch_bytes(dcsr_handle h);
// Rows staged elsewhere (row r: lens[r] entries at src_off[r]) become the
// matrix's content with policy capacities, in a pool allocated at cap_bound
// entries (an upper bound of the pool capacity the rows need); synchronises
// once at the end (pool top).  Uses the handle's scratch arena.
int load_from_rows(dcsr_handle h, const long long *src_off, const long long *lens, const int32_t *scols,
                   const void *svals, int64_t cap_bound, cudaStream_t s);

// Sort + group a COO batch (any order) into CSR form in the arena:
// MERGE: sorted by (row, col), duplicates summed in input order;
// APPEND: stably sorted by row.  *rp has n_rows+1 entries.  Sets BAD_INDEX in
// *bad (device int) for out-of-range input.
int coo_to_csr64(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz, bool merge,
                 Arena &ar, long long **rp, int32_t **ocols, void **ovals, int *bad, cudaStream_t s);
size_t coo_to_csr_scratch(dcsr_handle h, int64_t nnz);

// Per-call operators that take a scratch arena (default: the handle's own);
// a server passes its slot's arena so resident matrices keep no scratch.
int update_async(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                 cudaStream_t s, Arena *ar = nullptr);

// One matrix of a batched update (device-resident array element).
template <typename V>
struct BatchItem {
  Mat<V> m;
  const int32_t *rows, *cols;
  const V *vals;
  long long toff;  // first index of this matrix's triples in the batch
  long long T;     // its triple count
};
// Update `count` matrices at once (items_dev: device BatchItem<V>[count],
// toff prefix over T); gstat: batch-global status words.
int update_many(const void *items_dev, int dtype, int count, int64_t T, bool merge, int rb, int cb, long long *gstat,
                Arena &ar, cudaStream_t s);
size_t update_scratch_bytes(int64_t T, size_t vsize);
int compact(dcsr_handle h, cudaStream_t s);
int build_schedule(dcsr_handle h, cudaStream_t s, Arena *ar = nullptr);
int spmv_call(dcsr_handle h, const void *x, int32_t k, int64_t ldx, void *y, int64_t ldy, double alpha, double beta,
              cudaStream_t s, Arena *ar = nullptr);

// One matrix of a row pass (SpMV / reduction) over a set of matrices.
template <typename V>
struct RowItem {
  Mat<V> m;
  const int32_t *long_rows;
  const long long *long_off;
  const int2 *chunk_rl;   // per chunk: (row, long-row index)
  const int4 *chunk_desc; // per chunk: (row, length, layer-0 start, layer-0 capacity)
  const int4 *med_desc;   // per medium row: the same descriptor
  int32_t *info;  // [0] long rows, [1] chunks, [2] medium rows
  int32_t *long_cnt;
  double *part;
  const V *x;
  V *y;
  int64_t ldx, ldy;
  double alpha, beta;
  long long row0;             // first row of this matrix in the batch's row space
  int32_t short_max, long_min; // row classes: short <= short_max < medium <= long_min < long
  const int32_t *skip;        // batch: nonzero -> this matrix's pass is skipped (may be null)
  int32_t k, vec;             // runtime-k passes: right-hand sides, x rows loadable as vectors
};
// Rebuild the schedules of `count` matrices at once (items: device
// RowItem<V>[count] in row-space order; R = total rows).  Needs
// schedule_scratch_bytes(R) free in the arena.
int schedule_many(const void *items_dev, int dtype, int count, int64_t R, Arena &ar, cudaStream_t s);
size_t schedule_scratch_bytes(int64_t R);
// y = A x for `count` matrices (items: device RowItem<V>[count]) of one k
// family: kf = 1, 2, 4 or 8, every item's k <= kf (each item's own k / vec
// are read by the kernel); pref: device scratch of 3*(count+1)+2 long longs
// (the unit prefixes, then the k = 1 passes' counter words).
// prefixed: the group's unit prefixes were computed already (unit_prefix_many,
// with the same split); split: warps per 32-row block of short rows (short_split)
int spmv_many(const void *items_dev, int dtype, int count, int k, long long *pref, cudaStream_t s,
              bool prefixed = false, int split = 1);
// Warps per 32-row short-row block for an SpMV pass over `blocks` blocks with k RHS.
int short_split(int64_t blocks, int k);
// A k = 1 SpMV of a matrix of at most this many rows runs in the runtime-k
// (k <= 2) pass -- row groups of G lanes, blocks split across warps -- instead
// of the one-value stream, whose 32-row blocks leave a small matrix to a few
// dozen warps.  A per-matrix rule, so the per-call and batched paths agree.
constexpr int32_t K1_GROUP_ROWS = 32768;
// The unit prefixes of up to MAX_PREFIX_JOBS SpMV groups in one launch.
constexpr int MAX_PREFIX_JOBS = 8;
int unit_prefix_many(const void *const *items, const int *counts, long long *const *prefs, const int *splits, int n,
                     int dtype, cudaStream_t s);
template <typename V>
RowItem<V> row_item(dcsr_handle h, const void *x, void *y, int64_t ldx, int64_t ldy, double alpha, double beta);
// Size the handle's chunk table and chunk partials (K results per chunk).
int ensure_part(dcsr_handle h, int K, cudaStream_t s);
// Copy every row's logical entries to dst_off[r] (optionally COO row ids and
// an int32 row pointer); entries at positions >= limit are not written.
// Builds the schedule first if needed (so callers must not hold arena memory
// across this call unless the schedule is valid).
int copy_rows(dcsr_handle h, const long long *dst_off, int32_t *out_cols, void *out_vals, int32_t *out_rows,
              int32_t *out_rowptr, cudaStream_t s, int64_t limit = INT64_MAX);
// DCSR -> CSR writing at most `limit` entries (the row pointer is complete).
int export_csr(dcsr_handle h, int32_t *row_ptr, int32_t *cols, void *vals, int64_t limit, cudaStream_t s,
               Arena *ar = nullptr);
int reserve(dcsr_handle h, int64_t cap, cudaStream_t s);
// Pool capacity for a matrix whose pool top reached `need` and is nearly
// full: the policy's capacity for that top, and at least a quarter more than
// the current capacity (so the growth is never a no-op).
inline int64_t grow_target(dcsr_handle h, int64_t need) {
  const int64_t p = pool_capacity(h->o, need), q = h->pool_cap + h->pool_cap / 4;
  const int64_t t = p > q ? p : q;
  return t < 0x7fffffffLL ? t : 0x7fffffffLL;  // the pool's index range
}

// The device side of a batch (batch.cu): a plan over a set of
// dcsr_batch_items, their descriptor image, and the enqueue of the merged
// update + schedule rebuild + grouped SpMV.  Buffers grow, never shrink, so
// one core can serve many batches (the server re-plans one per slot).
struct BatchCore {
  struct Group {
    int k = 1;          // k family: 1, 2, 4 (k 3..4) or 8 (k 5..8)
    bool side = false;  // no update and a valid schedule: may run beside the update
    int split = 1;      // warps per 32-row short-row block (short_split of its rows)
    std::vector<int> idx;  // items of this group, in item order
    size_t off = 0;        // descriptor offset in the image
    size_t pref_off = 0;   // unit-prefix offset in pref
  };
  int count = 0, dtype = 0, mode = 0;
  int split_force = 0;  // > 0: warps per short-row block of every k >= 2 group (else short_split)
  std::vector<dcsr_batch_item> items;
  int64_t T = 0, R = 0;
  int rb = 1, cb = 1;
  std::vector<Group> groups;
  std::vector<int> sched;   // items whose schedules the run rebuilds
  std::vector<int> upd;     // items with update triples (the update pipeline's items)
  std::vector<int> upd_of;  // per item: its index in upd, or -1
  // image: BatchItem[upd] | RowItem[sched] (row space) | group RowItems
  size_t off_row = 0, img_bytes = 0, img_cap = 0;
  unsigned char *img_dev = nullptr;
  unsigned char *img_host = nullptr;  // pinned copy of the last upload
  cudaEvent_t up_ev = nullptr;        // recorded after the last upload from img_host
  std::vector<unsigned char> img_new;
  int cnt_cap = 0;
  int32_t *skip = nullptr;        // [upd] 1: the matrix's update was rejected this run
  long long *status_dev = nullptr;  // [2*upd] (status, pool top needed) per updated matrix
  size_t pref_cap = 0;
  long long *pref = nullptr;
  long long *gstat = nullptr;
  Arena ar;

  // Validate and plan `items` (one dtype and mode, each matrix once); grows
  // buffers with stream-ordered allocation on s.  all_schedules: every run
  // rebuilds every matrix's schedule (a captured graph must not depend on
  // host state); else only updated matrices and stale schedules.
  int plan(const dcsr_batch_item *items, int count, cudaStream_t s, bool all_schedules);
  // Size every matrix's schedule buffers for its pool (before an upload).
  int ensure_buffers(cudaStream_t s);
  // Size the image and per-item buffers for up to `items` items at once, so
  // later plans of that size allocate nothing (pinned host allocation and
  // release synchronise the device).
  int reserve_items(int items, int dtype, cudaStream_t s);
  // Rebuild the descriptor image from the handles and upload it if it changed.  sync=true waits for the
  // upload; otherwise the caller guarantees the previous upload of this core
  // has completed before the next call (the pinned image is reused).
  int upload(cudaStream_t s, bool sync, bool force = false);
  // Reserve the arena for this plan (before a capture: runs must not allocate).
  int reserve_scratch(cudaStream_t s);
  // Merged update, skip flags, schedule rebuild, grouped SpMV (capturable).
  // With a second stream s2 (and two events), the SpMVs of matrices without
  // an update and with a valid schedule run on s2 beside the update; s waits
  // for them before returning to the caller's stream order.
  int enqueue(cudaStream_t s, cudaStream_t s2 = nullptr, cudaEvent_t fork = nullptr, cudaEvent_t join = nullptr);
  // (status, needed pool top) of every updated matrix (item upd[j] -> words
  // 2j, 2j+1) into host memory (async); clears the device statuses.
  int status_async(long long *host, cudaStream_t s);
  void mark_scheduled();
  void release();
};

}  // namespace dcsr
