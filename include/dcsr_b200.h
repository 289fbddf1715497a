/*
 * dcsr_b200.h -- C ABI of the B200-native Dynamic-CSR (DCSR) library.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream passed as
 * `void *` (a cudaStream_t; NULL = the legacy default stream) and returns an
 * int status (dcsr_status).  Device pointers for inputs/outputs are owned by
 * the caller; the library owns each matrix's entry pool.  Calls on one handle
 * must come from one stream at a time; different handles are independent.
 *
 * The reference (Vizerai/DCSR) is a header-only C++/CUDA template library in
 * `namespace device` with no ABI; each function below names the reference
 * interface it replaces (file:line in the reference tree).
 *
 * Layout of a matrix in HBM (reference include/dcsr_matrix.h:9-73):
 *   row_sizes[n_rows+1]  logical row lengths; row_sizes[n_rows] = pool top
 *   seg[max_segs*pitch]  (start,end) pool ranges per row and segment layer:
 *                        seg[l*pitch + 2*r], seg[l*pitch + 2*r + 1];
 *                        pitch = align_up(2*n_rows, 32); unused = (-1,-1)
 *   cols[pool_cap] int32, vals[pool_cap] float|double: the entry pool
 * A row's entries are its segments' contents in layer order, up to its
 * logical length.  In MERGE mode every row is kept sorted by column with
 * unique columns; in APPEND mode entries keep insertion order (reference
 * behaviour).
 */
#ifndef DCSR_B200_H
#define DCSR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dcsr_matrix_s *dcsr_handle;

enum { DCSR_F32 = 0, DCSR_F64 = 1 };
enum { DCSR_MERGE = 0, DCSR_APPEND = 1 };

typedef enum {
  DCSR_OK = 0,
  DCSR_POOL_EXHAUSTED = 1, /* update rejected: pool too small (matrix unchanged) */
  DCSR_LAYER_OVERFLOW = 2, /* APPEND-mode update rejected: a row needs > max_segs segments */
  DCSR_BAD_INDEX = 3,      /* an input row/column index is out of range */
  DCSR_OOM = 4,            /* device allocation failed */
  DCSR_BAD_ARG = 5,        /* invalid argument (null handle, size, dtype ...) */
  DCSR_TIMEOUT = 6,        /* a bounded device wait gave up */
  DCSR_CUDA_ERROR = 7,     /* a CUDA runtime call failed */
  DCSR_NOT_SUPPORTED = 8
} dcsr_status;

/* Row-reduction operators for dcsr_row_reduce. */
enum { DCSR_REDUCE_SUM = 0, DCSR_REDUCE_MAX = 1, DCSR_REDUCE_MIN = 2, DCSR_REDUCE_COUNT = 3 };

/* Layout policy (all integers so the CPU oracle restates it exactly).
 * Row capacity on load/compaction: align_up(max(ceil(len*factor_x16/16),
 * min_cap, len), align).  A MERGE-mode row that outgrows its chain gets a new
 * segment of policy_cap(new_len) - current_capacity; an APPEND-mode row gets
 * rlB - free + alpha (reference include/sparse_update.inl:93-105).  The pool
 * is sized top + max(top*spare_x16/16, min_spare) on load. */
typedef struct {
  int32_t max_segs;   /* segment layers per row, 1..4 (reference MAX_OFFSET=4) */
  int32_t factor_x16; /* per-row slack factor in 1/16 (32 = 2x) */
  int32_t min_cap;    /* minimum row capacity */
  int32_t align;      /* capacity alignment in entries (power of two) */
  int32_t alpha;      /* APPEND-mode extra slack per new segment (reference: 4) */
  int32_t spare_x16;  /* pool spare capacity in 1/16 of the laid-out size */
  int32_t min_spare;  /* minimum pool spare, entries */
  int32_t mode;       /* DCSR_MERGE (canonical) or DCSR_APPEND (reference) */
  int32_t reloc_min;  /* MERGE: a row whose in-place merge would shift more than
                         reloc_min entries -- or that outgrows a chain already
                         max_segs segments long -- is instead merged out of
                         place into one fresh segment of policy_cap(new_len)
                         (chain reset); MERGE updates therefore never report
                         LAYER_OVERFLOW */
} dcsr_opts;

/* Snapshot of a matrix's device layout (device pointers). */
typedef struct {
  int32_t n_rows, n_cols, dtype, pitch;
  int64_t pool_cap;
  int32_t *row_sizes;
  int32_t *seg;
  int32_t *cols;
  void *vals;
  dcsr_opts opts;
} dcsr_info_t;

/* ------------------------------------------------------------ lifecycle */

/* Default policy for a mode: MERGE = 2x slack, 16-byte aligned segments;
 * APPEND = the reference's tight load/compaction with alpha = 4. */
void dcsr_default_opts(dcsr_opts *opts, int32_t mode);

/* Replaces dcsr_matrix::resize (reference include/dcsr_matrix.h:41-108) and
 * device::Initialize_Matrix (include/load.h:8-22).  opts may be NULL. */
int dcsr_create(dcsr_handle *out, int32_t n_rows, int32_t n_cols, int32_t dtype, const dcsr_opts *opts);
/* Replaces ~dcsr_matrix (include/dcsr_matrix.h:35-39). */
int dcsr_destroy(dcsr_handle h);
int dcsr_info(dcsr_handle h, dcsr_info_t *info);
/* Copy the layout (row_sizes[n_rows+1], seg[max_segs*pitch]) into caller
 * buffers (host or device; either pointer may be NULL).  Synchronises. */
int dcsr_get_layout(dcsr_handle h, int32_t *row_sizes, int32_t *seg, void *stream);

/* ----------------------------------------------------------- conversion */

/* CSR -> DCSR.  Replaces device::LoadMatrix(dcsr, csr) (include/load.h:207-227).
 * In MERGE mode unsorted rows / duplicate columns are canonicalised
 * (duplicates summed in input order).  Synchronises the stream once. */
int dcsr_from_csr(dcsr_handle h, const int32_t *row_ptr, const int32_t *cols, const void *vals, int64_t nnz,
                  void *stream);
/* COO -> DCSR (any order).  Replaces device::LoadMatrix(dcsr, rows, cols, vals, N)
 * (include/load.h:27-59, which required row-sorted input).  Synchronises once. */
int dcsr_from_coo(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                  void *stream);
/* HYB (ELL column-major with -1 padding + COO overflow) -> DCSR.  Replaces
 * the reference's HYB -> COO -> DCSR route (include/load.h:61-106,174-205). */
int dcsr_from_hyb(dcsr_handle h, const int32_t *ell_cols, const void *ell_vals, int32_t ell_width,
                  int64_t ell_pitch, const int32_t *coo_rows, const int32_t *coo_cols, const void *coo_vals,
                  int64_t coo_nnz, void *stream);

/* DCSR -> HYB (ELL + COO overflow, the reference's hyb_matrix and its
 * LoadMatrix(hyb, csr), include/dcsr_matrix.h:149-172, include/load.h:174-205).
 * Each row's first ell_width entries (in DCSR order) go to the ELL part,
 * column-major: slot k of row r at ell_cols[k*ell_pitch + r] (ell_pitch >=
 * n_rows); unused slots get column -1 and value 0.  The remaining entries go
 * to the COO part in row order; *coo_nnz (host) receives their count, and the
 * call returns DCSR_BAD_ARG without writing anything when it exceeds coo_cap
 * (dcsr_hyb_overflow gives the count first).  Synchronises once. */
int dcsr_hyb_overflow(dcsr_handle h, int32_t ell_width, int64_t *coo_nnz, void *stream);
int dcsr_to_hyb(dcsr_handle h, int32_t ell_width, int64_t ell_pitch, int32_t *ell_cols, void *ell_vals,
                int32_t *coo_rows, int32_t *coo_cols, void *coo_vals, int64_t coo_cap, int64_t *coo_nnz, void *stream);
/* y = alpha*A*x + beta*y for a HYB matrix in that layout (COO part sorted by
 * row; beta == 0 does not read y).  A row's ELL products are summed in slot
 * order, then its COO products in order.  Replaces device::spmv(hyb, x, y)
 * (include/spmv.h:36-94, spmv_hyb include/spmv.inl:105-156). */
int dcsr_hyb_spmv(int32_t n_rows, int32_t dtype, int32_t ell_width, int64_t ell_pitch, const int32_t *ell_cols,
                  const void *ell_vals, int64_t coo_nnz, const int32_t *coo_rows, const int32_t *coo_cols,
                  const void *coo_vals, const void *x, void *y, double alpha, double beta, void *stream);

/* Append update triples to a HYB matrix in that layout, in place (replaces
 * device::UpdateMatrix(hyb, rows, cols, vals, N), include/load.h:327-373,
 * kernel UpdateMatrix_hyb include/sparse_update.inl:321-366).  The triples
 * are taken in row order -- a stable sort by row, so a row's triples keep
 * their input order (the reference requires input sorted by row) -- and each
 * goes to its row's next free ELL slot (the ELL part's filled slots are a
 * prefix, as dcsr_to_hyb and this call leave them), or, once the row's ELL
 * part is full, to the COO part, which stays sorted by row with a row's
 * earlier COO entries first (the reference appends with atomics, then sorts
 * the COO part by row).  No duplicate check (the reference's HYB update
 * appends).  *coo_nnz: the COO part's entries, in and out.  DCSR_BAD_INDEX
 * for a row outside [0, n_rows) or a column outside [0, n_cols),
 * DCSR_POOL_EXHAUSTED when the COO part would exceed coo_cap (the reference
 * writes past its end); both leave the matrix unchanged.  Synchronises once. */
int dcsr_hyb_update(int32_t n_rows, int32_t n_cols, int32_t dtype, int32_t ell_width, int64_t ell_pitch,
                    int32_t *ell_cols, void *ell_vals, int32_t *coo_rows, int32_t *coo_cols, void *coo_vals,
                    int64_t coo_cap, int64_t *coo_nnz, const int32_t *rows, const int32_t *cols, const void *vals,
                    int64_t nnz, void *stream);

/* Number of stored entries (synchronises).  Use before dcsr_to_csr. */
int dcsr_nnz(dcsr_handle h, int64_t *nnz, void *stream);
/* DCSR -> CSR in row order, any state (chains followed).  Replaces
 * device::LoadMatrix(csr, dcsr) + DCSRtoCSROffsets (include/load.h:232-253,
 * include/sparse_update.inl:1101-1116).  Output arrays hold n_rows+1 / nnz. */
int dcsr_to_csr(dcsr_handle h, int32_t *row_ptr, int32_t *cols, void *vals, void *stream);
/* DCSR -> COO in row order (rows, cols, vals of length nnz). */
int dcsr_to_coo(dcsr_handle h, int32_t *rows, int32_t *cols, void *vals, void *stream);

/* Binary snapshot and restore (Matrix Market / checkpoint IO; the
 * reference keeps matrices in device memory only and reads text files with
 * ReadMatrixFile, include/load_matrix.h:48-119).  The image is a fixed
 * header (magic "DCSRSNP1", shape, dtype, layout policy, pitch, pool
 * capacity, pool top) followed by row_sizes[n_rows+1], seg[max_segs*pitch]
 * and the pool's cols/vals up to its top.  Restoring it reproduces the layout
 * bit for bit (row lengths, every segment pair, pool capacity and contents),
 * so a compacted or chained matrix comes back exactly as it was saved.
 * All three synchronise the stream; buffers are host memory. */
int dcsr_snapshot_bytes(dcsr_handle h, int64_t *bytes, void *stream);
int dcsr_snapshot(dcsr_handle h, void *host_buf, int64_t buf_bytes, void *stream);
/* Shape, dtype and policy stored in an image (to create the handle to
 * restore into); DCSR_BAD_ARG if the buffer is not a snapshot. */
int dcsr_snapshot_header(const void *host_buf, int64_t buf_bytes, int32_t *n_rows, int32_t *n_cols, int32_t *dtype,
                         dcsr_opts *opts);
/* Into a handle of the image's shape, dtype and max_segs (its policy is set
 * from the image); the handle's previous content is replaced. */
int dcsr_restore(dcsr_handle h, const void *host_buf, int64_t buf_bytes, void *stream);

/* -------------------------------------------------------------- updates */

/* In-place batch update with COO triples in any order.  Replaces
 * device::UpdateMatrix (include/load.h:258-325) + UpdateMatrix_dcsr
 * (include/sparse_update.inl:16-130).  MERGE: duplicate (row,col) pairs are
 * summed into the existing entry in batch order; APPEND: reference append.
 * Asynchronous: all-or-nothing, a rejection (POOL_EXHAUSTED, LAYER_OVERFLOW,
 * BAD_INDEX) leaves the matrix unchanged and is reported by dcsr_get_status. */
int dcsr_update(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                void *stream);
/* dcsr_update plus the repair policy: on rejection compact and retry, then
 * grow the pool and retry.  Synchronises; returns the final status. */
int dcsr_update_sync(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                     void *stream);
/* Read (and clear) the device status of the last asynchronous calls. */
int dcsr_get_status(dcsr_handle h, void *stream, int32_t *status);
/* Defragment into a fresh pool, rows in row order with policy capacities.
 * Replaces device::SortMatrixRow (include/load.h:404-581). */
int dcsr_compact(dcsr_handle h, void *stream);
/* Grow the pool to at least pool_cap entries (contents kept). */
int dcsr_reserve(dcsr_handle h, int64_t pool_cap, void *stream);
/* Recompute the SpMV row bins.  Replaces device::BinRows (include/load.h:583-610);
 * bins live in the handle (no process-global __constant__ table). */
int dcsr_bin_rows(dcsr_handle h, void *stream);
/* Row-class thresholds of the row passes (SpMV, reductions, export): rows of
 * at most short_max entries are streamed by 32-row blocks, rows above
 * long_min are split into CTA chunks, the others get a warp each.  Defaults
 * 64 / 512 (on a power-law graph rows of 512..4096 entries run about 1.3x
 * faster in CTA chunks than one warp each); 1 <= short_max <= 256,
 * max(short_max, 256) <= long_min <= 2^20.
 * The classes change only the order of floating-point additions: every path
 * (per call, batched, served) uses the handle's thresholds, so they agree
 * bit for bit.  The reference's bins are fixed (include/sparse_update.inl:1121-1150). */
int dcsr_set_row_classes(dcsr_handle h, int32_t short_max, int32_t long_min);
int dcsr_get_row_classes(dcsr_handle h, int32_t *short_max, int32_t *long_min);

/* ------------------------------------------------------------ operators */

/* Y = alpha*A*X + beta*Y with k (1..8) right-hand sides; X is n_cols x k
 * row-major with row stride ldx (X[c*ldx + j]), Y is n_rows x k with stride
 * ldy; values of the matrix dtype.  beta == 0 does not read Y.  Replaces
 * device::spmv(dcsr, x, y, streams) (include/spmv.h:121-248). */
int dcsr_spmv(dcsr_handle h, const void *x, int32_t k, int64_t ldx, void *y, int64_t ldy, double alpha,
              double beta, void *stream);
/* y[r] = op over row r's entries (sum / max / min / count).  The reference
 * computes row sums as SpMV with x = 1. */
int dcsr_row_reduce(dcsr_handle h, int32_t op, void *y, void *stream);
/* C = A*B.  C must be a handle created with n_rows = A.n_rows, n_cols =
 * B.n_cols and A's dtype; its content is replaced.  Rows sorted, explicit
 * zeros kept, all rows computed.  Replaces device::spmm (include/spmm.h:30-391).
 * Synchronises twice: after counting products (to size the staging area and
 * an upper bound of C's pool) and at the end (C's pool top); C's rows are
 * written straight into C's pool. */
int dcsr_spgemm(dcsr_handle A, dcsr_handle B, dcsr_handle C, void *stream);

/* Conjugate gradient on a symmetric positive definite matrix (square),
 * unpreconditioned: the solver the reference tree ships for its matrices
 * (cusp::krylov::cg, cusp/krylov/detail/cg.inl) with cusp::monitor's stop
 * rule (cusp/detail/monitor.inl: stop when ||r||_2 <= abs_tol +
 * rel_tol*||b||_2, tested before every iteration, or after max_iter
 * iterations; cusp's defaults are 500, 1e-5 and 0).  b and x are device
 * vectors of the matrix dtype; x holds the initial guess on entry and the
 * iterate on return.  *iters / *resid (host, may be NULL) receive the
 * iteration count and the last residual norm.  Every step runs on the device
 * (the SpMV is dcsr_spmv's); the host reads the stop flag between chunks of
 * iterations.  Synchronises. */
int dcsr_cg(dcsr_handle A, const void *b, void *x, int32_t max_iter, double rel_tol, double abs_tol, int32_t *iters,
            double *resid, void *stream);

/* X[I[n]] += 1 for a sorted index array I.  Replaces
 * device::count_sorted_indices (include/primitives.h:417-464). */
int dcsr_count_sorted_indices(const int32_t *I, int64_t n, int32_t *X, void *stream);
/* Reduce-by-key over sorted int32 keys; writes the unique count to *n_out
 * (device pointer).  Each run is summed in a fixed order: left to right
 * within pieces of at most 256 keys (a piece starts at the run's head or at
 * a multiple of 256), then the piece sums left to right -- deterministic,
 * and a long run is summed by many threads.  Replaces the CTA/global
 * reduce-by-key of include/reduce.inl:139-308, include/reduce_global.inl. */
int dcsr_reduce_by_key(const int32_t *keys, const void *vals, int64_t n, int32_t dtype, int32_t *keys_out,
                       void *vals_out, int64_t *n_out, void *stream);

/* ------------------------------------------------------- batched form */

/* One matrix's work in a batch: an update batch (nnz may be 0) followed by
 * Y = alpha*A*X + beta*Y (x == NULL: no SpMV).  Pointers are device pointers
 * that stay valid for the batch's lifetime (a captured graph replays them). */
typedef struct {
  dcsr_handle matrix;
  const int32_t *rows;
  const int32_t *cols;
  const void *vals;
  int64_t nnz;
  const void *x;
  void *y;
  int32_t k;
  int64_t ldx, ldy;
  double alpha, beta;
} dcsr_batch_item;

typedef struct dcsr_batch_s *dcsr_batch;

/* A batch over `count` matrices of one dtype and mode (each matrix at most
 * once).  The reference has no batched form; it would run count separate
 * UpdateMatrix + spmv sequences (include/load.h:258, include/spmv.h:121). */
int dcsr_batch_create(dcsr_batch *out, const dcsr_batch_item *items, int32_t count, void *stream);
/* Enqueue the batch: one merged update over all matrices (one sort, one
 * plan, one apply for the union of their triples) then one SpMV pass per
 * distinct k.  Asynchronous; per-matrix rejections are read with
 * dcsr_batch_status.  Results equal the per-call operators bit for bit. */
int dcsr_batch_run(dcsr_batch b, void *stream);
/* Capture dcsr_batch_run into a CUDA graph (instantiated once). */
int dcsr_batch_capture(dcsr_batch b, void *stream);
/* Launch the captured graph (one launch for the whole batch). */
int dcsr_batch_launch(dcsr_batch b, void *stream);
/* Per-matrix statuses of the last run (synchronises, clears them). */
int dcsr_batch_status(dcsr_batch b, int32_t *statuses, void *stream);
/* After dcsr_batch_status (and dcsr_batch_repair): grow, stream-ordered, the
 * pool of every matrix whose accepted update left less room than
 * max(pool / 8, 2 x run), run = the larger of the pool top's growth since the
 * previous call and its triple count (its next update has as many triples),
 * to twice that room, and the pool of every rejected (repaired) one by twice
 * its triple count, so the next runs' updates are not rejected for space and
 * need no repair.  Contents, row lengths, segment tables and the pool top
 * are unchanged; only the pool capacity grows.  *grown (may be NULL) =
 * matrices grown. */
int dcsr_batch_grow(dcsr_batch b, int32_t *grown, void *stream);
/* For matrices whose update was rejected: apply the repair policy
 * (compact, grow) and redo their update and SpMV per call.  Returns the
 * number of matrices repaired in *repaired (may be NULL). */
int dcsr_batch_repair(dcsr_batch b, const int32_t *statuses, int32_t *repaired, void *stream);
int dcsr_batch_destroy(dcsr_batch b);
/* Autotune the batch's row schedule: time the batch's schedule rebuild +
 * SpMV passes (outputs to scratch: the matrices' contents and the items' y
 * are not touched) for a grid of row-class thresholds (short_max x long_min),
 * then, under the best of those, for the warps per 32-row short-row block of
 * the k >= 2 passes (1, 2, 4, 8 against the automatic rule).  Sets the
 * fastest thresholds on every matrix and the split on the batch (a captured
 * graph must be captured again to use them), returns the thresholds
 * (best_us: the best time per run).  The split never changes a result; the
 * thresholds move rows between classes, which sum in different orders.
 * Synchronises. */
int dcsr_batch_autotune(dcsr_batch b, void *stream, int32_t *short_max, int32_t *long_min, float *best_us);
/* The short-row split the autotuner chose (0: the automatic rule, which
 * doubles warps per block up to 8 while the blocks stay under 12 warps per
 * SM). */
int dcsr_batch_short_split(dcsr_batch b, int32_t *split);

/* ------------------------------------------------------------ serving */

/* A request server over a table of resident matrices.  Requests (update,
 * SpMV, export) carry HOST buffers; worker threads admit queued requests
 * while their device memory fits the budget, coalesces them into batches
 * (merged update + grouped SpMV through the batched kernels, then exports),
 * keeps up to `depth` batches in flight on separate streams, and refills
 * slots as batches retire (continuous batching).  Per matrix, requests take
 * effect in submission order: a matrix is in at most one in-flight batch, and
 * within a batch its update precedes its SpMV.  A rejected update is repaired
 * (compact, grow, retry) before its result is reported, and pools nearing
 * full are grown ahead of the next update.  The reference has no serving
 * layer; its callers loop over UpdateMatrix / spmv (src/Fill_Test.inl). */
typedef struct dcsr_server_s *dcsr_server;

typedef struct {
  int32_t max_batch;   /* requests coalesced into one batch (default 256) */
  int32_t depth;       /* batches in flight, one stream each (default 8, at most 16) */
  int64_t mem_budget;  /* device bytes in-flight requests may hold; 0: free memory at creation - mem_reserve */
  int64_t mem_reserve; /* default 1 GiB */
  int32_t plain;       /* 1: no coalescing -- each request alone through the per-call operators */
  int32_t workers;     /* host threads forming and launching batches, each owning every workers-th
                          stream (default 2, 1..8, at most depth; plain uses 1) */
} dcsr_server_opts;

enum { DCSR_REQ_UPDATE = 0, DCSR_REQ_SPMV = 1, DCSR_REQ_EXPORT = 2 };

typedef struct {
  int32_t kind;   /* DCSR_REQ_* */
  int32_t matrix; /* index into the server's matrix table */
  /* UPDATE: nnz host triples (merged / appended by the matrix's mode) */
  const int32_t *rows;
  const int32_t *cols;
  const void *vals;
  int64_t nnz;
  /* SPMV: y = alpha*A*x + beta*y, host x [n_cols x k], y [n_rows x k] row-major */
  const void *x;
  void *y;
  int32_t k;
  double alpha, beta;
  /* EXPORT: host CSR of the matrix: row_ptr [n_rows+1], cols/vals with room for cap entries */
  int32_t *row_ptr;
  int32_t *out_cols;
  void *out_vals;
  int64_t cap;
  /* 1: every buffer of this request is device memory (no host staging) */
  int32_t on_device;
} dcsr_request;

typedef struct {
  int32_t status;     /* DCSR_OK, the update's final status, BAD_ARG if cap < nnz */
  int32_t batch_size; /* requests in the batch that served it */
  int64_t nnz;        /* EXPORT: entries of the matrix */
  double queue_us;    /* submit -> launch */
  double latency_us;  /* submit -> result in host memory */
} dcsr_result;

void dcsr_server_default_opts(dcsr_server_opts *o);
/* Host buffers of a request must stay valid (and unread / unwritten by the
 * caller) until its result is taken with dcsr_server_wait.  The matrices must
 * not be used outside the server while it runs. */
int dcsr_server_create(dcsr_server *out, const dcsr_handle *matrices, int32_t count, const dcsr_server_opts *opts);
/* Thread-safe, non-blocking: queue a request, return its ticket. */
int dcsr_server_submit(dcsr_server s, const dcsr_request *req, uint64_t *ticket);
/* Wait (at most timeout_us; < 0: forever) for a ticket's result and forget
 * the ticket.  DCSR_TIMEOUT if it has not completed. */
int dcsr_server_wait(dcsr_server s, uint64_t ticket, int64_t timeout_us, dcsr_result *out);
/* Counters: completed requests, batches launched, budget bytes in use. */
int dcsr_server_stats(dcsr_server s, int64_t *completed, int64_t *batches, int64_t *mem_in_use);
/* Drain the queue, stop the workers, release the server (not the matrices). */
int dcsr_server_destroy(dcsr_server s);
/* Load generator for measurements: submit requests[i] at arrival_us[i]
 * microseconds after the call starts (non-decreasing), then wait for all;
 * results[i] receives each result with its latency counted from the
 * scheduled arrival (a late submission is not forgiven); *wall_us = the time
 * from the start to the last completion. */
int dcsr_server_replay(dcsr_server s, const dcsr_request *requests, const double *arrival_us, int64_t count,
                       dcsr_result *results, double *wall_us);

/* Allocation-free reduce-by-key.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory at call time -- a process
 * that has carved the GPU's memory into fixed budgets up front, or code whose
 * allocator is not CUDA's and must not have the CUDA allocator (which can
 * synchronise the device) run underneath it.  Same result as
 * dcsr_reduce_by_key; its scratch is a static device array compiled into the
 * library (about 8 MiB per GPU that loads it, held until process exit), so
 * n is limited to DCSR_NOALLOC_MAX_KEYS (larger n returns DCSR_BAD_ARG
 * without touching the GPU).  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  The address is kept for
 * the life of the process: do not use this entry point on a device after
 * cudaDeviceReset there.  All calls share the one array: calls that overlap
 * on the GPU (different streams, or threads without ordering) race and must
 * be serialised by the caller. */
#define DCSR_NOALLOC_MAX_KEYS (1 << 20)
int dcsr_reduce_by_key_noalloc(const int32_t *keys, const void *vals, int64_t n, int32_t dtype, int32_t *keys_out,
                               void *vals_out, int64_t *n_out, void *stream);

/* ---------------------------------------------------------------- misc */

const char *dcsr_status_string(int status);
/* Number of CUDA kernels this library has launched in this process. */
uint64_t dcsr_launch_count(void);
/* Waits of the single-pass scan and sort kernels (decoupled look-back) on
 * the current device that reached their iteration limit and gave up, since
 * the library was loaded.  Each such wait is on an earlier tile that is
 * running or finished, so a non-zero count indicates a library bug (the
 * affected result is wrong; nothing hangs).  Synchronises the device.  No
 * counterpart in the reference (its scans and sorts come from Thrust/CUB). */
int dcsr_spin_faults(int64_t *count);
/* Failure-handling test hook (no counterpart in the reference).  Sets the
 * iteration limit of the look-back waits (spin_limit <= 0 restores the
 * default, about a second) and, with stall_first_tile != 0, keeps the first
 * tile of every single-pass scan and sort from publishing its prefix, so the
 * waits on it run out: each such wait gives up after the limit, the kernel
 * finishes (its result is wrong) and the operation's status word -- read by
 * dcsr_get_status, dcsr_batch_status, or returned by the synchronising
 * calls -- reports DCSR_TIMEOUT.  Nothing hangs and no GPU fault is raised.
 * For tests only; synchronises the device; not thread-safe with running
 * operations. */
int dcsr_debug_lookback(int32_t spin_limit, int32_t stall_first_tile);
/* Make sure at least `bytes` of device memory reserved for this library are
 * free on the current device: when the reserved regions have less free, a
 * new region of the difference is mapped (on `stream`, then synchronised)
 * and kept for the life of the process.  Every matrix pool, schedule,
 * scratch arena and staging buffer of the library is then carved from the
 * regions (best fit, 256-byte aligned); a block freed on one stream is
 * reused on another after an event wait on the device, with no host sync.
 * Only a request the regions cannot hold goes to the driver's
 * stream-ordered allocator (counted by dcsr_pool_usage).  Growing a matrix
 * (compaction, repair, grow-ahead) or staging a large batch then maps no
 * device memory: a driver allocation that maps new memory measured from 2 to
 * several hundred milliseconds on busy hosts.  Without a call, all
 * allocations go to the driver's allocator.  Regions are not used inside a
 * stream capture, and are kept for the life of the process: do not use the
 * library on a device after cudaDeviceReset there.  No counterpart in the
 * reference (host memory). */
int dcsr_pool_reserve(int64_t bytes, void *stream);
/* The current device's reserved regions: bytes mapped, bytes free (blocks
 * whose last user's work may still be running count as free), and how many
 * allocations the regions could not hold and the driver's allocator made
 * instead.  Any pointer may be null.  No counterpart in the reference. */
int dcsr_pool_usage(int64_t *reserved, int64_t *free_bytes, int64_t *fallback_allocs);
/* Measurement aid for the SpMV roofline (no counterpart in the reference):
 * reads n (column, value) entries -- e.g. a matrix's CSR export, FP32 --
 * coalesced and gathers x at every column, summing the products per block
 * into out[0 .. min(out_len, 8 * SMs)).  The memory traffic of a k = 1 SpMV
 * of those entries without its row bookkeeping: the time it takes is a floor
 * for that SpMV on this GPU (the random 4-byte reads of x are the part HBM
 * bandwidth does not cover).  Asynchronous. */
int dcsr_measure_gather(const int32_t *cols, const float *vals, int64_t n, const float *x, float *out,
                        int32_t out_len, void *stream);
/* Library version string. */
const char *dcsr_version(void);

#ifdef __cplusplus
}
#endif
#endif
