/*
 * dcsr_oracle.h -- CPU restatement of the Dynamic-CSR (DCSR) operators.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA library
 * in dcsr_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it; the product path never links or calls it.
 *
 * It restates the reference's DCSR algorithms (Vizerai/DCSR, include/ *.inl)
 * with the canonical semantics the library states where the reference is
 * defective (no duplicate merge, no overflow guard, stale bins, bin-ordered
 * compaction).  Every function cites the reference lines it follows.
 *
 * Parity pinning: the merge/append/SpMV/SpGEMM results are cross-checked
 * against the reference's own cusp host path (oracle/ref_cusp.cpp compiled
 * against the reference tree into oracle/_ref/) and against committed golden
 * vectors generated from it (tests/golden/make_golden.py).  The DCSR segment
 * layout itself (capacities, allocation addresses) has no runnable reference
 * (the GPU code does not build for sm_100a); it is restated from
 * include/sparse_update.inl and pinned only by this restatement.
 *
 * Layout (shared with the CUDA library, reference include/dcsr_matrix.h:9-73):
 *   row_sizes[n_rows+1]   logical row lengths; row_sizes[n_rows] = pool top
 *   seg[max_segs*pitch]   (start,end) pairs, seg[l*pitch + 2*r + {0,1}],
 *                         pitch = align_up(2*n_rows, 32); unused = (-1,-1)
 *   cols[pool_cap], vals[pool_cap]  the entry pool
 */
#ifndef DCSR_ORACLE_H
#define DCSR_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { OR_F32 = 0, OR_F64 = 1 };
enum { OR_MERGE = 0, OR_APPEND = 1 };
enum {
  OR_OK = 0,
  OR_POOL_EXHAUSTED = 1,
  OR_LAYER_OVERFLOW = 2,
  OR_BAD_INDEX = 3,
  OR_BAD_ARG = 5
};

typedef struct {
  int32_t max_segs;      /* segment layers per row (reference BINS=MAX_OFFSET=4) */
  int32_t factor_x16;    /* slack factor in 1/16 units (32 = 2x per-row slack) */
  int32_t min_cap;       /* minimum per-row capacity on load/compaction */
  int32_t align;         /* capacity alignment in entries (power of two) */
  int32_t alpha;         /* APPEND mode extra slack per new segment (ref: 4) */
  int32_t spare_x16;     /* pool spare beyond the laid-out capacity, 1/16 units */
  int32_t min_spare;     /* minimum pool spare, entries */
  int32_t mode;          /* OR_MERGE (canonical) or OR_APPEND (reference compat) */
  int32_t reloc_min;     /* MERGE: rows shifting > reloc_min entries relocate */
} or_opts;

typedef struct {
  int32_t n_rows, n_cols, dtype, pitch;
  or_opts o;
  int64_t pool_cap;
  int32_t *row_sizes;
  int32_t *seg;
  int32_t *cols;
  double *vals;   /* stored in double; F32 matrices round every op to float */
} or_dcsr;

void or_default_opts(or_opts *o, int mode);
or_dcsr *or_create(int32_t n_rows, int32_t n_cols, int32_t dtype, const or_opts *o);
void or_destroy(or_dcsr *m);

/* Policy helpers (exposed so tests can check the GPU side's arithmetic). */
int64_t or_policy_cap(const or_opts *o, int64_t len);
int64_t or_pool_capacity(const or_opts *o, int64_t top);

/* Load from CSR / COO.  Returns status. */
int or_load_csr(or_dcsr *m, const int32_t *row_ptr, const int32_t *cols, const double *vals);
int or_load_coo(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals, int64_t nnz);

/* One update attempt: all-or-nothing. *need (optional) = pool top required. */
int or_update(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals,
              int64_t nnz, int64_t *need);
/* Update with the library's repair policy: compact + retry, then grow + retry. */
int or_update_auto(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals,
                   int64_t nnz);
void or_compact(or_dcsr *m);
void or_grow(or_dcsr *m, int64_t new_cap);

int64_t or_nnz(const or_dcsr *m);
/* Export the logical content in row order: row_ptr[n+1], cols[nnz], vals[nnz]. */
void or_export_csr(const or_dcsr *m, int32_t *row_ptr, int32_t *cols, double *vals);

/* y[r*ldy+j] = alpha*sum_e a_e*x[c_e*ldx+j] + beta*y  (FP64 accumulate, FP64 out) */
void or_spmv(const or_dcsr *m, const double *x, int32_t k, int64_t ldx, double *y, int64_t ldy,
             double alpha, double beta);
/* op 0 = sum, 1 = max, 2 = min, 3 = count of stored entries */
void or_row_reduce(const or_dcsr *m, int32_t op, double *y);

/* C = A*B into a new matrix created with options *o (C layout per its policy).
 * Explicit zeros are kept; rows are sorted; sums run in product order. */
or_dcsr *or_spgemm(const or_dcsr *A, const or_dcsr *B, const or_opts *o, int *status);
/* Per-row product counts sum_{k in A_i} |B_k| (reference CalcSortSizes_SPMM). */
void or_spgemm_counts(const or_dcsr *A, const or_dcsr *B, int64_t *counts);

/* X[I[n]] += 1 for sorted I (reference include/primitives.h:417-464). */
void or_count_sorted_indices(const int32_t *I, int64_t n, int32_t *X);
/* Reduce-by-key over sorted keys: each run summed in pieces of 256 keys (from
 * its head and from each multiple of 256), left to right within a piece, then
 * the piece sums left to right.  Returns the unique count. */
int64_t or_reduce_by_key(const int32_t *keys, const double *vals, int64_t n, int32_t dtype,
                         int32_t *out_keys, double *out_vals);

/* Row bins {<2,<4,<8,<16,<32,<512,>=512} (reference SetBins,
 * include/sparse_update.inl:1121-1150); counts[7]. */
void or_bin_counts(const or_dcsr *m, int64_t *counts);

/* Structural self-check: returns 0 if consistent, else a negative code. */
int or_validate(const or_dcsr *m);

#ifdef __cplusplus
}
#endif
#endif
