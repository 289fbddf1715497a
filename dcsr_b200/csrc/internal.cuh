// internal.cuh -- cross-file internal API of the DCSR library.
#pragma once
#include "common.cuh"

namespace dcsr {

// Lay out a matrix from a CSR whose row_ptr is int64 on the device (rows
// already canonical for the handle's mode): policy capacities, fresh pool,
// content copy.  Synchronises once (pool size).
int load_from_csr64(dcsr_handle h, const long long *rp, const int32_t *cols, const void *vals, cudaStream_t s);
size_t load_scratch_bytes(dcsr_handle h);

// Sort + group a COO batch (any order) into CSR form in the arena:
// MERGE: sorted by (row, col), duplicates summed in input order;
// APPEND: stably sorted by row.  *rp has n_rows+1 entries.  Sets BAD_INDEX in
// *bad (device int) for out-of-range input.
int coo_to_csr64(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz, bool merge,
                 Arena &ar, long long **rp, int32_t **ocols, void **ovals, int *bad, cudaStream_t s);
size_t coo_to_csr_scratch(dcsr_handle h, int64_t nnz);

int update_async(dcsr_handle h, const int32_t *rows, const int32_t *cols, const void *vals, int64_t nnz,
                 cudaStream_t s);
int compact(dcsr_handle h, cudaStream_t s);
int build_schedule(dcsr_handle h, cudaStream_t s);
int ensure_part(dcsr_handle h, int K, cudaStream_t s);
// Copy every row's logical entries to dst_off[r] (optionally COO row ids and
// an int32 row pointer).  Builds the schedule first if needed (so callers
// must not hold arena memory across this call unless the schedule is valid).
int copy_rows(dcsr_handle h, const long long *dst_off, int32_t *out_cols, void *out_vals, int32_t *out_rows,
              int32_t *out_rowptr, cudaStream_t s);
int reserve(dcsr_handle h, int64_t cap, cudaStream_t s);

}  // namespace dcsr
