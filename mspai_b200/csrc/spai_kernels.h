// Launch interface of the batched MSPAI setup kernels (host side).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace mspai {

struct Problem;
struct Output;
struct Caps;

constexpr int kWarpKernelThreads = 256;  // 8 warps, one column each

// How columns are binned (see bucket_kernel).
struct BucketRule {
    int single_bucket;     // >= 0: every column goes to this bucket
    int allow_warp;        // tiny bucket enabled
    int warp_emax;         // tiny: entries of C(:,J) (after growth)
    int warp_nmax;         // tiny: |J| (after growth)
    int64_t smem_w_bytes;  // bucket 1 if the folded matrix fits in this
    int elem_bytes;        // 4 (mixed) or 8 (FP64)
    int grow_n;            // mn * ns
    int grow_e;            // mn * ns * max column nnz of C
    const int32_t* rep;    // reuse table: columns with rep[k] != k are skipped (nullable)
    int lo, hi;            // only problem columns [lo, hi) are binned
};

// Row structure (CSR) of a CSC matrix, in ascending column order within each
// row (apply.cu): tptr nrows + 1, tcol/tval nnz (tval may be null: structure
// only); keys_out, perm_in, perm_out nnz and cnt nrows are scratch; temp of
// rows_build_temp_bytes(nnz, nrows).
size_t rows_build_temp_bytes(int64_t nnz, int nrows);
cudaError_t launch_build_rows(const int64_t* ptr, const int32_t* idx, const double* val,
                              int ncols, int nrows, int64_t nnz, int64_t* tptr, int32_t* tcol,
                              double* tval, int32_t* keys_out, int32_t* perm_in, int32_t* perm_out,
                              int32_t* cnt, int64_t* scan_tmp, void* temp, size_t temp_bytes,
                              cudaStream_t st);
// y = M x from M's row structure, a fixed summation order per row
cudaError_t launch_csr_gather(const int64_t* tptr, const int32_t* tcol, const double* tval,
                              int nrows, const double* x, double* y, cudaStream_t st);

// Checks a CSC structure on the device (pointers, row range, sorted unique
// rows, optionally no empty column); the first error goes to err[0..2]
// (kind, column, row), which must start at zero.
cudaError_t launch_validate_csc(const int64_t* ptr, const int32_t* idx, int ncols, int nrows,
                                int64_t nnz, bool nonempty, int32_t* err, cudaStream_t st);

// E[k] = entries of C in the (scalar) columns of problem column k, nk[k] =
// its scalar pattern size (block pattern entries * bs)
cudaError_t launch_plan(const int64_t* cptr, const int64_t* pptr, const int32_t* pidx, int nprob,
                        int bs, int32_t* E, int32_t* nk, cudaStream_t st);
cudaError_t launch_bucket(const int32_t* E, const int32_t* nk, int n, const BucketRule& rule,
                          int32_t* counts, int32_t* maxE, int32_t* maxN, int32_t* lists,
                          cudaStream_t st);
size_t warp_slot_bytes(const Caps& cap, int elem_bytes);
// warp per column with the slots in global memory (scratch of
// warp_global_scratch_bytes; adaptive setups: cleared before the launch)
size_t warp_global_scratch_bytes(const Caps& cap, int elem_bytes, int count);
cudaError_t launch_warp_solve_global(int elem_bytes, const Problem& pb, const Caps& cap,
                                     const Output& out, const int32_t* list, int count,
                                     int32_t* counter, char* scratch, size_t scratch_bytes,
                                     cudaStream_t st, int* grid_out);
size_t cta_slot_bytes(const Caps& cap, int elem_bytes, bool w_smem);
size_t w_bytes(const Caps& cap, int elem_bytes);
// CTAs per SM of the solver for this element size and shared-memory area
int cta_per_sm(int elem_bytes, size_t smem_w_bytes);
size_t cta_scratch_needed(int elem_bytes, const Caps& cap, int count, size_t smem_w_bytes);
cudaError_t launch_warp_solve(int elem_bytes, const Problem& pb, const Caps& cap,
                              const Output& out, const int32_t* list, int count, int32_t* counter,
                              cudaStream_t st, int* grid_out);
// One CTA per column; the folded matrix of a column lives in `smem_w_bytes`
// of shared memory when it fits there, else in the CTA's global scratch slot.
// `blocked` selects the blocked Householder QR (16-column panels).
cudaError_t launch_cta_solve(int elem_bytes, size_t smem_w_bytes, bool blocked,
                             const Problem& pb, const Caps& cap, const Output& out,
                             const int32_t* list, int count, int32_t* counter, char* scratch,
                             size_t scratch_bytes, cudaStream_t st, int* grid_out);
// Fixed-pattern scalar solver (fixed_kernels.cu): columns list[0 .. count)
// (count from count_dev when not null, else count_host); columns that do not
// fit the arena of arena_bytes go to ovf_list / *ovf_count.  rglob: per-CTA
// areas of rglob_elems elements for R when it does not fit the arena (null:
// such columns overflow).
int fixed_ctas_per_sm(int arena_bytes);
int fixed_max_grid(int arena_bytes);
int64_t fixed_r_elems(int nmax);
cudaError_t launch_fixed_solve(int elem_bytes, int arena_bytes, const Problem& pb,
                               const Output& out, const int32_t* list, const int32_t* count_dev,
                               int count_host, int32_t* counter, int32_t* ovf_list,
                               int32_t* ovf_count, void* rglob, int64_t rglob_elems, int max_ctas,
                               cudaStream_t st, int* grid_out);
cudaError_t launch_scan_lengths(const int32_t* len, int n, int64_t* ptr, int64_t* tmp,
                                cudaStream_t st);
// len[k] = |P(:, k)| (|P(:, k)| + 1) / 2 (packed triangles of the kept R)
// Adds an order-independent 64-bit digest of a CSC structure (pointers and
// row indices) to *acc.
cudaError_t launch_structure_hash(const int64_t* ptr, const int32_t* idx, int ncols, int64_t nnz,
                                  unsigned long long salt, unsigned long long* acc,
                                  cudaStream_t st);
cudaError_t launch_tri_len(const int64_t* pptr, int n, int32_t* len, cudaStream_t st);
cudaError_t launch_capacity_len(const int64_t* pptr, int n, int bs, int grow, int32_t* len,
                                cudaStream_t st);
cudaError_t launch_compact(const int64_t* cap_ptr, const int32_t* cidx, const double* cval,
                           const int64_t* out_ptr, int32_t* oidx, double* oval, int n,
                           cudaStream_t st);
cudaError_t launch_max_len(const int64_t* ptr, int n, int32_t* out, cudaStream_t st);

int num_sms();

// Reuse of identical least-squares problems (reuse.cu).
struct ReuseTable {
    uint64_t* keys;         // mask + 1 slots, 0 = empty
    int32_t* rep_of_slot;   // smallest column with the slot's key
    int32_t* slot_of;       // per column: its slot or -1
    int32_t* nkeys;         // distinct keys stored
    uint32_t mask;          // slots - 1 (power of two)
    int32_t max_keys;       // cache size: at most this many distinct problems
};
size_t reuse_table_slots(int nprob, int max_keys);
// rep[k] = the column whose solution column k takes (k: solved itself);
// *nreused = columns with rep[k] != k
cudaError_t launch_reuse_keys(const Problem& pb, int nprob, const ReuseTable& t, int32_t* rep,
                              int32_t* nreused, cudaStream_t st);
cudaError_t launch_reuse_copy(const int32_t* rep, int nprob, int bs, const Output& out,
                              cudaStream_t st);

// Adjoint of the setup (adjoint.cu): problem columns read their pattern and
// solutions from the result M.
struct AdjointIO {
    const int64_t* mptr;  // M (the setup's result): n + 1 pointers, scalar columns
    const int32_t* midx;
    const double* mval;
    const double* gbar;   // nnz(M) or null (scalar setups)
    const void* rstore;   // R kept by the setup (packed by columns) or null
    const int64_t* roff;
    int r_elem;           // 4 or 8: the element size of rstore
    double wres;          // weight of the residual term ||C M - B||_F^2
    double* dC;           // nnz(C), zero on entry
    double* dB;           // nnz(B) or null
    double* loss;         // per problem column
};
// E[k], nk[k] of problem column k from the result's pattern
cudaError_t launch_adjoint_plan(const int64_t* cptr, const int64_t* mptr, const int32_t* midx,
                                int nprob, int bs, int32_t* E, int32_t* nk, cudaStream_t st);
// problem columns [lo, hi) of the last setup
cudaError_t launch_adjoint(const Problem& pb, const Caps& cap, const AdjointIO& io, int lo,
                           int hi, bool warp, char* scratch, size_t scratch_bytes,
                           int32_t* counter, cudaStream_t st);
size_t adjoint_scratch_bytes(const Caps& cap, int n, bool warp);

}  // namespace mspai
