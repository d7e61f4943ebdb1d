/*
 * mspai_b200 -- B200-native MSPAI preconditioner setup, C ABI.
 *
 * The setup computes a sparse M minimising ||C M - B||_F column by column:
 * for every column k it solves the small dense least-squares problem
 *     min || C(I_k, J_k) m_k - B(I_k, k) ||_2
 * where J_k is the pattern of column k of M and I_k the rows C(:, J_k)
 * touches, optionally growing J_k by the SPAI pattern-update rule.  Plain SPAI
 * is C = A, B = I; MSPAI's probing form appends p weighted rows:
 * C = [A; rho Ce], B = [I; rho Be] (Ce = e^T A, Be = e^T).
 *
 * This header replaces the reference's setup seam
 *     Spai<double>* alg = Switch_Algorithm<double>::Get_Algorithm(...);
 *     alg->SPAI_Algorithm(A, M, B, P, UP, epsilon, maxnew, ns, hash, use_mean,
 *                         pre_k, pre_max, count, verbose);
 * (reference src/imspai.cpp:818-833, src/Spai.h:89-102, src/Spai.imp:33-191)
 * with plain pointers and sizes.  Conventions follow the reference: 0 is
 * success; parameter checks mirror src/imspai.cpp:238-480.  No exception
 * crosses this boundary.  Calls on one handle are not thread-safe; handles on
 * different streams may run concurrently.
 */
#ifndef MSPAI_B200_H
#define MSPAI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes. */
typedef enum {
    MSPAI_OK = 0,
    MSPAI_ERR_PARAM = 1,        /* invalid option or option combination    */
    MSPAI_ERR_INPUT = 2,        /* malformed matrix / pattern, empty column */
    MSPAI_ERR_SINGULAR = 3,     /* some column's R had a zero diagonal      */
    MSPAI_ERR_CAPACITY = 4,     /* a problem exceeds the supported size     */
    MSPAI_ERR_CUDA = 5,         /* CUDA runtime error                       */
    MSPAI_ERR_NO_DEVICE = 6,    /* no usable CUDA device                    */
    MSPAI_ERR_STATE = 7,        /* call out of order (e.g. no setup yet)    */
    MSPAI_ERR_IO = 8,           /* file could not be read or written        */
    MSPAI_ERR_ALLOC = 9         /* device or host allocation failed         */
} mspai_status;

/* Where the arrays of a mspai_csc live. */
typedef enum { MSPAI_MEM_HOST = 0, MSPAI_MEM_DEVICE = 1 } mspai_mem;

/* Arithmetic of the per-column least-squares solve. */
typedef enum {
    MSPAI_PREC_FP64 = 0,   /* FP64 Householder QR and solve                   */
    MSPAI_PREC_MIXED = 1   /* FP32 QR/solve + FP64 residual refinement steps  */
} mspai_precision;

/* Per-column status codes (mspai_column_info). */
typedef enum {
    MSPAI_COL_OK = 0,
    MSPAI_COL_SINGULAR = 1,   /* zero diagonal in R: m_k = (Q^T b)(0:n), as the
                                 reference's dtrtrs leaves it                  */
    MSPAI_COL_NONFINITE = 2,  /* a non-finite value in m_k or the residual    */
    MSPAI_COL_CAPACITY = 3    /* problem exceeded its workspace (not solved)  */
} mspai_column_status;

/*
 * Compressed sparse column matrix (also used for patterns: values == NULL).
 * Row indices are sorted ascending and unique within each column.
 */
typedef struct {
    int32_t nrows;
    int32_t ncols;
    int64_t nnz;
    const int64_t* colptr; /* ncols + 1 */
    const int32_t* rowidx; /* nnz */
    const double* values;  /* nnz, or NULL for a pattern */
    int32_t mem;           /* mspai_mem */
} mspai_csc;

/*
 * Options.  Names and defaults follow the reference's command line
 * (src/Command_Line.cpp:192-225, src/imspai.cpp:57-218).
 */
typedef struct {
    double ep;        /* -ep  residual tolerance per column (0.4)             */
    int32_t mn;       /* -mn  max new indices per update step (5)             */
    int32_t ns;       /* -ns  max update steps (5); 0 = fixed pattern         */
    int32_t um;       /* -um  1: candidates need rho <= mean, 0: <= sum (1)   */
    int32_t hs;       /* -hs  remote-column hash size 0..6 (accepted, unused) */
    int32_t cs;       /* -cs  cache size (0); > 0: reuse table of <= cs problems */
    int32_t qr;       /* -qr  0..5 QR-update mode (accepted; dense on GPU)    */
    int32_t ch;       /* -ch  0/1 reuse table without a size limit            */
    double fg;        /* -fg  fill grade for -qr 1 (accepted)                  */
    int32_t pk;       /* -pk  prefetch count (accepted, unused on one GPU)    */
    int32_t pm;       /* -pm  prefetch all (accepted, unused on one GPU)      */
    int32_t schur;    /* -schur 0/1                                            */
    double rho;       /* -rho probing weight (already applied to C and B)     */
    int32_t bs;       /* -bs  block size (1 = scalar SPAI)                    */
    int32_t target;   /* 1: B = I (or [I; rho Be]) given by the caller or
                         implied; 0: arbitrary target matrix                  */
    int32_t probing;  /* 1: C has probing rows n..nrows-1 (-Ce/-Be given)    */
    int32_t prec;     /* mspai_precision (MSPAI_PREC_MIXED)                   */
    int32_t refine;   /* at most this many FP64 refinement steps in mixed
                         mode (4); a column stops when its correction is
                         below 2^-44 of its solution or stops contracting */
    int32_t batched;  /* 1: size-bucketed batched kernels (default);
                         0: the plain per-column path (one CTA per column,
                         FP64, no buckets) -- the throughput baseline         */
    int32_t verbose;  /* -vb                                                   */
    int32_t col_begin, col_end; /* solve only problem columns [begin, end)
                         (0, 0: all); M's other columns are left empty or
                         zero.  Used to shard the columns over several GPUs;
                         not in the reference (its column ranges come from
                         the MPI distribution, src/Distribution.cpp:48-71) */
    int32_t keep_factors; /* 1: keep every column's triangular factor R in the
                         handle (fixed scalar patterns) for mspai_adjoint's
                         gbar term and for re-setups (reuse_factors) (0)   */
    int32_t reuse_factors; /* > 0: re-setup from the kept factors.  When C, P
                         and B have the structure of the last setup that kept
                         its factors (keep_factors, same precision), every
                         column of the fixed-pattern solver starts from its
                         previous solution and R and takes at most this many
                         FP64 refinement steps against the new values; a
                         column that does not converge is factored again.
                         The reference's update path keeps each column's QR
                         across setups (src/Spai_Update.imp:45-325); 0
                         recomputes every column (0)                       */
} mspai_params;

/* Per-setup statistics. */
typedef struct {
    int64_t columns;          /* columns solved                              */
    int64_t ls_solves;        /* least-squares problems solved (all steps)   */
    int64_t nnz_m;            /* nonzeros of M                               */
    int64_t singular_columns; /* columns with MSPAI_COL_SINGULAR             */
    int64_t capacity_columns; /* columns with MSPAI_COL_CAPACITY             */
    int64_t bucket_columns[4];/* columns per size bucket                     */
    double flops;             /* algorithmic flops of the solved problems,
                                 on the folded least-squares matrices       */
    double flops_dense;       /* the same counted on dense C(I,J), as the
                                 reference's dgeqrf path would execute     */
    double gather_bytes;      /* algorithmic gather/assembly bytes           */
    double setup_ms;          /* device time of the last setup (CUDA events) */
    double kernel_ms[4];      /* device time per bucket kernel               */
    int64_t kernel_launches;  /* kernels this library launched in the setup  */
    double bucket_flops[4];   /* algorithmic (folded) flops per bucket kernel */
    int64_t reused_columns;   /* columns that took an identical column's solution (-cs/-ch) */
    int64_t factor_reuse_columns; /* columns that converged from their kept factor */
} mspai_stats;

typedef struct mspai_handle mspai_handle;

/* Fills *p with the reference defaults. */
void mspai_default_params(mspai_params* p);

/*
 * Checks an option set the way the reference does (src/imspai.cpp:238-480);
 * writes the reference's message into msg (if msg_len > 0) on failure.
 */
int mspai_validate_params(const mspai_params* p, char* msg, int32_t msg_len);

/* Creates a handle on CUDA device `device` using `stream` (NULL: own stream). */
int mspai_create(mspai_handle** h, int32_t device, void* stream);

/*
 * Runs the setup.  Replaces Spai<double>::SPAI_Algorithm
 * (reference src/Spai.imp:33-191).
 *   C      : nrows x n system matrix (rows >= n are probing rows).
 *   C_rows : row structure of C's first n rows as CSC of C^T restricted to
 *            those rows (i.e. CSR of C); used for pattern-update candidates.
 *            May be NULL (computed on the host when ns > 0).
 *   B      : target B (NULL: B = e_k, the reference's Spai_Unrestrained).
 *   P      : start pattern of M (n x n pattern).
 *   UP     : optional upper (maximal) pattern; NULL for none.
 * Inputs are borrowed for the call.  The result stays in the handle.
 */
int mspai_setup(mspai_handle* h, const mspai_csc* C, const mspai_csc* C_rows,
                const mspai_csc* B, const mspai_csc* P, const mspai_csc* UP,
                const mspai_params* prm);

/* nnz of the last result. */
int mspai_result_nnz(mspai_handle* h, int64_t* nnz);

/*
 * Copies the last result M (n x n CSC, rows sorted) into caller arrays of
 * size n+1 / nnz / nnz, on the host or the device (mem).
 */
int mspai_result_copy(mspai_handle* h, int64_t* colptr, int32_t* rowidx, double* values,
                      int32_t mem);

/*
 * Launch-shape knobs of a handle (no reference counterpart: the reference's
 * column loop has no launch shape).  The autotuner (mspai_tune, and the
 * persisted sweep of mspai_b200/tuner.py) chooses them; every setup of the
 * handle uses them.  Results do not depend on them beyond rounding.
 */
typedef struct {
    int32_t smem_kb;              /* shared-memory area per general-solver CTA, 16..220 (48) */
    int32_t fixed_arena_kb;       /* arena of the fixed-pattern solver's first launch,
                                     8..107 (two CTAs per SM) (107)                     */
    int32_t fixed_arena_large_kb; /* arena of its second launch, 8..212 (212)           */
    int32_t warp_emax;            /* tiny bucket (a warp per column): at most this many
                                     entries of C(:,J_k), 16..256 (64)                  */
    int32_t warp_nmax;            /* ... and |J_k| at most this, 4..32 (16)             */
    int32_t w_smem_kb;            /* general solver: a column whose folded matrix fits
                                     this goes to the shared-memory bucket, 16..220 (96) */
    int32_t warp_emax_adaptive;   /* adaptive scalar setups: a warp per column (slots in
                                     global memory) when the entries after the pattern
                                     updates are at most this, 16..4096 (256) ...       */
    int32_t warp_nmax_adaptive;   /* ... and |J_k| after the updates at most this, 4..64 (32) */
} mspai_tuning;

int mspai_get_tuning(mspai_handle* h, mspai_tuning* t);
/* Checks every field's range; MSPAI_ERR_PARAM and no change when one is out. */
int mspai_set_tuning(mspai_handle* h, const mspai_tuning* t);

/*
 * Autotuner (the reference has none: its column loop has no launch shape to
 * pick).  Times setups of problem columns [0, sample_cols) of the given
 * problem (20000 when sample_cols <= 0) with each candidate shared-memory
 * area per solver CTA -- 48, 32 and 24 KB, i.e. 4, 6 and 8 CTAs per SM --
 * keeps the fastest in the handle for its later setups and writes it (KB) to
 * *smem_kb_out when not NULL.  Leaves the handle without a result.
 */
int mspai_tune(mspai_handle* h, const mspai_csc* C, const mspai_csc* C_rows, const mspai_csc* B,
               const mspai_csc* P, const mspai_csc* UP, const mspai_params* prm,
               int32_t sample_cols, int32_t* smem_kb_out);

/*
 * y = M x with the last result M (the preconditioner application of
 * Apply_MSPAI, src/imspai.cpp:47-53, there a PETSc MatMult): x and y are
 * vectors of n doubles where `mem` says.  The first call after a setup builds
 * M's row structure on the device; every y_i is then summed over row i in a
 * fixed order, so repeated calls give bit-identical y.
 */
int mspai_apply(mspai_handle* h, const double* x, double* y, int32_t mem);

/* Per column: ||C(I,J) m - b||_2, LS solves, status (arrays of n; host). */
int mspai_column_info(mspai_handle* h, double* resnorm, int32_t* steps, int32_t* status);

/* Statistics of the last setup. */
int mspai_get_stats(mspai_handle* h, mspai_stats* s);

/*
 * Adjoint of the last setup for the loss
 *     L = ||C M - B||_F^2 + sum_k gbar_k^T m_k        (gbar optional)
 * at the pattern the setup chose (fixed, or the final pattern of the pattern
 * updates: the pattern is a discrete choice and carries no gradient), for
 * scalar and block setups (gbar: scalar setups only).  C and B must be the
 * matrices of that setup (B NULL: B = I).  Writes dL/dC at the nonzeros of C
 * (C's order, C->nnz values) and, if dB_values is not NULL, dL/dB at the
 * nonzeros of B; *loss receives L.  gbar_values (nnz(M) values in M's order)
 * may be NULL.  All value arrays live where `mem` says.  The residual term
 * needs no solve (M is stationary); the gbar term needs
 * lambda_k = R_k^-1 R_k^-T gbar_k: from the R that the setup kept
 * (keep_factors; refined in FP64 when R is FP32), else from R recomputed in
 * FP64.  Q is never stored.  Not in the reference.
 */
int mspai_adjoint(mspai_handle* h, const mspai_csc* C, const mspai_csc* B,
                  const double* gbar_values, double* dC_values, double* dB_values,
                  double* loss, int32_t mem);

/*
 * mspai_adjoint for L = w ||C M - B||_F^2 + sum_k gbar_k^T m_k with the
 * residual weight w = residual_weight (0: the sensitivity of gbar . M alone,
 * the backward pass of M as a function of C and B).
 */
int mspai_adjoint_weighted(mspai_handle* h, const mspai_csc* C, const mspai_csc* B,
                           const double* gbar_values, double residual_weight,
                           double* dC_values, double* dB_values, double* loss, int32_t mem);

/* Last error message of the handle ("" if none). */
const char* mspai_last_error(mspai_handle* h);

/* Releases the handle and its device memory. */
void mspai_free(mspai_handle* h);

/*
 * Measures the FP32 (fp64 == 0) or FP64 (fp64 == 1) fused-multiply-add
 * throughput of CUDA device `device` with independent register-resident FMA
 * chains on every SM: the CUDA-core roofline denominator of the
 * least-squares kernels.  Writes GFLOP/s (2 flops per FMA) to *gflops.
 */
int mspai_measure_fma_peak(int32_t device, int32_t fp64, double* gflops);

/*
 * Fixed-pattern setup that allocates nothing.  No counterpart in the
 * reference (which allocates per call, src/Matrix.imp:178-283).
 *
 * For callers that cannot call cudaMalloc when they need the preconditioner:
 * applications whose device memory is owned by their own pool or by another
 * framework, and latency-critical paths that must not pay for cudaMalloc /
 * cudaFree.  It runs the same column solver as mspai_setup with its scratch
 * in a fixed 64 MiB array inside the library (held by every GPU that loads the
 * library until the process exits) and calls no allocating routine.
 *
 * All of C, B (optional), P and the outputs are device arrays on the current
 * device: values_out receives M's values at P's nonzeros (M has P's pattern),
 * resnorm_out and status_out one entry per column.  Limits: ns = 0, bs = 1,
 * at most 1,048,576 columns, at most 512 entries of C(:, J_k) and |J_k| <= 64
 * per column; larger inputs are rejected with MSPAI_ERR_CAPACITY and a message
 * in msg.  The first call on a device looks up the array's device address;
 * make that call before any stream capture.  All calls share the array and it
 * keeps the last call's contents: calls whose kernels overlap on the GPU race
 * and must be serialised by the caller.  `stream` may be NULL (legacy stream).
 */
int mspai_setup_fixed_noalloc(const mspai_csc* C, const mspai_csc* B, const mspai_csc* P,
                              const mspai_params* prm, double* values_out, double* resnorm_out,
                              int32_t* status_out, void* stream, char* msg, int32_t msg_len);

/* Library version string. */
const char* mspai_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MSPAI_B200_H */
