// Per-column MSPAI solve, written once against the group interface of
// spai_device.cuh.  One call handles one column k of M:
//
//   repeat (step = -1 .. ns-1, as src/Spai_Unrestrained.imp:78-129):
//     1. gather the entries of C(:, J_k) and sort them by row      -> I_k
//        (replaces Get_I_Set's bit vector + std::sort, src/Spai_Sub.imp:65-122)
//     2. build the least-squares matrix from the sorted entries.  Rows of
//        C(I_k, J_k) with a single nonzero ("singleton rows") are folded, per
//        column, into one row of value ||s_j|| (an exact Householder
//        reflection inside that column's singleton rows); rows with two or
//        more nonzeros are kept as dense rows.  The folded matrix has the same
//        R factor and the same least-squares solution as the dense
//        C(I_k, J_k) of Create_Submatrix_AHat (src/Spai_Sub.imp:221-282).
//     3. Householder QR of the folded matrix and Q^T b, back substitution
//        (replaces dgeqrf / dormqr / dtrtrs, src/Spai_Unrestrained.imp:135-195)
//        in T = double (FP64 mode) or T = float (mixed mode);
//     4. mixed mode: `refine` steps x += R^-1 R^-T C^T (b - C x) with the
//        residual and C^T r in FP64 from the sparse entries;
//     5. FP64 residual r = b - C(I,J) m and ||r||_2 (Residual_Norm,
//        src/Spai_Sub.imp:915-941; the reference stores -r, same norm);
//     6. stop if ||r|| <= ep or the last step, else the pattern update of
//        Augment_Sparsity (src/Spai_Sub.imp:1010-1116): candidates from the
//        row structure of L = I u {k}, minus J, optionally within UP(:,k);
//        rho_j = sqrt(||r||^2 - (r^T a_j)^2 / ||a_j||^2) (Compute_Rhos,
//        src/Spai_Sub.imp:1231-1348); bound = mean (um=1) or sum of rho;
//        add up to mn candidates of smallest rho (ties by index) with
//        rho <= bound; keep J sorted.
#pragma once

#include "spai_blocked.cuh"
#include "spai_device.cuh"

namespace mspai {



// Read-only inputs of a setup (device pointers).
struct Problem {
    int n;                                   // columns of C and M
    int nrows;                               // rows of C (n + probing rows)
    const int64_t* cptr;
    const int32_t* cidx;
    const double* cval;
    const int64_t* rptr;                     // CSR structure of C's rows < n
    const int32_t* rcol;
    const int64_t* bptr;                     // target B (null: e_k)
    const int32_t* bidx;
    const double* bval;
    const int64_t* pptr;                     // start pattern
    const int32_t* pidx;
    const int64_t* upptr;                    // upper pattern (nullable)
    const int32_t* upidx;
    double ep;
    int mn, ns, um, refine;
    int bs;                                  // block size (1: scalar SPAI)
    int qru;                                 // 1: QR updates across pattern steps
};

// Results.  Column k's indices/values go to [optr[k], optr[k+1]).
struct Output {
    const int64_t* optr;   // capacity pointers (== pptr for fixed patterns)
    int32_t* oidx;         // may alias pidx for fixed patterns (then not written)
    double* oval;
    int32_t* olen;         // final |J_k|
    double* res;           // ||r_k||
    int32_t* steps;        // LS solves
    int32_t* status;       // mspai_column_status
    double* work;          // 3 per column: folded flops, dense-equivalent
                           // flops, gather bytes (accumulated over steps)
    int write_idx;         // 1: write oidx
    // optional (fixed scalar patterns): R of column k packed by columns,
    // R(i, j) at rstore + roff[k] + j (j + 1) / 2 + i, in the solve's precision
    void* rstore;
    const int64_t* roff;
    // re-setup from the kept factors (fixed-pattern solver): start from M's
    // previous values in oval and the R in rstore, at most reuse_steps FP64
    // refinement steps against the new values; a column that does not
    // converge is factored again.  reuse_count counts the columns that converged.
    int reuse_steps;
    int32_t* reuse_count;
};

// Capacities of one problem slot.
struct Caps {
    int emax;      // entries of C(:, J)
    int lsort;     // next_pow2(emax)
    int nmax;      // |J|
    int mwmax;     // rows of the folded matrix
    int cmax;      // candidate entries (row structure of L)
    int lcand;     // next_pow2(cmax)
    int nrhs;      // right-hand sides (the block size)
    int nbmap;     // words of the candidate bit vector (adaptive; 0 otherwise)
    int qru;       // 1: room for the QR-update state (dense W, row/column maps)
};

// Pointers of one problem slot's workspace.
template <class T>
struct Slot {
    int32_t* J;        // nmax
    int32_t* off;      // nmax + 1
    int32_t* ejj;      // emax   local column of entry e
    double* ev;        // emax   value of entry e
    int32_t* pos;      // emax   position in I of entry e
    uint64_t* keys;    // lsort  (row << 24) | e, sorted
    int32_t* I;        // emax   unique rows
    int32_t* rstart;   // emax + 1
    int32_t* tmp;      // emax + 1 (scan scratch; row classes)
    double* r;         // emax   residual on I (FP64)
    T* W;              // mwmax * nmax folded matrix (column-major, ld = mw)
    T* rhs;            // mwmax
    T* Wfast;          // optional shared-memory area for W (+ rhs) ...
    int wfast_elems;   // ... used when mw * n + mw <= wfast_elems; otherwise
                       // it stages the 16-column panels of the blocked QR
    BlockedScratch<T>* bsc;  // shared scratch of the blocked QR (CTA groups)
    double* x;         // nmax  solution
    double* gv;        // nmax  refinement right-hand side / correction
    double* rinv;      // nmax  1 / R(j, j) in FP64
    double* rs;        // (emax / 2 + 1) * nrhs  residual on the shared rows
    int32_t* srow;     // emax / 2 + 1  position in I of each shared row
    // QR-update state (cap.qru): W columns in the order they joined J, W rows
    // in the order their rows joined I
    int32_t* qcol;     // nmax  column of C of each W column
    int32_t* qpos;     // nmax  its position in the sorted J
    int32_t* qrow;     // emax  rows of I (sorted) ...
    int32_t* qwr;      // emax  ... and their W rows, from the previous step
    int32_t* qwu;      // emax  W row of each position of the current I
    double* qperm;     // nmax  vectors in W's column order
    int32_t* cand;     // lcand candidate column indices (adaptive)
    int32_t* ctmp;     // cmax + 1 candidate flags / scan
    uint32_t* bmap;    // nbmap words: bit vector over problem columns (adaptive)
    double* rho;       // cmax
};

template <class T>
__host__ __device__ inline size_t align_up(size_t v, size_t a)
{
    return (v + a - 1) / a * a;
}

// Byte layout of a slot (host and device agree on it).
template <class T>
struct SlotLayout {
    size_t o_J, o_off, o_ejj, o_ev, o_pos, o_keys, o_I, o_rstart, o_tmp, o_r, o_W, o_rhs, o_x,
        o_gv, o_rinv, o_rs, o_srow, o_qcol, o_qpos, o_qrow, o_qwr, o_qwu, o_qperm, o_cand, o_ctmp,
        o_rho, o_bmap, bytes;
    __host__ __device__ SlotLayout(const Caps& c, bool w_external)
    {
        size_t o = 0;
        auto take = [&](size_t bytes) {
            o = align_up<T>(o, 16);
            size_t at = o;
            o += bytes;
            return at;
        };
        o_keys = take(sizeof(uint64_t) * c.lsort);
        const int nr = c.nrhs > 0 ? c.nrhs : 1;
        o_ev = take(sizeof(double) * c.emax);
        o_r = take(sizeof(double) * static_cast<size_t>(c.emax) * nr);
        o_x = take(sizeof(double) * static_cast<size_t>(c.nmax) * nr);
        o_gv = take(sizeof(double) * static_cast<size_t>(c.nmax) * nr);
        o_rinv = take(sizeof(double) * c.nmax);
        o_rs = take(sizeof(double) * static_cast<size_t>(c.emax / 2 + 1) * nr);
        o_srow = take(sizeof(int32_t) * (c.emax / 2 + 1));
        const size_t qn = c.qru ? c.nmax : 1, qe = c.qru ? c.emax : 1;
        o_qcol = take(sizeof(int32_t) * qn);
        o_qpos = take(sizeof(int32_t) * qn);
        o_qrow = take(sizeof(int32_t) * qe);
        o_qwr = take(sizeof(int32_t) * qe);
        o_qwu = take(sizeof(int32_t) * qe);
        o_qperm = take(sizeof(double) * qn);
        o_rho = take(sizeof(double) * (c.cmax > 0 ? c.cmax : 1));
        o_J = take(sizeof(int32_t) * c.nmax);
        o_off = take(sizeof(int32_t) * (c.nmax + 1));
        o_ejj = take(sizeof(int32_t) * c.emax);
        o_pos = take(sizeof(int32_t) * (c.emax + 1));
        o_I = take(sizeof(int32_t) * c.emax);
        o_rstart = take(sizeof(int32_t) * (c.emax + 1));
        o_tmp = take(sizeof(int32_t) * (c.emax + 1));
        o_cand = take(sizeof(int32_t) * (c.lcand > 0 ? c.lcand : 1));
        o_ctmp = take(sizeof(int32_t) * (c.cmax + 1));
        o_bmap = take(sizeof(uint32_t) * (c.nbmap > 0 ? c.nbmap : 1));
        if (w_external) {
            o_W = o_rhs = 0;
        }
        else {
            // the dense folded matrix and its right-hand sides, or the
            // structured QR's shared rows + one panel and [R, Q^T b]
            // (QR updates: the dense C(I,J) with ld emax, nmax + 2 columns)
            size_t wel = static_cast<size_t>(c.mwmax + kPanel) * (c.nmax + nr);
            if (c.qru) {
                const size_t q = static_cast<size_t>(c.emax) * (c.nmax + 2);
                wel = q > wel ? q : wel;
            }
            o_W = take(sizeof(T) * wel);
            o_rhs = o_W;
        }
        bytes = align_up<T>(o, 128);
    }
    __host__ __device__ Slot<T> at(char* base, T* w_ext) const
    {
        Slot<T> s;
        s.J = reinterpret_cast<int32_t*>(base + o_J);
        s.off = reinterpret_cast<int32_t*>(base + o_off);
        s.ejj = reinterpret_cast<int32_t*>(base + o_ejj);
        s.ev = reinterpret_cast<double*>(base + o_ev);
        s.pos = reinterpret_cast<int32_t*>(base + o_pos);
        s.keys = reinterpret_cast<uint64_t*>(base + o_keys);
        s.I = reinterpret_cast<int32_t*>(base + o_I);
        s.rstart = reinterpret_cast<int32_t*>(base + o_rstart);
        s.tmp = reinterpret_cast<int32_t*>(base + o_tmp);
        s.r = reinterpret_cast<double*>(base + o_r);
        s.x = reinterpret_cast<double*>(base + o_x);
        s.gv = reinterpret_cast<double*>(base + o_gv);
        s.rinv = reinterpret_cast<double*>(base + o_rinv);
        s.rs = reinterpret_cast<double*>(base + o_rs);
        s.srow = reinterpret_cast<int32_t*>(base + o_srow);
        s.qcol = reinterpret_cast<int32_t*>(base + o_qcol);
        s.qpos = reinterpret_cast<int32_t*>(base + o_qpos);
        s.qrow = reinterpret_cast<int32_t*>(base + o_qrow);
        s.qwr = reinterpret_cast<int32_t*>(base + o_qwr);
        s.qwu = reinterpret_cast<int32_t*>(base + o_qwu);
        s.qperm = reinterpret_cast<double*>(base + o_qperm);
        s.cand = reinterpret_cast<int32_t*>(base + o_cand);
        s.ctmp = reinterpret_cast<int32_t*>(base + o_ctmp);
        s.bmap = reinterpret_cast<uint32_t*>(base + o_bmap);
        s.rho = reinterpret_cast<double*>(base + o_rho);
        if (w_ext) {
            s.W = w_ext;
        }
        else {
            s.W = reinterpret_cast<T*>(base + o_W);
        }
        s.rhs = nullptr;  // set by the caller from mw
        s.Wfast = nullptr;
        s.wfast_elems = 0;
        s.bsc = nullptr;
        return s;
    }
};

// Value of the target column b = B(:, col) at row `row`.
__device__ __forceinline__ double target_value(const Problem& pb, int col, int row)
{
    if (pb.bptr == nullptr)
        return row == col ? 1.0 : 0.0;
    int64_t lo = pb.bptr[col], hi = pb.bptr[col + 1];
    while (lo < hi) {  // binary search, rows sorted
        const int64_t mid = (lo + hi) >> 1;
        const int v = pb.bidx[mid];
        if (v == row)
            return pb.bval[mid];
        if (v < row)
            lo = mid + 1;
        else
            hi = mid;
    }
    return 0.0;
}

__device__ __forceinline__ int lower_bound_i32(const int32_t* a, int len, int v)
{
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Householder QR of W (mw x n, ld = mw) applied to the nrhs right-hand sides
// stored as columns n .. n + nrhs - 1 of W (same leading dimension); R
// overwrites the upper triangle.  Reflectors follow LAPACK's dlarfg
// convention: beta = -sign(alpha) * ||(alpha, x)||, tau = (beta - alpha) /
// beta, v = x / (alpha - beta), and tau = 0 (H = I) when x = 0.
template <class T, class G>
__device__ void group_householder(const G& g, T* W, int ld, int mw, int n, int nrhs)
{
    const int kmax = min(mw, n);
    const int lane = g.lane();
    for (int k = 0; k < kmax; k++) {
        T* wk = W + static_cast<size_t>(k) * ld;
        T part = 0;
        for (int i = k + 1 + g.rank(); i < mw; i += G::kSize)
            part += wk[i] * wk[i];
        const T xnorm2 = g.sum(part);
        if (xnorm2 == T(0))
            continue;  // tau = 0, H = I (xnorm2 is group-uniform)
        const T alpha = wk[k];
        const T beta = -copysign(tsqrt<T>(alpha * alpha + xnorm2), alpha);
        const T tau = (beta - alpha) / beta;
        const T scale = T(1) / (alpha - beta);
        g.sync();
        if (g.rank() == 0)
            wk[k] = beta;
        for (int i = k + 1 + g.rank(); i < mw; i += G::kSize)
            wk[i] *= scale;
        g.sync();
        // apply H = I - tau v v^T (v_k = 1) to the later columns and the rhs
        for (int c = k + 1 + g.warp(); c < n + nrhs; c += G::kWarps) {
            T* col = W + static_cast<size_t>(c) * ld;
            T d = (lane == 0) ? col[k] : T(0);
            for (int i = k + 1 + lane; i < mw; i += 32)
                d += wk[i] * col[i];
            d = warp_sum(d) * tau;
            if (lane == 0)
                col[k] -= d;
            for (int i = k + 1 + lane; i < mw; i += 32)
                col[i] -= d * wk[i];
        }
        g.sync();
    }
}

// Back substitution R y = rhs(0:n) by warp 0 of the group, result in x (FP64).
// Returns (group-uniformly) 1 if R has a zero diagonal; then x = rhs(0:n)
// unchanged, as LAPACK's dtrtrs leaves B when it reports info > 0.
template <class T, class G>
__device__ int group_back_substitute(const G& g, const T* W, int ld, int n, T* rhs, double* x)
{
    int singular = 0;
    for (int j = g.rank(); j < n; j += G::kSize)
        if (W[static_cast<size_t>(j) * ld + j] == T(0))
            singular = 1;
    singular = g.sum(singular) > 0;
    if (!singular && g.warp() == 0) {
        const int lane = g.lane();
        for (int j = n - 1; j >= 0; j--) {
            const T xj = rhs[j] / W[static_cast<size_t>(j) * ld + j];
            __syncwarp();
            if (lane == 0)
                rhs[j] = xj;
            const T* wj = W + static_cast<size_t>(j) * ld;
            for (int i = lane; i < j; i += 32)
                rhs[i] -= wj[i] * xj;
            __syncwarp();
        }
    }
    g.sync();
    for (int j = g.rank(); j < n; j += G::kSize)
        x[j] = static_cast<double>(rhs[j]);
    g.sync();
    return singular;
}

// delta = R^-1 R^-T gv (in place in gv), FP64 accumulation with R in T; warp 0.
template <class T, class G>
__device__ void group_normal_correction(const G& g, const T* W, int ld, int n, double* gv)
{
    if (g.warp() == 0) {
        const int lane = g.lane();
        // forward: R^T z = g
        for (int j = 0; j < n; j++) {
            const T* wj = W + static_cast<size_t>(j) * ld;
            double d = 0.0;
            for (int i = lane; i < j; i += 32)
                d += static_cast<double>(wj[i]) * gv[i];
            d = warp_sum(d);
            const double zj = (gv[j] - d) / static_cast<double>(wj[j]);
            __syncwarp();
            if (lane == 0)
                gv[j] = zj;
            __syncwarp();
        }
        // backward: R delta = z
        for (int j = n - 1; j >= 0; j--) {
            const T* wj = W + static_cast<size_t>(j) * ld;
            const double dj = gv[j] / static_cast<double>(wj[j]);
            __syncwarp();
            if (lane == 0)
                gv[j] = dj;
            for (int i = lane; i < j; i += 32)
                gv[i] -= static_cast<double>(wj[i]) * dj;
            __syncwarp();
        }
    }
    g.sync();
}

// FP64 residuals r_c = b_c - C(I,J) x_c on I for the nrhs right-hand sides
// (b_c = B(:, bs * col + c), x_c = x + c * n, r_c = r + c * m); returns the
// squared Frobenius norm.
template <class G>
__device__ double group_residual(const G& g, const Problem& pb, int col, const uint64_t* keys,
                                 const int32_t* I, const int32_t* rstart, const int32_t* ejj,
                                 const double* ev, const double* x, double* r, int m, int n,
                                 int nrhs)
{
    double part = 0.0;
    for (int t = g.rank(); t < m * nrhs; t += G::kSize) {
        const int c = t / m, u = t - c * m;
        double v = target_value(pb, pb.bs * col + c, I[u]);
        const double* xc = x + static_cast<size_t>(c) * n;
        for (int i = rstart[u]; i < rstart[u + 1]; i++) {
            const int e = static_cast<int>(keys[i] & kEntryMask);
            v -= ev[e] * xc[ejj[e]];
        }
        r[t] = v;
        part += v * v;
    }
    return g.sum(part);
}

// Householder QR of columns k0 .. n-1 of W (rows k0 .. m-1 of the trailing
// block; columns < k0 are already factored), LAPACK dlarfg convention,
// applied to the later columns and to the extra column `rhs`; tau[k] is kept
// (0: H = I) so that the reflectors can be applied to columns added later.
template <class T, class G>
__device__ void group_householder_from(const G& g, T* W, int ld, int m, int k0, int n, T* rhs,
                                       double* tau)
{
    const int lane = g.lane();
    const int kmax = min(m, n);
    for (int k = k0; k < kmax; k++) {
        T* wk = W + static_cast<size_t>(k) * ld;
        T part = 0;
        for (int i = k + 1 + g.rank(); i < m; i += G::kSize)
            part += wk[i] * wk[i];
        const T xnorm2 = g.sum(part);
        if (xnorm2 == T(0)) {
            if (g.rank() == 0)
                tau[k] = 0.0;
            g.sync();
            continue;
        }
        const T alpha = wk[k];
        const T beta = -copysign(tsqrt<T>(alpha * alpha + xnorm2), alpha);
        const T tk = (beta - alpha) / beta;
        const T scale = T(1) / (alpha - beta);
        g.sync();
        if (g.rank() == 0) {
            wk[k] = beta;
            tau[k] = static_cast<double>(tk);
        }
        for (int i = k + 1 + g.rank(); i < m; i += G::kSize)
            wk[i] *= scale;
        g.sync();
        for (int c = k + 1 + g.warp(); c <= n; c += G::kWarps) {
            T* col = c < n ? W + static_cast<size_t>(c) * ld : rhs;
            T d = (lane == 0) ? col[k] : T(0);
            for (int i = k + 1 + lane; i < m; i += 32)
                d += wk[i] * col[i];
            d = warp_sum(d) * tk;
            if (lane == 0)
                col[k] -= d;
            for (int i = k + 1 + lane; i < m; i += 32)
                col[i] -= d * wk[i];
        }
        g.sync();
    }
}

// One least-squares solve of the QR-update algorithm (the reference's
// Spai_QRUpdate::SPAI_Column with QR_Update, src/Spai_QRUpdate.imp:33-215,
// 341-377, qrupdates.cpp:164-327): the factorization of the previous pattern
// step is kept and extended instead of recomputed.
//
// W (ld emax, dense C(I,J), unfolded) holds its columns in the order they
// joined J (qcol) and its rows in the order they joined I.  The columns of
// the previous step are factored (reflectors below the diagonal, tau); a
// step adds the new rows at the bottom (zero in the old columns, so the old
// reflectors leave them alone) and the new columns at the right, applies the
// old reflectors to the new columns, factors the new columns below row
// n_old, and back-substitutes with R in W's column order.  Q^T b lives in
// column nmax + 1: its new rows get b's raw values.  x comes back in the
// sorted order of J (qpos).  Returns 1 (uniformly) if R is singular.
template <class T, class G>
__device__ int qr_update_solve(const G& g, const Problem& pb, const Caps& cap, Slot<T>& s, int col,
                               int m, int n, int& m_old, int& n_old)
{
    const int lane = g.lane();
    T* W = s.W;
    const int ld = cap.emax;
    T* qb = W + static_cast<size_t>(cap.nmax + 1) * ld;
    // W rows of the current I: old rows keep theirs, new rows follow in
    // sorted order
    for (int u = g.rank(); u < m; u += G::kSize) {
        const int row = s.I[u];
        const int q = lower_bound_i32(s.qrow, m_old, row);
        const bool old = q < m_old && s.qrow[q] == row;
        s.qwu[u] = old ? s.qwr[q] : -1;
        s.tmp[u] = old ? 0 : 1;
    }
    g.sync();
    group_exclusive_scan(g, s.tmp, m);
    for (int u = g.rank(); u < m; u += G::kSize) {
        if (s.qwu[u] < 0)
            s.qwu[u] = m_old + s.tmp[u];
        s.qrow[u] = s.I[u];
    }
    g.sync();
    for (int u = g.rank(); u < m; u += G::kSize)
        s.qwr[u] = s.qwu[u];
    // columns: the first step takes J as it is; later steps appended theirs
    // to qcol in the pattern update
    for (int t = g.rank(); t < n; t += G::kSize) {
        if (n_old == 0)
            s.qcol[t] = s.J[t];
        s.qpos[t] = lower_bound_i32(s.J, n, n_old == 0 ? s.J[t] : s.qcol[t]);
    }
    g.sync();
    // new rows of the old columns and of Q^T b; the new columns
    for (int i = g.rank(); i < (m - m_old) * n_old; i += G::kSize) {
        const int t = i / (m - m_old), r = m_old + i % (m - m_old);
        W[r + static_cast<size_t>(t) * ld] = T(0);
    }
    for (int i = g.rank(); i < m * (n - n_old); i += G::kSize) {
        const int t = n_old + i / m, r = i % m;
        W[r + static_cast<size_t>(t) * ld] = T(0);
    }
    for (int u = g.rank(); u < m; u += G::kSize)
        if (s.qwu[u] >= m_old)
            qb[s.qwu[u]] = static_cast<T>(target_value(pb, col, s.I[u]));
    g.sync();
    for (int t = n_old + g.warp(); t < n; t += G::kWarps) {
        const int jj = s.qpos[t];
        T* wc = W + static_cast<size_t>(t) * ld;
        for (int e = s.off[jj] + lane; e < s.off[jj + 1]; e += 32)
            wc[s.qwu[s.pos[e]]] = static_cast<T>(s.ev[e]);
    }
    g.sync();
    // the old reflectors on the new columns (a warp per column, in order)
    for (int t = n_old + g.warp(); t < n; t += G::kWarps) {
        T* wc = W + static_cast<size_t>(t) * ld;
        for (int k = 0; k < n_old; k++) {
            const T tk = static_cast<T>(s.rinv[k]);
            if (tk == T(0))
                continue;
            const T* wk = W + static_cast<size_t>(k) * ld;
            T d = (lane == 0) ? wc[k] : T(0);
            for (int i = k + 1 + lane; i < m; i += 32)
                d += wk[i] * wc[i];
            d = warp_sum(d) * tk;
            __syncwarp();
            if (lane == 0)
                wc[k] -= d;
            for (int i = k + 1 + lane; i < m; i += 32)
                wc[i] -= d * wk[i];
            __syncwarp();
        }
    }
    g.sync();
    // factor the new columns below the old R; tau kept in s.rinv
    group_householder_from<T>(g, W, ld, m, n_old, n, qb, s.rinv);
    // fewer rows than columns: R has no rows m..n-1 (rank deficient)
    for (int k = m + g.rank(); k < n; k += G::kSize)
        W[k + static_cast<size_t>(k) * ld] = T(0);
    g.sync();
    // back substitution on a copy of Q^T b (column n is free)
    T* rhs = W + static_cast<size_t>(n) * ld;
    for (int i = g.rank(); i < n; i += G::kSize)
        rhs[i] = qb[i];
    g.sync();
    const int sing = group_back_substitute<T>(g, W, ld, n, rhs, s.qperm);
    for (int t = g.rank(); t < n; t += G::kSize)
        s.x[s.qpos[t]] = s.qperm[t];
    g.sync();
    m_old = m;
    n_old = n;
    return sing;
}

// Fixed-pattern refinement residual: r = b - C(I,J) x in FP64 and the
// gradient gv = C(I,J)^T r, for the nrhs right-hand sides, in one pass over
// the entries (no pass over the rows of I).  `code[e]` is -1 for an entry that
// is alone in its row (its residual b_e - v_e x_j is formed in place, b_e in
// `eb[c * estride + e]`) and the dense shared-row number d otherwise; the S
// shared rows (positions srow[d] in I) are done first, one thread per row.
// A thread per column sums its entries in order, so the result does not
// depend on the schedule.  Returns ||r||_F^2.
template <class G>
__device__ double group_residual_gradient(const G& g, const Problem& pb, int col,
                                          const uint64_t* keys, const int32_t* I,
                                          const int32_t* rstart, const int32_t* srow,
                                          const int32_t* off, const int32_t* ejj,
                                          const double* ev, const int32_t* code,
                                          const double* eb, int estride, const double* x,
                                          double* rs, double* gv, int S, int n, int nrhs)
{
    double part = 0.0;
    for (int t = g.rank(); t < S * nrhs; t += G::kSize) {
        const int c = t / S, d = t - c * S;
        const int u = srow[d];
        double v = target_value(pb, pb.bs * col + c, I[u]);
        const double* xc = x + static_cast<size_t>(c) * n;
        for (int i = rstart[u]; i < rstart[u + 1]; i++) {
            const int e = static_cast<int>(keys[i] & kEntryMask);
            v -= ev[e] * xc[ejj[e]];
        }
        rs[t] = v;
        part += v * v;
    }
    g.sync();
    for (int t = g.rank(); t < n * nrhs; t += G::kSize) {
        const int c = t / n, jj = t - c * n;
        const double xj = x[t];
        const double* ebc = eb + static_cast<size_t>(c) * estride;
        const double* rsc = rs + static_cast<size_t>(c) * S;
        double acc = 0.0;
        const int e1 = off[jj + 1];
#pragma unroll 4
        for (int e = off[jj]; e < e1; e++) {
            const double v = ev[e];
            const int cd = code[e];
            double r;
            if (cd < 0) {
                r = ebc[e] - v * xj;
                part += r * r;
            }
            else {
                r = rsc[cd];
            }
            acc += v * r;
        }
        gv[t] = acc;
    }
    return g.sum(part);
}

// Largest constant block size of the block path.
constexpr int kMaxBlockSize = 8;

// Solves the bs x bs (bs <= kMaxBlockSize) SPD system G Y = N (column-major) by
// Cholesky in FP64 and returns sum(Y .* N), the block rho term
// <N, (A_j^T A_j)^-1 N> of Compute_Rhos_Block (src/Spai_Sub.imp:1350-1465).
__device__ __forceinline__ double block_rho_term(double* Gm, const double* N, int bs)
{
    constexpr int kMaxBs = kMaxBlockSize;
    double L[kMaxBs * kMaxBs];
    for (int j = 0; j < bs; j++) {
        double d = Gm[j + j * bs];
        for (int k = 0; k < j; k++)
            d -= L[j + k * kMaxBs] * L[j + k * kMaxBs];
        d = sqrt(d);
        L[j + j * kMaxBs] = d;
        for (int i = j + 1; i < bs; i++) {
            double v = Gm[i + j * bs];
            for (int k = 0; k < j; k++)
                v -= L[i + k * kMaxBs] * L[j + k * kMaxBs];
            L[i + j * kMaxBs] = v / d;
        }
    }
    double term = 0.0;
    for (int q = 0; q < bs; q++) {
        double y[kMaxBs];
        for (int i = 0; i < bs; i++) {  // L y = N(:, q)
            double v = N[i + q * bs];
            for (int k = 0; k < i; k++)
                v -= L[i + k * kMaxBs] * y[k];
            y[i] = v / L[i + i * kMaxBs];
        }
        for (int i = bs - 1; i >= 0; i--) {  // L^T z = y
            double v = y[i];
            for (int k = i + 1; k < bs; k++)
                v -= L[k + i * kMaxBs] * y[k];
            y[i] = v / L[i + i * kMaxBs];
        }
        for (int i = 0; i < bs; i++)
            term += y[i] * N[i + q * bs];
    }
    return term;
}

// Copies R (n x n upper triangle of the view) packed by columns to dst.
template <class T, class G>
__device__ void group_store_r(const G& g, RView<T> R, int n, T* dst)
{
    if (R.ld == 0) {
        for (int t = g.rank(); t < n * (n + 1) / 2; t += G::kSize)
            dst[t] = R.p[t];
    }
    else {
        group_pack_r<T>(g, R.p, R.ld, n, dst);
    }
}

// Solves problem column `col` (scalar column col, or block column col when
// pb.bs > 1; then the bs scalar columns bs*col .. bs*col+bs-1 of M share J,
// I and one QR, with bs right-hand sides).  Results go to `out`.
template <class T, class G>
__device__ void solve_column(const G& g, const Problem& pb, const Caps& cap, Slot<T> s,
                             const Output& out, int col)
{
    const int lane = g.lane();
    const int bs = pb.bs;
    const int nrhs = bs;
    // J <- P(:, col)   (block indices when bs > 1)
    const int64_t p0 = pb.pptr[col];
    int nbk = static_cast<int>(pb.pptr[col + 1] - p0);
    int status = 0;
    int steps = 0;
    double res = 0.0;
    if (nbk * bs > cap.nmax || nrhs > cap.nrhs) {
        status = 3;
        nbk = 0;
    }
    for (int t = g.rank(); t < nbk; t += G::kSize)
        s.J[t] = pb.pidx[p0 + t];
    g.sync();
    const double ep_eff = pb.ep * sqrt(static_cast<double>(bs));
    int n = 0;
    auto scol = [&](int jj) { return bs == 1 ? s.J[jj] : bs * s.J[jj / bs] + jj % bs; };

    // QR updates across the pattern steps (CTA groups, scalar, adaptive)
    const bool qru = pb.qru && cap.qru && bs == 1 && pb.ns > 0 && (G::kWarps > 1);
    int q_m_old = 0, q_n_old = 0;

    PHASE_BEGIN();
    for (int step = -1; step < pb.ns && status != 3; step++) {
        n = nbk * bs;
        // ---- 1. entries of C(:, J), sorted by row
        for (int jj = g.rank(); jj < n; jj += G::kSize) {
            const int j = scol(jj);
            s.off[jj] = static_cast<int>(pb.cptr[j + 1] - pb.cptr[j]);
        }
        g.sync();
        const int E = group_exclusive_scan(g, s.off, n);
        if (g.rank() == 0)
            s.off[n] = E;
        if (E > cap.emax) {
            status = 3;
            break;
        }
        g.sync();
        // the entries of each column of C are a run sorted by row; with room
        // for two key buffers and the run offsets in the shared area (free
        // until W is built) the runs are merged there
        const size_t merge_bytes = 2 * sizeof(uint64_t) * static_cast<size_t>(E) +
                                   sizeof(int) * static_cast<size_t>(n + 1);
        const bool merge = s.Wfast && E > 0 &&
                           merge_bytes <= static_cast<size_t>(s.wfast_elems) * sizeof(T);
        uint64_t* kdst = merge ? reinterpret_cast<uint64_t*>(s.Wfast) : s.keys;
        for (int jj = g.warp(); jj < n; jj += G::kWarps) {
            const int j = scol(jj);
            const int64_t base = pb.cptr[j];
            const int o = s.off[jj];
            const int len = s.off[jj + 1] - o;
            for (int t = lane; t < len; t += 32) {
                const int e = o + t;
                const int row = pb.cidx[base + t];
                s.ejj[e] = jj;
                s.ev[e] = pb.cval[base + t];
                kdst[e] = (static_cast<uint64_t>(row) << kEntryBits) | static_cast<uint64_t>(e);
            }
        }
        if (merge) {
            uint64_t* ka = kdst;
            uint64_t* kb = ka + E;
            int* offs = reinterpret_cast<int*>(kb + E);
            for (int i = g.rank(); i <= n; i += G::kSize)
                offs[i] = s.off[i];
            g.sync();
            const uint64_t* sorted = group_merge_runs(g, ka, kb, E, offs, n);
            for (int i = g.rank(); i < E; i += G::kSize)
                s.keys[i] = sorted[i];
            g.sync();
        }
        else {
            // bitonic sort of the keys padded to a power of two: in the
            // shared area when it fits, else in place in the global slot
            const int L = next_pow2(E > 0 ? E : 1);
            for (int i = E + g.rank(); i < L; i += G::kSize)
                s.keys[i] = ~uint64_t(0);
            g.sync();
            if (s.Wfast && static_cast<size_t>(L) * sizeof(uint64_t) <=
                               static_cast<size_t>(s.wfast_elems) * sizeof(T)) {
                uint64_t* ks = reinterpret_cast<uint64_t*>(s.Wfast);
                for (int i = g.rank(); i < L; i += G::kSize)
                    ks[i] = s.keys[i];
                g.sync();
                group_bitonic_sort(g, ks, L);
                for (int i = g.rank(); i < E; i += G::kSize)
                    s.keys[i] = ks[i];
                g.sync();
            }
            else {
                group_bitonic_sort(g, s.keys, L);
            }
        }

        PHASE_MARK(0);
        // ---- unique rows I, positions of entries, row runs
        for (int i = g.rank(); i < E; i += G::kSize)
            s.tmp[i] = (i == 0 || (s.keys[i] >> kEntryBits) != (s.keys[i - 1] >> kEntryBits)) ? 1 : 0;
        g.sync();
        const int m = group_exclusive_scan(g, s.tmp, E);
        for (int i = g.rank(); i < E; i += G::kSize) {
            const bool first = (i == 0 || (s.keys[i] >> kEntryBits) != (s.keys[i - 1] >> kEntryBits));
            const int u = first ? s.tmp[i] : s.tmp[i] - 1;
            s.pos[static_cast<int>(s.keys[i] & kEntryMask)] = u;
            if (first) {
                s.I[u] = static_cast<int>(s.keys[i] >> kEntryBits);
                s.rstart[u] = i;
            }
        }
        if (g.rank() == 0)
            s.rstart[m] = E;
        g.sync();
        // row classes: shared rows (>= 2 entries) get dense row numbers
        for (int u = g.rank(); u < m; u += G::kSize)
            s.tmp[u] = (s.rstart[u + 1] - s.rstart[u]) >= 2 ? 1 : 0;
        g.sync();
        const int S = group_exclusive_scan(g, s.tmp, m);
        // after the scan s.tmp[u] is the dense row of u if u is shared
        const int mw = S + n;
        if (mw > cap.mwmax) {
            status = 3;
            break;
        }
        PHASE_MARK(1);
        const int wcols = n + nrhs;
        const bool w_smem = !qru && s.Wfast && mw * wcols <= s.wfast_elems;
        // W in global memory (CTA groups): the structured blocked QR, which
        // keeps only the shared rows and one panel of diagonal rows (panels
        // staged in the shared area); W in shared memory: the dense blocked QR
        const bool structured = !qru && !w_smem && (G::kWarps > 1) && s.bsc != nullptr &&
                                s.Wfast && (kPanel + S) * kPanel <= s.wfast_elems;
        // (up to two panels the unblocked QR, a warp per trailing column, has
        // the shorter dependency chain)
        const bool blocked = !qru && (G::kWarps > 1) && s.bsc != nullptr &&
                             (structured || (w_smem && n > 2 * kPanel));
        T* W = w_smem ? s.Wfast : s.W;
        const int ld = qru ? cap.emax : (structured ? kPanel + S : mw);
        const int r0 = structured ? kPanel : 0;  // first shared row in W
        T* rhs = W + static_cast<size_t>(ld) * n;  // nrhs columns right after W
        // fixed pattern: per-entry codes, made before W is built (the build
        // and the refinement read them in entry order); `pos` is not needed
        // afterwards and takes the codes (-1 or the shared row), the residual
        // area holds the right-hand side of every singleton entry
        const bool fixed = (pb.ns == 0);
        if (fixed) {
            for (int e = g.rank(); e < E; e += G::kSize) {
                const int u = s.pos[e];
                const bool shared = (s.rstart[u + 1] - s.rstart[u]) >= 2;
                if (!shared)
                    for (int c = 0; c < nrhs; c++)
                        s.r[static_cast<size_t>(c) * cap.emax + e] =
                            target_value(pb, bs * col + c, s.I[u]);
                s.pos[e] = shared ? s.tmp[u] : -1;
            }
            for (int u = g.rank(); u < m; u += G::kSize)
                if (s.rstart[u + 1] - s.rstart[u] >= 2)
                    s.srow[s.tmp[u]] = u;
        }
        if (!qru) {
            if (structured) {
                for (int i = g.rank(); i < S * wcols; i += G::kSize) {
                    const int c = i / S, r = i - c * S;
                    W[r0 + r + static_cast<size_t>(c) * ld] = T(0);
                }
            }
            else {
                for (int i = g.rank(); i < mw * wcols; i += G::kSize)
                    W[i] = T(0);
            }
            g.sync();
            // shared entries
            if (fixed) {
                for (int e = g.rank(); e < E; e += G::kSize) {
                    const int cd = s.pos[e];
                    if (cd >= 0)
                        W[static_cast<size_t>(s.ejj[e]) * ld + r0 + cd] = static_cast<T>(s.ev[e]);
                }
                for (int t = g.rank(); t < S * nrhs; t += G::kSize) {
                    const int c = t / S, d = t - c * S;
                    rhs[r0 + d + static_cast<size_t>(c) * ld] =
                        static_cast<T>(target_value(pb, bs * col + c, s.I[s.srow[d]]));
                }
            }
            else {
                for (int i = g.rank(); i < E; i += G::kSize) {
                    const int e = static_cast<int>(s.keys[i] & kEntryMask);
                    const int u = s.pos[e];
                    if (s.rstart[u + 1] - s.rstart[u] >= 2) {
                        const int d = r0 + s.tmp[u];
                        W[static_cast<size_t>(s.ejj[e]) * ld + d] = static_cast<T>(s.ev[e]);
                        if (i == s.rstart[u])
                            for (int c = 0; c < nrhs; c++)
                                rhs[d + static_cast<size_t>(c) * ld] =
                                    static_cast<T>(target_value(pb, bs * col + c, s.I[u]));
                    }
                }
            }
            // singleton rows, folded per column (one warp per column)
            for (int jj = g.warp(); jj < n; jj += G::kWarps) {
                double sig = 0.0;
                double tb[kMaxBlockSize] = {};
                for (int e = s.off[jj] + lane; e < s.off[jj + 1]; e += 32) {
                    int u = 0;
                    const bool single =
                        fixed ? s.pos[e] < 0
                              : (u = s.pos[e], s.rstart[u + 1] - s.rstart[u] == 1);
                    if (single) {
                        const double v = s.ev[e];
                        sig += v * v;
#pragma unroll
                        for (int c = 0; c < kMaxBlockSize; c++)
                            if (c < nrhs)
                                tb[c] += v * (fixed ? s.r[static_cast<size_t>(c) * cap.emax + e]
                                                    : target_value(pb, bs * col + c, s.I[u]));
                    }
                }
                sig = warp_sum(sig);
#pragma unroll
                for (int c = 0; c < kMaxBlockSize; c++)
                    if (c < nrhs)
                        tb[c] = warp_sum(tb[c]);
                if (lane == 0) {
                    const double nrm = sqrt(sig);
                    if (structured) {
                        // diagonal rows kept apart: norms and right-hand sides
                        s.rinv[jj] = nrm;
                        for (int c = 0; c < nrhs; c++)
                            s.gv[jj + static_cast<size_t>(c) * n] = nrm > 0.0 ? tb[c] / nrm : 0.0;
                    }
                    else {
                        W[static_cast<size_t>(jj) * ld + S + jj] = static_cast<T>(nrm);
                        for (int c = 0; c < nrhs; c++)
                            rhs[S + jj + static_cast<size_t>(c) * ld] =
                                static_cast<T>(nrm > 0.0 ? tb[c] / nrm : 0.0);
                    }
                }
            }
        }
        g.sync();

        PHASE_MARK(2);
        // ---- 3. QR, Q^T b, back substitution (per right-hand side)
        int sing = 0;
        RView<T> rv{W, ld};
        T* rhs_s = rhs;
        int ldr = ld;  // leading dimension of the right-hand sides
        const int q_n_old_before = q_n_old;
        if (qru) {
            sing = qr_update_solve<T>(g, pb, cap, s, col, m, n, q_m_old, q_n_old);
            PHASE_MARK(3);
        }
        else if (structured) {
            T* Rg = W + static_cast<size_t>(ld) * wcols;  // [R, Q^T b], ld n
            group_householder_structured<T>(g, W, ld, S, n, nrhs, s.rinv, s.gv, Rg, s.Wfast,
                                            s.bsc);
            rv = RView<T>{Rg, n};
            rhs_s = Rg + static_cast<size_t>(n) * n;
            ldr = n;
            if (static_cast<size_t>(n) * (n + 1) / 2 + static_cast<size_t>(n) * nrhs <=
                static_cast<size_t>(s.wfast_elems)) {
                // R (packed) and the right-hand sides move to shared memory
                T* rp = s.Wfast;
                T* rh = s.Wfast + static_cast<size_t>(n) * (n + 1) / 2;
                group_pack_r<T>(g, Rg, n, n, rp);
                for (int t = g.rank(); t < n * nrhs; t += G::kSize)
                    rh[t] = rhs_s[t];
                g.sync();
                rv = RView<T>{rp, 0};
                rhs_s = rh;
            }
            if (out.rstore && pb.ns == 0 && bs == 1)
                group_store_r<T>(g, rv, n, static_cast<T*>(out.rstore) + out.roff[col]);
            PHASE_MARK(3);
            for (int c = 0; c < nrhs; c++)
                sing |= group_back_substitute_blocked<T>(g, rv, n, rhs_s + static_cast<size_t>(c) * ldr,
                                                         s.x + static_cast<size_t>(c) * n);
        }
        else if (blocked) {
            group_householder_blocked<T>(g, W, ld, mw, n, nrhs, w_smem, s.Wfast, s.bsc);
            if (!w_smem && static_cast<size_t>(n) * (n + 1) / 2 + static_cast<size_t>(n) * nrhs <=
                               static_cast<size_t>(s.wfast_elems)) {
                // R (packed) and the right-hand sides move to shared memory
                T* rp = s.Wfast;
                T* rh = s.Wfast + static_cast<size_t>(n) * (n + 1) / 2;
                group_pack_r<T>(g, W, ld, n, rp);
                for (int t = g.rank(); t < n * nrhs; t += G::kSize) {
                    const int c = t / n, i = t - c * n;
                    rh[t] = rhs[i + static_cast<size_t>(c) * ld];
                }
                g.sync();
                rv = RView<T>{rp, 0};
                rhs_s = rh;
                ldr = n;
            }
            if (out.rstore && pb.ns == 0 && bs == 1)
                group_store_r<T>(g, rv, n, static_cast<T*>(out.rstore) + out.roff[col]);
            PHASE_MARK(3);
            for (int c = 0; c < nrhs; c++)
                sing |= group_back_substitute_blocked<T>(g, rv, n, rhs_s + static_cast<size_t>(c) * ldr,
                                                         s.x + static_cast<size_t>(c) * n);
        }
        else {
            group_householder<T>(g, W, ld, mw, n, nrhs);
            if (out.rstore && pb.ns == 0 && bs == 1)
                group_store_r<T>(g, RView<T>{W, ld}, n, static_cast<T*>(out.rstore) + out.roff[col]);
            for (int c = 0; c < nrhs; c++)
                sing |= group_back_substitute<T>(g, W, ld, n, rhs + static_cast<size_t>(c) * ld,
                                                 s.x + static_cast<size_t>(c) * n);
        }
        steps++;
        status = sing ? 1 : 0;
        const int q_n_old_prev = qru ? q_n_old_before : 0;
        if (g.rank() == 0) {
            const double dn = n, dmw = mw, dm = m, dr = nrhs;
            double* wk = out.work + 3 * static_cast<size_t>(col);
            if (qru) {
                // the previous columns' reflectors on the new ones, then the
                // new block below the old R
                const double dk = q_n_old_prev, dd = dn - dk;
                wk[0] += 4.0 * dm * dk * dd + 2.0 * (dm - dk) * dd * dd -
                         (2.0 / 3.0) * dd * dd * dd + 4.0 * (dm - dk) * dd + dn * dn +
                         2.0 * E * dr;
            }
            else if (structured) {
                // panels of (nb + S) rows: factorization and trailing update
                double f = 0.0;
                for (int c0 = 0; c0 < n; c0 += kPanel) {
                    const double nb = min(kPanel, n - c0), mp = nb + S;
                    const double nc = n + nrhs - c0 - nb;
                    f += 2.0 * mp * nb * nb - (2.0 / 3.0) * nb * nb * nb +
                         (4.0 * mp * nb - 2.0 * nb * nb) * nc;
                }
                wk[0] += f + 2.0 * E * dr;
            }
            else {
                wk[0] += 2.0 * dmw * dn * dn - (2.0 / 3.0) * dn * dn * dn +
                         4.0 * dmw * dn * dr + 2.0 * E * dr;
            }
            wk[1] += 2.0 * dm * dn * dn - (2.0 / 3.0) * dn * dn * dn + 4.0 * dm * dn * dr +
                     2.0 * dm * dn * dr;
            wk[2] += 12.0 * E + 16.0 * dn + 8.0 * dm * dr;
        }

        PHASE_MARK(4);
        // ---- 4/5. refinement (mixed) and FP64 residual
        double r2 = 0.0;
        if (fixed) {
            // one pass over the entries gives ||r||^2 and C^T r
            const RView<T> rq = blocked ? rv : RView<T>{W, ld};
            auto resid_grad = [&]() {
                return group_residual_gradient(g, pb, col, s.keys, s.I, s.rstart, s.srow, s.off,
                                               s.ejj, s.ev, s.pos, s.r, cap.emax, s.x, s.rs,
                                               s.gv, S, n, nrhs);
            };
            r2 = resid_grad();
            if (!sing && pb.refine > 0) {
                group_diag_reciprocals<T>(g, rq, n, s.rinv);
                double d2_prev = 0.0;
                for (int it = 0; it < pb.refine; it++) {
                    for (int c = 0; c < nrhs; c++)
                        group_normal_correction_rl<T>(g, rq, n, s.rinv,
                                                      s.gv + static_cast<size_t>(c) * n);
                    double d2 = 0.0, x2 = 0.0;
                    for (int t = g.rank(); t < n * nrhs; t += G::kSize) {
                        const double x1 = s.x[t] + s.gv[t];
                        d2 += s.gv[t] * s.gv[t];
                        x2 += x1 * x1;
                        s.x[t] = x1;
                    }
                    d2 = g.sum(d2);
                    x2 = g.sum(x2);
                    r2 = resid_grad();
                    // converged, or no longer contracting
                    if (d2 <= 0x1p-88 * x2 || (it > 0 && d2 > 0.25 * d2_prev))
                        break;
                    d2_prev = d2;
                }
            }
        }
        else
            r2 = group_residual(g, pb, col, s.keys, s.I, s.rstart, s.ejj, s.ev, s.x, s.r, m, n,
                                nrhs);
        if (!sing && !fixed) {
            double d2_prev = 0.0;
            for (int it = 0; it < pb.refine; it++) {
                g.sync();
                for (int t = g.warp(); t < n * nrhs; t += G::kWarps) {
                    const int c = t / n, jj = t - c * n;
                    const double* rc = s.r + static_cast<size_t>(c) * m;
                    double d = 0.0;
                    for (int e = s.off[jj] + lane; e < s.off[jj + 1]; e += 32)
                        d += s.ev[e] * rc[s.pos[e]];
                    d = warp_sum(d);
                    if (lane == 0)
                        s.gv[t] = d;
                }
                g.sync();
                if (qru) {
                    // R is in W's column order: permute, correct, permute back
                    for (int t = g.rank(); t < n; t += G::kSize)
                        s.qperm[t] = s.gv[s.qpos[t]];
                    g.sync();
                    group_normal_correction<T>(g, W, ld, n, s.qperm);
                    for (int t = g.rank(); t < n; t += G::kSize)
                        s.gv[s.qpos[t]] = s.qperm[t];
                    g.sync();
                }
                else {
                    for (int c = 0; c < nrhs; c++) {
                        if (blocked)
                            group_normal_correction_blocked<T>(g, rv, n,
                                                               s.gv + static_cast<size_t>(c) * n);
                        else
                            group_normal_correction<T>(g, W, ld, n,
                                                       s.gv + static_cast<size_t>(c) * n);
                    }
                }
                double d2 = 0.0, x2 = 0.0;
                for (int t = g.rank(); t < n * nrhs; t += G::kSize) {
                    const double x1 = s.x[t] + s.gv[t];
                    d2 += s.gv[t] * s.gv[t];
                    x2 += x1 * x1;
                    s.x[t] = x1;
                }
                d2 = g.sum(d2);
                x2 = g.sum(x2);
                r2 = group_residual(g, pb, col, s.keys, s.I, s.rstart, s.ejj, s.ev, s.x, s.r, m,
                                    n, nrhs);
                // converged: ||delta|| <= 2^-44 ||x||; the next correction would be
                // smaller again by about kappa^2 * u_fp32, far below FP64 rounding.
                // No longer contracting: FP32 R is too far from this column's matrix
                if (d2 <= 0x1p-88 * x2 || (it > 0 && d2 > 0.25 * d2_prev))
                    break;
                d2_prev = d2;
            }
        }
        res = sqrt(r2);
        g.sync();
        PHASE_MARK(5);
        if (res <= ep_eff || step == pb.ns - 1)
            break;

        // ---- 6. pattern update (Augment_Sparsity / Augment_Sparsity_Block)
        // L = I u {col} in rows (bs == 1) or block rows (bs > 1); the
        // candidate entries are the row structure of L's rows
        int nl;
        int32_t* lrows;  // L as (block) row indices
        if (bs == 1) {
            int in_i = 0;
            {
                const int u = lower_bound_i32(s.I, m, col);
                in_i = (u < m && s.I[u] == col) ? 1 : 0;
            }
            nl = m + (in_i ? 0 : 1);
            lrows = s.I;
            if (!in_i && g.rank() == 0)
                s.pos[0] = col;  // the extra row, read as lrows[m] below
            g.sync();
        }
        else {
            // block rows of I (rows < n) are non-decreasing in u
            for (int u = g.rank(); u < m; u += G::kSize) {
                const int r = s.I[u];
                s.tmp[u] = (r < pb.n && (u == 0 || r / bs != s.I[u - 1] / bs)) ? 1 : 0;
            }
            g.sync();
            const int nb_i = group_exclusive_scan(g, s.tmp, m);
            for (int u = g.rank(); u < m; u += G::kSize) {
                const int r = s.I[u];
                if (r < pb.n && (u == 0 || r / bs != s.I[u - 1] / bs))
                    s.pos[s.tmp[u]] = r / bs;
            }
            g.sync();
            int in_l = 0;
            {
                const int q = lower_bound_i32(s.pos, nb_i, col);
                in_l = (q < nb_i && s.pos[q] == col) ? 1 : 0;
            }
            if (!in_l && g.rank() == 0)
                s.pos[nb_i] = col;
            nl = nb_i + (in_l ? 0 : 1);
            lrows = s.pos;
            g.sync();
        }
        // mark the candidate columns in the slot's bit vector; the first thread
        // to set a bit appends the column to the candidate list (the
        // reference's bit vector + reset list, src/Spai_Sub.imp:124-200)
        if (g.rank() == 0)
            g.sc->i[1] = 0;
        g.sync();
        for (int u = g.warp(); u < nl; u += G::kWarps) {
            int r0, r1;
            if (bs == 1) {
                const int l = (u < m) ? lrows[u] : s.pos[0];
                r0 = l;
                r1 = (l < pb.n) ? l + 1 : l;
            }
            else {
                const int l = lrows[u];
                r0 = l * bs;
                r1 = min(l * bs + bs, pb.n);
            }
            for (int r = r0; r < r1; r++) {
                const int64_t b0 = pb.rptr[r];
                const int len = static_cast<int>(pb.rptr[r + 1] - b0);
                for (int t = lane; t < len; t += 32) {
                    const int c = pb.rcol[b0 + t] / bs;
                    const uint32_t bit = 1u << (c & 31);
                    const uint32_t old = atomicOr(&s.bmap[c >> 5], bit);
                    if (!(old & bit)) {
                        const int idx = atomicAdd(&g.sc->i[1], 1);
                        if (idx < cap.cmax)
                            s.cand[idx] = c;
                    }
                }
            }
        }
        g.sync();
        const int nu = g.sc->i[1];
        const int T_c = min(nu, cap.cmax);
        // clear the bit vector for the next use (every set bit is listed)
        for (int t = g.rank(); t < T_c; t += G::kSize)
            s.bmap[s.cand[t] >> 5] = 0u;
        g.sync();
        if (nu > cap.cmax) {
            status = 3;
            break;
        }
        const int LC = next_pow2(T_c > 0 ? T_c : 1);
        for (int i = T_c + g.rank(); i < LC; i += G::kSize)
            s.cand[i] = 0x7fffffff;
        g.sync();
        group_bitonic_sort(g, s.cand, LC);
        // keep candidates not in J (and, scalar only, in UP(:,col))
        for (int i = g.rank(); i < T_c; i += G::kSize) {
            const int c = s.cand[i];
            int keep = 1;
            {
                const int q = lower_bound_i32(s.J, nbk, c);
                if (q < nbk && s.J[q] == c)
                    keep = 0;
            }
            if (keep && pb.upptr != nullptr && bs == 1) {
                const int64_t a = pb.upptr[col];
                const int len = static_cast<int>(pb.upptr[col + 1] - a);
                const int q = lower_bound_i32(pb.upidx + a, len, c);
                keep = (q < len && pb.upidx[a + q] == c) ? 1 : 0;
            }
            s.ctmp[i] = keep;
        }
        g.sync();
        const int nt = group_exclusive_scan(g, s.ctmp, T_c);
        if (g.rank() == 0)
            s.ctmp[T_c] = nt;
        g.sync();
        // compact (ascending) into rho[] used as int storage, then back to cand
        int32_t* jt = reinterpret_cast<int32_t*>(s.rho);
        for (int i = g.rank(); i < T_c; i += G::kSize)
            if (s.ctmp[i + 1] > s.ctmp[i])
                jt[s.ctmp[i]] = s.cand[i];
        g.sync();
        if (nt == 0)
            break;  // no candidates: Augment_Sparsity returns false
        for (int t = g.rank(); t < nt; t += G::kSize)
            s.cand[t] = jt[t];
        g.sync();
        // rho per candidate (one thread per candidate)
        const double res2 = res * res;
        for (int t = g.rank(); t < nt; t += G::kSize) {
            const int j = s.cand[t];
            if (bs == 1) {
                double a2 = 0.0, num = 0.0;
                for (int64_t p = pb.cptr[j]; p < pb.cptr[j + 1]; p++) {
                    const double v = pb.cval[p];
                    a2 += v * v;
                    const int u = lower_bound_i32(s.I, m, pb.cidx[p]);
                    if (u < m && s.I[u] == pb.cidx[p])
                        num += s.r[u] * v;
                }
                const double ajn = sqrt(a2);
                s.rho[t] = sqrt(res2 - (num * num) / (ajn * ajn));
            }
            else {
                // N = A_j(I)^T R (bs x bs), Gm = A_j^T A_j over the whole block column
                double N[kMaxBlockSize * kMaxBlockSize], Gm[kMaxBlockSize * kMaxBlockSize];
                for (int q = 0; q < bs * bs; q++)
                    N[q] = Gm[q] = 0.0;
                for (int a = 0; a < bs; a++) {
                    const int ca = j * bs + a;
                    for (int64_t p = pb.cptr[ca]; p < pb.cptr[ca + 1]; p++) {
                        const int u = lower_bound_i32(s.I, m, pb.cidx[p]);
                        if (u < m && s.I[u] == pb.cidx[p])
                            for (int b = 0; b < bs; b++)
                                N[a + b * bs] += pb.cval[p] * s.r[u + static_cast<size_t>(b) * m];
                    }
                    for (int a2 = a; a2 < bs; a2++) {
                        const int cb = j * bs + a2;
                        int64_t p = pb.cptr[ca], q = pb.cptr[cb];
                        double gsum = 0.0;
                        while (p < pb.cptr[ca + 1] && q < pb.cptr[cb + 1]) {
                            const int rp = pb.cidx[p], rq = pb.cidx[q];
                            if (rp < rq)
                                p++;
                            else if (rp > rq)
                                q++;
                            else
                                gsum += pb.cval[p++] * pb.cval[q++];
                        }
                        Gm[a + a2 * bs] = gsum;
                        Gm[a2 + a * bs] = gsum;
                    }
                }
                const double term = block_rho_term(Gm, N, bs);
                s.rho[t] = sqrt(res2 - term);
            }
        }
        {
            // algorithmic work of the candidate scan: 4 flops per entry
            int ce = 0;
            for (int t = g.rank(); t < nt; t += G::kSize)
                for (int a = 0; a < bs; a++)
                    ce += static_cast<int>(pb.cptr[s.cand[t] * bs + a + 1] -
                                           pb.cptr[s.cand[t] * bs + a]);
            ce = g.sum(ce);
            if (g.rank() == 0) {
                out.work[3 * static_cast<size_t>(col) + 0] += 4.0 * ce * nrhs;
                out.work[3 * static_cast<size_t>(col) + 1] += 4.0 * ce * nrhs;
                out.work[3 * static_cast<size_t>(col) + 2] += 12.0 * ce;
            }
        }
        g.sync();
        // bound: mean (um=1) or sum, summed in ascending index order
        if (g.rank() == 0) {
            double sum = 0.0;
            for (int t = 0; t < nt; t++)
                sum += s.rho[t];
            g.sc->d[0] = pb.um ? sum / static_cast<double>(nt) : sum;
        }
        g.sync();
        const double bound = g.sc->d[0];
        // select up to mn smallest rho <= bound (ties: smaller index), warp 0
        int added = 0;
        if (g.warp() == 0) {
            for (int sel = 0; sel < pb.mn && sel < nt; sel++) {
                double best = 0.0;
                int bj = 0x7fffffff, bt = -1;
                for (int t = lane; t < nt; t += 32) {
                    const double rv = s.rho[t];
                    const int j = s.cand[t];
                    if (j < 0)
                        continue;  // already taken
                    if (!(rv <= bound))
                        continue;  // includes NaN
                    if (bt < 0 || rv < best || (rv == best && j < bj)) {
                        best = rv;
                        bj = j;
                        bt = t;
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                    const int oj = __shfl_xor_sync(0xffffffffu, bj, o);
                    const int ot = __shfl_xor_sync(0xffffffffu, bt, o);
                    if (ot >= 0 && (bt < 0 || ob < best || (ob == best && oj < bj))) {
                        best = ob;
                        bj = oj;
                        bt = ot;
                    }
                }
                if (bt < 0)
                    break;
                if (lane == 0) {
                    s.J[nbk + added] = bj;
                    if (qru)
                        s.qcol[nbk + added] = bj;  // W's column order
                    s.cand[bt] = -1;
                }
                added++;
                __syncwarp();
            }
            if (lane == 0)
                g.sc->i[0] = added;
        }
        g.sync();
        added = g.sc->i[0];
        // keep J sorted (insertion of at most mn new entries, thread 0)
        if (g.rank() == 0) {
            for (int a = 0; a < added; a++) {
                int q = nbk + a;
                const int v = s.J[q];
                while (q > 0 && s.J[q - 1] > v) {
                    s.J[q] = s.J[q - 1];
                    q--;
                }
                s.J[q] = v;
            }
        }
        nbk += added;
        g.sync();
        if (nbk * bs > cap.nmax) {
            status = 3;
            break;
        }
    }
    n = nbk * bs;

    // ---- write the bs scalar columns of M for this problem column
    for (int c = 0; c < bs; c++) {
        const int sc_col = bs * col + c;
        const int64_t o0 = out.optr[sc_col];
        const int64_t ocap = out.optr[sc_col + 1] - o0;
        if (status == 3 || n > ocap) {
            if (g.rank() == 0) {
                // the status last: a caller may alias olen/steps with status
                out.olen[sc_col] = 0;
                out.res[sc_col] = 0.0;
                out.steps[sc_col] = steps;
                out.status[sc_col] = 3;
            }
            continue;
        }
        int nonfinite = 0;
        const double* xc = s.x + static_cast<size_t>(c) * n;
        for (int t = g.rank(); t < n; t += G::kSize) {
            const double v = xc[t];
            if (!isfinite(v))
                nonfinite = 1;
            out.oval[o0 + t] = v;
            if (out.write_idx)
                out.oidx[o0 + t] = scol(t);
        }
        nonfinite = g.sum(nonfinite);
        if (g.rank() == 0) {
            out.olen[sc_col] = n;
            out.res[sc_col] = res;
            out.steps[sc_col] = steps;
            out.status[sc_col] = (status == 1) ? 1 : ((nonfinite || !isfinite(res)) ? 2 : 0);
        }
    }
    PHASE_MARK(6);
    g.sync();
}

}  // namespace mspai
