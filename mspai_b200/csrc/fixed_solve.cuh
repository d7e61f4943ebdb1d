// Fixed-pattern column solver (ns = 0, scalar columns), one CTA per column,
// every per-column array in the CTA's shared-memory arena.
//
// It computes the same least-squares solutions as solve_column
// (spai_solve.cuh) -- the reference's Spai_Unrestrained::SPAI_Column with its
// Get_I_Set, Create_Submatrix_AHat, Create_ek_Hat / Create_bk_Hat,
// Approximative_Solution and Residual_Norm (src/Spai_Unrestrained.imp:78-132,
// src/Spai_Sub.imp:65-122, 221-282, 629-658, 735-775, 915-941) -- with a
// layout built for fixed patterns:
//
//  1. Rows of C(:, J_k): the sorted column runs are merged as plain row
//     numbers; a row that occurs in two or more columns of J_k is "shared",
//     every other row is a "singleton" row of one column.
//  2. Folding.  The singleton rows of column j fold into one diagonal row
//     d_j = ||s_j|| with right-hand side s_j^T b_s / d_j (an exact Householder
//     reflection inside those rows).  For the FP64 residual and its gradient
//     the singleton rows need no pass over their entries either:
//       sum over the singleton rows of column j with b = 0 of r_e^2 = x_j^2 d0_j,
//       their part of (C^T r)_j = -x_j d0_j   (d0_j = sum of their v_e^2),
//     and the few singleton entries with b != 0 are kept apart.  Only the
//     shared entries (about two per shared row) are visited per refinement.
//  3. Skyline QR.  Shared rows are ordered by their first column f (then by
//     row); row d is stored densely from column 16 floor(f_d / 16) on.  The
//     blocked Householder QR of [diag(d); shared rows] works on 16-column
//     panels; a shared row whose first column lies beyond the panel is zero in
//     the panel and is not touched by its reflectors, so panel p only involves
//     the panel's 16 diagonal rows and the shared rows that have started.
//     A panel of up to 64 rows is factored by one warp with its rows in
//     registers (one reduction per column for the norm, the dot products with
//     the later panel columns and V^T V), a taller one by the CTA (one barrier
//     per column); the later columns are updated with the compact WY form by
//     the whole CTA, two threads per column, V rows broadcast from shared
//     memory.
//  4. Back substitution and, in mixed mode, FP64 refinement steps
//     x += R^-1 R^-T C^T (b - C x): the residual and C^T r in FP64 (step 2),
//     the two triangular solves with the FP32 R.
//
// A column whose arrays do not fit the arena is appended to an overflow list
// and left to a later launch (a larger arena, then the general solver).
#pragma once

#include "spai_device.cuh"
#include "spai_solve.cuh"

namespace mspai {

#ifdef MSPAI_PHASE_TIMERS
#define FIX_SUB_BEGIN() long long _fx_t = clock64()
#define FIX_SUB(k)                                                                         \
    do {                                                                                   \
        if (threadIdx.x == 0) {                                                            \
            const long long _now = clock64();                                              \
            atomicAdd(&g_phase_cycles[k], static_cast<unsigned long long>(_now - _fx_t));  \
            _fx_t = _now;                                                                  \
        }                                                                                  \
    } while (0)
#else
#define FIX_SUB_BEGIN() \
    do {                \
    } while (0)
#define FIX_SUB(k) \
    do {           \
    } while (0)
#endif

constexpr int kFixPanel = 16;
constexpr int kFixMaxSpecial = 16;  // singleton entries with a nonzero target value

template <class T>
struct FixShared {
    GroupScratch sc;
    T tmat[kFixPanel * kFixPanel];  // T factor, column-major: T(i, j) at i + 16 j
    T vtv[kFixPanel * kFixPanel];   // V^T V: (j, k), j < k, at j + 16 k
    T tot[kFixPanel];               // reduced sums of one panel step
    T rowk[kFixPanel];              // scale of each panel column's reflector
    T rowk2[kFixPanel];             // row k of the panel at step k (warp panel)
    T tot2[kFixPanel];              // reduced sums of one step (warp panel)
    T tau[kFixPanel];
    T red[2][16][kFixPanel];        // per-warp column sums of one panel step (two buffers)
    T pkrow[2][kFixPanel];          // row k of the panel at step k (CTA panel, two buffers)
    int tg_row[kFixMaxSpecial];     // target column: rows and values
    double tg_val[kFixMaxSpecial];
    int nspec;
    int mcount;                     // distinct rows of C(:, J)
    int chol_fail;                  // a pivot of the Cholesky factorization was not positive
    T chol_rdiag[16];               // 1 / R(i, i) of the Cholesky's current diagonal block
    int spec_e[kFixMaxSpecial];
    int spec_jj[kFixMaxSpecial];
    double spec_v[kFixMaxSpecial];
    double spec_b[kFixMaxSpecial];
};

// Two-ended bump allocator over the arena: persistent arrays from the bottom,
// transient ones from the top.  Offsets are the same in every thread.
struct FixArena {
    char* base;
    int cap;
    int lo;
    int hi;
    template <class U>
    __device__ __forceinline__ U* low(int count)
    {
        lo = (lo + 15) & ~15;
        U* p = reinterpret_cast<U*>(base + lo);
        lo += count * static_cast<int>(sizeof(U));
        return p;
    }
    template <class U>
    __device__ __forceinline__ U* high(int count)
    {
        hi -= count * static_cast<int>(sizeof(U));
        hi &= ~15;
        return reinterpret_cast<U*>(base + hi);
    }
    __device__ __forceinline__ bool ok() const { return lo <= hi; }
};

// Position of `row` among the first m entries of q (rows with the shared flag
// in bit 31, sorted by row); m if absent.
__device__ __forceinline__ int fix_find_row(const int32_t* q, int m, int row)
{
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((q[mid] & 0x7fffffff) < row)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < m && (q[lo] & 0x7fffffff) == row) ? lo : m;
}

// Column jj of entry number e: off[jj] <= e < off[jj + 1].
__device__ __forceinline__ int fix_entry_column(const int32_t* off, int n, int e)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= e)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Target value B(row, col) (B == null: the identity column e_col).
__device__ __forceinline__ double fix_target(const Problem& pb, int col, int row)
{
    return target_value(pb, col, row);
}

// 16 partial sums per lane -> lane l holds the warp total of index
// fix_scatter_index(l) in acc[0] (lanes l and l ^ 1 hold the same index).
template <class T>
__device__ __forceinline__ void fix_reduce_scatter16(T (&acc)[16], int lane)
{
#pragma unroll
    for (int t = 0; t < 8; t++) {
        const bool up = (lane & 16) != 0;
        const T send = up ? acc[t] : acc[t + 8];
        const T keep = up ? acc[t + 8] : acc[t];
        acc[t] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const bool up = (lane & 8) != 0;
        const T send = up ? acc[t] : acc[t + 4];
        const T keep = up ? acc[t + 4] : acc[t];
        acc[t] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int t = 0; t < 2; t++) {
        const bool up = (lane & 4) != 0;
        const T send = up ? acc[t] : acc[t + 2];
        const T keep = up ? acc[t + 2] : acc[t];
        acc[t] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    {
        const bool up = (lane & 2) != 0;
        const T send = up ? acc[0] : acc[1];
        const T keep = up ? acc[1] : acc[0];
        acc[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], 1);
}

__device__ __forceinline__ int fix_scatter_index(int lane)
{
    return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}

// 16 consecutive elements from a 16-byte aligned address.
__device__ __forceinline__ void fix_load16(const float* p, float (&v)[16])
{
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float4 t = reinterpret_cast<const float4*>(p)[q];
        v[4 * q] = t.x;
        v[4 * q + 1] = t.y;
        v[4 * q + 2] = t.z;
        v[4 * q + 3] = t.w;
    }
}
__device__ __forceinline__ void fix_load16(const double* p, double (&v)[16])
{
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const double2 t = reinterpret_cast<const double2*>(p)[q];
        v[2 * q] = t.x;
        v[2 * q + 1] = t.y;
    }
}

// Reflector of one panel column (LAPACK dlarfg convention): from alpha and
// ||x||^2, beta = -sign(alpha) ||(alpha, x)||, tau = (beta - alpha) / beta and
// the scale 1 / (alpha - beta) of v.  FP32 (mixed mode, whose solution is
// refined in FP64) uses the fast square-root and reciprocal intrinsics; FP64
// the correctly rounded operations.
__device__ __forceinline__ void fix_reflector(float alpha, float x2, float& beta, float& tau,
                                              float& scale)
{
    const float nrm = __fsqrt_rn(fmaf(alpha, alpha, x2));
    beta = -copysignf(nrm, alpha);
    const float rb = __frcp_rn(beta);
    tau = (beta - alpha) * rb;
    scale = __frcp_rn(alpha - beta);
}
__device__ __forceinline__ void fix_reflector(double alpha, double x2, double& beta, double& tau,
                                              double& scale)
{
    beta = -copysign(sqrt(alpha * alpha + x2), alpha);
    tau = (beta - alpha) / beta;
    scale = 1.0 / (alpha - beta);
}

// Householder QR of the panel (mp <= 32 RL rows x nb <= 16 columns) by warp
// 0 alone, the rows in registers: lane l holds rows l, l + 32, ... (all 16
// columns each).  Per column one warp reduce-scatter of 16 partial sums (the
// norm of x, its dot products with the later columns and, for V^T V, with the
// finished reflectors); no CTA barrier and no shared-memory traffic inside
// the 16 steps.  Same reflectors, R, V, tau and V^T V as fix_panel_qr_rows.
template <class T, int RL>
__device__ void fix_panel_warp(FixShared<T>& fs, T* tb, const int32_t* prow, int nb, int mp)
{
    const int lane = threadIdx.x & 31;
    T v[RL][kFixPanel];
    int ro[RL];
#pragma unroll
    for (int r = 0; r < RL; r++) {
        const int i = lane + 32 * r;
        ro[r] = (i < mp) ? prow[i] : -1;
        if (ro[r] >= 0) {
            const T* p = tb + ro[r];
            if (nb == kFixPanel) {
                fix_load16(p, v[r]);
            }
            else {
#pragma unroll
                for (int c = 0; c < kFixPanel; c++)
                    v[r][c] = (c < nb) ? p[c] : T(0);
            }
        }
        else {
#pragma unroll
            for (int c = 0; c < kFixPanel; c++)
                v[r][c] = T(0);
        }
    }
#pragma unroll
    for (int k = 0; k < kFixPanel; k++) {
        if (k >= nb)
            break;
        T acc[kFixPanel];
#pragma unroll
        for (int c = 0; c < kFixPanel; c++)
            acc[c] = T(0);
#pragma unroll
        for (int r = 0; r < RL; r++) {
            const int i = lane + 32 * r;
            if (i > k && ro[r] >= 0) {
                const T x = v[r][k];
#pragma unroll
                for (int c = 0; c < kFixPanel; c++)
                    acc[c] += x * v[r][c];
            }
        }
        // row k is lane k's first row (k < 16 < 32)
        if (lane == k) {
#pragma unroll
            for (int c = 0; c < kFixPanel; c++)
                fs.rowk2[c] = v[0][c];
        }
        fix_reduce_scatter16<T>(acc, lane);
        if ((lane & 1) == 0)
            fs.tot2[fix_scatter_index(lane)] = acc[0];
        __syncwarp();
        const T alpha = fs.rowk2[k];
        const T x2 = fs.tot2[k];
        T tau = T(0), scale = T(0), beta = alpha;
        if (x2 != T(0))
            fix_reflector(alpha, x2, beta, tau, scale);
        T f[kFixPanel];
#pragma unroll
        for (int c = 0; c < kFixPanel; c++)
            f[c] = (c > k && c < nb) ? tau * (fs.rowk2[c] + scale * fs.tot2[c]) : T(0);
        if (lane == 0) {
            fs.tau[k] = tau;
#pragma unroll
            for (int c = 0; c < kFixPanel; c++)
                if (c < k)
                    fs.vtv[c + kFixPanel * k] = fs.rowk2[c] + scale * fs.tot2[c];
        }
        __syncwarp();  // rowk2 / tot2 are read before the next step writes them
#pragma unroll
        for (int r = 0; r < RL; r++) {
            const int i = lane + 32 * r;
            if (i > k && ro[r] >= 0) {
                const T sx = v[r][k] * scale;
#pragma unroll
                for (int c = 0; c < kFixPanel; c++)
                    if (c > k)
                        v[r][c] -= f[c] * sx;
                v[r][k] = sx;
            }
            else if (i == k) {
#pragma unroll
                for (int c = 0; c < kFixPanel; c++)
                    if (c > k)
                        v[r][c] -= f[c];
                v[r][k] = beta;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < RL; r++) {
        if (ro[r] >= 0) {
            T* p = tb + ro[r];
#pragma unroll
            for (int c = 0; c < kFixPanel; c++)
                if (c < nb)
                    p[c] = v[r][c];
        }
    }
}

// Householder QR of the panel (mp rows x nb <= 16 columns) by the whole CTA.
// Panel row i starts at tb + prow[i] (16 consecutive elements).  Thread
// (warp w, lane l) works on column c = l & 15 and the rows of group
// g = 2 w + (l >> 4) (rows congruent to g modulo 2 NW), so every load of a row
// is 16 consecutive elements; a column sum is one shuffle inside the warp and
// NW partial sums in shared memory.  LAPACK dlarfg reflectors (beta =
// -sign(alpha) ||(alpha, x)||, tau = (beta - alpha) / beta, v = x / (alpha -
// beta), tau = 0 when x = 0).  The scaling of each reflector by
// 1 / (alpha - beta) is deferred to the end of the panel: step k works with the
// unscaled x of the earlier columns (their scale factors enter the dot
// products and V^T V explicitly).  Two barriers per column.  Leaves R in the
// panel's upper triangle and V below it, and builds the T factor of the
// compact WY form I - V T V^T (dlarft, forward, columnwise) in fs.tmat.
template <class T, int NT, int RPL>
__device__ void fix_panel_qr_rows(FixShared<T>& fs, T* tb, const int32_t* prow, int nb, int mp)
{
    constexpr int NW = NT / 32;
    constexpr int G = 2 * NW;
    static_assert(G >= kFixPanel, "row k of the panel is the first row of group k");
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int c = lane & 15;
    const int grp = 2 * warp + (lane >> 4);
    // this lane's rows: grp, grp + G, ... (mp <= G * RPL); offsets from tb
    int ro[RPL];
#pragma unroll
    for (int q = 0; q < RPL; q++) {
        const int r = grp + q * G;
        ro[q] = (r < mp) ? prow[r] : -1;
    }
    FIX_SUB_BEGIN();
    // column sums of step 0 over the rows below the diagonal
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < RPL; q++) {
        const int r = grp + q * G;
        if (r > 0 && ro[q] >= 0) {
            const T* p = tb + ro[q];
            acc += p[0] * p[c];
        }
    }
    for (int k = 0; k < nb; k++) {
        // acc: x . col c over the rows below the diagonal (c == k: ||x||^2;
        // c > k: the dot products; c < k: against the earlier, unscaled
        // reflectors, for V^T V); per-warp sums, double-buffered by step
        acc += __shfl_xor_sync(0xffffffffu, acc, 16);
        T(*red)[kFixPanel] = fs.red[k & 1];
        if (lane < kFixPanel)
            red[warp][lane] = acc;
        // row k as it stands before step k, published with the sums: its
        // owner (group k, rows k, k + G, ...; k < 16 <= G) updates it in this
        // step while other warps may still be reading it
        if (grp == k)
            fs.pkrow[k & 1][c] = tb[ro[0] + c];
        __syncthreads();
        FIX_SUB(10);
        T tot = T(0), x2 = T(0);
#pragma unroll
        for (int w = 0; w < NW; w++) {
            tot += red[w][c];
            x2 += red[w][k];
        }
        const T alpha = fs.pkrow[k & 1][k];
        const T rkc = fs.pkrow[k & 1][c];
        T tau = T(0), scale = T(0), beta = alpha;
        if (x2 != T(0)) {
            beta = -copysign(tsqrt<T>(alpha * alpha + x2), alpha);
            tau = (beta - alpha) / beta;
            scale = T(1) / (alpha - beta);
        }
        if (threadIdx.x == 0) {
            fs.tau[k] = tau;
            fs.rowk[k] = scale;  // the deferred scale of reflector k
            fs.tot[k] = beta;
        }
        // V^T V (c, k) = v_c[k] + scale_k sum_{i>k} v_c[i] x_i, with v_c = scale_c x^(c)
        if (threadIdx.x < kFixPanel && c < k) {
            const T sc = fs.rowk[c];
            fs.vtv[c + kFixPanel * k] = sc * rkc + sc * scale * tot;
        }
        // update of the later columns (row k by f_c, rows below by f_c scale
        // x_i); then, row by row, the next step's sums: the lane of column
        // k + 1 in the same half-warp updated that column of the row (__syncwarp)
        const T f = (c > k && c < nb) ? tau * (rkc + scale * tot) : T(0);
        const T fsc = f * scale;
        const int kn = k + 1;
        T pcv[RPL];
#pragma unroll
        for (int q = 0; q < RPL; q++) {
            const int r = grp + q * G;
            pcv[q] = T(0);
            if (r >= k && ro[q] >= 0) {
                T* p = tb + ro[q];
                T pc = p[c];
                if (f != T(0)) {
                    pc -= (r == k) ? f : fsc * p[k];
                    p[c] = pc;
                }
                pcv[q] = pc;
            }
        }
        __syncwarp();
        acc = T(0);
        if (kn < nb) {
#pragma unroll
            for (int q = 0; q < RPL; q++) {
                const int r = grp + q * G;
                if (r > kn && ro[q] >= 0)
                    acc += tb[ro[q] + kn] * pcv[q];
            }
        }
    }
    __syncthreads();
    FIX_SUB(11);
    // deferred: v = scale * x below the diagonal, R(k, k) = beta
    if (c < nb) {
        const T sc = fs.rowk[c];
#pragma unroll
        for (int q = 0; q < RPL; q++) {
            const int r = grp + q * G;
            if (r > c && ro[q] >= 0)
                tb[ro[q] + c] *= sc;
            else if (r == c && ro[q] >= 0)
                tb[ro[q] + c] = fs.tot[c];
        }
    }
}

// Householder QR of the panel (mp rows x nb <= 16 columns) by the whole CTA.
// Panel row i starts at tb + prow[i] (16 consecutive elements).  Thread
// (warp w, lane l) works on column c = l & 15 and the rows of group
// g = 2 w + (l >> 4) (rows congruent to g modulo 2 NW, the same rows for all
// the panel's columns), so every load of a row is 16 consecutive elements; a
// column sum is one shuffle inside the warp and NW partial sums in shared
// memory, one barrier per column.  LAPACK dlarfg reflectors (beta =
// -sign(alpha) ||(alpha, x)||, tau = (beta - alpha) / beta, v = x / (alpha -
// beta), tau = 0 when x = 0).  The scaling of each reflector by
// 1 / (alpha - beta) is deferred to the end of the panel: step k works with the
// unscaled x of the earlier columns (their scale factors enter the dot
// products and V^T V explicitly).  Leaves R in the panel's upper triangle and
// V below it, and builds the T factor of the compact WY form I - V T V^T
// (dlarft, forward, columnwise) in fs.tmat.  Returns false (uniformly) when
// the panel has more rows than the register tiling holds.
template <class T, int NT>
__device__ bool fix_panel_qr(FixShared<T>& fs, T* tb, const int32_t* prow, int nb, int mp)
{
    constexpr int G = 2 * (NT / 32);
    // up to 64 rows the warp panel (two rows per lane); taller panels by the
    // CTA (four rows per lane in one warp measured slower than the CTA panel)
    constexpr int kWarpRows = 64;
    if (mp <= kWarpRows) {
        if (threadIdx.x < 32)
            fix_panel_warp<T, 2>(fs, tb, prow, nb, mp);
        __syncthreads();
    }
    else if (mp <= 16 * G)
        fix_panel_qr_rows<T, NT, 16>(fs, tb, prow, nb, mp);
    else if (mp <= 32 * G)
        fix_panel_qr_rows<T, NT, 32>(fs, tb, prow, nb, mp);
    else
        return false;
    // T factor: T(k, k) = tau_k, T(0:k, k) = -tau_k T(0:k, 0:k) (V^T V)(0:k, k);
    // thread i < 16 builds row i
    if (threadIdx.x < kFixPanel) {
        const int li = threadIdx.x;
        T tr[kFixPanel];
#pragma unroll
        for (int k = 0; k < kFixPanel; k++) {
            const T tk = (k < nb) ? fs.tau[k] : T(0);
            T sum = T(0);
#pragma unroll
            for (int j = 0; j < kFixPanel; j++)
                if (j < k && j >= li)
                    sum += tr[j] * fs.vtv[j + kFixPanel * k];
            tr[k] = (k >= nb) ? T(0) : (li < k ? -tk * sum : (li == k ? tk : T(0)));
        }
#pragma unroll
        for (int k = 0; k < kFixPanel; k++)
            fs.tmat[li + kFixPanel * k] = tr[k];
    }
    __syncthreads();
    return true;
}

// Trailing update of columns [c0 + nb, n] (n: the right-hand side) with the
// panel's reflectors: X <- X - V (T^T (V^T X)).  Two threads per column
// (lanes l and l ^ 16 of a warp, 16 columns per warp): each sums V^T X over
// the rows of its parity, the two partial sums are added with shuffles, both
// form z = T^T y, and each updates the rows of its parity.  Panel row i
// (column c0 on) starts at tb + prow[i]; the diagonal rows' part of V is the
// identity (a diagonal row is untouched by the reflectors before its own).
template <class T, int NT>
__device__ void fix_trailing(const FixShared<T>& fs, T* tb, const int32_t* prow, int nb, int c0,
                             int mp, int n)
{
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int h = lane >> 4;
    FIX_SUB_BEGIN();
    const int first = c0 + nb;
    // warp-uniform trip count (the shuffles inside)
    for (int base = first + 16 * warp; base <= n; base += 16 * NW) {
        const int c = base + (lane & 15);
        const bool act = c <= n;
        const int cc = act ? c - c0 : 0;
        T y[kFixPanel];
#pragma unroll
        for (int j = 0; j < kFixPanel; j++)
            y[j] = T(0);
        if (act) {
            if (h == 0) {
#pragma unroll
                for (int i = 0; i < kFixPanel; i++)
                    if (i < nb)
                        y[i] += tb[prow[i] + cc];
            }
            if (nb == kFixPanel) {
#pragma unroll 2
                for (int i = nb + h; i < mp; i += 2) {
                    const T* pr = tb + prow[i];
                    const T x = pr[cc];
                    T v[kFixPanel];
                    fix_load16(pr, v);
#pragma unroll
                    for (int j = 0; j < kFixPanel; j++)
                        y[j] += v[j] * x;
                }
            }
            else {
                for (int i = nb + h; i < mp; i += 2) {
                    const T* pr = tb + prow[i];
                    const T x = pr[cc];
#pragma unroll
                    for (int j = 0; j < kFixPanel; j++)
                        if (j < nb)
                            y[j] += pr[j] * x;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kFixPanel; j++)
            y[j] += __shfl_xor_sync(0xffffffffu, y[j], 16);
        FIX_SUB(12);
        if (!act)
            continue;
        // z = T^T y (T upper triangular, zero beyond nb)
        T z[kFixPanel];
#pragma unroll
        for (int j = 0; j < kFixPanel; j++) {
            T acc = T(0);
#pragma unroll
            for (int i = 0; i <= j; i++)
                acc += fs.tmat[i + kFixPanel * j] * y[i];
            z[j] = acc;
        }
        if (h == 0) {
#pragma unroll
            for (int i = 0; i < kFixPanel; i++)
                if (i < nb)
                    tb[prow[i] + cc] -= z[i];
        }
        if (nb == kFixPanel) {
#pragma unroll 2
            for (int i = nb + h; i < mp; i += 2) {
                T* pr = tb + prow[i];
                T v[kFixPanel];
                fix_load16(pr, v);
                T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
#pragma unroll
                for (int j = 0; j < kFixPanel; j += 4) {
                    a0 += v[j] * z[j];
                    a1 += v[j + 1] * z[j + 1];
                    a2 += v[j + 2] * z[j + 2];
                    a3 += v[j + 3] * z[j + 3];
                }
                pr[cc] -= (a0 + a1) + (a2 + a3);
            }
        }
        else {
            for (int i = nb + h; i < mp; i += 2) {
                T* pr = tb + prow[i];
                T acc = T(0);
#pragma unroll
                for (int j = 0; j < kFixPanel; j++)
                    if (j < nb)
                        acc += pr[j] * z[j];
                pr[cc] -= acc;
            }
        }
        FIX_SUB(13);
    }
}

// Packed upper-triangular storage of [R, Q^T b]: row i holds columns i .. n
// (column n is Q^T b), starting at fix_rs(i, n).
__device__ __forceinline__ int fix_rs(int i, int n)
{
    return i * (n + 1) - (i * (i - 1)) / 2;
}

// R y = rhs in place (y: n values in T), blocked by 16 rows from the bottom.
template <class T, int NT>
__device__ void fix_back_substitute(const CtaGroup<NT>& g, const T* R, int n, T* y)
{
    const int lane = threadIdx.x & 31;
    FIX_SUB_BEGIN();
    for (int b1 = n; b1 > 0; b1 -= kFixPanel) {
        const int b0 = b1 > kFixPanel ? b1 - kFixPanel : 0;
        const int nbk = b1 - b0;
        if (threadIdx.x < 32) {
            const int i = b0 + lane;
            T yi = lane < nbk ? y[i] : T(0);
            T rr[kFixPanel];  // R(i, b0 + j)
#pragma unroll
            for (int j = 0; j < kFixPanel; j++)
                rr[j] = (lane < nbk && j < nbk && j >= lane) ? R[fix_rs(i, n) + (b0 + j - i)] : T(0);
#pragma unroll
            for (int j = kFixPanel - 1; j >= 0; j--) {
                if (j < nbk) {
                    if (lane == j)
                        yi = yi / rr[j];
                    const T xj = __shfl_sync(0xffffffffu, yi, j);
                    if (lane < j)
                        yi -= rr[j] * xj;
                }
            }
            if (lane < nbk)
                y[i] = yi;
        }
        g.sync();
        FIX_SUB(14);
        for (int i = threadIdx.x; i < b0; i += NT) {
            const T* ri = R + fix_rs(i, n) - i;
            T s = T(0);
            for (int j = b0; j < b1; j++)
                s += ri[j] * y[j];
            y[i] -= s;
        }
        g.sync();
        FIX_SUB(15);
    }
}

// R^T z = rhs in place, blocked by 16 rows from the top.
template <class T, int NT>
__device__ void fix_forward_substitute(const CtaGroup<NT>& g, const T* R, int n, T* z)
{
    const int lane = threadIdx.x & 31;
    for (int b0 = 0; b0 < n; b0 += kFixPanel) {
        const int b1 = min(n, b0 + kFixPanel);
        const int nbk = b1 - b0;
        if (threadIdx.x < 32) {
            const int i = b0 + lane;
            T zi = lane < nbk ? z[i] : T(0);
            T rc[kFixPanel];  // R(b0 + j, i) for j <= lane
#pragma unroll
            for (int j = 0; j < kFixPanel; j++)
                rc[j] = (lane < nbk && j <= lane) ? R[fix_rs(b0 + j, n) + (i - b0 - j)] : T(0);
#pragma unroll
            for (int j = 0; j < kFixPanel; j++) {
                if (j < nbk) {
                    if (lane == j)
                        zi = zi / rc[j];
                    const T zj = __shfl_sync(0xffffffffu, zi, j);
                    if (lane > j)
                        zi -= rc[j] * zj;
                }
            }
            if (lane < nbk)
                z[i] = zi;
        }
        g.sync();
        for (int j = b1 + threadIdx.x; j < n; j += NT) {
            T s = T(0);
            for (int i = b0; i < b1; i++)
                s += R[fix_rs(i, n) + (j - i)] * z[i];
            z[j] -= s;
        }
        g.sync();
    }
}

// Warp-level factorization of the 16 x 16 diagonal block at c0 (nb rows) in
// place, the reciprocals of its diagonal into rdiag and the factored block
// into r11 (16 x 16 row-major, zero below the diagonal); returns true (on
// every lane) when a pivot is not positive.
template <class T>
__device__ __forceinline__ bool fix_chol_diag(T* R, int n, int c0, int nb, int lane, T* rdiag,
                                              T* r11)
{
    T a[kFixPanel];
#pragma unroll
    for (int j = 0; j < kFixPanel; j++)
        a[j] = (lane < nb && j >= lane && j < nb) ? R[fix_rs(c0 + lane, n) + (j - lane)] : T(0);
    bool bad = false;
#pragma unroll
    for (int k = 0; k < kFixPanel; k++) {
        if (k < nb) {
            const T piv = __shfl_sync(0xffffffffu, a[k], k);
            bad = bad || !(piv > T(0));
            const T rkk = bad ? T(1) : sqrt(piv);
            const T inv = T(1) / rkk;
            if (lane == k) {
                rdiag[k] = inv;
#pragma unroll
                for (int j = 0; j < kFixPanel; j++)
                    a[j] = (j == k) ? rkk : (j > k ? a[j] * inv : a[j]);
            }
            T rk[kFixPanel];
#pragma unroll
            for (int j = 0; j < kFixPanel; j++)
                rk[j] = __shfl_sync(0xffffffffu, a[j], k);
            if (lane > k && lane < nb) {
#pragma unroll
                for (int j = 0; j < kFixPanel; j++)
                    if (j >= lane)
                        a[j] -= rk[lane] * rk[j];
            }
        }
    }
    if (lane < nb) {
#pragma unroll
        for (int j = 0; j < kFixPanel; j++)
            if (j >= lane && j < nb)
                R[fix_rs(c0 + lane, n) + (j - lane)] = a[j];
    }
    if (lane < kFixPanel) {
#pragma unroll
        for (int j = 0; j < kFixPanel; j++)
            r11[lane * kFixPanel + j] = a[j];
    }
    return bad;
}

// Cholesky factorization G = R^T R in place, R upper triangular in the packed
// rows of fix_rs (row i holds columns i .. n - 1 of G's upper triangle on
// entry, of R on return).  Right-looking by 16 columns with look-ahead: a
// thread per later column solves R11^T X = G12 for its 16 entries of the
// block row; the trailing update of the next block row runs first (a thread
// per column); then warp 0 factors the next diagonal block in registers while
// the other warps update the rows below it.  Three barriers per block, and
// the diagonal factorization off the critical path while the trailing
// triangle is large.  Every element of G sees the same operations in the same
// order as in the plain right-looking order.  Returns false (uniformly) when
// a pivot is not positive (G not numerically positive definite in T).
// tile: 16 n elements, 16-byte aligned (the block row of R right of the
// diagonal block, 16 consecutive values per column); r11: 256 elements,
// 16-byte aligned (the current diagonal block of R, dense).
template <class T, int NT>
__device__ bool fix_cholesky(const CtaGroup<NT>& g, FixShared<T>& fs, T* R, int n, T* tile,
                             T* r11)
{
    static_assert(NT > 32, "the look-ahead needs warps besides warp 0");
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid < 32) {
        const bool bad = fix_chol_diag<T>(R, n, 0, min(kFixPanel, n), lane, fs.chol_rdiag, r11);
        if (lane == 0)
            fs.chol_fail = bad ? 1 : 0;
    }
    g.sync();
    if (fs.chol_fail)
        return false;
    for (int c0 = 0; c0 + kFixPanel < n; c0 += kFixPanel) {
        const int nb = kFixPanel;  // every block but the last is full
        const int c1 = c0 + nb;
        // R(c0:c1, j) for j >= c1: forward substitution with R11^T, one column
        // per thread, R11 row by row from the dense copy (broadcast 16-byte
        // loads) and its diagonal as reciprocals from the factor step; each
        // entry takes its terms in the order l = 0, 1, ... as a column-wise
        // substitution would
        for (int j = c1 + tid; j < n; j += NT) {
            T x[kFixPanel];
#pragma unroll
            for (int i = 0; i < kFixPanel; i++)
                x[i] = R[fix_rs(c0 + i, n) + (j - c0 - i)];
#pragma unroll
            for (int l = 0; l < kFixPanel; l++) {
                x[l] = x[l] * fs.chol_rdiag[l];
                T rl[kFixPanel];
                fix_load16(r11 + l * kFixPanel, rl);
#pragma unroll
                for (int i = 0; i < kFixPanel; i++)
                    if (i > l)
                        x[i] -= rl[i] * x[l];
            }
            T* tj = tile + static_cast<size_t>(j - c1) * kFixPanel;
#pragma unroll
            for (int i = 0; i < kFixPanel; i++) {
                R[fix_rs(c0 + i, n) + (j - c0 - i)] = x[i];
                tj[i] = x[i];
            }
        }
        g.sync();
        const int nb2 = min(kFixPanel, n - c1);
        const int c2 = c1 + nb2;
        // trailing update of the next block row: G(i, j) -= sum_l R(c0 + l, i) R(c0 + l, j),
        // c1 <= i < c2, i <= j < n
        for (int j = c1 + tid; j < n; j += NT) {
            T rj[kFixPanel];
            fix_load16(tile + static_cast<size_t>(j - c1) * kFixPanel, rj);
            T* gj = R + j;
            const int iend = min(j, c2 - 1);
            for (int i = c1; i <= iend; i++) {
                T v[kFixPanel];
                fix_load16(tile + static_cast<size_t>(i - c1) * kFixPanel, v);
                T s0 = T(0), s1 = T(0);
#pragma unroll
                for (int l = 0; l < kFixPanel; l += 2) {
                    s0 += v[l] * rj[l];
                    s1 += v[l + 1] * rj[l + 1];
                }
                gj[fix_rs(i, n) - i] -= s0 + s1;
            }
        }
        g.sync();
        if (tid < 32) {
            // the next diagonal block is final: factor it
            const bool bad = fix_chol_diag<T>(R, n, c1, nb2, lane, fs.chol_rdiag, r11);
            if (lane == 0 && bad)
                fs.chol_fail = 1;
        } else {
            // ... while the other warps update the rows below it
            for (int j = c2 + tid - 32; j < n; j += NT - 32) {
                T rj[kFixPanel];
                fix_load16(tile + static_cast<size_t>(j - c1) * kFixPanel, rj);
                T* gj = R + j;
                for (int i = c2; i <= j; i++) {
                    T v[kFixPanel];
                    fix_load16(tile + static_cast<size_t>(i - c1) * kFixPanel, v);
                    T s0 = T(0), s1 = T(0);
#pragma unroll
                    for (int l = 0; l < kFixPanel; l += 2) {
                        s0 += v[l] * rj[l];
                        s1 += v[l + 1] * rj[l + 1];
                    }
                    gj[fix_rs(i, n) - i] -= s0 + s1;
                }
            }
        }
        g.sync();
        if (fs.chol_fail)
            return false;
    }
    return true;
}

// Inverses of the 16 x 16 diagonal blocks of R (packed rows, fix_rs), block b
// at Dinv + 256 b, column-major (D(r, c) at r + 16 c, zero below the
// diagonal).  Thread (b, i) solves U x = e_i for column i of block b.  R must
// have a nonzero diagonal.
template <class T, int NT>
__device__ void fix_invert_diag(const T* R, int n, T* Dinv)
{
    const int nblk = (n + kFixPanel - 1) / kFixPanel;
    for (int t = threadIdx.x; t < nblk * kFixPanel; t += NT) {
        const int b = t / kFixPanel, i = t % kFixPanel;
        const int b0 = kFixPanel * b;
        const int nbk = min(kFixPanel, n - b0);
        T col[kFixPanel];
#pragma unroll
        for (int r = kFixPanel - 1; r >= 0; r--) {
            T acc = T(0);
            if (r < i && i < nbk) {
                const T* ur = R + fix_rs(b0 + r, n) - (b0 + r);  // ur[b0 + k] = U(r, k)
#pragma unroll
                for (int k = 0; k < kFixPanel; k++)
                    if (k > r && k <= i)
                        acc += ur[b0 + k] * col[k];
            }
            const T urr = (r < nbk) ? R[fix_rs(b0 + r, n)] : T(1);
            col[r] = (i >= nbk || r > i) ? T(0) : (r == i ? T(1) / urr : -acc / urr);
        }
        T* D = Dinv + kFixPanel * kFixPanel * b;
#pragma unroll
        for (int r = 0; r < kFixPanel; r++)
            D[r + kFixPanel * i] = col[r];
    }
}

// R y = rhs in place with the inverted diagonal blocks: per block (from the
// bottom) y_b = D_b^-1 y_b by warp 0, then the rows above update.
template <class T, int NT>
__device__ void fix_back_inv(const CtaGroup<NT>& g, const T* R, const T* Dinv, int n, T* y)
{
    const int lane = threadIdx.x & 31;
    const int nblk = (n + kFixPanel - 1) / kFixPanel;
    FIX_SUB_BEGIN();
    for (int b = nblk - 1; b >= 0; b--) {
        const int b0 = kFixPanel * b;
        const int b1 = min(n, b0 + kFixPanel);
        const int nbk = b1 - b0;
        if (threadIdx.x < 32) {
            const T* D = Dinv + kFixPanel * kFixPanel * b;
            T acc0 = T(0), acc1 = T(0);
            if (lane < nbk) {
#pragma unroll
                for (int k = 0; k < kFixPanel; k += 2) {
                    if (k >= lane && k < nbk)
                        acc0 += D[lane + kFixPanel * k] * y[b0 + k];
                    if (k + 1 >= lane && k + 1 < nbk)
                        acc1 += D[lane + kFixPanel * (k + 1)] * y[b0 + k + 1];
                }
            }
            __syncwarp();
            if (lane < nbk)
                y[b0 + lane] = acc0 + acc1;
        }
        g.sync();
        FIX_SUB(14);
        for (int i = threadIdx.x; i < b0; i += NT) {
            const T* ri = R + fix_rs(i, n) - i;
            T s0 = T(0), s1 = T(0);
            int j = b0;
            for (; j + 1 < b1; j += 2) {
                s0 += ri[j] * y[j];
                s1 += ri[j + 1] * y[j + 1];
            }
            if (j < b1)
                s0 += ri[j] * y[j];
            y[i] -= s0 + s1;
        }
        g.sync();
        FIX_SUB(15);
    }
}

// R^T z = rhs in place with the inverted diagonal blocks, from the top.
template <class T, int NT>
__device__ void fix_forward_inv(const CtaGroup<NT>& g, const T* R, const T* Dinv, int n, T* z)
{
    const int lane = threadIdx.x & 31;
    const int nblk = (n + kFixPanel - 1) / kFixPanel;
    for (int b = 0; b < nblk; b++) {
        const int b0 = kFixPanel * b;
        const int b1 = min(n, b0 + kFixPanel);
        const int nbk = b1 - b0;
        if (threadIdx.x < 32) {
            const T* D = Dinv + kFixPanel * kFixPanel * b;
            T acc0 = T(0), acc1 = T(0);
            if (lane < nbk) {
#pragma unroll
                for (int k = 0; k < kFixPanel; k += 2) {
                    if (k <= lane)
                        acc0 += D[k + kFixPanel * lane] * z[b0 + k];
                    if (k + 1 <= lane)
                        acc1 += D[k + 1 + kFixPanel * lane] * z[b0 + k + 1];
                }
            }
            __syncwarp();
            if (lane < nbk)
                z[b0 + lane] = acc0 + acc1;
        }
        g.sync();
        for (int j = b1 + threadIdx.x; j < n; j += NT) {
            T s0 = T(0), s1 = T(0);
            int i = b0;
            for (; i + 1 < b1; i += 2) {
                s0 += R[fix_rs(i, n) + (j - i)] * z[i];
                s1 += R[fix_rs(i + 1, n) + (j - i - 1)] * z[i + 1];
            }
            if (i < b1)
                s0 += R[fix_rs(i, n) + (j - i)] * z[i];
            z[j] -= s0 + s1;
        }
        g.sync();
    }
}

// Solves fixed-pattern column `col`.  Returns false (uniformly) when the
// column's arrays do not fit the arena; nothing of the column is written then.
// rglob: this CTA's global area for R when R does not fit the arena
// (rglob_elems elements).
template <class T, int NT>
__device__ bool fixed_solve_column(const CtaGroup<NT>& g, FixShared<T>& fs, const Problem& pb,
                                   const Output& out, int col, char* arena_base, int arena_cap,
                                   T* rglob, int64_t rglob_elems)
{
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t p0 = pb.pptr[col];
    const int n = static_cast<int>(pb.pptr[col + 1] - p0);
    FixArena a{arena_base, arena_cap, 0, arena_cap};
    PHASE_BEGIN();

    // ---- column starts and lengths of C(:, J), entry offsets
    int32_t* off = a.low<int32_t>(n + 1);
    double* x = a.low<double>(n);
    double* d0sq = a.low<double>(n);
    int64_t* cbase = a.high<int64_t>(n);  // transient: start of C(:, J(t))
    if (!a.ok())
        return false;
    for (int t = tid; t < n; t += NT) {
        const int j = pb.pidx[p0 + t];
        const int64_t b0 = pb.cptr[j];
        cbase[t] = b0;
        off[t] = static_cast<int>(pb.cptr[j + 1] - b0);
    }
    // the target column: e_col, or B(:, col) (at most kFixMaxSpecial entries)
    const int ntg = pb.bptr ? static_cast<int>(pb.bptr[col + 1] - pb.bptr[col]) : 1;
    if (ntg > kFixMaxSpecial)
        return false;
    if (tid < ntg) {
        if (pb.bptr) {
            fs.tg_row[tid] = pb.bidx[pb.bptr[col] + tid];
            fs.tg_val[tid] = pb.bval[pb.bptr[col] + tid];
        }
        else {
            fs.tg_row[0] = col;
            fs.tg_val[0] = 1.0;
        }
    }
    g.sync();
    const int E = group_exclusive_scan(g, off, n);
    if (tid == 0) {
        off[n] = E;
        fs.nspec = 0;
    }
    g.sync();

    // ---- entries: rows and values in entry order; the rows counted in a
    // shared-memory hash table (open addressing, linear probing).  A row with
    // two or more entries is shared; only the shared entries are sorted later.
    const int hbits = 32 - __clz(max(64, E + E / 2) - 1);  // >= 1.5 E slots
    const int HS = 1 << hbits;
    // slot: -1 empty, else the row, with bit 31 set once a second entry of the
    // row arrives (rows are < 2^31 - 1)
    int32_t* hkey = a.high<int32_t>(HS);
    int32_t* erow = a.high<int32_t>(E + 1);
    int32_t* se = a.high<int32_t>(E + 1);   // shared flag -> q(e)
    double* V = a.high<double>(E);
    if (!a.ok())
        return false;
    for (int i = tid; i < HS; i += NT)
        hkey[i] = -1;
    if (tid == 0)
        fs.mcount = 0;
    FIX_SUB_BEGIN();
    for (int e = tid; e < E; e += NT) {
        const int jj = fix_entry_column(off, n, e);
        const int64_t q = cbase[jj] + (e - off[jj]);
        erow[e] = pb.cidx[q];
        V[e] = pb.cval[q];
    }
    g.sync();
    FIX_SUB(8);
    for (int e = tid; e < E; e += NT) {
        const int row = erow[e];
        uint32_t h = (static_cast<uint32_t>(row) * 2654435761u) >> (32 - hbits);
        for (int probe = 0; probe < HS; probe++) {
            const int old = atomicCAS(&hkey[h], -1, row);
            if (old == -1) {
                atomicAdd(&fs.mcount, 1);
                break;
            }
            if ((old & 0x7fffffff) == row) {
                atomicOr(&hkey[h], static_cast<int>(0x80000000u));
                break;
            }
            h = (h + 1) & (HS - 1);
        }
    }
    g.sync();
    FIX_SUB(9);
    PHASE_MARK(0);
    // shared flags; singleton entries whose row is a target row are kept
    // apart (their values leave V)
    for (int e = tid; e < E; e += NT) {
        const int row = erow[e];
        uint32_t h = (static_cast<uint32_t>(row) * 2654435761u) >> (32 - hbits);
        while ((hkey[h] & 0x7fffffff) != row)
            h = (h + 1) & (HS - 1);
        const int sh = (hkey[h] < 0) ? 1 : 0;
        se[e] = sh;
        if (!sh) {
            for (int t = 0; t < ntg; t++) {
                if (fs.tg_row[t] == row) {
                    const int k = atomicAdd(&fs.nspec, 1);
                    if (k < kFixMaxSpecial) {
                        fs.spec_e[k] = e;
                        fs.spec_jj[k] = fix_entry_column(off, n, e);
                        fs.spec_v[k] = V[e];
                        fs.spec_b[k] = fs.tg_val[t];
                    }
                    V[e] = 0.0;  // not part of the singleton sums d0
                }
            }
        }
    }
    g.sync();
    const int m = fs.mcount;  // |I_k|
    const int nspec = fs.nspec;
    if (nspec > kFixMaxSpecial)
        return false;
    if (tid == 0) {
        // entry order (the atomic order above is not fixed)
        for (int s2 = 1; s2 < nspec; s2++) {
            const int e = fs.spec_e[s2], jj = fs.spec_jj[s2];
            const double v = fs.spec_v[s2], b = fs.spec_b[s2];
            int q = s2;
            while (q > 0 && fs.spec_e[q - 1] > e) {
                fs.spec_e[q] = fs.spec_e[q - 1];
                fs.spec_jj[q] = fs.spec_jj[q - 1];
                fs.spec_v[q] = fs.spec_v[q - 1];
                fs.spec_b[q] = fs.spec_b[q - 1];
                q--;
            }
            fs.spec_e[q] = e;
            fs.spec_jj[q] = jj;
            fs.spec_v[q] = v;
            fs.spec_b[q] = b;
        }
    }
    // singleton sums per column: d0_j = sum of v^2 over the column's singleton
    // entries (a warp per column, lanes in entry order)
    for (int jj = warp; jj < n; jj += NW) {
        double s0 = 0.0;
        for (int e = off[jj] + lane; e < off[jj + 1]; e += 32)
            if (!se[e])
                s0 += V[e] * V[e];
        s0 = warp_sum(s0);
        if (lane == 0)
            d0sq[jj] = s0;
    }
    g.sync();
    const int SEn = group_exclusive_scan(g, se, E);  // se[e] = q(e): place in column order
    if (tid == 0)
        se[E] = SEn;
    // shared entries as (row << 32 | e) keys, sorted: row order
    const int LSE = next_pow2(SEn > 0 ? SEn : 1);
    uint64_t* SEk = a.high<uint64_t>(LSE);
    if (!a.ok())
        return false;
    g.sync();
    for (int e = tid; e < E; e += NT)
        if (se[e + 1] > se[e])
            SEk[se[e]] = (static_cast<uint64_t>(erow[e]) << 32) | static_cast<uint32_t>(e);
    for (int i = SEn + tid; i < LSE; i += NT)
        SEk[i] = ~uint64_t(0);
    g.sync();
    group_bitonic_sort(g, SEk, LSE);
    const uint64_t* Z = SEk;
    auto krow = [&](int i) { return static_cast<int>(Z[i] >> 32); };

    // ---- shared entries: column order (q) and row order (t, the sorted keys)
    int32_t* cstart = a.low<int32_t>(n + 1);
    double* csh_v = a.low<double>(SEn);
    int32_t* csh_jj = a.low<int32_t>(SEn);
    int32_t* csh_d = a.low<int32_t>(SEn);
    int32_t* rq = a.low<int32_t>(SEn);
    int32_t* gtmp = a.high<int32_t>(SEn + 1);  // row-group flags -> group numbers
    if (!a.ok())
        return false;
    for (int t = tid; t < SEn; t += NT) {
        const int e = static_cast<int>(Z[t] & 0xffffffffu);
        const int q = se[e];
        rq[t] = q;
        csh_v[q] = V[e];
        csh_jj[q] = fix_entry_column(off, n, e);
        gtmp[t] = (t == 0 || krow(t - 1) != krow(t)) ? 1 : 0;
    }
    for (int jj = tid; jj < n; jj += NT)
        cstart[jj] = se[off[jj]];
    if (tid == 0)
        cstart[n] = SEn;
    g.sync();
    const int S = group_exclusive_scan(g, gtmp, SEn);  // group of t = gtmp[t + 1] - 1
    if (tid == 0)
        gtmp[SEn] = S;
    int32_t* gstart = a.low<int32_t>(S + 1);
    int32_t* sof = a.low<int32_t>(S);      // group of row d
    int32_t* rowoff = a.low<int32_t>(S);   // skyline offset of row d
    int32_t* c0row = a.low<int32_t>(S);    // first stored column of row d
    double* bd = a.low<double>(S);         // target value of row d
    double* rd = a.low<double>(S);         // FP64 residual of row d
    if (S + kFixPanel > 32 * 2 * (NT / 32))
        return false;  // taller panels than the register tiling of fix_panel_qr
    const int LS = next_pow2(S > 0 ? S : 1);
    uint64_t* RK = a.high<uint64_t>(LS);
    int32_t* dof = a.high<int32_t>(S);     // d of group s
    double* btmp = a.high<double>(S);      // target value of group s
    if (!a.ok())
        return false;
    g.sync();
    // one thread per shared row: its first entry (smallest entry number, so
    // the smallest column) gives the key (first column, group)
    for (int t = tid; t < SEn; t += NT) {
        if (!(t == 0 || krow(t - 1) != krow(t)))
            continue;
        const int row = krow(t);
        const int sgrp = gtmp[t];
        const int e = static_cast<int>(Z[t] & 0xffffffffu);
        gstart[sgrp] = t;
        RK[sgrp] = (static_cast<uint64_t>(fix_entry_column(off, n, e)) << 32) |
                   static_cast<uint32_t>(sgrp);
        double b = 0.0;
        for (int q = 0; q < ntg; q++)
            if (fs.tg_row[q] == row)
                b = fs.tg_val[q];
        btmp[sgrp] = b;
    }
    for (int i = S + tid; i < LS; i += NT)
        RK[i] = ~uint64_t(0);
    if (tid == 0)
        gstart[S] = SEn;
    g.sync();
    group_bitonic_sort(g, RK, LS);
    for (int d = tid; d < S; d += NT) {
        const int sgrp = static_cast<int>(RK[d] & 0xffffffffu);
        const int f = static_cast<int>(RK[d] >> 32);
        sof[d] = sgrp;
        dof[sgrp] = d;
        c0row[d] = (f / kFixPanel) * kFixPanel;
        bd[d] = btmp[sgrp];
    }
    g.sync();
    // d of every shared entry (column order)
    for (int t = tid; t < SEn; t += NT)
        csh_d[rq[t]] = dof[gtmp[t + 1] - 1];
    g.sync();
    PHASE_MARK(1);

    // FP64 residual r = b - C(I, J) x on the shared rows, its squared norm
    // with the singleton rows' part from d0 and the target entries kept
    // apart; with grad, C^T r into gv (in T)
    auto residual = [&](bool grad, T* gv) -> double {
        double part = 0.0;
        for (int d = tid; d < S; d += NT) {
            const int s = sof[d];
            double v = bd[d];
            for (int t = gstart[s]; t < gstart[s + 1]; t++) {
                const int q = rq[t];
                v -= csh_v[q] * x[csh_jj[q]];
            }
            rd[d] = v;
            part += v * v;
        }
        for (int jj = tid; jj < n; jj += NT)
            part += x[jj] * x[jj] * d0sq[jj];
        if (tid == 0)
            for (int s = 0; s < nspec; s++) {
                const double r = fs.spec_b[s] - fs.spec_v[s] * x[fs.spec_jj[s]];
                part += r * r;
            }
        const double r2 = g.sum(part);  // includes a barrier: rd is complete
        if (grad) {
            for (int jj = tid; jj < n; jj += NT) {
                double acc = -x[jj] * d0sq[jj];
                for (int q = cstart[jj]; q < cstart[jj + 1]; q++)
                    acc += csh_v[q] * rd[csh_d[q]];
                for (int s = 0; s < nspec; s++)
                    if (fs.spec_jj[s] == jj)
                        acc += fs.spec_v[s] * (fs.spec_b[s] - fs.spec_v[s] * x[jj]);
                gv[jj] = static_cast<T>(acc);
            }
            g.sync();
        }
        return r2;
    };
    // Refinement x += R^-1 R^-T C^T (b - C x), gv holding C^T r on entry, at
    // most max_steps steps; r2 is updated.  Returns true when the last
    // correction fell below 2^-44 of the solution (converged); stops early
    // when the corrections no longer contract.
    int ref_steps = 0;  // refinement steps taken
    auto refine = [&](const T* R, const T* Dinv, T* gv, int max_steps, double& r2) -> bool {
        double d2_prev = 0.0;
        for (int it = 0; it < max_steps; it++) {
            ref_steps++;
            if (Dinv) {
                fix_forward_inv<T, NT>(g, R, Dinv, n, gv);
                fix_back_inv<T, NT>(g, R, Dinv, n, gv);
            }
            else {
                fix_forward_substitute<T, NT>(g, R, n, gv);
                fix_back_substitute<T, NT>(g, R, n, gv);
            }
            double d2 = 0.0, x2 = 0.0;
            for (int i = tid; i < n; i += NT) {
                const double dl = static_cast<double>(gv[i]);
                const double x1 = x[i] + dl;
                d2 += dl * dl;
                x2 += x1 * x1;
                x[i] = x1;
            }
            d2 = g.sum(d2);
            x2 = g.sum(x2);
            // converged (correction below 2^-44 of the solution), or no
            // longer contracting (R too far from this column's matrix)
            const bool conv = d2 <= 0x1p-88 * x2;
            const bool last = conv || (it + 1 == max_steps) || (it > 0 && d2 > 0.25 * d2_prev);
            d2_prev = d2;
            r2 = residual(!last, gv);
            if (last)
                return conv;
        }
        return false;
    };
    // outputs (M has P's pattern: values only); fwork: the folded flops done
    auto finish = [&](double r2, int sing, double fwork) {
        const double res = sqrt(r2);
        int nonfinite = 0;
        for (int t = tid; t < n; t += NT) {
            const double v = x[t];
            if (!isfinite(v))
                nonfinite = 1;
            out.oval[p0 + t] = v;
        }
        nonfinite = g.sum(nonfinite);
        if (tid == 0) {
            const double dn = n, dm = m;
            double* wk = out.work + 3 * static_cast<size_t>(col);
            wk[0] += fwork;
            wk[1] += 2.0 * dm * dn * dn - (2.0 / 3.0) * dn * dn * dn + 4.0 * dm * dn + 2.0 * dm * dn;
            wk[2] += 12.0 * E + 16.0 * dn + 8.0 * dm;
            out.olen[col] = n;
            out.res[col] = res;
            out.steps[col] = 1;
            out.status[col] = sing ? 1 : ((nonfinite || !isfinite(res)) ? 2 : 0);
        }
        g.sync();
    };

    // ---- re-setup from the kept factor: the previous solution and R, FP64
    // refinement against the new values; not converged -> factored below
    if (out.reuse_steps > 0 && out.rstore) {
        FixArena b2 = a;
        b2.hi = arena_cap;  // the transient arrays are dead
        const int r_el = fix_rs(n, n);
        T* gv = b2.low<T>(n);
        T* Rr = nullptr;
        if (b2.ok()) {
            FixArena b3 = b2;
            T* rr = b3.low<T>(r_el);
            if (b3.ok()) {
                Rr = rr;
                b2 = b3;
            }
            else if (rglob != nullptr && rglob_elems >= r_el) {
                Rr = rglob;
            }
        }
        if (Rr != nullptr) {
            const T* src = static_cast<const T*>(out.rstore) + out.roff[col];
            for (int t = tid; t < n * (n + 1) / 2; t += NT) {
                int j = static_cast<int>((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
                while (j * (j + 1) / 2 > t)
                    j--;
                while ((j + 1) * (j + 2) / 2 <= t)
                    j++;
                const int i = t - j * (j + 1) / 2;
                Rr[fix_rs(i, n) + (j - i)] = src[t];
            }
            for (int t = tid; t < n; t += NT)
                x[t] = out.oval[p0 + t];
            g.sync();
            int zero = 0;
            for (int i = tid; i < n; i += NT)
                if (Rr[fix_rs(i, n)] == T(0))
                    zero = 1;
            zero = g.sum(zero);
            if (!zero) {
                T* Dr = nullptr;
                const int nblk = (n + kFixPanel - 1) / kFixPanel;
                FixArena b4 = b2;
                T* dd = b4.low<T>(kFixPanel * kFixPanel * nblk);
                const bool r_smem = reinterpret_cast<char*>(Rr) >= arena_base &&
                                    reinterpret_cast<char*>(Rr) < arena_base + arena_cap;
                if (r_smem && b4.ok()) {
                    Dr = dd;
                    fix_invert_diag<T, NT>(Rr, n, Dr);
                    g.sync();
                }
                double r2 = residual(true, gv);
                if (refine(Rr, Dr, gv, out.reuse_steps, r2)) {
                    // per step: two triangular solves, the residual and C^T r
                    finish(r2, 0, (ref_steps + 1.0) * (2.0 * n * n + 4.0 * SEn + 3.0 * n));
                    if (tid == 0)
                        atomicAdd(out.reuse_count, 1);
                    return true;
                }
            }
            g.sync();  // every thread is done with the kept factor's arrays
        }
    }

    // ---- mixed mode: R from the Cholesky factorization of C^T C, formed in
    // T from the sparse entries (the folded diagonal in FP64), then the FP64
    // refinement from x = 0 (its first step is the normal-equations solve).
    // The factor only preconditions the refinement: R^T R equals C^T C to
    // O(u_T ||C||^2), as the R of the Householder QR in T does, so the
    // corrections contract alike; the refinement ends at the least-squares
    // solution in FP64.  A column whose Cholesky meets a pivot <= 0 or whose
    // refinement does not converge takes the Householder path below.  (FP64
    // mode has no refinement and keeps the Householder QR.)
    if constexpr (sizeof(T) == 4) if (pb.refine > 0) {
        FixArena b2 = a;
        b2.hi = arena_cap;  // the transient arrays are dead
        const int r_el = fix_rs(n, n);
        const int nblk = (n + kFixPanel - 1) / kFixPanel;
        T* gv = b2.low<T>(n);
        T* Gs = b2.low<T>(r_el);
        // the tile is dead once the factorization ends: the inverted diagonal
        // blocks take its place
        T* tile = b2.low<T>(max(kFixPanel * n, kFixPanel * kFixPanel * nblk));
        T* Dr = tile;
        T* r11 = b2.low<T>(kFixPanel * kFixPanel);  // the current diagonal block
        if (b2.ok()) {
            // G = C^T C: column j of G's lower triangle (= row j of its upper
            // triangle, packed as R) by one thread, in entry order
            for (int j = tid; j < n; j += NT) {
                T* row = Gs + fix_rs(j, n) - j;  // row[c] = G(j, c), c >= j
                for (int c = j; c <= n; c++)
                    row[c] = T(0);
                double dd = d0sq[j];
                for (int sp = 0; sp < nspec; sp++)
                    if (fs.spec_jj[sp] == j)
                        dd += fs.spec_v[sp] * fs.spec_v[sp];
                for (int q = cstart[j]; q < cstart[j + 1]; q++) {
                    const double vq = csh_v[q];
                    const int grp_s = sof[csh_d[q]];
                    for (int t = gstart[grp_s]; t < gstart[grp_s + 1]; t++) {
                        const int q2 = rq[t];
                        const int j2 = csh_jj[q2];
                        if (j2 > j)
                            row[j2] += static_cast<T>(vq * csh_v[q2]);
                        else if (j2 == j)
                            dd += vq * csh_v[q2];
                    }
                }
                row[j] = static_cast<T>(dd);
            }
            g.sync();
            PHASE_MARK(2);
            const bool factored = fix_cholesky<T, NT>(g, fs, Gs, n, tile, r11);
            PHASE_MARK(3);
            if (factored) {
                fix_invert_diag<T, NT>(Gs, n, Dr);
                for (int t = tid; t < n; t += NT)
                    x[t] = 0.0;
                g.sync();
                PHASE_MARK(6);
                double r2 = residual(true, gv);  // gv = C^T b
                ref_steps = 0;
                const bool conv = refine(Gs, Dr, gv, pb.refine + 2, r2);
                PHASE_MARK(7);
                if (conv) {
                    if (out.rstore) {
                        T* dst = static_cast<T*>(out.rstore) + out.roff[col];
                        for (int t = tid; t < n * (n + 1) / 2; t += NT) {
                            int j = static_cast<int>((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
                            while (j * (j + 1) / 2 > t)
                                j--;
                            while ((j + 1) * (j + 2) / 2 <= t)
                                j++;
                            const int i = t - j * (j + 1) / 2;
                            dst[t] = Gs[fix_rs(i, n) + (j - i)];
                        }
                    }
                    const double dn = n;
                    finish(r2, 0,
                           dn * dn * dn / 3.0 + 2.0 * SEn + ref_steps * (2.0 * dn * dn + 4.0 * SEn));
                    return true;
                }
            }
            g.sync();  // every thread is done with the factor's arrays
        }
    }

    // ---- skyline of the shared rows, diagonal rows H, [R, Q^T b]
    const int ldw = (n + 1 + 3) & ~3;
    for (int d = tid; d < S; d += NT)
        rowoff[d] = ldw - c0row[d];
    g.sync();
    const int sky_total = group_exclusive_scan(g, rowoff, S);
    a.hi = arena_cap;  // the transient arrays are dead
    T* dv = a.low<T>(n);   // folded diagonal d_j
    T* tv = a.low<T>(n);   // folded right-hand side t_j
    T* yv = a.low<T>(n);   // triangular-solve vector
    T* sky = a.low<T>(sky_total + kFixPanel);
    T* H = a.low<T>(kFixPanel * ldw + kFixPanel);
    int32_t* prow = a.low<int32_t>(S + kFixPanel);  // panel rows: element offsets from tb
    if (!a.ok())
        return false;
    T* tb = reinterpret_cast<T*>(arena_base);
    const int r_elems = fix_rs(n, n);  // n(n+1)/2 + n
    T* Rst;
    bool r_in_smem;
    {
        FixArena b2 = a;
        T* rs = b2.low<T>(r_elems);
        r_in_smem = b2.ok();
        Rst = r_in_smem ? rs : rglob;
        if (r_in_smem)
            a = b2;
        else if (rglob == nullptr || rglob_elems < r_elems)
            return false;
    }
    // folded diagonal rows (FP64 sums, stored in T)
    for (int jj = tid; jj < n; jj += NT) {
        double dd = d0sq[jj], tb = 0.0;
        for (int s = 0; s < nspec; s++) {
            if (fs.spec_jj[s] == jj) {
                dd += fs.spec_v[s] * fs.spec_v[s];
                tb += fs.spec_v[s] * fs.spec_b[s];
            }
        }
        const double nrm = sqrt(dd);
        dv[jj] = static_cast<T>(nrm);
        tv[jj] = static_cast<T>(nrm > 0.0 ? tb / nrm : 0.0);
    }
    for (int i = tid; i < sky_total + kFixPanel; i += NT)
        sky[i] = T(0);
    for (int i = tid; i < kFixPanel * ldw + kFixPanel; i += NT)
        H[i] = T(0);
    g.sync();
    for (int q = tid; q < SEn; q += NT) {
        const int d = csh_d[q];
        sky[rowoff[d] + (csh_jj[q] - c0row[d])] = static_cast<T>(csh_v[q]);
    }
    for (int d = tid; d < S; d += NT)
        sky[rowoff[d] + (n - c0row[d])] = static_cast<T>(bd[d]);
    g.sync();
    PHASE_MARK(2);

    // ---- QR by panels
    const int npan = (n + kFixPanel - 1) / kFixPanel;
    int Ap = 0;
    for (int p = 0; p < npan; p++) {
        const int c0 = p * kFixPanel;
        const int nb = min(kFixPanel, n - c0);
        while (Ap < S && c0row[Ap] <= c0)  // uniform: every thread reads the same
            Ap++;
        const int mp = nb + Ap;
        // diagonal rows c0 .. c0 + nb - 1 over columns c0 .. n; the row table
        for (int i = 0; i < nb; i++) {
            T* hr = H + static_cast<size_t>(i) * ldw;
            for (int c = c0 + tid; c <= n; c += NT)
                hr[c] = (c == c0 + i) ? dv[c0 + i] : (c == n ? tv[c0 + i] : T(0));
        }
        for (int i = tid; i < mp; i += NT)
            prow[i] = (i < nb) ? static_cast<int32_t>(H - tb) + i * ldw + c0
                               : static_cast<int32_t>(sky - tb) + rowoff[i - nb] + (c0 - c0row[i - nb]);
        g.sync();
        PHASE_MARK(5);
        if (!fix_panel_qr<T, NT>(fs, tb, prow, nb, mp))
            return false;  // not reached: the panel height was checked above
        PHASE_MARK(3);
        fix_trailing<T, NT>(fs, tb, prow, nb, c0, mp, n);
        g.sync();
        PHASE_MARK(4);
        // rows c0 .. c0 + nb - 1 of [R, Q^T b]
        for (int i = 0; i < nb; i++) {
            const int r = c0 + i;
            const T* hr = H + static_cast<size_t>(i) * ldw;
            T* dst = Rst + fix_rs(r, n) - r;
            for (int c = r + tid; c <= n; c += NT)
                dst[c] = hr[c];
        }
        g.sync();
        PHASE_MARK(5);
    }

    // the caller keeps R (packed by columns) for the adjoint
    if (out.rstore) {
        T* dst = static_cast<T*>(out.rstore) + out.roff[col];
        for (int t = tid; t < n * (n + 1) / 2; t += NT) {
            int j = static_cast<int>((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
            while (j * (j + 1) / 2 > t)
                j--;
            while ((j + 1) * (j + 2) / 2 <= t)
                j++;
            const int i = t - j * (j + 1) / 2;
            dst[t] = Rst[fix_rs(i, n) + (j - i)];
        }
    }

    // R in global memory: move it into the skyline's region, dead after the QR
    if (!r_in_smem && reinterpret_cast<char*>(sky + r_elems) <= arena_base + arena_cap) {
        for (int i = tid; i < r_elems; i += NT)
            sky[i] = Rst[i];
        g.sync();
        Rst = sky;
    }

    // ---- back substitution; R singular -> x = (Q^T b)(0:n) (dtrtrs leaves B)
    int sing = 0;
    for (int i = tid; i < n; i += NT) {
        yv[i] = Rst[fix_rs(i, n) + (n - i)];
        if (Rst[fix_rs(i, n)] == T(0))
            sing = 1;
    }
    sing = g.sum(sing) > 0;
    // inverted diagonal blocks of R, in shared memory after R when there is room
    T* Dinv = nullptr;
    if (!sing) {
        const int nblk = (n + kFixPanel - 1) / kFixPanel;
        char* rend = reinterpret_cast<char*>(Rst + r_elems);
        char* dbeg = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(rend) + 15) & ~uintptr_t(15));
        const bool r_smem = reinterpret_cast<char*>(Rst) >= arena_base &&
                            reinterpret_cast<char*>(Rst) < arena_base + arena_cap;
        if (r_smem && dbeg + sizeof(T) * kFixPanel * kFixPanel * nblk <= arena_base + arena_cap) {
            Dinv = reinterpret_cast<T*>(dbeg);
            fix_invert_diag<T, NT>(Rst, n, Dinv);
            g.sync();
        }
    }
    if (!sing) {
        if (Dinv)
            fix_back_inv<T, NT>(g, Rst, Dinv, n, yv);
        else
            fix_back_substitute<T, NT>(g, Rst, n, yv);
    }
    for (int i = tid; i < n; i += NT)
        x[i] = static_cast<double>(yv[i]);
    g.sync();
    PHASE_MARK(6);

    // ---- FP64 residual (and refinement in mixed mode)
    double r2 = residual(!sing && pb.refine > 0, yv);
    if (!sing)
        refine(Rst, Dinv, yv, pb.refine, r2);
    PHASE_MARK(7);
    // algorithmic work: the skyline QR (panel factorization and compact-WY
    // update), Q^T b, the solve and the FP64 residual
    double fwork = 0.0;
    {
        int ap = 0;
        for (int p = 0; p < npan; p++) {
            const int c0 = p * kFixPanel;
            const double nb = min(kFixPanel, n - c0);
            while (ap < S && c0row[ap] <= c0)
                ap++;
            const double mp = nb + ap, nc = n + 1 - c0 - nb;
            fwork += 2.0 * mp * nb * nb - (2.0 / 3.0) * nb * nb * nb + 4.0 * mp * nb * nc;
        }
        fwork += static_cast<double>(n) * n + 2.0 * E;
    }
    finish(r2, sing, fwork);
    return true;
}

}  // namespace mspai
