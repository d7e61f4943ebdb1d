// Blocked Householder QR and blocked triangular solves for one CTA.
//
// The folded least-squares matrix W (mw x n, column-major, ld = mw) lives in
// shared memory when it fits, else in the CTA's global scratch slot.  The QR
// follows LAPACK's dgeqrf: 16-column panels are factored with unblocked
// Householder reflectors (dgeqr2), the panel's reflectors are accumulated into
// the compact WY form H_0...H_{nb-1} = I - V T V^T (dlarft, forward,
// columnwise), and the trailing columns plus the right-hand side are updated
// as W2 <- W2 - V (T^T (V^T W2)) (dlarfb, transposed).  The trailing update is
// a register-tiled mini-GEMM: one warp owns 4 trailing columns, lanes split
// the rows, the 4 x 16 partial dot products are combined with a warp
// reduce-scatter, and the rank-16 update reuses every V element for 4
// columns.  When W is in global memory the panel is staged in shared memory,
// so only the trailing update touches global memory (twice per panel instead
// of twice per column).
#pragma once

#include "spai_device.cuh"

namespace mspai {

constexpr int kPanel = 16;     // panel width
constexpr int kTileCols = 2;   // trailing columns per warp tile
constexpr int kTileVals = kTileCols * kPanel;  // partial sums per lane
constexpr int kPerLane = kTileVals / 32;        // reduced sums per lane

// Shared-memory scratch of the blocked routines (besides the W/panel area).
template <class T>
struct BlockedScratch {
    T tmat[kPanel * kPanel];  // T factor (upper triangular, column-major)
    T tau[kPanel];
    T vtv[kPanel * kPanel];   // V^T V (strictly upper part used)
    T scale[kPanel];          // 1 / (alpha - beta) of each panel column
    T beta[kPanel];           // R(k, k) of each panel column
    T nrm2[kPanel + 1];       // squared norm below the diagonal, next column
};

// V(r, i) of the panel: unit lower trapezoidal, explicit below the diagonal.
template <class T>
__device__ __forceinline__ T vpanel(const T* P, int ldp, int r, int i)
{
    const T v = P[r + static_cast<size_t>(i) * ldp];
    return r > i ? v : (r == i ? T(1) : T(0));
}

// Unblocked Householder QR of the panel P (mp x nb, ld ldp); tau[k] = 0 when
// the column below the diagonal is zero (H = I), as LAPACK's dlarfg.
template <class T, class G>
__device__ void panel_qr(const G& g, T* P, int ldp, int mp, int nb, T* tau)
{
    const int lane = g.lane();
    for (int k = 0; k < nb; k++) {
        T* pk = P + static_cast<size_t>(k) * ldp;
        T part = 0;
        for (int i = k + 1 + g.rank(); i < mp; i += G::kSize)
            part += pk[i] * pk[i];
        const T xnorm2 = g.sum(part);
        if (xnorm2 == T(0) || k >= mp) {
            if (g.rank() == 0)
                tau[k] = T(0);
            g.sync();
            continue;
        }
        const T alpha = pk[k];
        const T beta = -copysign(tsqrt<T>(alpha * alpha + xnorm2), alpha);
        const T tk = (beta - alpha) / beta;
        const T scale = T(1) / (alpha - beta);
        g.sync();
        if (g.rank() == 0) {
            pk[k] = beta;
            tau[k] = tk;
        }
        for (int i = k + 1 + g.rank(); i < mp; i += G::kSize)
            pk[i] *= scale;
        g.sync();
        for (int c = k + 1 + g.warp(); c < nb; c += G::kWarps) {
            T* col = P + static_cast<size_t>(c) * ldp;
            T d = (lane == 0) ? col[k] : T(0);
            for (int i = k + 1 + lane; i < mp; i += 32)
                d += pk[i] * col[i];
            d = warp_sum(d) * tk;
            if (lane == 0)
                col[k] -= d;
            for (int i = k + 1 + lane; i < mp; i += 32)
                col[i] -= d * pk[i];
        }
        g.sync();
    }
}

// T factor of the panel (dlarft, forward, columnwise):
//   T(k,k) = tau_k,  T(0:k, k) = -tau_k T(0:k, 0:k) V(:, 0:k)^T v_k.
template <class T, class G>
__device__ void panel_tfactor(const G& g, const T* P, int ldp, int mp, int nb,
                              BlockedScratch<T>* bs)
{
    // V^T V for j < k: (j, k) pairs spread over the warps, lanes over rows >= k
    const int lane = g.lane();
    const int pairs = nb * (nb - 1) / 2;
    for (int q = g.warp(); q < pairs; q += G::kWarps) {
        // decode q -> (j, k), j < k
        int k = 1, base = 0;
        while (base + k <= q) {
            base += k;
            k++;
        }
        const int j = q - base;
        T d = 0;
        for (int r = k + lane; r < mp; r += 32)
            d += vpanel(P, ldp, r, j) * vpanel(P, ldp, r, k);
        d = warp_sum(d);
        if (lane == 0)
            bs->vtv[j + k * kPanel] = d;
    }
    g.sync();
    if (g.warp() == 0) {
        for (int k = 0; k < nb; k++) {
            const T tk = bs->tau[k];
            // T(i, k) for i < k: -tau_k sum_{j=i}^{k-1} T(i, j) vtv(j, k)
            T v = 0;
            if (lane < k) {
                for (int j = lane; j < k; j++)
                    v += bs->tmat[lane + j * kPanel] * bs->vtv[j + k * kPanel];
                v = -tk * v;
            }
            __syncwarp();
            if (lane < k)
                bs->tmat[lane + k * kPanel] = v;
            if (lane == k)
                bs->tmat[k + k * kPanel] = tk;
            if (lane > k && lane < kPanel)
                bs->tmat[lane + k * kPanel] = T(0);
            __syncwarp();
        }
    }
    g.sync();
}

// Trailing update of `ncols` columns starting at W2 (ld ldw, rows aligned with
// the panel's rows; the right-hand sides are the last columns):
//   X <- X - V (T^T (V^T X)).
template <class T, class G>
__device__ void trailing_update(const G& g, const T* P, int ldp, int mp, int nb,
                                const BlockedScratch<T>* bs, T* W2, int ldw, int ncols)
{
    const int lane = g.lane();
    const int total = ncols;
    for (int cb = g.warp() * kTileCols; cb < total; cb += G::kWarps * kTileCols) {
        T* col[kTileCols];
#pragma unroll
        for (int c = 0; c < kTileCols; c++) {
            const int cc = cb + c;
            col[c] = (cc < ncols) ? W2 + static_cast<size_t>(cc) * ldw : nullptr;
        }
        // Y = V^T X (partial sums per lane over its rows).  Rows are taken four
        // at a time so that 16 independent loads of X are in flight per lane
        // (X may be in global memory).
        T acc[kTileVals];
#pragma unroll
        for (int t = 0; t < kTileVals; t++)
            acc[t] = T(0);
        constexpr int kRows = 4;
        int r0 = lane;
        for (; r0 + 32 * (kRows - 1) < mp; r0 += 32 * kRows) {
            T x[kRows][kTileCols];
#pragma unroll
            for (int q = 0; q < kRows; q++)
#pragma unroll
                for (int c = 0; c < kTileCols; c++)
                    x[q][c] = col[c] ? col[c][r0 + 32 * q] : T(0);
#pragma unroll
            for (int q = 0; q < kRows; q++) {
                const int r = r0 + 32 * q;
#pragma unroll
                for (int i = 0; i < kPanel; i++) {
                    const T v = (i < nb) ? vpanel(P, ldp, r, i) : T(0);
#pragma unroll
                    for (int c = 0; c < kTileCols; c++)
                        acc[c * kPanel + i] += v * x[q][c];
                }
            }
        }
        for (int r = r0; r < mp; r += 32) {
            T x[kTileCols];
#pragma unroll
            for (int c = 0; c < kTileCols; c++)
                x[c] = col[c] ? col[c][r] : T(0);
#pragma unroll
            for (int i = 0; i < kPanel; i++) {
                const T v = (i < nb) ? vpanel(P, ldp, r, i) : T(0);
#pragma unroll
                for (int c = 0; c < kTileCols; c++)
                    acc[c * kPanel + i] += v * x[c];
            }
        }
        // warp reduce-scatter: lane l ends with the sums of entries
        // kPerLane * l .. kPerLane * l + kPerLane - 1
#pragma unroll
        for (int level = 0; level < 5; level++) {
            const int half = kTileVals >> (level + 1);
            const int bit = 16 >> level;
            const bool upper = (lane & bit) != 0;
#pragma unroll
            for (int t = 0; t < kTileVals / 2; t++) {
                if (t < half) {
                    const T mine = upper ? acc[half + t] : acc[t];
                    const T other = upper ? acc[t] : acc[half + t];
                    acc[t] = mine + __shfl_xor_sync(0xffffffffu, other, bit);
                }
            }
        }
        // Y -> Z = T^T Y via a shared exchange of Y (one row per warp)
        __shared__ T ybuf_all[G::kWarps][kTileVals];
        T* ybuf = ybuf_all[g.warp()];
#pragma unroll
        for (int h = 0; h < kPerLane; h++)
            ybuf[kPerLane * lane + h] = acc[h];
        __syncwarp();
        T zl[kPerLane];
#pragma unroll
        for (int h = 0; h < kPerLane; h++) {
            const int idx = kPerLane * lane + h;
            const int c = idx / kPanel, i = idx % kPanel;
            T z = 0;
            for (int j = 0; j <= i && j < nb; j++)
                z += bs->tmat[j + i * kPanel] * ybuf[c * kPanel + j];
            zl[h] = (i < nb) ? z : T(0);
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < kPerLane; h++)
            ybuf[kPerLane * lane + h] = zl[h];
        __syncwarp();
        T zr[kTileVals];
#pragma unroll
        for (int t = 0; t < kTileVals; t++)
            zr[t] = ybuf[t];
        // X -= V Z (four rows per lane at a time: loads first, then stores)
        int r1 = lane;
        for (; r1 + 32 * (kRows - 1) < mp; r1 += 32 * kRows) {
            T x[kRows][kTileCols];
#pragma unroll
            for (int q = 0; q < kRows; q++)
#pragma unroll
                for (int c = 0; c < kTileCols; c++)
                    x[q][c] = col[c] ? col[c][r1 + 32 * q] : T(0);
#pragma unroll
            for (int q = 0; q < kRows; q++) {
                const int r = r1 + 32 * q;
#pragma unroll
                for (int i = 0; i < kPanel; i++) {
                    const T v = (i < nb) ? vpanel(P, ldp, r, i) : T(0);
#pragma unroll
                    for (int c = 0; c < kTileCols; c++)
                        x[q][c] -= v * zr[c * kPanel + i];
                }
            }
#pragma unroll
            for (int q = 0; q < kRows; q++)
#pragma unroll
                for (int c = 0; c < kTileCols; c++)
                    if (col[c])
                        col[c][r1 + 32 * q] = x[q][c];
        }
        for (int r = r1; r < mp; r += 32) {
            T x[kTileCols];
#pragma unroll
            for (int c = 0; c < kTileCols; c++)
                x[c] = col[c] ? col[c][r] : T(0);
#pragma unroll
            for (int i = 0; i < kPanel; i++) {
                const T v = (i < nb) ? vpanel(P, ldp, r, i) : T(0);
#pragma unroll
                for (int c = 0; c < kTileCols; c++)
                    x[c] -= v * zr[c * kPanel + i];
            }
#pragma unroll
            for (int c = 0; c < kTileCols; c++)
                if (col[c])
                    col[c][r] = x[c];
        }
        __syncwarp();
    }
}

// Unblocked Householder QR of the panel P (mp x nb, ld ldp) with one group
// barrier per column: the norm of column k+1 below its diagonal is computed by
// the warp that updates column k+1 during step k, the dot products of step k
// use the unscaled column k (v = scale * x), and the scaling of every panel
// column and its diagonal entry beta are applied once after the last step.
// Same reflectors as panel_qr (LAPACK dlarfg convention).
template <class T, class G>
__device__ void panel_qr_fast(const G& g, T* P, int ldp, int mp, int nb, BlockedScratch<T>* bs)
{
    const int lane = g.lane();
    {
        T part = 0;
        for (int i = 1 + g.rank(); i < mp; i += G::kSize)
            part += P[i] * P[i];
        const T x2 = g.sum(part);
        if (g.rank() == 0)
            bs->nrm2[0] = x2;
    }
    g.sync();
    for (int k = 0; k < nb; k++) {
        const T* pk = P + static_cast<size_t>(k) * ldp;
        const T alpha = pk[k];
        const T x2 = bs->nrm2[k];
        T tau = 0, scale = 0, beta = alpha;
        if (x2 != T(0)) {
            beta = -copysign(tsqrt<T>(alpha * alpha + x2), alpha);
            tau = (beta - alpha) / beta;
            scale = T(1) / (alpha - beta);
        }
        for (int c = k + 1 + g.warp(); c < nb; c += G::kWarps) {
            T* col = P + static_cast<size_t>(c) * ldp;
            if (tau != T(0)) {
                T d = 0;
                for (int i = k + 1 + lane; i < mp; i += 32)
                    d += pk[i] * col[i];
                d = (col[k] + scale * warp_sum(d)) * tau;
                if (lane == 0)
                    col[k] -= d;
                const T ds = d * scale;
                for (int i = k + 1 + lane; i < mp; i += 32)
                    col[i] -= ds * pk[i];
            }
            if (c == k + 1) {
                T q = 0;
                for (int i = k + 2 + lane; i < mp; i += 32)
                    q += col[i] * col[i];
                q = warp_sum(q);
                if (lane == 0)
                    bs->nrm2[k + 1] = q;
            }
        }
        if (g.rank() == 0) {
            bs->tau[k] = tau;
            bs->scale[k] = scale;
            bs->beta[k] = beta;
        }
        g.sync();
    }
    // deferred: v = scale * x below the diagonal, R(k, k) = beta
    for (int t = g.rank(); t < nb * mp; t += G::kSize) {
        const int k = t / mp, i = t - k * mp;
        T* pk = P + static_cast<size_t>(k) * ldp;
        if (i > k && bs->tau[k] != T(0))
            pk[i] *= bs->scale[k];
        else if (i == k)
            pk[i] = bs->beta[k];
    }
    g.sync();
}

// Applies the panel's reflectors H_0 .. H_{nb-1} (V unit lower trapezoidal in
// P, tau in bs) to `ncols` columns of W2 (ld ldw; right-hand sides included).
// One warp owns NC columns and holds them in registers (Q rows per lane, rows
// lane + 32 q) for all nb reflectors: each column is read and written once
// per panel, and every V element loaded from shared memory serves NC columns.
template <class T, class G, int Q, int NC>
__device__ void trailing_apply_q(const G& g, const T* P, int ldp, int mp, int nb,
                                 const BlockedScratch<T>* bs, T* W2, int ldw, int ncols)
{
    const int lane = g.lane();
    for (int cb = g.warp() * NC; cb < ncols; cb += G::kWarps * NC) {
        T* cp[NC];
#pragma unroll
        for (int c = 0; c < NC; c++)
            cp[c] = (cb + c < ncols) ? W2 + static_cast<size_t>(cb + c) * ldw : nullptr;
        T x[NC][Q];
#pragma unroll
        for (int q = 0; q < Q; q++) {
            const int r = lane + 32 * q;
#pragma unroll
            for (int c = 0; c < NC; c++)
                x[c][q] = (cp[c] && r < mp) ? cp[c][r] : T(0);
        }
        for (int k = 0; k < nb; k++) {
            const T tau = bs->tau[k];
            if (tau == T(0))
                continue;
            const T* pk = P + static_cast<size_t>(k) * ldp;
            T vq[Q];
            // row lane of the first 32 holds the unit diagonal / zeros above
            vq[0] = (lane > k && lane < mp) ? pk[lane] : (lane == k ? T(1) : T(0));
#pragma unroll
            for (int q = 1; q < Q; q++) {
                const int r = lane + 32 * q;
                vq[q] = (r < mp) ? pk[r] : T(0);
            }
            T d[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) {
                T a = 0;
#pragma unroll
                for (int q = 0; q < Q; q++)
                    a += vq[q] * x[c][q];
                d[c] = a;
            }
#pragma unroll
            for (int c = 0; c < NC; c++)
                d[c] = warp_sum(d[c]) * tau;
#pragma unroll
            for (int c = 0; c < NC; c++)
#pragma unroll
                for (int q = 0; q < Q; q++)
                    x[c][q] -= d[c] * vq[q];
        }
#pragma unroll
        for (int q = 0; q < Q; q++) {
            const int r = lane + 32 * q;
            if (r < mp) {
#pragma unroll
                for (int c = 0; c < NC; c++)
                    if (cp[c])
                        cp[c][r] = x[c][q];
            }
        }
    }
}

// Dispatch on the rows per lane: the smallest Q (in steps of 4) with
// 32 Q >= mp; four columns per warp tile for short panels, two otherwise.
template <class T, class G>
__device__ bool trailing_apply(const G& g, const T* P, int ldp, int mp, int nb,
                               const BlockedScratch<T>* bs, T* W2, int ldw, int ncols)
{
    const int q = (mp + 31) / 32;
    if (q <= 4)
        trailing_apply_q<T, G, 4, 4>(g, P, ldp, mp, nb, bs, W2, ldw, ncols);
    else if (q <= 8)
        trailing_apply_q<T, G, 8, 4>(g, P, ldp, mp, nb, bs, W2, ldw, ncols);
    else if (q <= 12)
        trailing_apply_q<T, G, 12, 2>(g, P, ldp, mp, nb, bs, W2, ldw, ncols);
    else if (q <= 16)
        trailing_apply_q<T, G, 16, 2>(g, P, ldp, mp, nb, bs, W2, ldw, ncols);
    else if (q <= 24)
        trailing_apply_q<T, G, 24, 1>(g, P, ldp, mp, nb, bs, W2, ldw, ncols);
    else
        return false;
    return true;
}

// Blocked Householder QR of W (mw x n, ld) applied to the nrhs right-hand
// sides stored as the next columns of W.  `region` is a shared-memory area of
// at least mw * kPanel elements used to stage panels when W is not itself in
// shared memory (w_in_smem == false).
template <class T, class G>
__device__ void group_householder_blocked(const G& g, T* W, int ld, int mw, int n, int nrhs,
                                          bool w_in_smem, T* region, BlockedScratch<T>* bs)
{
    const int kmax = min(mw, n);
    for (int c0 = 0; c0 < kmax; c0 += kPanel) {
        const int nb = min(kPanel, kmax - c0);
        const int mp = mw - c0;
        T* P;
        int ldp;
        T* Wc = W + static_cast<size_t>(c0) * ld + c0;
        if (w_in_smem) {
            P = Wc;
            ldp = ld;
        }
        else {
            P = region;
            ldp = mp;
            for (int t = g.rank(); t < mp * nb; t += G::kSize) {
                const int c = t / mp, r = t - c * mp;
                P[r + c * mp] = Wc[r + static_cast<size_t>(c) * ld];
            }
            g.sync();
        }
        panel_qr_fast<T>(g, P, ldp, mp, nb, bs);
        const bool reg_path = mp <= 32 * 24;
        if (!reg_path)
            panel_tfactor<T>(g, P, ldp, mp, nb, bs);  // compact WY for tall panels
        if (!w_in_smem) {
            // only R (rows < nb of the panel) is needed later
            for (int t = g.rank(); t < nb * nb; t += G::kSize) {
                const int c = t / nb, r = t - c * nb;
                if (r <= c)
                    Wc[r + static_cast<size_t>(c) * ld] = P[r + c * mp];
            }
        }
        T* W2 = W + static_cast<size_t>(c0 + nb) * ld + c0;
        const int ncols = n - c0 - nb + nrhs;
        if (!reg_path || !trailing_apply<T>(g, P, ldp, mp, nb, bs, W2, ld, ncols))
            trailing_update<T>(g, P, ldp, mp, nb, bs, W2, ld, ncols);
        g.sync();
    }
}

// Blocked Householder QR of the folded matrix [Sm; diag(d)] that never
// touches the structural zeros of the diagonal part.
//
// Sm (S shared rows) lives in rows kPanel .. kPanel+S-1 of Wp (ld ldp =
// kPanel + S, n + nrhs columns, the right-hand sides last); d holds the
// folded norms and t (n x nrhs, ld n) the folded right-hand sides of the
// diagonal rows.  Reflector j only involves diagonal row j and the rows of
// Sm: every other diagonal row is zero in column j and stays zero (a
// reflector whose vector is zero on a row leaves that row unchanged).  So
// panel [c0, c0+nb) works on the (nb + S)-row matrix [H; Sm], where H holds
// diagonal rows c0..c0+nb-1 (rows kPanel-nb .. kPanel-1 of Wp, written fresh
// for the panel); after the panel and its trailing update H is the finished
// rows c0..c0+nb-1 of [R, Q^T b], copied to Rg (ld n).  Flops: about
// 2 (16 + S) n^2 instead of 2 (S + n) n^2 - 2/3 n^3 for the dense folded
// matrix.  Panels are staged in `region` (>= (kPanel + S) * kPanel elements,
// shared memory).
template <class T, class G>
__device__ void group_householder_structured(const G& g, T* Wp, int ldp, int S, int n, int nrhs,
                                             const double* d, const double* t, T* Rg, T* region,
                                             BlockedScratch<T>* bs)
{
    const int wcols = n + nrhs;
    SUBPHASE_BEGIN();
    for (int c0 = 0; c0 < n; c0 += kPanel) {
        const int nb = min(kPanel, n - c0);
        const int h0 = kPanel - nb;  // first row of H in Wp
        const int mp = nb + S;
        // H: diagonal rows c0..c0+nb-1 over columns c0 .. wcols-1
        for (int idx = g.rank(); idx < nb * (wcols - c0); idx += G::kSize) {
            const int c = c0 + idx / nb, i = idx % nb;
            T v;
            if (c < n)
                v = (c == c0 + i) ? static_cast<T>(d[c0 + i]) : T(0);
            else
                v = static_cast<T>(t[(c0 + i) + static_cast<size_t>(c - n) * n]);
            Wp[h0 + i + static_cast<size_t>(c) * ldp] = v;
        }
        g.sync();
        // stage the panel [H; Sm](:, c0 .. c0+nb-1) and factor it
        const T* Wc = Wp + static_cast<size_t>(c0) * ldp + h0;
        T* P = region;
        for (int idx = g.rank(); idx < mp * nb; idx += G::kSize) {
            const int c = idx / mp, r = idx - c * mp;
            P[r + c * mp] = Wc[r + static_cast<size_t>(c) * ldp];
        }
        g.sync();
        SUBPHASE_MARK(8);
        panel_qr_fast<T>(g, P, mp, mp, nb, bs);
        const bool reg_path = mp <= 32 * 24;
        if (!reg_path)
            panel_tfactor<T>(g, P, mp, mp, nb, bs);
        SUBPHASE_MARK(9);
        // R(c0.., c0..c0+nb-1): the panel's upper triangle
        for (int idx = g.rank(); idx < nb * nb; idx += G::kSize) {
            const int c = idx / nb, r = idx - c * nb;
            if (r <= c)
                Rg[(c0 + r) + static_cast<size_t>(c0 + c) * n] = P[r + c * mp];
        }
        const int ncols = wcols - c0 - nb;
        T* W2 = Wp + static_cast<size_t>(c0 + nb) * ldp + h0;
        if (!reg_path || !trailing_apply<T>(g, P, mp, mp, nb, bs, W2, ldp, ncols))
            trailing_update<T>(g, P, mp, mp, nb, bs, W2, ldp, ncols);
        g.sync();
        SUBPHASE_MARK(10);
        // H is now rows c0..c0+nb-1 of [R, Q^T b] over the trailing columns
        for (int idx = g.rank(); idx < nb * ncols; idx += G::kSize) {
            const int c = c0 + nb + idx / nb, i = idx % nb;
            Rg[(c0 + i) + static_cast<size_t>(c) * n] = Wp[h0 + i + static_cast<size_t>(c) * ldp];
        }
        g.sync();
        SUBPHASE_MARK(11);
    }
}

// Read-only view of the triangular factor R: column-major with leading
// dimension ld, or packed by columns (R(i, j) at j (j + 1) / 2 + i) when ld == 0.
template <class T>
struct RView {
    const T* p;
    int ld;
    __device__ __forceinline__ T operator()(int i, int j) const
    {
        return ld > 0 ? p[static_cast<size_t>(j) * ld + i]
                      : p[static_cast<size_t>(j) * (j + 1) / 2 + i];
    }
};

// Copies the upper triangle of W (n x n part, ld) into `dst` packed by columns.
template <class T, class G>
__device__ void group_pack_r(const G& g, const T* W, int ld, int n, T* dst)
{
    const int total = n * (n + 1) / 2;
    for (int t = g.rank(); t < total; t += G::kSize) {
        // invert t = j (j + 1) / 2 + i, 0 <= i <= j
        int j = static_cast<int>((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
        while (j * (j + 1) / 2 > t)
            j--;
        while ((j + 1) * (j + 2) / 2 <= t)
            j++;
        const int i = t - j * (j + 1) / 2;
        dst[t] = W[static_cast<size_t>(j) * ld + i];
    }
    g.sync();
}

// Back substitution R y = rhs(0:n) (R = upper triangle of W), blocked by 16
// columns from the right; x (FP64) receives y.  Returns (uniformly) 1 if R has
// a zero diagonal, in which case x = rhs(0:n) unchanged (LAPACK dtrtrs).
template <class T, class G>
__device__ int group_back_substitute_blocked(const G& g, RView<T> R, int n, T* rhs, double* x)
{
    int singular = 0;
    for (int j = g.rank(); j < n; j += G::kSize)
        if (R(j, j) == T(0))
            singular = 1;
    singular = g.sum(singular) > 0;
    if (!singular) {
        const int lane = g.lane();
        for (int c1 = n; c1 > 0; c1 -= kPanel) {
            const int c0 = max(0, c1 - kPanel);
            if (g.warp() == 0) {
                for (int j = c1 - 1; j >= c0; j--) {
                    const T xj = rhs[j] / R(j, j);
                    __syncwarp();
                    if (lane == 0)
                        rhs[j] = xj;
                    for (int i = c0 + lane; i < j; i += 32)
                        rhs[i] -= R(i, j) * xj;
                    __syncwarp();
                }
            }
            g.sync();
            for (int i = g.rank(); i < c0; i += G::kSize) {
                T s = 0;
                for (int j = c0; j < c1; j++)
                    s += R(i, j) * rhs[j];
                rhs[i] -= s;
            }
            g.sync();
        }
    }
    for (int j = g.rank(); j < n; j += G::kSize)
        x[j] = static_cast<double>(rhs[j]);
    g.sync();
    return singular;
}

// gv <- R^-1 R^-T gv (FP64 accumulation, R in T), blocked by 16 columns.
template <class T, class G>
__device__ void group_normal_correction_blocked(const G& g, RView<T> R, int n, double* gv)
{
    const int lane = g.lane();
    // forward R^T z = g
    for (int c0 = 0; c0 < n; c0 += kPanel) {
        const int c1 = min(n, c0 + kPanel);
        for (int j = c0 + g.warp(); j < c1; j += G::kWarps) {
            double d = 0.0;
            for (int i = lane; i < c0; i += 32)
                d += static_cast<double>(R(i, j)) * gv[i];
            d = warp_sum(d);
            if (lane == 0)
                gv[j] -= d;
        }
        g.sync();
        if (g.warp() == 0) {
            for (int j = c0; j < c1; j++) {
                double d = 0.0;
                for (int i = c0 + lane; i < j; i += 32)
                    d += static_cast<double>(R(i, j)) * gv[i];
                d = warp_sum(d);
                const double zj = (gv[j] - d) / static_cast<double>(R(j, j));
                __syncwarp();
                if (lane == 0)
                    gv[j] = zj;
                __syncwarp();
            }
        }
        g.sync();
    }
    // backward R delta = z
    for (int c1 = n; c1 > 0; c1 -= kPanel) {
        const int c0 = max(0, c1 - kPanel);
        if (g.warp() == 0) {
            for (int j = c1 - 1; j >= c0; j--) {
                const double dj = gv[j] / static_cast<double>(R(j, j));
                __syncwarp();
                if (lane == 0)
                    gv[j] = dj;
                for (int i = c0 + lane; i < j; i += 32)
                    gv[i] -= static_cast<double>(R(i, j)) * dj;
                __syncwarp();
            }
        }
        g.sync();
        for (int i = g.rank(); i < c0; i += G::kSize) {
            double s2 = 0.0;
            for (int j = c0; j < c1; j++)
                s2 += static_cast<double>(R(i, j)) * gv[j];
            gv[i] -= s2;
        }
        g.sync();
    }
}

// rinv[j] = 1 / R(j, j) in FP64 (R nonsingular), for the corrections below.
template <class T, class G>
__device__ void group_diag_reciprocals(const G& g, RView<T> R, int n, double* rinv)
{
    for (int j = g.rank(); j < n; j += G::kSize)
        rinv[j] = 1.0 / static_cast<double>(R(j, j));
    g.sync();
}

// gv <- R^-1 R^-T gv in FP64 (R in T, rinv = 1 / diag(R)), right-looking by
// 16-column blocks: one warp solves a block's diagonal triangle with the
// block's values in lanes (a shuffle and an FMA per step, the block's column
// of R prefetched into registers), then every thread updates one remaining
// entry with the block's 16 solved values.  Two barriers per block.
template <class T, class G>
__device__ void group_normal_correction_rl(const G& g, RView<T> R, int n, const double* rinv,
                                           double* gv)
{
    const int lane = g.lane();
    // forward R^T z = g: z_j = (g_j - sum_{i<j} R(i,j) z_i) / R(j,j)
    for (int c0 = 0; c0 < n; c0 += kPanel) {
        const int nb = min(kPanel, n - c0);
        if (g.warp() == 0) {
            const int i = c0 + lane;  // this lane's entry (lanes < nb)
            double gi = lane < nb ? gv[i] : 0.0;
            double rc[kPanel];        // R(c0 + j, i) for j < lane
#pragma unroll
            for (int j = 0; j < kPanel; j++)
                rc[j] = (j < lane && lane < nb) ? static_cast<double>(R(c0 + j, i)) : 0.0;
            const double ri = lane < nb ? rinv[i] : 0.0;
#pragma unroll
            for (int j = 0; j < kPanel; j++) {
                if (j >= nb)
                    break;
                if (lane == j)
                    gi *= ri;
                const double zj = __shfl_sync(0xffffffffu, gi, j);
                if (lane > j)
                    gi -= rc[j] * zj;
            }
            if (lane < nb)
                gv[i] = gi;
        }
        g.sync();
        const int c1 = c0 + nb;
        for (int j = c1 + g.rank(); j < n; j += G::kSize) {
            double acc = 0.0;
#pragma unroll 4
            for (int i = c0; i < c1; i++)
                acc += static_cast<double>(R(i, j)) * gv[i];
            gv[j] -= acc;
        }
        g.sync();
    }
    // backward R d = z: d_j = (z_j - sum_{i>j} R(j,i) d_i) / R(j,j)
    for (int c1 = n; c1 > 0; c1 -= kPanel) {
        const int c0 = max(0, c1 - kPanel);
        const int nb = c1 - c0;
        if (g.warp() == 0) {
            const int i = c0 + lane;
            double zi = lane < nb ? gv[i] : 0.0;
            double rr[kPanel];        // R(i, c0 + j) for j > lane
#pragma unroll
            for (int j = 0; j < kPanel; j++)
                rr[j] = (j > lane && j < nb) ? static_cast<double>(R(i, c0 + j)) : 0.0;
            const double ri = lane < nb ? rinv[i] : 0.0;
#pragma unroll
            for (int j = kPanel - 1; j >= 0; j--) {
                if (j >= nb)
                    continue;
                if (lane == j)
                    zi *= ri;
                const double dj = __shfl_sync(0xffffffffu, zi, j);
                if (lane < j)
                    zi -= rr[j] * dj;
            }
            if (lane < nb)
                gv[i] = zi;
        }
        g.sync();
        for (int i = g.rank(); i < c0; i += G::kSize) {
            double acc = 0.0;
#pragma unroll 4
            for (int j = c0; j < c1; j++)
                acc += static_cast<double>(R(i, j)) * gv[j];
            gv[i] -= acc;
        }
        g.sync();
    }
}

}  // namespace mspai
