// Adjoint of the setup (no reference counterpart).
//
// For problem column k (a scalar column, or a block column of bs scalar
// columns sharing J_k) with C_k = C(I_k, J_k), the right-hand sides b_k,c =
// B(I_k, bs k + c), the solutions m_k,c of the setup (read from its result M)
// and r_k,c = b_k,c - C_k m_k,c, the loss
//     L = w ||C M - B||_F^2 + sum_k gbar_k^T m_k      (gbar: scalar columns)
// has, at the pattern the setup chose (fixed, or the final pattern of the
// updates: the pattern is a discrete choice and carries no gradient):
//     dL/dC_k  = sum_c -2w r_k,c m_k,c^T  +  r_k lambda_k^T - (C_k lambda_k) m_k^T
//     dL/db_k,c = 2w r_k,c  +  C_k lambda_k
//     lambda_k = (C_k^T C_k)^-1 gbar_k = R_k^-1 R_k^-T gbar_k
// (envelope theorem for the squared residual -- M is stationary, so no
// re-solve is needed for it -- and the least-squares sensitivity for gbar),
// plus dL/dB(i, .) = 2w B(i, .) for target entries outside I_k.  lambda_k comes
// from two triangular solves with the R the setup kept (keep_factors), refined
// in FP64 against C_k^T C_k from the sparse entries when R is FP32; without a
// kept R the folded Householder QR is recomputed here in FP64.  Q is never
// formed or stored.  Every column adds its part to the nonzeros of C(:, J_k)
// with FP64 atomics.
#include "mspai_b200.h"
#include "spai_kernels.h"
#include "spai_solve.cuh"

#include <algorithm>
#include <vector>

namespace mspai {

// FP64 q = C(I, J) v on I (the sorted entries' runs), in q[0 .. m).
template <class G>
__device__ void adj_apply_c(const G& g, const Slot<double>& s, int m, const double* v, double* q)
{
    for (int u = g.rank(); u < m; u += G::kSize) {
        double acc = 0.0;
        for (int i = s.rstart[u]; i < s.rstart[u + 1]; i++) {
            const int e = static_cast<int>(s.keys[i] & kEntryMask);
            acc += s.ev[e] * v[s.ejj[e]];
        }
        q[u] = acc;
    }
    g.sync();
}

// lambda (in gv) = (C^T C)^-1 gbar with the kept R (packed by columns, TR):
// two triangular solves, then FP64 refinement steps gv += R^-1 R^-T (gbar -
// C^T C gv) when TR is FP32.  q (m entries) and tmp (n) are scratch.
template <class TR, class G>
__device__ void adj_lambda_kept(const G& g, const Slot<double>& s, const TR* R, int m, int n,
                                const double* gbar, double* gv, double* q, double* tmp)
{
    for (int jj = g.rank(); jj < n; jj += G::kSize)
        gv[jj] = gbar[jj];
    g.sync();
    const RView<TR> rv{R, 0};
    group_normal_correction_blocked<TR>(g, rv, n, gv);
    const int steps = sizeof(TR) == 4 ? 2 : 0;
    for (int it = 0; it < steps; it++) {
        adj_apply_c(g, s, m, gv, q);
        // tmp = gbar - C^T q, a warp per column over its entries
        for (int jj = g.warp(); jj < n; jj += G::kWarps) {
            double acc = 0.0;
            for (int e = s.off[jj] + g.lane(); e < s.off[jj + 1]; e += 32)
                acc += s.ev[e] * q[s.pos[e]];
            acc = warp_sum(acc);
            if (g.lane() == 0)
                tmp[jj] = gbar[jj] - acc;
        }
        g.sync();
        group_normal_correction_blocked<TR>(g, rv, n, tmp);
        for (int jj = g.rank(); jj < n; jj += G::kSize)
            gv[jj] += tmp[jj];
        g.sync();
    }
}

template <class TR, class G>
__device__ void adjoint_column(const G& g, const Problem& pb, const Caps& cap, Slot<double> s,
                               const AdjointIO& io, int kb)
{
    const int lane = g.lane();
    const int bs = pb.bs;
    const int sc0 = bs * kb;                 // first scalar column of the problem
    const int64_t p0 = io.mptr[sc0];
    const int n = static_cast<int>(io.mptr[sc0 + 1] - p0);
    if (n > cap.nmax || bs > cap.nrhs)
        return;
    // J and the solutions from the setup's result (the bs scalar columns of a
    // block column share J)
    for (int t = g.rank(); t < n; t += G::kSize) {
        const int j = io.midx[p0 + t];
        s.J[t] = j;
        s.off[t] = static_cast<int>(pb.cptr[j + 1] - pb.cptr[j]);
        for (int c = 0; c < bs; c++)
            s.x[static_cast<size_t>(c) * n + t] = io.mval[io.mptr[sc0 + c] + t];
    }
    g.sync();
    const int E = group_exclusive_scan(g, s.off, n);
    if (g.rank() == 0)
        s.off[n] = E;
    if (E > cap.emax)
        return;
    g.sync();
    for (int jj = g.warp(); jj < n; jj += G::kWarps) {
        const int j = s.J[jj];
        const int64_t base = pb.cptr[j];
        const int o = s.off[jj];
        const int len = s.off[jj + 1] - o;
        for (int t = lane; t < len; t += 32) {
            const int e = o + t;
            s.ejj[e] = jj;
            s.ev[e] = pb.cval[base + t];
            s.keys[e] = (static_cast<uint64_t>(pb.cidx[base + t]) << kEntryBits) |
                        static_cast<uint64_t>(e);
        }
    }
    const int L = next_pow2(E > 0 ? E : 1);
    for (int i = E + g.rank(); i < L; i += G::kSize)
        s.keys[i] = ~uint64_t(0);
    g.sync();
    group_bitonic_sort(g, s.keys, L);
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
    // r_c = b_c - C m_c on I (s.r + c m), ||r||_F^2
    const double r2 =
        group_residual(g, pb, kb, s.keys, s.I, s.rstart, s.ejj, s.ev, s.x, s.r, m, n, bs);
    g.sync();
    // lambda = R^-1 R^-T gbar_k (scalar columns with a gbar)
    double gx = 0.0;
    double* q = s.rho;     // C lambda on I (cmax >= emax doubles)
    const bool lam = io.gbar != nullptr && bs == 1;
    if (lam) {
        const double* gb = io.gbar + io.mptr[kb];
        for (int jj = g.rank(); jj < n; jj += G::kSize)
            gx += gb[jj] * s.x[jj];
        if (io.rstore) {
            adj_lambda_kept<TR>(g, s, static_cast<const TR*>(io.rstore) + io.roff[kb], m, n, gb,
                                s.gv, q, s.rinv);
        }
        else {
            // recompute R: the folded Householder QR of the forward, in FP64
            for (int u = g.rank(); u < m; u += G::kSize)
                s.tmp[u] = (s.rstart[u + 1] - s.rstart[u]) >= 2 ? 1 : 0;
            g.sync();
            const int S = group_exclusive_scan(g, s.tmp, m);
            const int mw = S + n;
            if (mw > cap.mwmax)
                return;
            double* W = s.W;
            const int ld = mw;
            for (int i = g.rank(); i < mw * n; i += G::kSize)
                W[i] = 0.0;
            g.sync();
            for (int i = g.rank(); i < E; i += G::kSize) {
                const int e = static_cast<int>(s.keys[i] & kEntryMask);
                const int u = s.pos[e];
                if (s.rstart[u + 1] - s.rstart[u] >= 2)
                    W[static_cast<size_t>(s.ejj[e]) * ld + s.tmp[u]] = s.ev[e];
            }
            for (int jj = g.warp(); jj < n; jj += G::kWarps) {
                double sig = 0.0;
                for (int e = s.off[jj] + lane; e < s.off[jj + 1]; e += 32) {
                    const int u = s.pos[e];
                    if (s.rstart[u + 1] - s.rstart[u] == 1)
                        sig += s.ev[e] * s.ev[e];
                }
                sig = warp_sum(sig);
                if (lane == 0)
                    W[static_cast<size_t>(jj) * ld + S + jj] = sqrt(sig);
            }
            g.sync();
            group_householder<double>(g, W, ld, mw, n, 0);
            for (int jj = g.rank(); jj < n; jj += G::kSize)
                s.gv[jj] = gb[jj];
            g.sync();
            group_normal_correction<double>(g, W, ld, n, s.gv);
        }
        adj_apply_c(g, s, m, s.gv, q);
    }
    gx = g.sum(gx);
    // dL/dC at the nonzeros of C(:, J_k)
    for (int jj = g.warp(); jj < n; jj += G::kWarps) {
        const int j = s.J[jj];
        const int64_t base = pb.cptr[j];
        const int o = s.off[jj];
        const int len = s.off[jj + 1] - o;
        const double lj = lam ? s.gv[jj] : 0.0;
        for (int t = lane; t < len; t += 32) {
            const int u = s.pos[o + t];
            double gval = 0.0;
            for (int c = 0; c < bs; c++)
                gval -= s.r[static_cast<size_t>(c) * m + u] * s.x[static_cast<size_t>(c) * n + jj];
            gval *= 2.0 * io.wres;
            if (lam)
                gval += s.r[u] * lj - q[u] * s.x[jj];
            atomicAdd(&io.dC[base + t], gval);
        }
    }
    // dL/dB at the target entries, and the loss of the target outside I_k
    double outside = 0.0;
    for (int c = 0; c < bs; c++) {
        const int col = sc0 + c;
        if (pb.bptr) {
            const int64_t b0 = pb.bptr[col], b1 = pb.bptr[col + 1];
            for (int64_t p = b0 + g.rank(); p < b1; p += G::kSize) {
                const int row = pb.bidx[p];
                const int u = lower_bound_i32(s.I, m, row);
                double gbv;
                if (u < m && s.I[u] == row) {
                    gbv = 2.0 * io.wres * s.r[static_cast<size_t>(c) * m + u] +
                          (lam ? q[u] : 0.0);
                }
                else {
                    gbv = 2.0 * io.wres * pb.bval[p];
                    outside += pb.bval[p] * pb.bval[p];
                }
                if (io.dB)
                    io.dB[p] = gbv;
            }
        }
        else if (g.rank() == 0) {
            const int u = lower_bound_i32(s.I, m, col);
            if (!(u < m && s.I[u] == col))
                outside += 1.0;  // e_col has its 1 outside I_k
        }
    }
    outside = g.sum(outside);
    if (g.rank() == 0)
        io.loss[kb] = io.wres * (r2 + outside) + gx;
    g.sync();
}

// E[k] = entries of C(:, J_k), nk[k] = |J_k| for problem column k, J_k the
// pattern of scalar column bs k of the result
__global__ void adjoint_plan_kernel(const int64_t* __restrict__ cptr,
                                    const int64_t* __restrict__ mptr,
                                    const int32_t* __restrict__ midx, int nprob, int bs,
                                    int32_t* __restrict__ E, int32_t* __restrict__ nk)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int kb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; kb < nprob; kb += warps) {
        const int64_t a = mptr[bs * kb], b = mptr[bs * kb + 1];
        int64_t e = 0;
        for (int64_t p = a + lane; p < b; p += 32) {
            const int j = midx[p];
            e += cptr[j + 1] - cptr[j];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            e += __shfl_xor_sync(0xffffffffu, e, o);
        if (lane == 0) {
            E[kb] = static_cast<int32_t>(e > 0x7fffffff ? 0x7fffffff : e);
            nk[kb] = static_cast<int32_t>(b - a);
        }
    }
}

cudaError_t launch_adjoint_plan(const int64_t* cptr, const int64_t* mptr, const int32_t* midx,
                                int nprob, int bs, int32_t* E, int32_t* nk, cudaStream_t st)
{
    if (nprob <= 0)
        return cudaSuccess;
    const int blocks = std::max(1, std::min((nprob + 7) / 8, num_sms() * 16));
    adjoint_plan_kernel<<<blocks, 256, 0, st>>>(cptr, mptr, midx, nprob, bs, E, nk);
    return cudaGetLastError();
}

template <class TR, int NT>
__global__ void __launch_bounds__(NT)
    adjoint_cta_kernel(Problem pb, Caps cap, AdjointIO io, int lo, int hi, char* scratch,
                       size_t slot_bytes, int32_t* counter)
{
    __shared__ GroupScratch sc;
    CtaGroup<NT> g{&sc};
    SlotLayout<double> lay(cap, false);
    Slot<double> s = lay.at(scratch + static_cast<size_t>(blockIdx.x) * slot_bytes, nullptr);
    while (true) {
        if (threadIdx.x == 0)
            sc.i[5] = lo + atomicAdd(counter, 1);
        __syncthreads();
        const int col = sc.i[5];
        __syncthreads();
        if (col >= hi)
            break;
        adjoint_column<TR>(g, pb, cap, s, io, col);
    }
}

template <class TR>
__global__ void __launch_bounds__(kWarpKernelThreads)
    adjoint_warp_kernel(Problem pb, Caps cap, AdjointIO io, int lo, int hi, char* scratch,
                        size_t slot_bytes, int32_t* counter)
{
    __shared__ GroupScratch sc[kWarpKernelThreads / 32];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    WarpGroup g{&sc[w]};
    SlotLayout<double> lay(cap, false);
    const size_t slot_id = static_cast<size_t>(blockIdx.x) * (kWarpKernelThreads / 32) + w;
    Slot<double> s = lay.at(scratch + slot_id * slot_bytes, nullptr);
    while (true) {
        int col = 0;
        if (lane == 0)
            col = lo + atomicAdd(counter, 1);
        col = __shfl_sync(0xffffffffu, col, 0);
        if (col >= hi)
            break;
        adjoint_column<TR>(g, pb, cap, s, io, col);
    }
}

template <class TR>
static void launch_adjoint_t(const Problem& pb, const Caps& cap, const AdjointIO& io, int lo,
                             int hi, bool warp, char* scratch, size_t scratch_bytes,
                             int32_t* counter, cudaStream_t st)
{
    const int n = hi - lo;  // columns of this launch
    const size_t slot = SlotLayout<double>(cap, false).bytes;
    const int sms = num_sms();
    if (warp) {
        const int per_block = kWarpKernelThreads / 32;
        int grid = std::min<int>(sms * 8, (n + per_block - 1) / per_block);
        grid = std::max(1, std::min<int>(grid, static_cast<int>(scratch_bytes / (slot * per_block))));
        adjoint_warp_kernel<TR><<<grid, kWarpKernelThreads, 0, st>>>(pb, cap, io, lo, hi, scratch,
                                                                     slot, counter);
    }
    else {
        int grid = std::min(sms * 4, n);
        grid = std::max(1, std::min<int>(grid, static_cast<int>(scratch_bytes / slot)));
        adjoint_cta_kernel<TR, 128><<<grid, 128, 0, st>>>(pb, cap, io, lo, hi, scratch, slot,
                                                          counter);
    }
}

cudaError_t launch_adjoint(const Problem& pb, const Caps& cap, const AdjointIO& io, int lo,
                           int hi, bool warp, char* scratch, size_t scratch_bytes,
                           int32_t* counter, cudaStream_t st)
{
    if (io.rstore && io.r_elem == 4)
        launch_adjoint_t<float>(pb, cap, io, lo, hi, warp, scratch, scratch_bytes, counter, st);
    else
        launch_adjoint_t<double>(pb, cap, io, lo, hi, warp, scratch, scratch_bytes, counter, st);
    return cudaGetLastError();
}

size_t adjoint_scratch_bytes(const Caps& cap, int n, bool warp)
{
    const size_t slot = SlotLayout<double>(cap, false).bytes;
    const int sms = num_sms();
    const size_t slots = warp ? static_cast<size_t>(std::min(sms * 8, (n + 7) / 8)) * 8
                              : static_cast<size_t>(std::min(sms * 4, n));
    return slot * std::max<size_t>(slots, 1);
}

}  // namespace mspai
