// Adjoint of the fixed-pattern setup (no reference counterpart).
//
// For column k with C_k = C(I_k, J_k), b_k = B(I_k, k), m_k = argmin
// ||C_k m - b_k|| and r_k = b_k - C_k m_k, the loss
//     L = ||C M - B||_F^2 + sum_k gbar_k^T m_k
// has, per column (envelope theorem for the squared residual; the least-
// squares sensitivity dm = (C^T C)^-1 (dC^T r - C^T dC m + C^T db) for gbar):
//     lambda_k = R_k^-1 R_k^-T gbar_k            (two triangular solves)
//     dL/dC_k  = -2 r_k m_k^T + r_k lambda_k^T - (C_k lambda_k) m_k^T
//     dL/db_k  =  2 r_k + C_k lambda_k
// plus dL/dB(i,k) = 2 B(i,k) for the rows of B(:,k) outside I_k (where the
// residual is -B).  dL/dC is only needed at the nonzeros of C; every column k
// adds its part to the nonzeros of C(:, J_k) with FP64 atomics.  R_k comes from
// the same folded Householder QR as the forward solve, recomputed in FP64 in
// this kernel; Q is never formed or stored.
#include "mspai_b200.h"
#include "spai_kernels.h"
#include "spai_solve.cuh"

#include <algorithm>
#include <vector>

namespace mspai {

template <class G>
__device__ void adjoint_column(const G& g, const Problem& pb, const Caps& cap, Slot<double> s,
                               const AdjointIO& io, int col)
{
    const int lane = g.lane();
    const int64_t p0 = pb.pptr[col];
    const int n = static_cast<int>(pb.pptr[col + 1] - p0);
    if (n > cap.nmax)
        return;
    for (int t = g.rank(); t < n; t += G::kSize)
        s.J[t] = pb.pidx[p0 + t];
    for (int jj = g.rank(); jj < n; jj += G::kSize) {
        const int j = pb.pidx[p0 + jj];
        s.off[jj] = static_cast<int>(pb.cptr[j + 1] - pb.cptr[j]);
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
    for (int u = g.rank(); u < m; u += G::kSize)
        s.tmp[u] = (s.rstart[u + 1] - s.rstart[u]) >= 2 ? 1 : 0;
    g.sync();
    const int S = group_exclusive_scan(g, s.tmp, m);
    const int mw = S + n;
    if (mw > cap.mwmax)
        return;
    double* W = s.W;
    double* rhs = s.W + static_cast<size_t>(mw) * n;
    const int ld = mw;
    for (int i = g.rank(); i < mw * n + mw; i += G::kSize)
        W[i] = 0.0;
    g.sync();
    for (int i = g.rank(); i < E; i += G::kSize) {
        const int e = static_cast<int>(s.keys[i] & kEntryMask);
        const int u = s.pos[e];
        if (s.rstart[u + 1] - s.rstart[u] >= 2) {
            const int d = s.tmp[u];
            W[static_cast<size_t>(s.ejj[e]) * ld + d] = s.ev[e];
            if (i == s.rstart[u])
                rhs[d] = target_value(pb, col, s.I[u]);
        }
    }
    for (int jj = g.warp(); jj < n; jj += G::kWarps) {
        double sig = 0.0, tb = 0.0;
        for (int e = s.off[jj] + lane; e < s.off[jj + 1]; e += 32) {
            const int u = s.pos[e];
            if (s.rstart[u + 1] - s.rstart[u] == 1) {
                const double v = s.ev[e];
                sig += v * v;
                tb += v * target_value(pb, col, s.I[u]);
            }
        }
        sig = warp_sum(sig);
        tb = warp_sum(tb);
        if (lane == 0) {
            const double nrm = sqrt(sig);
            W[static_cast<size_t>(jj) * ld + S + jj] = nrm;
            rhs[S + jj] = nrm > 0.0 ? tb / nrm : 0.0;
        }
    }
    g.sync();
    group_householder<double>(g, W, ld, mw, n, 1);
    group_back_substitute<double>(g, W, ld, n, rhs, s.x);
    // r = b - C m on I
    const double r2 =
        group_residual(g, pb, col, s.keys, s.I, s.rstart, s.ejj, s.ev, s.x, s.r, m, n, 1);
    // lambda = R^-1 R^-T gbar_k
    double gx = 0.0;
    if (io.gbar) {
        for (int jj = g.rank(); jj < n; jj += G::kSize) {
            const double gb = io.gbar[io.mptr[col] + jj];
            s.gv[jj] = gb;
            gx += gb * s.x[jj];
        }
        g.sync();
        group_normal_correction<double>(g, W, ld, n, s.gv);
    }
    else {
        for (int jj = g.rank(); jj < n; jj += G::kSize)
            s.gv[jj] = 0.0;
        g.sync();
    }
    gx = g.sum(gx);
    // q = C lambda on I (stored in rho[], emax doubles)
    double* q = s.rho;
    for (int u = g.rank(); u < m; u += G::kSize) {
        double v = 0.0;
        for (int i = s.rstart[u]; i < s.rstart[u + 1]; i++) {
            const int e = static_cast<int>(s.keys[i] & kEntryMask);
            v += s.ev[e] * s.gv[s.ejj[e]];
        }
        q[u] = v;
    }
    g.sync();
    // dL/dC at the nonzeros of C(:, J_k)
    for (int jj = g.warp(); jj < n; jj += G::kWarps) {
        const int j = s.J[jj];
        const int64_t base = pb.cptr[j];
        const int o = s.off[jj];
        const int len = s.off[jj + 1] - o;
        const double xj = s.x[jj];
        const double lj = s.gv[jj];
        for (int t = lane; t < len; t += 32) {
            const int u = s.pos[o + t];
            const double gval = -2.0 * s.r[u] * xj + s.r[u] * lj - q[u] * xj;
            atomicAdd(&io.dC[base + t], gval);
        }
    }
    // dL/dB(:, k) and the part of the loss outside I_k
    double outside = 0.0;
    if (pb.bptr) {
        const int64_t b0 = pb.bptr[col], b1 = pb.bptr[col + 1];
        for (int64_t p = b0 + g.rank(); p < b1; p += G::kSize) {
            const int row = pb.bidx[p];
            const int u = lower_bound_i32(s.I, m, row);
            double gb;
            if (u < m && s.I[u] == row) {
                gb = 2.0 * s.r[u] + q[u];
            }
            else {
                gb = 2.0 * pb.bval[p];
                outside += pb.bval[p] * pb.bval[p];
            }
            if (io.dB)
                io.dB[p] = gb;
        }
    }
    else {
        if (g.rank() == 0) {
            const int u = lower_bound_i32(s.I, m, col);
            if (!(u < m && s.I[u] == col))
                outside = 1.0;  // e_k has its 1 outside I_k
        }
    }
    outside = g.sum(outside);
    if (g.rank() == 0)
        io.loss[col] = r2 + outside + gx;
    g.sync();
}

template <int NT>
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
        adjoint_column(g, pb, cap, s, io, col);
    }
}

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
        adjoint_column(g, pb, cap, s, io, col);
    }
}

cudaError_t launch_adjoint(const Problem& pb, const Caps& cap, const AdjointIO& io, int lo,
                           int hi, bool warp, char* scratch, size_t scratch_bytes,
                           int32_t* counter, cudaStream_t st)
{
    const int n = hi - lo;  // columns of this launch
    const size_t slot = SlotLayout<double>(cap, false).bytes;
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (warp) {
        const int per_block = kWarpKernelThreads / 32;
        int grid = std::min<int>(sms * 8, (n + per_block - 1) / per_block);
        grid = std::max(1, std::min<int>(grid, static_cast<int>(scratch_bytes / (slot * per_block))));
        adjoint_warp_kernel<<<grid, kWarpKernelThreads, 0, st>>>(pb, cap, io, lo, hi, scratch,
                                                                 slot, counter);
    }
    else {
        int grid = std::min(sms * 4, n);
        grid = std::max(1, std::min<int>(grid, static_cast<int>(scratch_bytes / slot)));
        adjoint_cta_kernel<128><<<grid, 128, 0, st>>>(pb, cap, io, lo, hi, scratch, slot, counter);
    }
    return cudaGetLastError();
}

size_t adjoint_scratch_bytes(const Caps& cap, int n, bool warp)
{
    const size_t slot = SlotLayout<double>(cap, false).bytes;
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t slots = warp ? static_cast<size_t>(std::min(sms * 8, (n + 7) / 8)) * 8
                              : static_cast<size_t>(std::min(sms * 4, n));
    return slot * std::max<size_t>(slots, 1);
}

}  // namespace mspai
