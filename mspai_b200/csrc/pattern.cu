// Start pattern of the square of A on the device, with small entries dropped
// per column: P(:, k) = { i : |(A^2)(i, k)| >= drop * max_i |(A^2)(i, k)| }.
//
// The reference builds its power patterns with PETSc (To_Pattern_Powers /
// To_Pattern_Power, src/Matrix.imp:359-470, src/Matrix.cpp:602-636: MatMatMult
// of the sparsified matrix, then Sparsify keeps a count of the largest entries
// per column).  This is the same family with a relative drop tolerance (the
// pattern of the ragged benchmark workload).  A is the first n rows of C
// (probing rows are not part of it).
//
// One CTA per column k: the products A(i, l) A(l, k) of every entry (l, k)
// with every entry (i, l) of column l go to shared memory as (row, value)
// pairs, are bitonic-sorted by row, summed per row, and the rows that pass
// the tolerance are counted (pass 1) or written in row order (pass 2, after
// a scan of the counts).  Up to kMaxProducts products per column.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mspai_b200.h"
#include "mspai_b200_io.h"
#include "spai_kernels.h"

namespace mspai {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxProducts = 8192;  // 8192 x 12 bytes of shared memory

__device__ void block_sort_pairs(int* key, double* val, int L)
{
    for (int k = 2; k <= L; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < L; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const int a = key[i], b = key[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        key[i] = b;
                        key[ixj] = a;
                        const double t = val[i];
                        val[i] = val[ixj];
                        val[ixj] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// pass 0: counts (cnt[k]); pass 1: rows into out_idx at out_ptr[k]
__global__ void __launch_bounds__(kThreads)
    power_pattern_kernel(const int64_t* __restrict__ cp, const int32_t* __restrict__ ci,
                         const double* __restrict__ cv, int n, double drop, int pass,
                         int32_t* __restrict__ cnt, const int64_t* __restrict__ out_ptr,
                         int32_t* __restrict__ out_idx, int32_t* __restrict__ err)
{
    extern __shared__ __align__(16) char smem[];
    double* val = reinterpret_cast<double*>(smem);
    int* key = reinterpret_cast<int*>(val + kMaxProducts);
    __shared__ int s_pos[kThreads / 32 + 1];
    __shared__ double s_max[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        // products of column k: a warp per entry (l, k) of column k, at the
        // offset of the entry's column l among the column's products (a fixed
        // order, so the sums below do not depend on the schedule)
        int64_t total = 0;
        for (int64_t p = cp[k]; p < cp[k + 1] && ci[p] < n; p++)
            total += cp[ci[p] + 1] - cp[ci[p]];
        if (total > kMaxProducts) {
            if (threadIdx.x == 0)
                atomicExch(err, k + 1);
            continue;  // uniform across the block
        }
        for (int64_t p = cp[k] + warp; p < cp[k + 1]; p += kThreads / 32) {
            const int l = ci[p];
            if (l >= n)
                break;  // probing rows come last
            const double alk = cv[p];
            const int64_t b0 = cp[l], b1 = cp[l + 1];
            int base = 0;
            for (int64_t q = cp[k]; q < p; q++)
                base += static_cast<int>(cp[ci[q] + 1] - cp[ci[q]]);
            for (int64_t q = b0 + lane; q < b1; q += 32) {
                const int i = ci[q];
                key[base + (q - b0)] = i < n ? i : 0x7fffffff;  // probing rows sort last
                val[base + (q - b0)] = i < n ? cv[q] * alk : 0.0;
            }
        }
        __syncthreads();
        const int T = static_cast<int>(total);
        int L = 1;
        while (L < T)
            L <<= 1;
        for (int i = T + threadIdx.x; i < L; i += kThreads) {
            key[i] = 0x7fffffff;
            val[i] = 0.0;
        }
        __syncthreads();
        block_sort_pairs(key, val, L);
        // sums per row: the first entry of each run sums its run (runs are
        // short: rows shared by few columns l)
        double mx = 0.0;
        for (int i = threadIdx.x; i < T; i += kThreads) {
            if (key[i] == 0x7fffffff || (i > 0 && key[i - 1] == key[i]))
                continue;
            double s = 0.0;
            for (int q = i; q < T && key[q] == key[i]; q++)
                s += val[q];
            mx = fmax(mx, fabs(s));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0)
            s_max[warp] = mx;
        __syncthreads();
        mx = 0.0;
        for (int w = 0; w < kThreads / 32; w++)
            mx = fmax(mx, s_max[w]);
        const double thr = drop * mx;
        // keep flags in row order: count per thread chunk, then positions
        const int chunk = (T + kThreads - 1) / kThreads;
        const int lo = min(T, static_cast<int>(threadIdx.x) * chunk), hi = min(T, lo + chunk);
        int c = 0;
        for (int i = lo; i < hi; i++) {
            if (key[i] == 0x7fffffff || (i > 0 && key[i - 1] == key[i]))
                continue;
            double s = 0.0;
            for (int q = i; q < T && key[q] == key[i]; q++)
                s += val[q];
            c += fabs(s) >= thr ? 1 : 0;
        }
        // block exclusive scan of c
        int v = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o)
                v += t;
        }
        if (lane == 31)
            s_pos[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            int run = 0;
            for (int w = 0; w < kThreads / 32; w++) {
                const int t = s_pos[w];
                s_pos[w] = run;
                run += t;
            }
            s_pos[kThreads / 32] = run;
        }
        __syncthreads();
        if (pass == 0) {
            if (threadIdx.x == 0)
                cnt[k] = s_pos[kThreads / 32];
        }
        else {
            int64_t o = out_ptr[k] + s_pos[warp] + v - c;
            for (int i = lo; i < hi; i++) {
                if (key[i] == 0x7fffffff || (i > 0 && key[i - 1] == key[i]))
                    continue;
                double s = 0.0;
                for (int q = i; q < T && key[q] == key[i]; q++)
                    s += val[q];
                if (fabs(s) >= thr)
                    out_idx[o++] = key[i];
            }
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace mspai

extern "C" int mspai_pattern_power2(const mspai_csc* C, double drop, int32_t device,
                                    mspai_matrix* P_out, char* msg, int32_t msg_len)
{
    auto fail = [&](int rc, const char* what) {
        if (msg && msg_len > 0)
            std::snprintf(msg, static_cast<size_t>(msg_len), "%s", what);
        return rc;
    };
    if (!P_out)
        return fail(MSPAI_ERR_PARAM, "P_out is required");
    std::memset(P_out, 0, sizeof(*P_out));
    // !(drop >= 0) also refuses a NaN drop tolerance
    if (!C || C->mem != MSPAI_MEM_HOST || !C->colptr || !(drop >= 0.0) || !std::isfinite(drop) ||
        (C->nnz > 0 && (!C->values || !C->rowidx)))
        return fail(MSPAI_ERR_PARAM, "host C with values and a finite drop >= 0 are required");
    const int n = C->ncols;
    // the kernel assumes a well-formed square-or-taller CSC with sorted rows:
    // check it here, on the host where the arrays are
    if (n < 0 || C->nrows < n || C->nnz < 0)
        return fail(MSPAI_ERR_INPUT, "C must have at least as many rows as columns");
    if (C->colptr[0] != 0 || C->colptr[n] != C->nnz)
        return fail(MSPAI_ERR_INPUT, "C: column pointers do not match nnz");
    for (int k = 0; k < n; k++) {
        const int64_t a = C->colptr[k], b = C->colptr[k + 1];
        if (b < a || a < 0 || b > C->nnz) {
            char buf[128];
            std::snprintf(buf, sizeof(buf), "C: column pointers decrease at column %d", k);
            return fail(MSPAI_ERR_INPUT, buf);
        }
        int prev = -1;
        for (int64_t q = a; q < b; q++) {
            const int r = C->rowidx[q];
            if (r < 0 || r >= C->nrows) {
                char buf[128];
                std::snprintf(buf, sizeof(buf), "C: row index %d out of range in column %d", r, k);
                return fail(MSPAI_ERR_INPUT, buf);
            }
            if (r <= prev) {
                char buf[128];
                std::snprintf(buf, sizeof(buf), "C: row indices not sorted/unique in column %d", k);
                return fail(MSPAI_ERR_INPUT, buf);
            }
            prev = r;
        }
    }
    if (cudaSetDevice(device) != cudaSuccess)
        return fail(MSPAI_ERR_NO_DEVICE, "no usable CUDA device");
    cudaStream_t st = nullptr;
    int64_t* dcp = nullptr;
    int32_t *dci = nullptr, *dcnt = nullptr, *didx = nullptr, *derr = nullptr;
    double* dcv = nullptr;
    int64_t* dptr = nullptr;
    int rc = MSPAI_OK;
    std::vector<int32_t> cnt(static_cast<size_t>(std::max(n, 1)));
    std::vector<int64_t> ptr(static_cast<size_t>(n) + 1, 0);
    const size_t smem = mspai::kMaxProducts * (sizeof(double) + sizeof(int));
    int grid = 0, err = 0;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == MSPAI_OK)
            rc = e == cudaErrorMemoryAllocation ? MSPAI_ERR_ALLOC : MSPAI_ERR_CUDA;
        return rc == MSPAI_OK;
    };
    if (!ok(cudaStreamCreate(&st)) || !ok(cudaMalloc(&dcp, sizeof(int64_t) * (n + 1))) ||
        !ok(cudaMalloc(&dci, sizeof(int32_t) * std::max<int64_t>(C->nnz, 1))) ||
        !ok(cudaMalloc(&dcv, sizeof(double) * std::max<int64_t>(C->nnz, 1))) ||
        !ok(cudaMalloc(&dcnt, sizeof(int32_t) * std::max(n, 1))) ||
        !ok(cudaMalloc(&dptr, sizeof(int64_t) * (n + 1))) || !ok(cudaMalloc(&derr, sizeof(int32_t))))
        goto done;
    if (!ok(cudaMemcpyAsync(dcp, C->colptr, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st)) ||
        !ok(cudaMemcpyAsync(dci, C->rowidx, sizeof(int32_t) * C->nnz, cudaMemcpyHostToDevice, st)) ||
        !ok(cudaMemcpyAsync(dcv, C->values, sizeof(double) * C->nnz, cudaMemcpyHostToDevice, st)) ||
        !ok(cudaMemsetAsync(derr, 0, sizeof(int32_t), st)) ||
        !ok(cudaFuncSetAttribute(mspai::power_pattern_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem))))
        goto done;
    grid = std::max(1, std::min(n, mspai::num_sms() * 2));
    mspai::power_pattern_kernel<<<grid, mspai::kThreads, smem, st>>>(dcp, dci, dcv, n, drop, 0, dcnt,
                                                                     nullptr, nullptr, derr);
    if (!ok(cudaGetLastError()) ||
        !ok(cudaMemcpyAsync(cnt.data(), dcnt, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st)) ||
        !ok(cudaMemcpyAsync(&err, derr, sizeof(int32_t), cudaMemcpyDeviceToHost, st)) ||
        !ok(cudaStreamSynchronize(st)))
        goto done;
    if (err) {
        rc = MSPAI_ERR_CAPACITY;
        if (msg && msg_len > 0)
            std::snprintf(msg, static_cast<size_t>(msg_len),
                          "column %d has more than %d products of A(:, l) A(l, k)", err - 1,
                          mspai::kMaxProducts);
        goto done;
    }
    for (int k = 0; k < n; k++)
        ptr[k + 1] = ptr[k] + cnt[k];
    if (!ok(cudaMalloc(&didx, sizeof(int32_t) * std::max<int64_t>(ptr[n], 1))) ||
        !ok(cudaMemcpyAsync(dptr, ptr.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st)))
        goto done;
    mspai::power_pattern_kernel<<<grid, mspai::kThreads, smem, st>>>(dcp, dci, dcv, n, drop, 1, dcnt,
                                                                     dptr, didx, derr);
    P_out->nrows = n;
    P_out->ncols = n;
    P_out->nnz = ptr[n];
    P_out->colptr = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * (n + 1)));
    P_out->rowidx = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max<int64_t>(ptr[n], 1)));
    P_out->values = nullptr;
    if (!P_out->colptr || !P_out->rowidx) {
        rc = MSPAI_ERR_ALLOC;
        goto done;
    }
    std::memcpy(P_out->colptr, ptr.data(), sizeof(int64_t) * (n + 1));
    if (!ok(cudaGetLastError()) ||
        !ok(cudaMemcpyAsync(P_out->rowidx, didx, sizeof(int32_t) * ptr[n], cudaMemcpyDeviceToHost, st)) ||
        !ok(cudaStreamSynchronize(st)))
        goto done;
done:
    if (rc != MSPAI_OK) {
        if (msg && msg_len > 0 && rc != MSPAI_ERR_CAPACITY && rc != MSPAI_ERR_PARAM)
            std::snprintf(msg, static_cast<size_t>(msg_len), "CUDA error in the pattern kernel");
        mspai_matrix_free(P_out);
    }
    cudaFree(dcp);
    cudaFree(dci);
    cudaFree(dcv);
    cudaFree(dcnt);
    cudaFree(dptr);
    cudaFree(didx);
    cudaFree(derr);
    if (st)
        cudaStreamDestroy(st);
    return rc;
}
