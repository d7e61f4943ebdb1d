// Application of the preconditioner, y = M x (the reference's Apply_MSPAI,
// src/imspai.cpp:47-53, a PETSc MatMult with M).
//
// M comes out of the setup as CSC.  A scatter over its columns would need
// atomics on y, whose order of additions varies from call to call; instead the
// row structure of M (CSR) is built once per result and every y_i is a gather
// over row i in ascending column order, so y is the same, bit for bit, on every
// call.
//
//   build: a stable radix sort of the entries by row (CUB) gives, per row, the
//          entry numbers in CSC order -- which is ascending column order;
//          row lengths by a histogram, row pointers by a scan
//   apply: a warp per row, lanes stride the row's entries, then a fixed
//          butterfly reduction
#include "spai_kernels.h"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>

namespace mspai {

namespace {

__global__ void iota_kernel(int32_t* __restrict__ v, int64_t nnz)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nnz;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        v[i] = static_cast<int32_t>(i);
}

__global__ void row_count_kernel(const int32_t* __restrict__ idx, int64_t nnz,
                                 int32_t* __restrict__ cnt)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nnz;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        atomicAdd(&cnt[idx[i]], 1);
}

// Entry t of the row-sorted order: the CSC entry e = perm[t]; its column is
// found by a binary search of the column pointers.
__global__ void gather_rows_kernel(const int64_t* __restrict__ ptr, int ncols,
                                   const double* __restrict__ val, const int32_t* __restrict__ perm,
                                   int64_t nnz, int32_t* __restrict__ tcol,
                                   double* __restrict__ tval)
{
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < nnz;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = perm[t];
        int lo = 0, hi = ncols - 1;  // the column j with ptr[j] <= e < ptr[j + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (ptr[mid] <= e)
                lo = mid;
            else
                hi = mid - 1;
        }
        tcol[t] = lo;
        if (tval)
            tval[t] = val[e];
    }
}

__global__ void csr_gather_kernel(const int64_t* __restrict__ tptr, const int32_t* __restrict__ tcol,
                                  const double* __restrict__ tval, int nrows,
                                  const double* __restrict__ x, double* __restrict__ y)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nrows; i += warps) {
        double s = 0.0;
        for (int64_t t = tptr[i] + lane; t < tptr[i + 1]; t += 32)
            s += tval[t] * x[tcol[t]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
            y[i] = s;
    }
}

int grid_for(int64_t work, int per_block)
{
    const int64_t b = (work + per_block - 1) / per_block;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, num_sms() * 16)));
}

}  // namespace

size_t rows_build_temp_bytes(int64_t nnz, int nrows)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, static_cast<const int32_t*>(nullptr),
                                    static_cast<int32_t*>(nullptr),
                                    static_cast<const int32_t*>(nullptr),
                                    static_cast<int32_t*>(nullptr), static_cast<int>(nnz), 0,
                                    std::max(1, 32 - __builtin_clz(std::max(nrows, 1))));
    return bytes;
}

cudaError_t launch_build_rows(const int64_t* ptr, const int32_t* idx, const double* val,
                              int ncols, int nrows, int64_t nnz, int64_t* tptr, int32_t* tcol,
                              double* tval, int32_t* keys_out, int32_t* perm_in, int32_t* perm_out,
                              int32_t* cnt, int64_t* scan_tmp, void* temp, size_t temp_bytes,
                              cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int32_t) * std::max(nrows, 1), st);
    if (e != cudaSuccess)
        return e;
    if (nnz > 0) {
        iota_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(perm_in, nnz);
        row_count_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(idx, nnz, cnt);
        size_t bytes = temp_bytes;
        e = cub::DeviceRadixSort::SortPairs(temp, bytes, idx, keys_out, perm_in, perm_out,
                                            static_cast<int>(nnz), 0,
                                            std::max(1, 32 - __builtin_clz(std::max(nrows, 1))),
                                            st);
        if (e != cudaSuccess)
            return e;
        gather_rows_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(ptr, ncols, val, perm_out, nnz,
                                                               tcol, tval);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    return launch_scan_lengths(cnt, nrows, tptr, scan_tmp, st);
}

cudaError_t launch_csr_gather(const int64_t* tptr, const int32_t* tcol, const double* tval,
                              int nrows, const double* x, double* y, cudaStream_t st)
{
    if (nrows <= 0)
        return cudaSuccess;
    csr_gather_kernel<<<grid_for(static_cast<int64_t>(nrows) * 32, 256), 256, 0, st>>>(
        tptr, tcol, tval, nrows, x, y);
    return cudaGetLastError();
}

}  // namespace mspai
