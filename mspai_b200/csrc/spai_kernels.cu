// Kernels of the batched MSPAI setup and their launchers.
//
//   plan_kernel      per column: |J_k| and the number of entries of C(:, J_k)
//                    (the size that decides the bucket), warp per column
//   bucket_kernel    size-binned work lists (atomic append per bucket) and
//                    per-bucket maxima of the sizes
//   warp_solve       one warp per column, whole workspace in shared memory
//                    (tiny problems: |C(:,J)| <= 64 entries, |J| <= 16)
//   cta_solve        one CTA per column from a work queue (persistent grid);
//                    the folded least-squares matrix lives in shared memory
//                    (W_SMEM) or in a per-CTA global scratch slot
//   compact_kernel   gathers per-column results into M's CSC arrays
//
// The column loop of the reference (src/Spai.imp:160-167 with
// Load_Balance::Grab_M_Col, src/Load_Balance.imp:33-69) becomes these work
// queues: an atomic counter per bucket hands out columns.
#include "spai_kernels.h"
#include "spai_solve.cuh"

#include <algorithm>
#include <cstdio>

namespace mspai {

#ifdef MSPAI_PHASE_TIMERS
extern "C" int mspai_profile_phase_cycles(unsigned long long* out, int reset)
{
    cudaMemcpyFromSymbol(out, g_phase_cycles, sizeof(unsigned long long) * 16);
    if (reset) {
        unsigned long long z[16] = {};
        cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z));
    }
    return 0;
}
#endif

// ------------------------------------------------------------------ planning
__global__ void plan_kernel(const int64_t* __restrict__ cptr, const int64_t* __restrict__ pptr,
                            const int32_t* __restrict__ pidx, int nprob, int bs,
                            int32_t* __restrict__ E, int32_t* __restrict__ nk)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; col < nprob; col += warps) {
        const int64_t a = pptr[col], b = pptr[col + 1];
        int64_t e = 0;
        for (int64_t p = a + lane; p < b; p += 32) {
            const int j = pidx[p];
            for (int c = 0; c < bs; c++)
                e += cptr[bs * j + c + 1] - cptr[bs * j + c];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            e += __shfl_xor_sync(0xffffffffu, e, o);
        if (lane == 0) {
            E[col] = static_cast<int32_t>(e > 0x7fffffff ? 0x7fffffff : e);
            nk[col] = static_cast<int32_t>((b - a) * bs);
        }
    }
}

// bucket ids: 0 warp (tiny), 1 CTA + shared-memory W, 2 CTA + global W
__global__ void bucket_kernel(const int32_t* __restrict__ E, const int32_t* __restrict__ nk, int n,
                              BucketRule rule, int32_t* __restrict__ counts,
                              int32_t* __restrict__ maxE, int32_t* __restrict__ maxN,
                              int32_t* __restrict__ lists)
{
    for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n;
         col += gridDim.x * blockDim.x) {
        if (col < rule.lo || col >= rule.hi)
            continue;  // outside the requested column range
        if (rule.rep && rule.rep[col] != col)
            continue;  // solved by its representative
        // sizes after at most ns pattern updates
        const int64_t nf = static_cast<int64_t>(nk[col]) + rule.grow_n;
        const int64_t ef = static_cast<int64_t>(E[col]) + rule.grow_e;
        int b;
        if (rule.single_bucket >= 0)
            b = rule.single_bucket;
        else if (rule.allow_warp && ef <= rule.warp_emax && nf <= rule.warp_nmax)
            b = 0;
        else {
            const int64_t mw = ef / 2 + nf;
            const int64_t wbytes = (mw * nf + mw) * rule.elem_bytes;
            b = (wbytes <= rule.smem_w_bytes) ? 1 : 2;
        }
        const int slot = atomicAdd(&counts[b], 1);
        lists[static_cast<int64_t>(b) * n + slot] = col;
        atomicMax(&maxE[b], static_cast<int32_t>(ef > 0x7fffffff ? 0x7fffffff : ef));
        atomicMax(&maxN[b], static_cast<int32_t>(nf));
    }
}

// ------------------------------------------------------------------ solvers
template <class T>
__global__ void __launch_bounds__(kWarpKernelThreads)
    warp_solve_kernel(Problem pb, Caps cap, Output out, const int32_t* __restrict__ list,
                      int count, int32_t* __restrict__ counter, int slot_bytes)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ GroupScratch sc[kWarpKernelThreads / 32];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    WarpGroup g{&sc[w]};
    SlotLayout<T> lay(cap, false);
    Slot<T> s = lay.at(smem + static_cast<size_t>(w) * slot_bytes, nullptr);
    while (true) {
        int t = 0;
        if (lane == 0)
            t = atomicAdd(counter, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= count)
            break;
        solve_column<T>(g, pb, cap, s, out, list[t]);
    }
}

// A warp per column with the slot in global memory (scratch + slot_bytes per
// warp): the tiny bucket of adaptive setups, whose candidate bit vector over
// all problem columns does not fit a shared-memory slot.
template <class T>
__global__ void __launch_bounds__(kWarpKernelThreads)
    warp_solve_global_kernel(Problem pb, Caps cap, Output out, const int32_t* __restrict__ list,
                             int count, int32_t* __restrict__ counter, char* __restrict__ scratch,
                             size_t slot_bytes)
{
    __shared__ GroupScratch sc[kWarpKernelThreads / 32];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    WarpGroup g{&sc[w]};
    SlotLayout<T> lay(cap, false);
    const size_t slot_id = static_cast<size_t>(blockIdx.x) * (kWarpKernelThreads / 32) + w;
    Slot<T> s = lay.at(scratch + slot_id * slot_bytes, nullptr);
    while (true) {
        int t = 0;
        if (lane == 0)
            t = atomicAdd(counter, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= count)
            break;
        solve_column<T>(g, pb, cap, s, out, list[t]);
    }
}

// The solver is latency bound: throughput grows with the columns in flight
// per SM.  MINB CTAs of 128 threads per SM bound the registers per thread
// (128 for 4, 64 for 8); the shared-memory area per CTA is chosen with it.
template <class T, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    cta_solve_kernel(Problem pb, Caps cap, Output out, const int32_t* __restrict__ list, int count,
                     int32_t* __restrict__ counter, char* __restrict__ scratch, size_t slot_bytes,
                     int wfast_elems, int blocked)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ GroupScratch sc;
    __shared__ BlockedScratch<T> bsc;
    CtaGroup<NT> g{&sc};
    SlotLayout<T> lay(cap, false);
    Slot<T> s = lay.at(scratch + static_cast<size_t>(blockIdx.x) * slot_bytes, nullptr);
    s.Wfast = wfast_elems > 0 ? reinterpret_cast<T*>(smem) : nullptr;
    s.wfast_elems = wfast_elems;
    s.bsc = blocked ? &bsc : nullptr;
    while (true) {
        if (threadIdx.x == 0)
            sc.i[5] = atomicAdd(counter, 1);
        __syncthreads();
        const int t = sc.i[5];
        __syncthreads();
        if (t >= count)
            break;
        solve_column<T>(g, pb, cap, s, out, list[t]);
    }
}

// ------------------------------------------------------------------ assembly
__global__ void compact_kernel(const int64_t* __restrict__ cap_ptr, const int32_t* __restrict__ cidx,
                               const double* __restrict__ cval, const int64_t* __restrict__ out_ptr,
                               int32_t* __restrict__ oidx, double* __restrict__ oval, int n)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; col < n; col += warps) {
        const int64_t a = cap_ptr[col];
        const int64_t o = out_ptr[col];
        const int len = static_cast<int>(out_ptr[col + 1] - o);
        for (int t = lane; t < len; t += 32) {
            oidx[o + t] = cidx[a + t];
            oval[o + t] = cval[a + t];
        }
    }
}

// exclusive scan of int32 lengths into int64 pointers (3-phase, device-wide)
__global__ void scan_blocks_kernel(const int32_t* __restrict__ len, int n, int64_t* __restrict__ out,
                                   int64_t* __restrict__ block_sums)
{
    __shared__ int64_t sh[1024];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t v = (i < n) ? len[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
        int64_t t = (threadIdx.x >= o) ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n)
        out[i] = sh[threadIdx.x] - v;
    if (threadIdx.x == blockDim.x - 1)
        block_sums[blockIdx.x] = sh[threadIdx.x];
}

__global__ void scan_add_kernel(int64_t* __restrict__ out, int n, const int64_t* __restrict__ block_off)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] += block_off[blockIdx.x];
}

__global__ void scan_serial_kernel(int64_t* __restrict__ v, int nb)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int64_t run = 0;
        for (int i = 0; i < nb; i++) {
            const int64_t t = v[i];
            v[i] = run;
            run += t;
        }
        v[nb] = run;
    }
}

__global__ void finish_ptr_kernel(int64_t* __restrict__ ptr, int n, const int32_t* __restrict__ len)
{
    // ptr[n] = ptr[n-1] + len[n-1]
    if (blockIdx.x == 0 && threadIdx.x == 0)
        ptr[n] = (n > 0) ? ptr[n - 1] + len[n - 1] : 0;
}

// entries of a packed triangle of |P(:, k)|: n_k (n_k + 1) / 2
// Order-independent 64-bit digest of a CSC structure: the wrapping sum of a
// mix of (position, value) over the column pointers and the row indices, so
// that the result does not depend on the launch shape or the order of the
// atomic adds.
__device__ __forceinline__ unsigned long long struct_mix(unsigned long long v)
{
    // SplitMix64 finaliser
    v += 0x9e3779b97f4a7c15ull;
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
    return v ^ (v >> 31);
}

__global__ void structure_hash_kernel(const int64_t* __restrict__ ptr,
                                      const int32_t* __restrict__ idx, int ncols, int64_t nnz,
                                      unsigned long long salt, unsigned long long* acc)
{
    unsigned long long part = 0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= ncols;
         i += stride)
        part += struct_mix(salt ^ (static_cast<unsigned long long>(i) << 1) ^
                           (static_cast<unsigned long long>(ptr[i]) * 0x100000001b3ull));
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
         i += stride)
        part += struct_mix(~salt ^ (static_cast<unsigned long long>(i) << 1) ^
                           (static_cast<unsigned long long>(static_cast<uint32_t>(idx[i])) << 33));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(acc, part);
}

cudaError_t launch_structure_hash(const int64_t* ptr, const int32_t* idx, int ncols, int64_t nnz,
                                  unsigned long long salt, unsigned long long* acc,
                                  cudaStream_t st)
{
    const int blocks = std::max(1, std::min<int>(num_sms() * 8,
                                                 static_cast<int>((nnz + ncols + 255) / 256)));
    structure_hash_kernel<<<blocks, 256, 0, st>>>(ptr, idx, ncols, nnz, salt, acc);
    return cudaGetLastError();
}

__global__ void tri_len_kernel(const int64_t* __restrict__ pptr, int n, int32_t* __restrict__ len)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int64_t nk = pptr[k + 1] - pptr[k];
        len[k] = static_cast<int32_t>(nk * (nk + 1) / 2);
    }
}

cudaError_t launch_tri_len(const int64_t* pptr, int n, int32_t* len, cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    int blocks = std::min((n + 255) / 256, num_sms() * 8);
    tri_len_kernel<<<blocks, 256, 0, st>>>(pptr, n, len);
    return cudaGetLastError();
}

// capacity of scalar column sc: bs * (|P(:, sc / bs)| + grow) entries
__global__ void capacity_len_kernel(const int64_t* __restrict__ pptr, int n, int bs, int grow,
                                    int32_t* __restrict__ len)
{
    for (int sc = blockIdx.x * blockDim.x + threadIdx.x; sc < n; sc += gridDim.x * blockDim.x) {
        const int kb = sc / bs;
        len[sc] = static_cast<int32_t>((pptr[kb + 1] - pptr[kb] + grow) * bs);
    }
}

__global__ void max_len_kernel(const int64_t* __restrict__ ptr, int n, int32_t* __restrict__ out)
{
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = max(m, static_cast<int>(ptr[i + 1] - ptr[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(out, m);
}

// ------------------------------------------------------------------ input checks
// First error found in a CSC structure: err[0] = kind (1 pointers do not match
// nnz, 2 pointers decrease, 3 row out of range, 4 rows not sorted/unique,
// 5 empty column), err[1] = column, err[2] = row.  Pointers are checked
// before any entry of their column is read.
__global__ void validate_csc_kernel(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                    int ncols, int nrows, int64_t nnz, int nonempty,
                                    int32_t* __restrict__ err)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    auto report = [&](int kind, int c, int r) {
        if (atomicCAS(err, 0, kind) == 0) {
            err[1] = c;
            err[2] = r;
        }
    };
    if (tid == 0 && (ptr[0] != 0 || ptr[ncols] != nnz))
        report(1, -1, 0);
    for (int c = tid; c < ncols; c += gridDim.x * blockDim.x) {
        const int64_t a = ptr[c], b = ptr[c + 1];
        if (a < 0 || b > nnz || b < a) {
            report(b < a ? 2 : 1, c, 0);
            continue;
        }
        if (nonempty && a == b)
            report(5, c, 0);
        int prev = -1;
        for (int64_t p = a; p < b; p++) {
            const int r = idx[p];
            if (r < 0 || r >= nrows) {
                report(3, c, r);
                break;
            }
            if (r <= prev) {
                report(4, c, r);
                break;
            }
            prev = r;
        }
    }
}

// ------------------------------------------------------------------ launchers
namespace {
int g_num_sms = 0;
}  // namespace

int num_sms()
{
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0)
            g_num_sms = 1;
    }
    return g_num_sms;
}

cudaError_t launch_validate_csc(const int64_t* ptr, const int32_t* idx, int ncols, int nrows,
                                int64_t nnz, bool nonempty, int32_t* err, cudaStream_t st)
{
    const int blocks = std::max(1, std::min((ncols + 255) / 256, num_sms() * 8));
    validate_csc_kernel<<<blocks, 256, 0, st>>>(ptr, idx, ncols, nrows, nnz, nonempty ? 1 : 0,
                                                err);
    return cudaGetLastError();
}

cudaError_t launch_plan(const int64_t* cptr, const int64_t* pptr, const int32_t* pidx, int nprob,
                        int bs, int32_t* E, int32_t* nk, cudaStream_t st)
{
    if (nprob <= 0)
        return cudaSuccess;
    const int threads = 256;
    int blocks = (nprob + 7) / 8;
    blocks = std::min(blocks, num_sms() * 16);
    plan_kernel<<<blocks, threads, 0, st>>>(cptr, pptr, pidx, nprob, bs, E, nk);
    return cudaGetLastError();
}

cudaError_t launch_bucket(const int32_t* E, const int32_t* nk, int n, const BucketRule& rule,
                          int32_t* counts, int32_t* maxE, int32_t* maxN, int32_t* lists,
                          cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    int blocks = std::min((n + 255) / 256, num_sms() * 8);
    bucket_kernel<<<blocks, 256, 0, st>>>(E, nk, n, rule, counts, maxE, maxN, lists);
    return cudaGetLastError();
}

size_t warp_slot_bytes(const Caps& cap, int elem_bytes)
{
    if (elem_bytes == 4)
        return SlotLayout<float>(cap, false).bytes;
    return SlotLayout<double>(cap, false).bytes;
}

size_t cta_slot_bytes(const Caps& cap, int elem_bytes, bool w_smem)
{
    if (elem_bytes == 4)
        return SlotLayout<float>(cap, w_smem).bytes;
    return SlotLayout<double>(cap, w_smem).bytes;
}

size_t w_bytes(const Caps& cap, int elem_bytes)
{
    return static_cast<size_t>(cap.mwmax) * (cap.nmax + std::max(1, cap.nrhs)) * elem_bytes;
}

template <class T>
static cudaError_t launch_warp_t(const Problem& pb, const Caps& cap, const Output& out,
                                 const int32_t* list, int count, int32_t* counter, cudaStream_t st,
                                 int* grid_out)
{
    const int slot = static_cast<int>(SlotLayout<T>(cap, false).bytes);
    const size_t smem = static_cast<size_t>(slot) * (kWarpKernelThreads / 32);
    cudaError_t e = cudaFuncSetAttribute(warp_solve_kernel<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, warp_solve_kernel<T>,
                                                      kWarpKernelThreads, smem);
    if (e != cudaSuccess)
        return e;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    int grid = per_sm * num_sms();
    const int need = (count + kWarpKernelThreads / 32 - 1) / (kWarpKernelThreads / 32);
    grid = std::max(1, std::min(grid, need));
    *grid_out = grid;
    warp_solve_kernel<T><<<grid, kWarpKernelThreads, smem, st>>>(pb, cap, out, list, count,
                                                                   counter, slot);
    return cudaGetLastError();
}

template <class T>
static int warp_global_grid(int count)
{
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, warp_solve_global_kernel<T>,
                                                  kWarpKernelThreads, 0);
    const int need = (count + kWarpKernelThreads / 32 - 1) / (kWarpKernelThreads / 32);
    return std::max(1, std::min(std::max(per_sm, 1) * num_sms(), need));
}

size_t warp_global_scratch_bytes(const Caps& cap, int elem_bytes, int count)
{
    const int grid = elem_bytes == 4 ? warp_global_grid<float>(count) : warp_global_grid<double>(count);
    return warp_slot_bytes(cap, elem_bytes) * static_cast<size_t>(grid) * (kWarpKernelThreads / 32);
}

template <class T>
static cudaError_t launch_warp_global_t(const Problem& pb, const Caps& cap, const Output& out,
                                        const int32_t* list, int count, int32_t* counter,
                                        char* scratch, size_t scratch_bytes, cudaStream_t st,
                                        int* grid_out)
{
    const size_t slot = SlotLayout<T>(cap, false).bytes;
    int grid = warp_global_grid<T>(count);
    grid = std::max(1, std::min<int>(grid, static_cast<int>(
                                               scratch_bytes / (slot * (kWarpKernelThreads / 32)))));
    *grid_out = grid;
    warp_solve_global_kernel<T><<<grid, kWarpKernelThreads, 0, st>>>(pb, cap, out, list, count,
                                                                     counter, scratch, slot);
    return cudaGetLastError();
}

cudaError_t launch_warp_solve_global(int elem_bytes, const Problem& pb, const Caps& cap,
                                     const Output& out, const int32_t* list, int count,
                                     int32_t* counter, char* scratch, size_t scratch_bytes,
                                     cudaStream_t st, int* grid_out)
{
    if (elem_bytes == 4)
        return launch_warp_global_t<float>(pb, cap, out, list, count, counter, scratch,
                                           scratch_bytes, st, grid_out);
    return launch_warp_global_t<double>(pb, cap, out, list, count, counter, scratch,
                                        scratch_bytes, st, grid_out);
}

cudaError_t launch_warp_solve(int elem_bytes, const Problem& pb, const Caps& cap,
                              const Output& out, const int32_t* list, int count, int32_t* counter,
                              cudaStream_t st, int* grid_out)
{
    if (elem_bytes == 4)
        return launch_warp_t<float>(pb, cap, out, list, count, counter, st, grid_out);
    return launch_warp_t<double>(pb, cap, out, list, count, counter, st, grid_out);
}

template <class T, int NT, int MINB>
static cudaError_t launch_cta_t(const Problem& pb, const Caps& cap, const Output& out,
                                const int32_t* list, int count, int32_t* counter, char* scratch,
                                size_t scratch_bytes, size_t smem, int blocked, cudaStream_t st,
                                int* grid_out)
{
    const size_t slot = SlotLayout<T>(cap, false).bytes;
    cudaError_t e = cudaFuncSetAttribute(cta_solve_kernel<T, NT, MINB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cta_solve_kernel<T, NT, MINB>, NT,
                                                      smem);
    if (e != cudaSuccess)
        return e;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    int grid = std::min(per_sm, MINB) * num_sms();
    grid = std::max(1, std::min(grid, count));
    const size_t slots_fit = slot > 0 ? scratch_bytes / slot : 0;
    if (slots_fit < 1)
        return cudaErrorMemoryAllocation;
    grid = static_cast<int>(std::min<size_t>(grid, slots_fit));
    *grid_out = grid;
    const int wfast = static_cast<int>(smem / sizeof(T));
    cta_solve_kernel<T, NT, MINB><<<grid, NT, smem, st>>>(pb, cap, out, list, count, counter,
                                                          scratch, slot, wfast, blocked);
    return cudaGetLastError();
}

cudaError_t launch_cta_solve(int elem_bytes, size_t smem_w_bytes, bool blocked,
                             const Problem& pb, const Caps& cap, const Output& out,
                             const int32_t* list, int count, int32_t* counter, char* scratch,
                             size_t scratch_bytes, cudaStream_t st, int* grid_out)
{
    const int per_sm = cta_per_sm(elem_bytes, smem_w_bytes);
    if (elem_bytes == 4) {
        if (per_sm == 8)
            return launch_cta_t<float, 128, 8>(pb, cap, out, list, count, counter, scratch,
                                               scratch_bytes, smem_w_bytes, blocked ? 1 : 0, st,
                                               grid_out);
        if (per_sm == 6)
            return launch_cta_t<float, 128, 6>(pb, cap, out, list, count, counter, scratch,
                                               scratch_bytes, smem_w_bytes, blocked ? 1 : 0, st,
                                               grid_out);
        return launch_cta_t<float, 128, 4>(pb, cap, out, list, count, counter, scratch,
                                           scratch_bytes, smem_w_bytes, blocked ? 1 : 0, st,
                                           grid_out);
    }
    return launch_cta_t<double, 128, 4>(pb, cap, out, list, count, counter, scratch,
                                        scratch_bytes, smem_w_bytes, blocked ? 1 : 0, st,
                                        grid_out);
}

int cta_per_sm(int elem_bytes, size_t smem_w_bytes)
{
    if (elem_bytes != 4)
        return 4;
    if (smem_w_bytes <= 24 * 1024)
        return 8;
    if (smem_w_bytes <= 32 * 1024)
        return 6;
    return 4;
}

size_t cta_scratch_needed(int elem_bytes, const Caps& cap, int count, size_t smem_w_bytes)
{
    const size_t slot = cta_slot_bytes(cap, elem_bytes, false);
    const size_t slots =
        static_cast<size_t>(std::min(count, cta_per_sm(elem_bytes, smem_w_bytes) * num_sms()));
    return slot * std::max<size_t>(slots, 1);
}

cudaError_t launch_scan_lengths(const int32_t* len, int n, int64_t* ptr, int64_t* tmp,
                                cudaStream_t st)
{
    // ptr has n+1 entries; tmp has >= nb + 1 entries
    if (n <= 0) {
        return cudaMemsetAsync(ptr, 0, sizeof(int64_t), st);
    }
    const int bs = 1024;
    const int nb = (n + bs - 1) / bs;
    scan_blocks_kernel<<<nb, bs, 0, st>>>(len, n, ptr, tmp);
    scan_serial_kernel<<<1, 1, 0, st>>>(tmp, nb);
    scan_add_kernel<<<nb, bs, 0, st>>>(ptr, n, tmp);
    finish_ptr_kernel<<<1, 1, 0, st>>>(ptr, n, len);
    return cudaGetLastError();
}

cudaError_t launch_capacity_len(const int64_t* pptr, int n, int bs, int grow, int32_t* len,
                                cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    int blocks = std::min((n + 255) / 256, num_sms() * 8);
    capacity_len_kernel<<<blocks, 256, 0, st>>>(pptr, n, bs, grow, len);
    return cudaGetLastError();
}

cudaError_t launch_compact(const int64_t* cap_ptr, const int32_t* cidx, const double* cval,
                           const int64_t* out_ptr, int32_t* oidx, double* oval, int n,
                           cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    int blocks = std::min((n + 7) / 8, num_sms() * 16);
    compact_kernel<<<blocks, 256, 0, st>>>(cap_ptr, cidx, cval, out_ptr, oidx, oval, n);
    return cudaGetLastError();
}

cudaError_t launch_max_len(const int64_t* ptr, int n, int32_t* out, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(int32_t), st);
    if (e != cudaSuccess || n <= 0)
        return e;
    int blocks = std::min((n + 255) / 256, num_sms() * 8);
    max_len_kernel<<<blocks, 256, 0, st>>>(ptr, n, out);
    return cudaGetLastError();
}

}  // namespace mspai
