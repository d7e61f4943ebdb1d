// A fixed-pattern setup that allocates no device or host memory.
//
// Some callers cannot allocate GPU memory at the point where they need the
// preconditioner: applications whose device memory is reserved up front by
// their own pool or by another framework (cudaMalloc would fail or would
// fragment the pool), and latency-critical code paths that must not pay for
// cudaMalloc/cudaFree and the device synchronisation they can imply.  For
// them, mspai_setup_fixed_noalloc runs the same per-column solver as
// mspai_setup on inputs and outputs the caller already holds in device
// memory, with its scratch in a file-scope device array of fixed size.
//
// The array (kNoAllocScratchBytes) is part of the library image: every GPU
// that loads the library holds it until the process exits.  All calls share
// it and it keeps the last call's contents; the work counters that must start
// at zero are cleared at the start of every call.  Calls whose kernels overlap
// on the GPU (different streams, or different host threads) race on the same
// array and must be serialised by the caller.
#include "mspai_b200.h"
#include "spai_kernels.h"
#include "spai_solve.cuh"

#include <algorithm>
#include <cstdio>
#include <mutex>

namespace {

using mspai::Caps;
using mspai::CtaGroup;
using mspai::GroupScratch;
using mspai::Output;
using mspai::Problem;
using mspai::Slot;
using mspai::SlotLayout;

// Size limits of the no-allocation path.  With them the folded least-squares
// matrix of every column fits the CTA's shared-memory area, and one scratch
// slot per resident CTA fits kNoAllocScratchBytes.
constexpr int kNoAllocMaxEntries = 512;     // entries of C(:, J_k) per column
constexpr int kNoAllocMaxPattern = 64;      // |J_k|
constexpr int kNoAllocMaxColumns = 1 << 20; // columns per call
constexpr int kNoAllocThreads = 256;
// 64 MiB: 40 MiB of per-CTA slots, then 24 bytes per column of solver
// bookkeeping (the algorithmic-work counters the solver keeps per column).
constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
constexpr size_t kNoAllocSlotBytes = size_t(40) << 20;

static __device__ __align__(256) char g_noalloc_scratch[kNoAllocScratchBytes];
// [0] work counter, [1] max entries, [2] max |J|, [3] columns over the limits
static __device__ __align__(16) int g_noalloc_counters[4];
// first error of the structure checks of C, P and B (4 ints each: kind,
// column, row, unused), cleared on every call
static __device__ __align__(16) int g_noalloc_checks[12];

struct DeviceAddrs {
    char* scratch = nullptr;
    int* counters = nullptr;
    int* checks = nullptr;
    bool ready = false;
};
constexpr int kMaxDevices = 64;
DeviceAddrs g_addrs[kMaxDevices];
std::mutex g_addrs_mu;

// Per-device set-up: the device addresses of the file-scope arrays.  Host code
// may not use the arrays' names as device pointers; it asks the runtime once
// per device, with that device current.
int device_addrs(int device, DeviceAddrs* out)
{
    if (device < 0 || device >= kMaxDevices)
        return MSPAI_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_addrs_mu);
    DeviceAddrs& a = g_addrs[device];
    if (!a.ready) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess)
            return MSPAI_ERR_CUDA;
        a.scratch = static_cast<char*>(p);
        p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_counters) != cudaSuccess)
            return MSPAI_ERR_CUDA;
        a.counters = static_cast<int*>(p);
        p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_checks) != cudaSuccess)
            return MSPAI_ERR_CUDA;
        a.checks = static_cast<int*>(p);
        a.ready = true;
    }
    *out = a;
    return MSPAI_OK;
}

// Largest entry count and pattern size over all columns.
__global__ void noalloc_sizes_kernel(const int64_t* __restrict__ cptr,
                                     const int64_t* __restrict__ pptr,
                                     const int32_t* __restrict__ pidx, int n, int* counters)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; col < n; col += warps) {
        const int64_t a = pptr[col], b = pptr[col + 1];
        int64_t e = 0;
        for (int64_t p = a + lane; p < b; p += 32) {
            const int j = pidx[p];
            e += cptr[j + 1] - cptr[j];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            e += __shfl_xor_sync(0xffffffffu, e, o);
        if (lane == 0) {
            const int ei = static_cast<int>(e > 0x7fffffff ? 0x7fffffff : e);
            const int ni = static_cast<int>(b - a);
            atomicMax(&counters[1], ei);
            atomicMax(&counters[2], ni);
            if (ei > kNoAllocMaxEntries || ni > kNoAllocMaxPattern)
                atomicAdd(&counters[3], 1);
        }
    }
}

// One CTA per column from the shared work counter; the slot of CTA b is
// scratch + b * slot_bytes, the folded matrix lives in dynamic shared memory.
template <class T>
__global__ void __launch_bounds__(kNoAllocThreads)
    noalloc_solve_kernel(Problem pb, Caps cap, Output out, int n, char* __restrict__ scratch,
                         size_t slot_bytes, int* counters, int wfast_elems)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ GroupScratch sc;
    __shared__ mspai::BlockedScratch<T> bsc;
    CtaGroup<kNoAllocThreads> g{&sc};
    SlotLayout<T> lay(cap, false);
    Slot<T> s = lay.at(scratch + static_cast<size_t>(blockIdx.x) * slot_bytes, nullptr);
    s.Wfast = reinterpret_cast<T*>(smem);
    s.wfast_elems = wfast_elems;
    s.bsc = &bsc;
    while (true) {
        if (threadIdx.x == 0)
            sc.i[5] = atomicAdd(&counters[0], 1);
        __syncthreads();
        const int col = sc.i[5];
        __syncthreads();
        if (col >= n)
            break;
        mspai::solve_column<T>(g, pb, cap, s, out, col);
    }
}

template <class T>
int launch_noalloc(const Problem& pb, const Caps& cap, const Output& out, int n,
                   const DeviceAddrs& a, cudaStream_t st)
{
    // slots live in the first kNoAllocSlotBytes of the array
    const size_t slot = SlotLayout<T>(cap, false).bytes;
    const size_t smem = (static_cast<size_t>(cap.mwmax) * cap.nmax + cap.mwmax) * sizeof(T);
    if (cudaFuncSetAttribute(noalloc_solve_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
        return MSPAI_ERR_CUDA;
    int per_sm = 0, dev = 0, sms = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, noalloc_solve_kernel<T>,
                                                      kNoAllocThreads, smem) != cudaSuccess ||
        per_sm < 1)
        return MSPAI_ERR_CUDA;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t grid = std::min<size_t>(static_cast<size_t>(per_sm) * sms, static_cast<size_t>(n));
    grid = std::min(grid, kNoAllocSlotBytes / slot);
    if (grid < 1)
        return MSPAI_ERR_CAPACITY;
    noalloc_solve_kernel<T><<<static_cast<unsigned>(grid), kNoAllocThreads, smem, st>>>(
        pb, cap, out, n, a.scratch, slot, a.counters, static_cast<int>(smem / sizeof(T)));
    return cudaGetLastError() == cudaSuccess ? MSPAI_OK : MSPAI_ERR_CUDA;
}

}  // namespace

extern "C" int mspai_setup_fixed_noalloc(const mspai_csc* C, const mspai_csc* B,
                                         const mspai_csc* P, const mspai_params* prm,
                                         double* values_out, double* resnorm_out,
                                         int32_t* status_out, void* stream, char* msg,
                                         int32_t msg_len)
{
    auto fail = [&](int code, const char* text) {
        if (msg && msg_len > 0) {
            int i = 0;
            for (; text[i] && i < msg_len - 1; i++)
                msg[i] = text[i];
            msg[i] = '\0';
        }
        return code;
    };
    if (msg && msg_len > 0)
        msg[0] = '\0';
    if (!C || !P || !prm || !values_out || !resnorm_out || !status_out)
        return fail(MSPAI_ERR_PARAM, "C, P, params and the three output arrays are required");
    char vmsg[512];
    const int vrc = mspai_validate_params(prm, vmsg, sizeof(vmsg));
    if (vrc != MSPAI_OK)
        return fail(vrc, vmsg);
    if (prm->ns != 0 || prm->bs != 1)
        return fail(MSPAI_ERR_PARAM, "the no-allocation setup is fixed-pattern and scalar: "
                                     "ns must be 0 and bs 1");
    if (C->mem != MSPAI_MEM_DEVICE || P->mem != MSPAI_MEM_DEVICE ||
        (B && B->mem != MSPAI_MEM_DEVICE))
        return fail(MSPAI_ERR_PARAM, "the no-allocation setup takes device arrays only");
    const int n = C->ncols;
    if (P->ncols != n || P->nrows != n || C->nrows < n ||
        (B && (B->ncols != n || B->nrows != C->nrows)))
        return fail(MSPAI_ERR_INPUT, "matrix dimensions do not match");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess)
        return fail(MSPAI_ERR_NO_DEVICE, "no CUDA device");
    DeviceAddrs a;
    if (device_addrs(device, &a) != MSPAI_OK)
        return fail(MSPAI_ERR_CUDA, "cudaGetSymbolAddress failed for the scratch array");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n == 0)
        return MSPAI_OK;
    if (n > kNoAllocMaxColumns)
        return fail(MSPAI_ERR_CAPACITY, "more columns than the no-allocation limit (1048576)");
    if (C->nnz < 0 || P->nnz < 0 || (B && B->nnz < 0) || !C->colptr || !P->colptr ||
        (C->nnz > 0 && (!C->rowidx || !C->values)) || (P->nnz > 0 && !P->rowidx) ||
        (B && (!B->colptr || (B->nnz > 0 && (!B->rowidx || !B->values)))))
        return fail(MSPAI_ERR_INPUT, "missing arrays");

    // structure of C, P and B (pointers, row range, sorted unique rows, no empty
    // column of C), checked before any kernel indexes with them
    if (cudaMemsetAsync(a.checks, 0, 12 * sizeof(int), st) != cudaSuccess)
        return fail(MSPAI_ERR_CUDA, "cudaMemsetAsync failed");
    if (mspai::launch_validate_csc(C->colptr, C->rowidx, n, C->nrows, C->nnz, true, a.checks,
                                   st) != cudaSuccess ||
        mspai::launch_validate_csc(P->colptr, P->rowidx, n, n, P->nnz, false, a.checks + 4,
                                   st) != cudaSuccess ||
        (B && mspai::launch_validate_csc(B->colptr, B->rowidx, n, C->nrows, B->nnz, false,
                                         a.checks + 8, st) != cudaSuccess))
        return fail(MSPAI_ERR_CUDA, "input check launch failed");
    {
        int hv[12] = {};
        if (cudaMemcpyAsync(hv, a.checks, sizeof(hv), cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return fail(MSPAI_ERR_CUDA, "input checks failed");
        static const char* names[3] = {"C", "P", "B"};
        for (int i = 0; i < 3; i++) {
            const int kind = hv[4 * i], c = hv[4 * i + 1], r = hv[4 * i + 2];
            if (kind == 0)
                continue;
            char buf[256];
            switch (kind) {
            case 1: std::snprintf(buf, sizeof(buf), "%s: column pointers do not match nnz", names[i]); break;
            case 2: std::snprintf(buf, sizeof(buf), "%s: column pointers decrease", names[i]); break;
            case 3:
                std::snprintf(buf, sizeof(buf), "%s: row index %d out of range in column %d",
                              names[i], r, c);
                break;
            case 4:
                std::snprintf(buf, sizeof(buf), "%s: row indices not sorted/unique in column %d",
                              names[i], c);
                break;
            default:
                std::snprintf(buf, sizeof(buf), "Matrix is singular: column %d of C is empty", c);
            }
            return fail(MSPAI_ERR_INPUT, buf);
        }
    }

    // sizes (counters start at zero on every call)
    if (cudaMemsetAsync(a.counters, 0, 4 * sizeof(int), st) != cudaSuccess)
        return fail(MSPAI_ERR_CUDA, "cudaMemsetAsync failed");
    int sms = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    noalloc_sizes_kernel<<<std::min((n + 7) / 8, sms * 16), 256, 0, st>>>(
        C->colptr, P->colptr, P->rowidx, n, a.counters);
    int hc[4] = {0, 0, 0, 0};
    if (cudaMemcpyAsync(hc, a.counters, sizeof(hc), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(MSPAI_ERR_CUDA, "size pass failed");
    if (hc[3] > 0) {
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "%d columns exceed the no-allocation limits (largest: %d entries of "
                      "C(:,J), |J| = %d; limits %d and %d); use mspai_setup",
                      hc[3], hc[1], hc[2], kNoAllocMaxEntries, kNoAllocMaxPattern);
        return fail(MSPAI_ERR_CAPACITY, buf);
    }
    Problem pb{};
    pb.n = n;
    pb.nrows = C->nrows;
    pb.cptr = C->colptr;
    pb.cidx = C->rowidx;
    pb.cval = C->values;
    pb.pptr = P->colptr;
    pb.pidx = P->rowidx;
    if (B) {
        pb.bptr = B->colptr;
        pb.bidx = B->rowidx;
        pb.bval = B->values;
    }
    pb.bs = 1;
    pb.ep = prm->ep;
    pb.mn = prm->mn;
    pb.ns = 0;
    pb.um = prm->um;
    const bool mixed = prm->prec == MSPAI_PREC_MIXED;
    pb.refine = mixed ? std::max(0, prm->refine) : 0;
    Caps cap{};
    cap.emax = std::max(1, hc[1]);
    cap.nmax = std::max(1, hc[2]);
    cap.lsort = mspai::next_pow2(cap.emax);
    cap.mwmax = cap.emax / 2 + cap.nmax;
    cap.cmax = 0;
    cap.lcand = 0;
    cap.nrhs = 1;
    cap.nbmap = 0;
    Output out{};
    out.optr = P->colptr;  // M has P's pattern: only the values are written
    out.oidx = nullptr;
    out.write_idx = 0;
    out.oval = values_out;
    out.res = resnorm_out;
    out.status = status_out;
    // the solver also records |J_k| and the LS-solve count per column.  They
    // share the caller's status array: solve_column writes a column's length
    // and step count before its status, from the same thread, in every branch,
    // so the status is the value that remains
    out.olen = status_out;
    out.steps = status_out;
    // per-column work counters: the array's tail, cleared for this call
    out.work = reinterpret_cast<double*>(a.scratch + kNoAllocSlotBytes);
    if (cudaMemsetAsync(out.work, 0, static_cast<size_t>(n) * 3 * sizeof(double), st) !=
        cudaSuccess)
        return fail(MSPAI_ERR_CUDA, "cudaMemsetAsync failed");
    const int rc = mixed ? launch_noalloc<float>(pb, cap, out, n, a, st)
                         : launch_noalloc<double>(pb, cap, out, n, a, st);
    if (rc != MSPAI_OK)
        return fail(rc, "kernel launch failed");
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return fail(MSPAI_ERR_CUDA, "kernel failed");
    return MSPAI_OK;
}
