// Launchers of the fixed-pattern column solver (fixed_solve.cuh).
//
// fixed_solve_kernel takes columns from a work list with an atomic counter
// (a persistent grid: the reference's column loop, src/Spai.imp:160-167, as a
// device work queue); a column whose arrays do not fit the CTA's arena goes
// to the overflow list, which a later launch with a larger arena (and after
// that the general solver) works through.  The number of listed columns may
// come from device memory (the previous launch's overflow count), so the
// launches follow each other on the stream without a host round trip.
#include "spai_kernels.h"
#include "fixed_solve.cuh"

#include <algorithm>

namespace mspai {

#ifdef MSPAI_PHASE_TIMERS
// cycle counters of the fixed-pattern solver's phases (profiling builds only)
extern "C" int mspai_profile_fixed_cycles(unsigned long long* out, int reset)
{
    cudaMemcpyFromSymbol(out, g_phase_cycles, sizeof(unsigned long long) * 16);
    if (reset) {
        unsigned long long z[16] = {};
        cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z));
    }
    return 0;
}
#endif

template <class T, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    fixed_solve_kernel(Problem pb, Output out, const int32_t* __restrict__ list,
                       const int32_t* __restrict__ count_dev, int count_host,
                       int32_t* __restrict__ counter, int32_t* __restrict__ ovf_list,
                       int32_t* __restrict__ ovf_count, int arena_bytes, T* __restrict__ rglob,
                       int64_t rglob_elems)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ FixShared<T> fs;
    CtaGroup<NT> g{&fs.sc};
    const int count = count_dev ? *count_dev : count_host;
    T* rg = rglob ? rglob + static_cast<int64_t>(blockIdx.x) * rglob_elems : nullptr;
    while (true) {
        if (threadIdx.x == 0)
            fs.sc.i[5] = atomicAdd(counter, 1);
        __syncthreads();
        const int t = fs.sc.i[5];
        __syncthreads();
        if (t >= count)
            break;
        const int col = list[t];
        const bool done =
            fixed_solve_column<T, NT>(g, fs, pb, out, col, smem, arena_bytes, rg, rglob_elems);
        if (!done && threadIdx.x == 0)
            ovf_list[atomicAdd(ovf_count, 1)] = col;
        __syncthreads();
    }
}

namespace {

template <class T, int NT, int MINB>
cudaError_t launch_fixed_t(int arena_bytes, const Problem& pb, const Output& out,
                           const int32_t* list, const int32_t* count_dev, int count_host,
                           int32_t* counter, int32_t* ovf_list, int32_t* ovf_count, void* rglob,
                           int64_t rglob_elems, int max_ctas, cudaStream_t st, int* grid_out)
{
    auto kern = fixed_solve_kernel<T, NT, MINB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         arena_bytes);
    if (e != cudaSuccess)
        return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, arena_bytes);
    if (e != cudaSuccess)
        return e;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    int grid = std::min(per_sm, MINB) * num_sms();
    if (count_dev == nullptr)
        grid = std::min(grid, std::max(count_host, 1));
    grid = std::min(grid, max_ctas);
    *grid_out = grid;
    kern<<<grid, NT, arena_bytes, st>>>(pb, out, list, count_dev, count_host, counter, ovf_list,
                                        ovf_count, arena_bytes, static_cast<T*>(rglob),
                                        rglob_elems);
    return cudaGetLastError();
}

}  // namespace

int fixed_ctas_per_sm(int arena_bytes)
{
    // two CTAs of 256 threads per SM (128 registers per thread), or one CTA
    // of 256 threads with the largest arena (measured faster than 512 threads:
    // the barriers of the panel steps wait for half as many warps)
    return arena_bytes <= 107 * 1024 ? 2 : 1;
}

int fixed_max_grid(int arena_bytes) { return fixed_ctas_per_sm(arena_bytes) * num_sms(); }

int64_t fixed_r_elems(int nmax)
{
    return static_cast<int64_t>(nmax) * (nmax + 1) / 2 + nmax + 16;
}

cudaError_t launch_fixed_solve(int elem_bytes, int arena_bytes, const Problem& pb,
                               const Output& out, const int32_t* list, const int32_t* count_dev,
                               int count_host, int32_t* counter, int32_t* ovf_list,
                               int32_t* ovf_count, void* rglob, int64_t rglob_elems, int max_ctas,
                               cudaStream_t st, int* grid_out)
{
    const int per_sm = fixed_ctas_per_sm(arena_bytes);
    if (elem_bytes == 4) {
        if (per_sm >= 2)
            return launch_fixed_t<float, 256, 2>(arena_bytes, pb, out, list, count_dev, count_host,
                                                 counter, ovf_list, ovf_count, rglob, rglob_elems,
                                                 max_ctas, st, grid_out);
        return launch_fixed_t<float, 256, 1>(arena_bytes, pb, out, list, count_dev, count_host,
                                             counter, ovf_list, ovf_count, rglob, rglob_elems,
                                             max_ctas, st, grid_out);
    }
    if (per_sm >= 2)
        return launch_fixed_t<double, 256, 2>(arena_bytes, pb, out, list, count_dev, count_host,
                                              counter, ovf_list, ovf_count, rglob, rglob_elems,
                                              max_ctas, st, grid_out);
    return launch_fixed_t<double, 256, 1>(arena_bytes, pb, out, list, count_dev, count_host,
                                          counter, ovf_list, ovf_count, rglob, rglob_elems,
                                          max_ctas, st, grid_out);
}

}  // namespace mspai
