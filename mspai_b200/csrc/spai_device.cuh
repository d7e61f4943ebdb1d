// Device building blocks of the batched MSPAI column solver (sm_100a).
//
// A "group" is the set of threads that cooperates on one column problem:
// either one warp (WarpGroup, tiny problems, everything in shared memory) or
// one CTA (CtaGroup<NT>, larger problems, workspace in global scratch that
// stays resident in L2).  All routines below are written against the group
// interface, so the same per-column algorithm runs at both granularities.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mspai {

// Optional per-phase cycle counters (profiling builds only: -DMSPAI_PHASE_TIMERS).
#ifdef MSPAI_PHASE_TIMERS
static __device__ unsigned long long g_phase_cycles[16];
#define PHASE_BEGIN() long long _ph_t = clock64()
#define PHASE_MARK(k)                                                        \
    do {                                                                     \
        if (g.rank() == 0) {                                                 \
            const long long _now = clock64();                                \
            atomicAdd(&g_phase_cycles[k], static_cast<unsigned long long>(_now - _ph_t)); \
            _ph_t = _now;                                                    \
        }                                                                    \
    } while (0)
// sub-phases inside a phase, counted separately in slots 8..15
#define SUBPHASE_BEGIN() long long _sph_t = clock64()
#define SUBPHASE_MARK(k)                                                     \
    do {                                                                     \
        if (g.rank() == 0) {                                                 \
            const long long _now = clock64();                                \
            atomicAdd(&g_phase_cycles[k], static_cast<unsigned long long>(_now - _sph_t)); \
            _sph_t = _now;                                                   \
        }                                                                    \
    } while (0)
#else
#define SUBPHASE_BEGIN() \
    do {                 \
    } while (0)
#define SUBPHASE_MARK(k) \
    do {                 \
    } while (0)
#define PHASE_BEGIN() \
    do {              \
    } while (0)
#define PHASE_MARK(k) \
    do {              \
    } while (0)
#endif


constexpr int kEntryBits = 24;  // sort key = (row << 24) | entry index
constexpr uint64_t kEntryMask = (uint64_t(1) << kEntryBits) - 1;
constexpr int kMaxEntries = 1 << kEntryBits;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ int warp_sum(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class T>
__device__ __forceinline__ T tsqrt(T v);
template <>
__device__ __forceinline__ float tsqrt<float>(float v)
{
    return sqrtf(v);
}
template <>
__device__ __forceinline__ double tsqrt<double>(double v)
{
    return sqrt(v);
}

// Shared scratch a group needs for reductions and broadcasts.
struct GroupScratch {
    double red[32];  // reductions (two halves of 16, see CtaGroup::sum)
    double d[4];
    int i[8];
    int scan[32];    // per-warp totals of group_exclusive_scan
};

struct WarpGroup {
    GroupScratch* sc;
    static constexpr int kSize = 32;
    static constexpr int kWarps = 1;
    __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
    __device__ __forceinline__ int warp() const { return 0; }
    __device__ __forceinline__ int lane() const { return threadIdx.x & 31; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    template <class T>
    __device__ __forceinline__ T sum(T v) const
    {
        return warp_sum(v);
    }
    __device__ __forceinline__ int bcast(int v) const { return __shfl_sync(0xffffffffu, v, 0); }
};

template <int NT>
struct CtaGroup {
    GroupScratch* sc;
    static constexpr int kSize = NT;
    static constexpr int kWarps = NT / 32;
    // reductions alternate between two halves of sc->red so that one barrier
    // per reduction suffices (a warp cannot overwrite a half that a slower warp
    // is still reading: the next reduction's barrier lies in between)
    mutable int parity = 0;
    __device__ __forceinline__ int rank() const { return threadIdx.x; }
    __device__ __forceinline__ int warp() const { return threadIdx.x >> 5; }
    __device__ __forceinline__ int lane() const { return threadIdx.x & 31; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    template <class T>
    __device__ __forceinline__ T sum(T v) const
    {
        static_assert(kWarps <= 16, "two halves of 16 partial sums");
        v = warp_sum(v);
        double* half = sc->red + 16 * parity;
        parity ^= 1;
        if (lane() == 0)
            half[warp()] = static_cast<double>(v);
        __syncthreads();
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; w++)
            t += half[w];
        return static_cast<T>(t);
    }
    __device__ __forceinline__ int bcast(int v) const
    {
        if (threadIdx.x == 0)
            sc->i[7] = v;
        __syncthreads();
        int r = sc->i[7];
        __syncthreads();
        return r;
    }
};

// Exclusive prefix sum of a[0..len) in place; returns the total.  Each thread
// scans a contiguous chunk; the thread totals are scanned with warp shuffles.
template <class G>
__device__ int group_exclusive_scan(const G& g, int* a, int len)
{
    const int chunk = (len + G::kSize - 1) / G::kSize;
    const int lo = min(g.rank() * chunk, len);
    const int hi = min(lo + chunk, len);
    int s = 0;
    for (int i = lo; i < hi; i++)
        s += a[i];
    // inclusive warp scan of the thread totals
    int v = s;
    const int lane = g.lane();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o)
            v += t;
    }
    int* part = g.sc->scan;
    if constexpr (G::kWarps > 1) {
        if (lane == 31)
            part[g.warp()] = v;
        g.sync();
        if (g.rank() == 0) {
            int run = 0;
            for (int w = 0; w < G::kWarps; w++) {
                const int t = part[w];
                part[w] = run;
                run += t;
            }
            g.sc->i[6] = run;
        }
        g.sync();
        int run = part[g.warp()] + v - s;
        for (int i = lo; i < hi; i++) {
            const int t = a[i];
            a[i] = run;
            run += t;
        }
        const int total = g.sc->i[6];
        g.sync();
        return total;
    }
    else {
        const int total = __shfl_sync(0xffffffffu, v, 31);
        int run = v - s;
        for (int i = lo; i < hi; i++) {
            const int t = a[i];
            a[i] = run;
            run += t;
        }
        __syncwarp();
        return total;
    }
}

// Bitonic sort of keys[0..L), L a power of two (pad with the maximum key).
template <class G, class K>
__device__ void group_bitonic_sort(const G& g, K* keys, int L)
{
    for (int k = 2; k <= L; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = g.rank(); i < L; i += G::kSize) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const K a = keys[i];
                    const K b = keys[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[ixj] = a;
                    }
                }
            }
            g.sync();
        }
    }
}

// Sorts E distinct keys made of n ascending runs (run r occupies
// [off[r], off[r + 1])) by merging pairs of runs, ceil(log2 n) rounds.  Each
// thread writes a contiguous chunk of the output: it finds the pair that holds
// its first output position, then its split between the pair's two halves by
// the merge-path binary search (Odeh, Green, Mwassi, Shmueli and Birk, "Merge
// Path - parallel merging made simple", IPDPSW 2012), and merges sequentially.
// a and b are two buffers of E keys; returns the one that holds the result.
template <class K, class G>
__device__ K* group_merge_runs(const G& g, K* a, K* b, int E, const int* off, int n)
{
    const int chunk = (E + G::kSize - 1) / G::kSize;
    for (int w = 1; w < n; w <<= 1) {
        const int npairs = (n + 2 * w - 1) / (2 * w);
        int o = min(E, g.rank() * chunk);
        const int oe = min(E, o + chunk);
        while (o < oe) {
            // the last pair whose output starts at or before o
            int lo = 0, hi = npairs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (off[min(2 * mid * w, n)] <= o)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const int s0 = off[min(2 * lo * w, n)];
            const int s1 = off[min((2 * lo + 1) * w, n)];
            const int s2 = off[min((2 * lo + 2) * w, n)];
            const int la = s1 - s0, lb = s2 - s1, d = o - s0;
            // keys of the first half among the pair's first d outputs
            int ilo = max(0, d - lb), ihi = min(d, la);
            while (ilo < ihi) {
                const int i = (ilo + ihi) >> 1;
                if (a[s0 + i] <= a[s1 + d - i - 1])
                    ilo = i + 1;
                else
                    ihi = i;
            }
            int ia = s0 + ilo, ib = s1 + (d - ilo);
            const int end = min(oe, s2);
            for (; o < end; o++) {
                const bool take_a = ib >= s2 || (ia < s1 && a[ia] <= a[ib]);
                b[o] = take_a ? a[ia++] : a[ib++];
            }
        }
        g.sync();
        K* t = a;
        a = b;
        b = t;
    }
    return a;
}

__host__ __device__ inline int next_pow2(int v)
{
    int p = 1;
    while (p < v)
        p <<= 1;
    return p;
}

}  // namespace mspai
