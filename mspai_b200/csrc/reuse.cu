// Reuse of identical least-squares problems (the reference's `-cs` cache,
// Spai_Caching::SPAI_Column, src/Spai_Caching.imp:45-332, and `-ch` hash
// table, src/Spai_Hashing.imp): columns whose problems C(I_k,J_k) m = b_k are
// identical are solved once and the solution is copied.
//
// The reference keys its cache on a hash of the dense values of Â and compares
// Â exactly on a hit (Cache.imp:66-104).  Here a column's problem is described
// by its canonical stream, built from the sparse data without forming Â:
//   |J_k|; for every j in J_k (sorted): j - k, nnz(C(:,j)), and every entry
//   (row, value) of C(:,j); then every entry of B(:,k) when B is given.
// Rows below n are written relative to k (r - k); probing rows (r >= n) are
// written absolute, since they do not move with k.  A block problem column k
// (fixed block patterns, bs > 1) streams its bs scalar columns per block of
// J_k, relative to its first scalar column bs k, and B's bs columns.  Two columns with equal
// streams have the same I_k - k, J_k - k, the same Â (same row and column
// order) and the same right-hand side, so the same solution, bit for bit.
// Equal streams are a sufficient condition for equal Â: columns whose Â agree
// by accident of values but not of relative structure are solved separately,
// which changes nothing in M.
//
// Device side, three kernels:
//  1. reuse_key_kernel: a warp per column hashes its stream (a sum of
//     position-tagged 64-bit mixes, so lanes hash in parallel) and inserts the
//     key into an open-addressing table (linear probing, atomicCAS on the
//     key); the smallest column index with that key becomes the slot's
//     representative (atomicMin).
//  2. reuse_verify_kernel: every other column compares its stream with its
//     representative's word by word; equal -> rep[k] = representative, else
//     (a 64-bit hash collision) rep[k] = k and it is solved itself.
//  3. reuse_copy_kernel (after the solves): members copy the representative's
//     values, residual, step count, status and work counters.
// The bucket kernel skips members, so only representatives are solved.
#include "spai_kernels.h"
#include "spai_solve.cuh"

namespace mspai {
namespace {

// SplitMix64 finaliser (Steele, Lea and Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// a word of the stream at position tag
__device__ __forceinline__ uint64_t tagged(uint64_t word, uint64_t tag)
{
    return mix64(word ^ mix64(tag * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull));
}

__device__ __forceinline__ uint64_t enc_row(int r, int k, int n)
{
    return r < n ? (static_cast<uint64_t>(static_cast<int64_t>(r) - k) << 1)
                 : ((static_cast<uint64_t>(r) << 1) | 1ull);
}

__device__ __forceinline__ uint64_t dbits(double v)
{
    return static_cast<uint64_t>(__double_as_longlong(v));
}

// tags: (q + 1) << 32 | 2 * t (+1 for the value) for entry t of the q-th
// scalar column of J (q = bs jj + c for the c-th scalar column of the jj-th
// block of J); q = bs n_k + c for the entries of B(:, bs k + c);
// (q + 1) << 32 | 0xffffffff for a column's header (j - bs k, nnz); 0 for |J_k|.
// Rows below n are relative to bs k, the first scalar column of problem k.
__device__ uint64_t column_hash(const Problem& pb, int k, int lane)
{
    const int bs = pb.bs;
    const int64_t p0 = pb.pptr[k], p1 = pb.pptr[k + 1];
    const int nk = static_cast<int>(p1 - p0);
    const int k0 = bs * k;
    uint64_t h = (lane == 0) ? tagged(static_cast<uint64_t>(nk), 0) : 0;
    for (int jj = 0; jj < nk; jj++) {
        for (int c = 0; c < bs; c++) {
            const int j = bs * pb.pidx[p0 + jj] + c;
            const int64_t c0 = pb.cptr[j], c1 = pb.cptr[j + 1];
            const uint64_t base = static_cast<uint64_t>(bs * jj + c + 1) << 32;
            if (lane == 0)
                h += tagged((static_cast<uint64_t>(static_cast<int64_t>(j) - k0) << 32) ^
                                static_cast<uint64_t>(c1 - c0),
                            base | 0xffffffffull);
            for (int64_t e = c0 + lane; e < c1; e += 32) {
                const uint64_t t = static_cast<uint64_t>(e - c0);
                h += tagged(enc_row(pb.cidx[e], k0, pb.n), base | (2 * t));
                h += tagged(dbits(pb.cval[e]), base | (2 * t + 1));
            }
        }
    }
    if (pb.bptr) {
        for (int c = 0; c < bs; c++) {
            const int64_t b0 = pb.bptr[k0 + c], b1 = pb.bptr[k0 + c + 1];
            const uint64_t base = static_cast<uint64_t>(bs * nk + c + 1) << 32;
            if (lane == 0)
                h += tagged(static_cast<uint64_t>(b1 - b0), base | 0xffffffffull);
            for (int64_t e = b0 + lane; e < b1; e += 32) {
                const uint64_t t = static_cast<uint64_t>(e - b0);
                h += tagged(enc_row(pb.bidx[e], k0, pb.n), base | (2 * t));
                h += tagged(dbits(pb.bval[e]), base | (2 * t + 1));
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        h += __shfl_xor_sync(0xffffffffu, h, o);
    return h | 1ull;  // 0 marks an empty slot
}

// 1 if the entries of scalar columns ja (problem a) and jb (problem b) are
// equal relative to their problems' first scalar columns a0, b0 (warp-uniform)
__device__ int same_entries(const int64_t* ptr, const int32_t* idx, const double* val, int ja,
                            int jb, int a0, int b0, int n, int lane)
{
    const int64_t s0 = ptr[ja], t0 = ptr[jb];
    const int64_t len = ptr[ja + 1] - s0;
    if (len != ptr[jb + 1] - t0)
        return 0;
    int diff = 0;
    for (int64_t t = lane; t < len; t += 32)
        diff |= (enc_row(idx[s0 + t], a0, n) != enc_row(idx[t0 + t], b0, n)) ||
                (dbits(val[s0 + t]) != dbits(val[t0 + t]));
    return __any_sync(0xffffffffu, diff) ? 0 : 1;
}

// 1 if the streams of problem columns a and b are equal (warp-uniform result)
__device__ int same_stream(const Problem& pb, int a, int b, int lane)
{
    const int bs = pb.bs;
    const int64_t pa = pb.pptr[a], pbb = pb.pptr[b];
    const int na = static_cast<int>(pb.pptr[a + 1] - pa);
    if (na != static_cast<int>(pb.pptr[b + 1] - pbb))
        return 0;
    const int a0 = bs * a, b0 = bs * b;
    for (int jj = 0; jj < na; jj++) {
        const int ja = pb.pidx[pa + jj], jb = pb.pidx[pbb + jj];
        if (static_cast<int64_t>(ja) - a != static_cast<int64_t>(jb) - b)
            return 0;
        for (int c = 0; c < bs; c++)
            if (!same_entries(pb.cptr, pb.cidx, pb.cval, bs * ja + c, bs * jb + c, a0, b0, pb.n,
                              lane))
                return 0;
    }
    if (pb.bptr)
        for (int c = 0; c < bs; c++)
            if (!same_entries(pb.bptr, pb.bidx, pb.bval, a0 + c, b0 + c, a0, b0, pb.n, lane))
                return 0;
    return 1;
}

__global__ void reuse_key_kernel(Problem pb, int nprob, ReuseTable t)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < nprob; k += warps) {
        const uint64_t h = column_hash(pb, k, lane);
        if (lane == 0) {
            int slot = -1;
            uint32_t s = static_cast<uint32_t>(h ^ (h >> 32)) & t.mask;
            // at most max_keys distinct problems are stored (the cache size);
            // a column that finds no place is solved on its own.  Best effort:
            // a column that sees its key's slot still empty while the table
            // is full (the key being inserted at that moment) also solves on
            // its own, which changes no result.
            for (uint32_t probe = 0; probe <= t.mask; probe++) {
                // read through L2: other warps insert concurrently
                const unsigned long long cur = __ldcg(
                    reinterpret_cast<const unsigned long long*>(t.keys) + s);
                if (cur == h) {
                    slot = static_cast<int>(s);
                    break;
                }
                if (cur == 0) {
                    if (atomicAdd(t.nkeys, 0) >= t.max_keys)
                        break;
                    const unsigned long long old = atomicCAS(
                        reinterpret_cast<unsigned long long*>(t.keys) + s, 0ull,
                        static_cast<unsigned long long>(h));
                    if (old == 0ull) {
                        atomicAdd(t.nkeys, 1);
                        slot = static_cast<int>(s);
                        break;
                    }
                    if (old == h) {
                        slot = static_cast<int>(s);
                        break;
                    }
                }
                s = (s + 1) & t.mask;
            }
            t.slot_of[k] = slot;
            if (slot >= 0)
                atomicMin(t.rep_of_slot + slot, k);
        }
    }
}

__global__ void reuse_verify_kernel(Problem pb, int nprob, ReuseTable t, int32_t* __restrict__ rep,
                                    int32_t* __restrict__ nreused)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    int mine = 0;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < nprob; k += warps) {
        const int slot = t.slot_of[k];
        int r = k;
        if (slot >= 0) {
            const int cand = t.rep_of_slot[slot];
            if (cand != k && same_stream(pb, cand, k, lane))
                r = cand;
        }
        if (lane == 0) {
            rep[k] = r;
            mine += (r != k);
        }
    }
    if (lane == 0 && mine)
        atomicAdd(nreused, mine);
}

__global__ void reuse_copy_kernel(const int32_t* __restrict__ rep, int nprob, int bs,
                                  Output out)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < nprob; k += warps) {
        const int r = rep[k];
        if (r == k)
            continue;
        // the bs scalar columns of the problem; a block problem's rows move
        // with it (J_k = J_r + (k - r) blocks)
        for (int c = 0; c < bs; c++) {
            const int sk = bs * k + c, sr = bs * r + c;
            const int64_t dst = out.optr[sk], src = out.optr[sr];
            const int len = out.olen[sr];
            for (int t = lane; t < len; t += 32) {
                out.oval[dst + t] = out.oval[src + t];
                if (out.write_idx)
                    out.oidx[dst + t] = out.oidx[src + t] + bs * (k - r);
            }
            if (lane == 0) {
                out.olen[sk] = len;
                out.res[sk] = out.res[sr];
                out.steps[sk] = out.steps[sr];
                out.status[sk] = out.status[sr];
                // the work was done once, for the representative
                out.work[3 * static_cast<size_t>(sk)] = 0.0;
                out.work[3 * static_cast<size_t>(sk) + 1] = 0.0;
                out.work[3 * static_cast<size_t>(sk) + 2] = 0.0;
            }
        }
    }
}

int grid_for(int nprob)
{
    const int warps_per_block = 8;
    const int need = (nprob + warps_per_block - 1) / warps_per_block;
    const int cap = num_sms() * 8;
    return need < 1 ? 1 : (need < cap ? need : cap);
}

}  // namespace

size_t reuse_table_slots(int nprob, int max_keys)
{
    const int64_t want = 2 * static_cast<int64_t>(max_keys < nprob ? max_keys : nprob);
    size_t s = 64;
    while (static_cast<int64_t>(s) < want)
        s <<= 1;
    return s;
}

cudaError_t launch_reuse_keys(const Problem& pb, int nprob, const ReuseTable& t, int32_t* rep,
                              int32_t* nreused, cudaStream_t st)
{
    if (nprob <= 0)
        return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(t.keys, 0, sizeof(uint64_t) * (t.mask + 1ull), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(t.rep_of_slot, 0x7f, sizeof(int32_t) * (t.mask + 1ull), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(t.nkeys, 0, sizeof(int32_t), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(nreused, 0, sizeof(int32_t), st);
    if (e != cudaSuccess)
        return e;
    const int grid = grid_for(nprob);
    reuse_key_kernel<<<grid, 256, 0, st>>>(pb, nprob, t);
    reuse_verify_kernel<<<grid, 256, 0, st>>>(pb, nprob, t, rep, nreused);
    return cudaGetLastError();
}

cudaError_t launch_reuse_copy(const int32_t* rep, int nprob, int bs, const Output& out,
                              cudaStream_t st)
{
    if (nprob <= 0)
        return cudaSuccess;
    reuse_copy_kernel<<<grid_for(nprob), 256, 0, st>>>(rep, nprob, bs, out);
    return cudaGetLastError();
}

}  // namespace mspai
