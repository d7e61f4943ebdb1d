// Power patterns of A with the reference's count-based sparsification, on
// the device: the pattern the reference's To_Pattern_Powers builds through
// PETSc (src/Matrix.imp:359-470):
//
//   S = Sparsify(|A|);  repeat nb_pw times { S = Sparsify(S) (not the first
//   time);  S = S S };  S = Sparsify(S);  P = pattern(S)
//
// Sparsify (src/Matrix.imp:471-620) keeps, per column k, the lfill_k largest
// entries by magnitude (lfill_k = the number of entries of A(:, k)), all
// entries equal in magnitude to the smallest kept one, and the diagonal: when
// the diagonal is not among the kept entries it takes the place of the
// smallest of them (with its value, 0 when A has no diagonal entry there).
// The stored values are magnitudes, so the products have no cancellation.
//
// One CTA per column for both steps.  Products: the products S(i, l) S(l, k)
// go to shared memory at fixed offsets, are bitonic-sorted by row and summed
// per row (a fixed order).  Sparsify: the column's entries are sorted by
// magnitude, larger first and equal magnitudes in row order (the order of
// a stable sort of the row-ordered column), marked, and written back in row
// order.  Each step runs a counting pass and, after a scan, a writing pass.
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

constexpr int kPwThreads = 256;
constexpr int kPwMax = 8192;  // products (or entries) of one column in shared memory

// ascending bitonic sort of (key, val) by key
__device__ void pw_sort_by_key(int* key, double* val, int L)
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

// sort of positions pos[] by (val[pos] descending, pos ascending)
__device__ void pw_sort_by_magnitude(int* pos, const double* val, int L, int len)
{
    auto before = [&](int a, int b) {  // a strictly before b; padding (>= len) last
        if (a >= len || b >= len)
            return a < b;
        return val[a] > val[b] || (val[a] == val[b] && a < b);
    };
    for (int k = 2; k <= L; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < L; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const int a = pos[i], b = pos[ixj];
                    const bool up = (i & k) == 0;
                    if (before(b, a) == up) {
                        pos[i] = b;
                        pos[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// S S, a CTA per column: pass 0 counts the rows of each column, pass 1
// writes rows and summed values at out_ptr[k]
__global__ void __launch_bounds__(kPwThreads)
    pw_product_kernel(const int64_t* __restrict__ sp, const int32_t* __restrict__ si,
                      const double* __restrict__ sv, int n, int pass, int32_t* __restrict__ cnt,
                      const int64_t* __restrict__ out_ptr, int32_t* __restrict__ out_idx,
                      double* __restrict__ out_val, int32_t* __restrict__ err)
{
    extern __shared__ __align__(16) char smem[];
    double* val = reinterpret_cast<double*>(smem);
    int* key = reinterpret_cast<int*>(val + kPwMax);
    __shared__ int s_pos[kPwThreads / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        int64_t total = 0;
        for (int64_t p = sp[k]; p < sp[k + 1]; p++)
            total += sp[si[p] + 1] - sp[si[p]];
        if (total > kPwMax) {
            if (threadIdx.x == 0)
                atomicExch(err, k + 1);
            continue;  // uniform across the block
        }
        for (int64_t p = sp[k] + warp; p < sp[k + 1]; p += kPwThreads / 32) {
            const int l = si[p];
            const double alk = sv[p];
            int base = 0;
            for (int64_t q = sp[k]; q < p; q++)
                base += static_cast<int>(sp[si[q] + 1] - sp[si[q]]);
            for (int64_t q = sp[l] + lane; q < sp[l + 1]; q += 32) {
                key[base + (q - sp[l])] = si[q];
                val[base + (q - sp[l])] = sv[q] * alk;
            }
        }
        __syncthreads();
        const int T = static_cast<int>(total);
        int L = 1;
        while (L < T)
            L <<= 1;
        for (int i = T + threadIdx.x; i < L; i += kPwThreads) {
            key[i] = 0x7fffffff;
            val[i] = 0.0;
        }
        __syncthreads();
        pw_sort_by_key(key, val, L);
        // one output per run of equal rows, in row order
        const int chunk = (T + kPwThreads - 1) / kPwThreads;
        const int lo = min(T, static_cast<int>(threadIdx.x) * chunk), hi = min(T, lo + chunk);
        int c = 0;
        for (int i = lo; i < hi; i++)
            c += (i == 0 || key[i - 1] != key[i]) ? 1 : 0;
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
            for (int w = 0; w < kPwThreads / 32; w++) {
                const int t = s_pos[w];
                s_pos[w] = run;
                run += t;
            }
            s_pos[kPwThreads / 32] = run;
        }
        __syncthreads();
        if (pass == 0) {
            if (threadIdx.x == 0)
                cnt[k] = s_pos[kPwThreads / 32];
        }
        else {
            int64_t o = out_ptr[k] + s_pos[warp] + v - c;
            for (int i = lo; i < hi; i++) {
                if (!(i == 0 || key[i - 1] != key[i]))
                    continue;
                double s = 0.0;
                for (int q = i; q < T && key[q] == key[i]; q++)
                    s += val[q];
                out_idx[o] = key[i];
                out_val[o] = s;
                o++;
            }
        }
        __syncthreads();
    }
}

// Sparsify, a CTA per column (see the file comment): pass 0 counts, pass 1
// writes rows and values at out_ptr[k]
__global__ void __launch_bounds__(kPwThreads)
    pw_sparsify_kernel(const int64_t* __restrict__ sp, const int32_t* __restrict__ si,
                       const double* __restrict__ sv, const int32_t* __restrict__ lfill, int n,
                       int pass, int32_t* __restrict__ cnt, const int64_t* __restrict__ out_ptr,
                       int32_t* __restrict__ out_idx, double* __restrict__ out_val,
                       int32_t* __restrict__ err)
{
    extern __shared__ __align__(16) char smem[];
    double* val = reinterpret_cast<double*>(smem);
    int* pos = reinterpret_cast<int*>(val + kPwMax);
    int* keep = pos + kPwMax;
    __shared__ int s_diag_in, s_diag_pos;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int64_t a = sp[k];
        const int len = static_cast<int>(sp[k + 1] - a);
        if (len > kPwMax) {
            if (threadIdx.x == 0)
                atomicExch(err, k + 1);
            continue;
        }
        int L = 1;
        while (L < len)
            L <<= 1;
        for (int i = threadIdx.x; i < L; i += kPwThreads) {
            pos[i] = i;
            if (i < len)
                val[i] = fabs(sv[a + i]);
            keep[i] = 0;
        }
        if (threadIdx.x == 0) {
            s_diag_in = 0;
            s_diag_pos = -1;
        }
        __syncthreads();
        pw_sort_by_magnitude(pos, val, L, len);
        // the lfill largest (at least one, at most the column), the diagonal
        const int nk = len == 0 ? 0 : min(len, max(lfill[k], 1));
        for (int r = threadIdx.x; r < len; r += kPwThreads) {
            if (si[a + r] == k)
                s_diag_pos = r;
        }
        for (int t = threadIdx.x; t < nk; t += kPwThreads) {
            keep[pos[t]] = 1;
            if (si[a + pos[t]] == k)
                s_diag_in = 1;
        }
        __syncthreads();
        if (threadIdx.x == 0 && !s_diag_in && nk > 0) {
            // the diagonal takes the place of the smallest kept entry
            keep[pos[nk - 1]] = 0;
            if (s_diag_pos >= 0)
                keep[s_diag_pos] = 1;
        }
        __syncthreads();
        // entries equal in magnitude to the (originally) smallest kept one
        if (nk > 0) {
            const double vcut = val[pos[nk - 1]];
            for (int t = nk + threadIdx.x; t < len; t += kPwThreads) {
                bool tie = true;  // sorted positions nk .. t all tie
                for (int u = nk; u <= t && tie; u++)
                    tie = val[pos[u]] == vcut;
                if (tie)
                    keep[pos[t]] = 1;
            }
        }
        __syncthreads();
        // the diagonal missing from the column is inserted with the value 0
        const bool ins = (nk > 0 || len == 0) && !s_diag_in && s_diag_pos < 0;
        if (pass == 0) {
            if (threadIdx.x == 0) {
                int c = ins ? 1 : 0;
                for (int r = 0; r < len; r++)
                    c += keep[r];
                cnt[k] = c;
            }
        }
        else if (threadIdx.x == 0) {
            int64_t o = out_ptr[k];
            bool done_ins = !ins;
            for (int r = 0; r < len; r++) {
                if (!done_ins && si[a + r] > k) {
                    out_idx[o] = k;
                    out_val[o] = 0.0;
                    o++;
                    done_ins = true;
                }
                if (keep[r]) {
                    out_idx[o] = si[a + r];
                    out_val[o] = val[r];
                    o++;
                }
            }
            if (!done_ins) {
                out_idx[o] = k;
                out_val[o] = 0.0;
            }
        }
        __syncthreads();
    }
}

struct DevCsc {
    int64_t* ptr = nullptr;
    int32_t* idx = nullptr;
    double* val = nullptr;
    int64_t nnz = 0;
    void release()
    {
        cudaFree(ptr);
        cudaFree(idx);
        cudaFree(val);
        ptr = nullptr;
        idx = nullptr;
        val = nullptr;
    }
};

}  // namespace
}  // namespace mspai

extern "C" int mspai_pattern_powers(const mspai_csc* A, int32_t nb_pw, int32_t device,
                                    mspai_matrix* P_out, char* msg, int32_t msg_len)
{
    using mspai::DevCsc;
    auto fail = [&](int rc, const char* what) {
        if (msg && msg_len > 0)
            std::snprintf(msg, static_cast<size_t>(msg_len), "%s", what);
        return rc;
    };
    if (!P_out)
        return fail(MSPAI_ERR_PARAM, "P_out is required");
    std::memset(P_out, 0, sizeof(*P_out));
    if (!A || A->mem != MSPAI_MEM_HOST || !A->colptr || nb_pw < 0 || nb_pw > 4 ||
        (A->nnz > 0 && (!A->values || !A->rowidx)))
        return fail(MSPAI_ERR_PARAM, "host A with values and 0 <= nb_pw <= 4 are required");
    const int n = A->ncols;
    if (n < 0 || A->nrows != n || A->nnz < 0)
        return fail(MSPAI_ERR_INPUT, "A must be square (pass A without probing rows)");
    if (A->colptr[0] != 0 || A->colptr[n] != A->nnz)
        return fail(MSPAI_ERR_INPUT, "A: column pointers do not match nnz");
    for (int k = 0; k < n; k++) {
        const int64_t a = A->colptr[k], b = A->colptr[k + 1];
        if (b < a || a < 0 || b > A->nnz) {
            char buf[128];
            std::snprintf(buf, sizeof(buf), "A: column pointers decrease at column %d", k);
            return fail(MSPAI_ERR_INPUT, buf);
        }
        int prev = -1;
        for (int64_t q = a; q < b; q++) {
            const int r = A->rowidx[q];
            if (r < 0 || r >= n || r <= prev) {
                char buf[128];
                std::snprintf(buf, sizeof(buf),
                              "A: row indices out of range or not sorted/unique in column %d", k);
                return fail(MSPAI_ERR_INPUT, buf);
            }
            prev = r;
        }
    }
    if (cudaSetDevice(device) != cudaSuccess)
        return fail(MSPAI_ERR_NO_DEVICE, "no usable CUDA device");
    int rc = MSPAI_OK;
    cudaStream_t st = nullptr;
    DevCsc S, T;
    int32_t *dlf = nullptr, *dcnt = nullptr, *derr = nullptr;
    std::vector<int32_t> lf(static_cast<size_t>(std::max(n, 1))), cnt(lf.size());
    std::vector<int64_t> ptr(static_cast<size_t>(n) + 1, 0);
    const size_t smem = mspai::kPwMax * (sizeof(double) + 2 * sizeof(int));
    const int grid = std::max(1, std::min(n, mspai::num_sms() * 2));
    int err = 0;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == MSPAI_OK)
            rc = e == cudaErrorMemoryAllocation ? MSPAI_ERR_ALLOC : MSPAI_ERR_CUDA;
        return rc == MSPAI_OK;
    };
    // one step: count, scan on the host, allocate T, write; T becomes S
    auto step = [&](bool product) -> bool {
        if (!ok(cudaMemsetAsync(derr, 0, sizeof(int32_t), st)))
            return false;
        if (product)
            mspai::pw_product_kernel<<<grid, mspai::kPwThreads, smem, st>>>(
                S.ptr, S.idx, S.val, n, 0, dcnt, nullptr, nullptr, nullptr, derr);
        else
            mspai::pw_sparsify_kernel<<<grid, mspai::kPwThreads, smem, st>>>(
                S.ptr, S.idx, S.val, dlf, n, 0, dcnt, nullptr, nullptr, nullptr, derr);
        if (!ok(cudaGetLastError()) ||
            !ok(cudaMemcpyAsync(cnt.data(), dcnt, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                                st)) ||
            !ok(cudaMemcpyAsync(&err, derr, sizeof(int32_t), cudaMemcpyDeviceToHost, st)) ||
            !ok(cudaStreamSynchronize(st)))
            return false;
        if (err) {
            rc = MSPAI_ERR_CAPACITY;
            if (msg && msg_len > 0)
                std::snprintf(msg, static_cast<size_t>(msg_len),
                              "column %d has more than %d products or entries", err - 1,
                              mspai::kPwMax);
            return false;
        }
        for (int k = 0; k < n; k++)
            ptr[k + 1] = ptr[k] + cnt[k];
        T.nnz = ptr[n];
        if (!ok(cudaMalloc(&T.ptr, sizeof(int64_t) * (n + 1))) ||
            !ok(cudaMalloc(&T.idx, sizeof(int32_t) * std::max<int64_t>(T.nnz, 1))) ||
            !ok(cudaMalloc(&T.val, sizeof(double) * std::max<int64_t>(T.nnz, 1))) ||
            !ok(cudaMemcpyAsync(T.ptr, ptr.data(), sizeof(int64_t) * (n + 1),
                                cudaMemcpyHostToDevice, st)))
            return false;
        if (product)
            mspai::pw_product_kernel<<<grid, mspai::kPwThreads, smem, st>>>(
                S.ptr, S.idx, S.val, n, 1, dcnt, T.ptr, T.idx, T.val, derr);
        else
            mspai::pw_sparsify_kernel<<<grid, mspai::kPwThreads, smem, st>>>(
                S.ptr, S.idx, S.val, dlf, n, 1, dcnt, T.ptr, T.idx, T.val, derr);
        if (!ok(cudaGetLastError()) || !ok(cudaStreamSynchronize(st)))
            return false;
        S.release();
        S = T;
        T = DevCsc{};
        return true;
    };
    for (int k = 0; k < n; k++)
        lf[k] = static_cast<int32_t>(A->colptr[k + 1] - A->colptr[k]);
    S.nnz = A->nnz;
    if (!ok(cudaStreamCreate(&st)) || !ok(cudaMalloc(&S.ptr, sizeof(int64_t) * (n + 1))) ||
        !ok(cudaMalloc(&S.idx, sizeof(int32_t) * std::max<int64_t>(A->nnz, 1))) ||
        !ok(cudaMalloc(&S.val, sizeof(double) * std::max<int64_t>(A->nnz, 1))) ||
        !ok(cudaMalloc(&dlf, sizeof(int32_t) * std::max(n, 1))) ||
        !ok(cudaMalloc(&dcnt, sizeof(int32_t) * std::max(n, 1))) ||
        !ok(cudaMalloc(&derr, sizeof(int32_t))))
        goto done;
    if (!ok(cudaMemcpyAsync(S.ptr, A->colptr, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice,
                            st)) ||
        !ok(cudaMemcpyAsync(S.idx, A->rowidx, sizeof(int32_t) * A->nnz, cudaMemcpyHostToDevice,
                            st)) ||
        !ok(cudaMemcpyAsync(S.val, A->values, sizeof(double) * A->nnz, cudaMemcpyHostToDevice,
                            st)) ||
        !ok(cudaMemcpyAsync(dlf, lf.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st)) ||
        !ok(cudaFuncSetAttribute(mspai::pw_product_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem))) ||
        !ok(cudaFuncSetAttribute(mspai::pw_sparsify_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem))))
        goto done;
    if (!step(false))  // Sparsify(|A|)
        goto done;
    for (int k = 0; k < nb_pw; k++) {
        if (k >= 1 && !step(false))
            goto done;
        if (!step(true))
            goto done;
    }
    if (!step(false))
        goto done;
    P_out->nrows = n;
    P_out->ncols = n;
    P_out->nnz = S.nnz;
    P_out->colptr = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * (n + 1)));
    P_out->rowidx = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max<int64_t>(S.nnz, 1)));
    P_out->values = static_cast<double*>(std::malloc(sizeof(double) * std::max<int64_t>(S.nnz, 1)));
    if (!P_out->colptr || !P_out->rowidx || !P_out->values) {
        rc = MSPAI_ERR_ALLOC;
        goto done;
    }
    if (!ok(cudaMemcpyAsync(P_out->colptr, S.ptr, sizeof(int64_t) * (n + 1),
                            cudaMemcpyDeviceToHost, st)) ||
        !ok(cudaMemcpyAsync(P_out->rowidx, S.idx, sizeof(int32_t) * S.nnz,
                            cudaMemcpyDeviceToHost, st)) ||
        !ok(cudaMemcpyAsync(P_out->values, S.val, sizeof(double) * S.nnz,
                            cudaMemcpyDeviceToHost, st)) ||
        !ok(cudaStreamSynchronize(st)))
        goto done;
done:
    if (rc != MSPAI_OK) {
        if (msg && msg_len > 0 && rc != MSPAI_ERR_CAPACITY && rc != MSPAI_ERR_PARAM)
            std::snprintf(msg, static_cast<size_t>(msg_len), "CUDA error in the pattern kernels");
        mspai_matrix_free(P_out);
    }
    S.release();
    T.release();
    cudaFree(dlf);
    cudaFree(dcnt);
    cudaFree(derr);
    if (st)
        cudaStreamDestroy(st);
    return rc;
}
