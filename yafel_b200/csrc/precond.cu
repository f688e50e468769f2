// precond.cu -- Jacobi and ILU(0) preconditioners.
//
// Jacobi replaces JacobiPreconditioner (solver/iterative/JacobiPreconditioner.hpp:11-54):
// z_i = r_i / a_ii with the scalar diagonal; a zero diagonal gives inf, as the
// reference computes 1/0 (its warning text says otherwise).  Inside PCG it is
// fused into the vector kernels (krylov.cu) and never launched on its own.
//
// ILU(0) replaces ILUPreconditioner (ILUPreconditioner.hpp:96-329): incomplete
// LU without pivoting on the scalar pattern of A (a BCSR matrix is expanded to
// its full B*B entries per block), zero pivots skipped.  The reference walks
// pivots (KIJ, O(N^2) row scans); here rows are factored in IKJ order, which
// applies to every entry the same updates in the same order.  Rows are grouped
// into dependency levels on the host (level = 1 + max level of the rows it
// depends on); the factorization and each triangular solve are one persistent
// launch walking the levels with a grid-wide barrier between them, a warp per
// row.
#include "internal.h"
#include "device_common.cuh"

#include <algorithm>
#include <cmath>

namespace yg {

int stream_grid(yg_context ctx, int64_t n);

__global__ void k_jacobi_build(int64_t nbrows, int B, const int32_t *__restrict__ diag, const double *__restrict__ val,
                               double *__restrict__ dinv, int *__restrict__ zeros) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nbrows * B; r += (int64_t)gridDim.x * blockDim.x) {
        int64_t I = r / B, i = r % B;
        int32_t d = diag[I];
        double a = d >= 0 ? val[(int64_t)d * B * B + i * B + i] : 0.0;
        dinv[r] = 1.0 / a;
        if (a == 0) atomicAdd(zeros, 1);
    }
}

__global__ void k_jacobi_apply(int64_t n, const double *__restrict__ dinv, const double *__restrict__ r,
                               double *__restrict__ z) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        z[i] = r[i] * dinv[i];
}

// Scalar CSR expansion of a BCSR pattern: row I*B+i lists columns J*B+j.
__global__ void k_expand_rowptr(int64_t nbrows, int B, const int32_t *__restrict__ brp, int32_t *__restrict__ rp) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= nbrows * B; r += (int64_t)gridDim.x * blockDim.x) {
        if (r == nbrows * B) { rp[r] = brp[nbrows] * B * B; continue; }
        int64_t I = r / B, i = r % B;
        int32_t len = brp[I + 1] - brp[I];
        rp[r] = brp[I] * B * B + (int32_t)i * len * B;
    }
}
__global__ void k_expand_vals(int64_t nbrows, int B, const int32_t *__restrict__ brp, const int32_t *__restrict__ bcol,
                              const double *__restrict__ bval, const int32_t *__restrict__ rp, int32_t *__restrict__ col,
                              double *__restrict__ val) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nbrows * B; r += (int64_t)gridDim.x * blockDim.x) {
        int64_t I = r / B, i = r % B;
        int32_t pos = rp[r];
        for (int32_t k = brp[I]; k < brp[I + 1]; ++k)
            for (int j = 0; j < B; ++j) {
                col[pos] = bcol[k] * B + j;
                val[pos] = bval[(int64_t)k * B * B + i * B + j];
                ++pos;
            }
    }
}

__global__ void k_scalar_diag(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                              int32_t *__restrict__ diag) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int lo = rp[r], hi = rp[r + 1] - 1, pos = -1;
        while (lo <= hi) {
            int mid = (lo + hi) >> 1;
            if (col[mid] == r) { pos = mid; break; }
            if (col[mid] < r) lo = mid + 1; else hi = mid - 1;
        }
        diag[r] = pos;
    }
}

__device__ __forceinline__ int find_col(const int32_t *__restrict__ col, int lo, int hi, int c) {
    --hi;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int v = col[mid];
        if (v == c) return mid;
        if (v < c) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// Persistent level sweeps.  One cooperative launch per factorization and per
// triangular solve: the grid walks the levels in order with a grid-wide barrier
// between them, instead of one launch per level (the levels of a 3-D mesh in
// natural order number ~78 per cell layer, so launch latency dominated).  Values
// written in earlier levels by other blocks are read through L2 (__ldcg).  The
// barrier is bounded: after kSpinLimit polls a block records YG_TIMEOUT in the
// context's error word and returns, so a sweep can only end.
struct GridBarrier {
    unsigned count, gen;
};

__device__ bool grid_barrier(GridBarrier *b) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned g = atomicAdd(&b->gen, 0u);
        __threadfence();
        if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            long long spins = 0;
            while (atomicAdd(&b->gen, 0u) == g)
                if (++spins > kSpinLimit) { ok = 0; break; }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// Factorization (IKJ): a warp per row of the level, pivots in ascending order,
// the lanes share the updates of one pivot row.
__global__ void __launch_bounds__(kThreads)
k_ilu_factor_sweep(const int32_t *__restrict__ lev_ptr, int nlev, const int32_t *__restrict__ rows,
                   const int32_t *__restrict__ rp, const int32_t *__restrict__ col, const int32_t *__restrict__ diag,
                   double *__restrict__ lu, int *__restrict__ zero_pivots, GridBarrier *bar, int32_t *err) {
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int l = 0; l < nlev; ++l) {
        for (int t = lev_ptr[l] + w; t < lev_ptr[l + 1]; t += nw) {
            const int i = rows[t];
            const int rs = rp[i], re = rp[i + 1];
            for (int kk = rs; kk < re; ++kk) {
                const int k = col[kk];
                if (k >= i) break;
                const int dk = diag[k];
                const double piv = dk >= 0 ? __ldcg(lu + dk) : 0.0;
                if (piv == 0) {
                    if (lane == 0) atomicAdd(zero_pivots, 1);
                    continue;
                }
                __syncwarp();
                const double m = lu[kk] / piv;
                const int ke = rp[k + 1];
                for (int q = dk + 1 + lane; q < ke; q += 32) {
                    const int pos = find_col(col, kk + 1, re, col[q]);
                    if (pos >= 0) lu[pos] -= m * __ldcg(lu + q);
                }
                __syncwarp();
                if (lane == 0) lu[kk] = m;
                __syncwarp();
            }
        }
        if (l + 1 < nlev && !grid_barrier(bar)) {
            if (threadIdx.x == 0) atomicExch(err, (int32_t)YG_TIMEOUT);
            return;
        }
    }
}

// Forward substitution with unit L (f_subst, ILUPreconditioner.hpp:201-221).
__global__ void __launch_bounds__(kThreads)
k_ilu_lower_sweep(const int32_t *__restrict__ lev_ptr, int nlev, const int32_t *__restrict__ rows,
                  const int32_t *__restrict__ rp, const int32_t *__restrict__ col, const int32_t *__restrict__ diag,
                  const double *__restrict__ lu, double *__restrict__ z, GridBarrier *bar, int32_t *err) {
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int l = 0; l < nlev; ++l) {
        for (int t = lev_ptr[l] + w; t < lev_ptr[l + 1]; t += nw) {
            const int i = rows[t];
            const int rs = rp[i];
            const int re = diag[i] >= 0 ? diag[i] : rp[i + 1];
            double s = 0;
            for (int k = rs + lane; k < re; k += 32) {
                const int c = col[k];
                if (c < i) s += lu[k] * __ldcg(z + c);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) z[i] = __ldcg(z + i) - s;
        }
        if (l + 1 < nlev && !grid_barrier(bar)) {
            if (threadIdx.x == 0) atomicExch(err, (int32_t)YG_TIMEOUT);
            return;
        }
    }
}

// Backward substitution (b_subst, ILUPreconditioner.hpp:226-253); a row
// without a diagonal uses its first entry, as the reference does.
__global__ void __launch_bounds__(kThreads)
k_ilu_upper_sweep(const int32_t *__restrict__ lev_ptr, int nlev, const int32_t *__restrict__ rows,
                  const int32_t *__restrict__ rp, const int32_t *__restrict__ col, const int32_t *__restrict__ diag,
                  const double *__restrict__ lu, double *__restrict__ z, GridBarrier *bar, int32_t *err) {
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int l = 0; l < nlev; ++l) {
        for (int t = lev_ptr[l] + w; t < lev_ptr[l + 1]; t += nw) {
            const int i = rows[t];
            const int id = diag[i] >= 0 ? diag[i] : rp[i];
            const int re = rp[i + 1];
            double s = 0;
            for (int k = id + 1 + lane; k < re; k += 32) s += lu[k] * __ldcg(z + col[k]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) z[i] = (__ldcg(z + i) - s) / lu[id];
        }
        if (l + 1 < nlev && !grid_barrier(bar)) {
            if (threadIdx.x == 0) atomicExch(err, (int32_t)YG_TIMEOUT);
            return;
        }
    }
}

// One block per SM: every block of the cooperative launch is resident at once.
template <typename K, typename... Args>
static yg_status launch_sweep(yg_context ctx, K kern, GridBarrier *bar, Args... args) {
    YG_CUDA(cudaMemsetAsync(bar, 0, sizeof(GridBarrier), ctx->stream));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctx->num_sms);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    YG_CUDA(cudaLaunchKernelEx(&cfg, kern, args..., bar, ctx->d_err));
    YG_LAUNCHED(ctx);
    return YG_OK;
}

static yg_status build_ilu(yg_precond M) {
    yg_matrix A = M->A;
    yg_context ctx = A->ctx;
    const int B = A->block;
    const int64_t n = A->rows();
    const int64_t nnz = A->nnzb * B * B;
    if (nnz >= INT32_MAX) return fail(YG_UNSUPPORTED, "ILU(0): too many entries for 32-bit indices");
    M->n = n;
    M->nnz = nnz;
    YG_TRY(dev_alloc_t(ctx, &M->d_csr_rowptr, n + 1));
    YG_TRY(dev_alloc_t(ctx, &M->d_csr_col, nnz));
    YG_TRY(dev_alloc_t(ctx, &M->d_csr_diag, n));
    YG_TRY(dev_alloc_t(ctx, &M->d_lu, nnz));
    YG_TRY(dev_alloc_t(ctx, &M->d_tmp, 1));
    cudaStream_t st = ctx->stream;
    k_expand_rowptr<<<stream_grid(ctx, n + 1), kThreads, 0, st>>>(A->nbrows, B, A->d_rowptr, M->d_csr_rowptr);
    YG_LAUNCHED(ctx);
    k_expand_vals<<<stream_grid(ctx, n), kThreads, 0, st>>>(A->nbrows, B, A->d_rowptr, A->d_col, A->d_val,
                                                            M->d_csr_rowptr, M->d_csr_col, M->d_lu);
    YG_LAUNCHED(ctx);
    k_scalar_diag<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, M->d_csr_rowptr, M->d_csr_col, M->d_csr_diag);
    YG_LAUNCHED(ctx);
    YG_CUDA(cudaGetLastError());
    // dependency levels on the host
    std::vector<int32_t> rp(n + 1), col(nnz);
    YG_CUDA(cudaMemcpyAsync(rp.data(), M->d_csr_rowptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
    YG_CUDA(cudaMemcpyAsync(col.data(), M->d_csr_col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
    YG_CUDA(cudaStreamSynchronize(st));
    std::vector<int32_t> lev(n, 0), ulev(n, 0);
    int32_t maxl = 0, maxu = 0;
    for (int64_t i = 0; i < n; ++i) {
        int32_t l = 0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            int32_t c = col[k];
            if (c >= i) break;
            l = std::max(l, lev[c] + 1);
        }
        lev[i] = l;
        maxl = std::max(maxl, l);
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        int32_t l = 0;
        for (int32_t k = rp[i + 1] - 1; k >= rp[i]; --k) {
            int32_t c = col[k];
            if (c <= i) break;
            l = std::max(l, ulev[c] + 1);
        }
        ulev[i] = l;
        maxu = std::max(maxu, l);
    }
    auto group = [&](const std::vector<int32_t> &L, int32_t nl, std::vector<int32_t> &ptr, std::vector<int32_t> &rows) {
        ptr.assign(nl + 2, 0);
        for (int64_t i = 0; i < n; ++i) ptr[L[i] + 1]++;
        for (int32_t l = 0; l <= nl; ++l) ptr[l + 1] += ptr[l];
        rows.resize(n);
        std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
        for (int64_t i = 0; i < n; ++i) rows[fill[L[i]]++] = (int32_t)i;
    };
    std::vector<int32_t> lrows, urows;
    group(lev, maxl, M->lower_level_ptr, lrows);
    group(ulev, maxu, M->upper_level_ptr, urows);
    YG_TRY(dev_alloc_t(ctx, &M->d_lower_levels, n));
    YG_TRY(dev_alloc_t(ctx, &M->d_upper_levels, n));
    YG_CUDA(cudaMemcpyAsync(M->d_lower_levels, lrows.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    YG_CUDA(cudaMemcpyAsync(M->d_upper_levels, urows.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    // level pointers on the device for the persistent sweeps
    YG_TRY(dev_alloc_t(ctx, &M->d_lower_ptr, M->lower_level_ptr.size()));
    YG_TRY(dev_alloc_t(ctx, &M->d_upper_ptr, M->upper_level_ptr.size()));
    YG_TRY(dev_alloc_t(ctx, &M->d_bar, 4));
    YG_CUDA(cudaMemcpyAsync(M->d_lower_ptr, M->lower_level_ptr.data(), sizeof(int32_t) * M->lower_level_ptr.size(),
                            cudaMemcpyHostToDevice, st));
    YG_CUDA(cudaMemcpyAsync(M->d_upper_ptr, M->upper_level_ptr.data(), sizeof(int32_t) * M->upper_level_ptr.size(),
                            cudaMemcpyHostToDevice, st));
    // factor the levels in one persistent launch
    int *d_zero = reinterpret_cast<int *>(M->d_tmp);
    YG_CUDA(cudaMemsetAsync(d_zero, 0, sizeof(int), st));
    GridBarrier *bar = reinterpret_cast<GridBarrier *>(M->d_bar);
    YG_TRY(launch_sweep(ctx, k_ilu_factor_sweep, bar, (const int32_t *)M->d_lower_ptr,
                        (int)M->lower_level_ptr.size() - 1, (const int32_t *)M->d_lower_levels,
                        (const int32_t *)M->d_csr_rowptr, (const int32_t *)M->d_csr_col,
                        (const int32_t *)M->d_csr_diag, M->d_lu, d_zero));
    YG_CUDA(cudaGetLastError());
    int zeros = 0;
    YG_CUDA(cudaMemcpyAsync(&zeros, d_zero, sizeof(int), cudaMemcpyDeviceToHost, st));
    YG_CUDA(cudaStreamSynchronize(st));
    M->zero_pivots = zeros;
    return YG_OK;
}

yg_status precond_apply_dev(yg_precond M, const double *r, double *z) {
    yg_context ctx = M->A->ctx;
    cudaStream_t st = ctx->stream;
    const int64_t n = M->A->rows();
    if (M->kind == YG_PRECOND_IDENTITY) {
        if (z != r) YG_CUDA(cudaMemcpyAsync(z, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        return YG_OK;
    }
    if (M->kind == YG_PRECOND_JACOBI) {
        k_jacobi_apply<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, M->d_dinv, r, z);
        YG_LAUNCHED(ctx);
        return YG_OK;
    }
    if (z != r) YG_CUDA(cudaMemcpyAsync(z, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    GridBarrier *bar = reinterpret_cast<GridBarrier *>(M->d_bar);
    YG_TRY(launch_sweep(ctx, k_ilu_lower_sweep, bar, (const int32_t *)M->d_lower_ptr, (int)M->lower_level_ptr.size() - 1,
                        (const int32_t *)M->d_lower_levels, (const int32_t *)M->d_csr_rowptr,
                        (const int32_t *)M->d_csr_col, (const int32_t *)M->d_csr_diag, (const double *)M->d_lu, z));
    YG_TRY(launch_sweep(ctx, k_ilu_upper_sweep, bar, (const int32_t *)M->d_upper_ptr, (int)M->upper_level_ptr.size() - 1,
                        (const int32_t *)M->d_upper_levels, (const int32_t *)M->d_csr_rowptr,
                        (const int32_t *)M->d_csr_col, (const int32_t *)M->d_csr_diag, (const double *)M->d_lu, z));
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

bool precond_fusable(yg_precond M) { return !M || M->kind == YG_PRECOND_IDENTITY || M->kind == YG_PRECOND_JACOBI; }
const double *precond_dinv(yg_precond M) { return (M && M->kind == YG_PRECOND_JACOBI) ? M->d_dinv : nullptr; }

}  // namespace yg

using namespace yg;

extern "C" yg_status yg_precond_create(yg_matrix A, int32_t kind, yg_precond *out) {
    if (!A || !out) return fail(YG_BAD_ARG, "yg_precond_create: NULL argument");
    if (A->rows() != A->cols()) return fail(YG_BAD_ARG, "preconditioner needs a square matrix");
    *out = nullptr;
    auto *M = new yg_precond_t();
    M->A = A;
    M->ctx = A->ctx;
    M->kind = kind;
    yg_context ctx = A->ctx;
    yg_status s = YG_OK;
    if (kind == YG_PRECOND_JACOBI) {
        const int64_t n = A->rows();
        if ((s = dev_alloc_t(ctx, &M->d_dinv, n)) == YG_OK && (s = dev_alloc_t(ctx, &M->d_tmp, 1)) == YG_OK) {
            int *d_zero = reinterpret_cast<int *>(M->d_tmp);
            cudaMemsetAsync(d_zero, 0, sizeof(int), ctx->stream);
            k_jacobi_build<<<stream_grid(ctx, n), kThreads, 0, ctx->stream>>>(A->nbrows, A->block, A->d_diag, A->d_val,
                                                                             M->d_dinv, d_zero);
            YG_LAUNCHED(ctx);
            int zeros = 0;
            cudaMemcpyAsync(&zeros, d_zero, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
            cudaError_t e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) s = fail(YG_CUDA_ERROR, "Jacobi build: %s", cudaGetErrorString(e));
            M->zero_pivots = zeros;
        }
    } else if (kind == YG_PRECOND_ILU0) {
        s = build_ilu(M);
    } else if (kind != YG_PRECOND_IDENTITY) {
        s = fail(YG_BAD_ARG, "unknown preconditioner kind %d", kind);
    }
    if (s != YG_OK) { yg_precond_destroy(M); return s; }
    *out = M;
    return YG_OK;
}

extern "C" yg_status yg_precond_apply(yg_precond M, yg_vector z) {
    if (!M || !z || z->n != M->A->rows()) return fail(YG_BAD_ARG, "yg_precond_apply: size mismatch");
    return precond_apply_dev(M, z->d, z->d);
}

extern "C" yg_status yg_precond_destroy(yg_precond M) {
    if (!M) return YG_OK;
    yg_context ctx = M->ctx;
    for (void *p : {(void *)M->d_dinv, (void *)M->d_lu, (void *)M->d_lower_levels, (void *)M->d_upper_levels,
                    (void *)M->d_csr_rowptr, (void *)M->d_csr_col, (void *)M->d_csr_diag, (void *)M->d_tmp,
                    (void *)M->d_lower_ptr, (void *)M->d_upper_ptr, (void *)M->d_bar})
        dev_free(ctx, p);
    delete M;
    return YG_OK;
}

extern "C" int64_t yg_precond_zero_pivots(yg_precond M) { return M ? M->zero_pivots : -1; }

extern "C" yg_status yg_precond_levels(yg_precond M, int64_t *lower, int64_t *upper) {
    if (!M || !lower || !upper) return fail(YG_BAD_ARG, "yg_precond_levels: NULL argument");
    *lower = M->lower_level_ptr.empty() ? 0 : (int64_t)M->lower_level_ptr.size() - 1;
    *upper = M->upper_level_ptr.empty() ? 0 : (int64_t)M->upper_level_ptr.size() - 1;
    return YG_OK;
}
