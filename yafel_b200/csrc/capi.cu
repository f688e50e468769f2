// capi.cu -- context, error reporting, device vectors and matrix import/export
// of the C ABI declared in include/yafel_gpu.h.
#include "internal.h"
#include "device_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <numeric>

namespace yg {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

yg_status fail(yg_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

// Released blocks are kept, up to kCacheTotal bytes per context, and handed out
// again for an allocation of the same size: solver work vectors, iterates,
// Dirichlet scratch and re-assembled matrices are allocated and freed over and
// over, and cudaMalloc / cudaFree would otherwise map and unmap pages and
// synchronise the device each time.  A cudaMalloc that fails releases the
// cached blocks and tries again.
constexpr size_t kCacheBlock = 16ull << 30, kCacheTotal = 32ull << 30;

void flush_alloc_cache(yg_context ctx) {
    for (auto &kv : ctx->cache) {
        cudaEventSynchronize(kv.second.ev);
        cudaEventDestroy(kv.second.ev);
        cudaFree(kv.second.p);
    }
    ctx->cache.clear();
    ctx->cached_bytes = 0;
}

yg_status dev_alloc(yg_context ctx, void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (ctx->budget && ctx->in_use + bytes > ctx->budget)
        return fail(YG_OVER_BUDGET, "allocation of %zu bytes exceeds the HBM budget (%llu of %llu in use)",
                    bytes, (unsigned long long)ctx->in_use, (unsigned long long)ctx->budget);
    auto hit = ctx->cache.find(bytes);
    if (hit != ctx->cache.end()) {
        yg_context_t::CachedBlock b = hit->second;
        ctx->cache.erase(hit);
        ctx->cached_bytes -= bytes;
        cudaEventSynchronize(b.ev);
        cudaEventDestroy(b.ev);
        *p = b.p;
    } else {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess && !ctx->cache.empty()) {  // give the cached blocks back and retry
            cudaGetLastError();
            flush_alloc_cache(ctx);
            e = cudaMalloc(p, bytes);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            return fail(YG_OUT_OF_MEMORY, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        }
    }
    ctx->in_use += bytes;
    ctx->allocs[*p] = bytes;
    return YG_OK;
}

void dev_free(yg_context ctx, void *p) {
    if (!p) return;
    auto it = ctx->allocs.find(p);
    size_t bytes = 0;
    if (it != ctx->allocs.end()) {
        bytes = it->second;
        ctx->in_use -= bytes;
        ctx->allocs.erase(it);
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->stream, &cs);
    if (bytes && bytes <= kCacheBlock && ctx->cached_bytes + bytes <= kCacheTotal && cs == cudaStreamCaptureStatusNone) {
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
            cudaEventRecord(ev, ctx->stream);
            ctx->cache.insert({bytes, {p, ev}});
            ctx->cached_bytes += bytes;
            return;
        }
        cudaGetLastError();
    }
    cudaFree(p);
}

// ------------------------------------------------------------ small kernels

__global__ void k_fill(double *__restrict__ v, int64_t n, double val) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = val;
}

__global__ void k_axpy(double alpha, const double *__restrict__ x, double *__restrict__ y, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += alpha * x[i];
}

__global__ void __launch_bounds__(kThreads) k_dot_partials(const double *__restrict__ a, const double *__restrict__ b,
                                                           int64_t n, double *__restrict__ partials) {
    __shared__ double sm[kThreads / 32];
    double s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += a[i] * b[i];
    s = block_sum<kThreads>(s, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_sum_partials(const double *__restrict__ partials, int np,
                                                           double *__restrict__ out) {
    __shared__ double sm[kThreads / 32];
    double s = 0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
    s = block_sum<kThreads>(s, sm);
    if (threadIdx.x == 0) out[0] = s;
}

__global__ void k_find_diag(int64_t nbrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                            int32_t *__restrict__ diag) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nbrows; r += (int64_t)gridDim.x * blockDim.x) {
        int lo = rowptr[r], hi = rowptr[r + 1] - 1, pos = -1;
        while (lo <= hi) {
            int mid = (lo + hi) >> 1;
            int c = col[mid];
            if (c == r) { pos = mid; break; }
            if (c < r) lo = mid + 1; else hi = mid - 1;
        }
        diag[r] = pos;
    }
}

__global__ void k_to_fp32(const double *__restrict__ v, float *__restrict__ o, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        o[i] = (float)v[i];
}

// Row-sum correction of the FP32 values: corr[r][i][k] = sum over the blocks
// j of block row r of (A_rj[i][k] - fl32(A_rj[i][k])), in FP64.  A warp per
// block row; each lane sums its blocks (lane-strided), then a fixed butterfly,
// so the result does not change from run to run.  With it, A32 x + C x_r is
// exact on fields that are constant per component (A's block row sums are
// kept), which removes most of the FP32 rounding seen by the smooth error
// components that limit the mixed-precision solvers.
template <int B>
__global__ void k_fp32_correction(int64_t nbrows, const int32_t *__restrict__ rowptr, const double *__restrict__ v,
                                  double *__restrict__ corr) {
    constexpr int B2 = B * B;
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < nbrows; r += nw) {
        double s[B2];
#pragma unroll
        for (int e = 0; e < B2; ++e) s[e] = 0;
        const int rs = rowptr[r], re = rowptr[r + 1];
        for (int j = rs + lane; j < re; j += 32) {
#pragma unroll
            for (int e = 0; e < B2; ++e) {
                const double a = v[(int64_t)j * B2 + e];
                s[e] += a - (double)(float)a;
            }
        }
#pragma unroll
        for (int e = 0; e < B2; ++e) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s[e] += __shfl_xor_sync(0xffffffffu, s[e], o);
        }
        if (lane == 0)
#pragma unroll
            for (int e = 0; e < B2; ++e) corr[r * B2 + e] = s[e];
    }
}

// x rounded to FP32 in the node-padded gather layout of the FP32-value SpMV
// (xs floats per node of B values; the padding stays zero).
__global__ void k_to_x32(const double *__restrict__ x, float *__restrict__ x32, int64_t n, int B, int xs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x32[(i / B) * xs + i % B] = (float)x[i];
}

// A kernel whose bounded wait expired leaves YG_TIMEOUT in the context's error
// word; report it (once) and clear it.
yg_status check_device_error(yg_context ctx) {
    int32_t e = 0;
    YG_CUDA(cudaMemcpy(&e, ctx->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (e != 0) {
        cudaMemset(ctx->d_err, 0, sizeof(int32_t));
        return fail((yg_status)e, "a device wait expired (status %d); results of that launch are invalid", e);
    }
    return YG_OK;
}

int stream_grid(yg_context ctx, int64_t n) {
    int64_t g = (n + kThreads - 1) / kThreads;
    int64_t cap = (int64_t)ctx->num_sms * 8;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

yg_status vector_dot(yg_context ctx, const double *a, const double *b, int64_t n, double *out) {
    int g = stream_grid(ctx, n);
    if (g > kMaxReduceBlocks) g = kMaxReduceBlocks;
    k_dot_partials<<<g, kThreads, 0, ctx->stream>>>(a, b, n, ctx->d_partials);
    YG_LAUNCHED(ctx);
    k_sum_partials<<<1, kThreads, 0, ctx->stream>>>(ctx->d_partials, g, ctx->d_partials + kMaxReduceBlocks);
    YG_LAUNCHED(ctx);
    YG_CUDA(cudaGetLastError());
    YG_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_partials + kMaxReduceBlocks, sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = ctx->h_pinned[0];
    return YG_OK;
}

yg_status matrix_build_diag(yg_matrix A) {
    yg_context ctx = A->ctx;
    if (!A->d_diag) YG_TRY(dev_alloc_t(ctx, &A->d_diag, A->nbrows + 1));
    k_find_diag<<<stream_grid(ctx, A->nbrows), kThreads, 0, ctx->stream>>>(A->nbrows, A->d_rowptr, A->d_col, A->d_diag);
    YG_LAUNCHED(ctx);
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

// Upload a host block-CSR (int64 indices) into a new device matrix.
static yg_status upload_bcsr(yg_context ctx, int32_t block, int64_t nbrows, int64_t nbcols,
                             const std::vector<int64_t> &rp, const std::vector<int64_t> &col,
                             const double *vals, yg_matrix *out) {
    int64_t nnzb = rp[nbrows];
    if (nnzb >= INT32_MAX || nbrows >= INT32_MAX || nbcols >= INT32_MAX)
        return fail(YG_UNSUPPORTED, "matrix too large for 32-bit indices (nnzb=%lld)", (long long)nnzb);
    if ((int64_t)nnzb * block * block >= ((int64_t)1 << 40))
        return fail(YG_UNSUPPORTED, "matrix too large");
    auto *A = new yg_matrix_t();
    A->ctx = ctx;
    A->block = block;
    A->nbrows = nbrows;
    A->nbcols = nbcols;
    A->nnzb = nnzb;
    std::vector<int32_t> rp32(nbrows + 1), col32(nnzb);
    for (int64_t i = 0; i <= nbrows; ++i) rp32[i] = (int32_t)rp[i];
    for (int64_t i = 0; i < nnzb; ++i) col32[i] = (int32_t)col[i];
    yg_status s;
    if ((s = dev_alloc_t(ctx, &A->d_rowptr, nbrows + 1)) != YG_OK ||
        (s = dev_alloc_t(ctx, &A->d_col, nnzb)) != YG_OK ||
        (s = dev_alloc_t(ctx, &A->d_val, nnzb * block * block)) != YG_OK) {
        yg_matrix_destroy(A);
        return s;
    }
    cudaMemcpyAsync(A->d_rowptr, rp32.data(), sizeof(int32_t) * (nbrows + 1), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(A->d_col, col32.data(), sizeof(int32_t) * nnzb, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(A->d_val, vals, sizeof(double) * nnzb * block * block, cudaMemcpyHostToDevice, ctx->stream);
    if ((s = matrix_build_diag(A)) != YG_OK) { yg_matrix_destroy(A); return s; }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { yg_matrix_destroy(A); return fail(YG_CUDA_ERROR, "upload: %s", cudaGetErrorString(e)); }
    spmv_autotune(A);
    *out = A;
    return YG_OK;
}

}  // namespace yg

using namespace yg;

// ================================================================ context

extern "C" yg_status yg_context_create(int32_t device, uint64_t hbm_budget_bytes, yg_context *out) {
    if (!out) return fail(YG_BAD_ARG, "yg_context_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(YG_CUDA_ERROR, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return fail(YG_BAD_ARG, "device %d out of range (%d devices)", device, ndev);
    YG_CUDA(cudaSetDevice(device));
    auto *ctx = new yg_context_t();
    ctx->device = device;
    ctx->budget = hbm_budget_bytes;
    cudaDeviceProp prop;
    YG_CUDA(cudaGetDeviceProperties(&prop, device));
    ctx->num_sms = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    ctx->reduce_blocks = ctx->num_sms * 4;
    YG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    yg_status s;
    if ((s = dev_alloc_t(ctx, &ctx->d_partials, 8 * kMaxReduceBlocks)) != YG_OK ||
        (s = dev_alloc_t(ctx, &ctx->d_scalars, 4)) != YG_OK || (s = dev_alloc_t(ctx, &ctx->d_err, 4)) != YG_OK) {
        yg_context_destroy(ctx);
        return s;
    }
    cudaMemset(ctx->d_err, 0, sizeof(int32_t));
    e = cudaMallocHost(&ctx->h_pinned, 64 * sizeof(double));
    if (e != cudaSuccess) {
        yg_context_destroy(ctx);
        return fail(YG_OUT_OF_MEMORY, "cudaMallocHost: %s", cudaGetErrorString(e));
    }
    *out = ctx;
    return YG_OK;
}

extern "C" yg_status yg_context_destroy(yg_context ctx) {
    if (!ctx) return YG_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    flush_alloc_cache(ctx);
    for (auto &kv : ctx->allocs) cudaFree(kv.first);
    ctx->allocs.clear();
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return YG_OK;
}

extern "C" yg_status yg_context_synchronize(yg_context ctx) {
    if (!ctx) return fail(YG_BAD_ARG, "NULL context");
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_device_error(ctx);
}

extern "C" yg_status yg_context_memory(yg_context ctx, uint64_t *in_use, uint64_t *budget) {
    if (!ctx) return fail(YG_BAD_ARG, "NULL context");
    if (in_use) *in_use = ctx->in_use;
    if (budget) *budget = ctx->budget;
    return YG_OK;
}

extern "C" int64_t yg_context_launches(yg_context ctx) { return ctx ? ctx->launches : 0; }

extern "C" const char *yg_last_error(void) { return g_last_error.c_str(); }

extern "C" const char *yg_status_string(yg_status s) {
    switch (s) {
    case YG_OK: return "ok";
    case YG_NOT_CONVERGED: return "not converged";
    case YG_BREAKDOWN: return "breakdown";
    case YG_NAN: return "non-finite value";
    case YG_TIMEOUT: return "timeout";
    case YG_OUT_OF_MEMORY: return "out of memory";
    case YG_OVER_BUDGET: return "over HBM budget";
    case YG_BAD_ARG: return "bad argument";
    case YG_CUDA_ERROR: return "CUDA error";
    case YG_UNSUPPORTED: return "unsupported";
    case YG_ZERO_PIVOT: return "zero pivot";
    case YG_RUNNING: return "running";
    }
    return "unknown status";
}

// ================================================================ vectors

extern "C" yg_status yg_vector_create(yg_context ctx, int64_t n, yg_vector *out) {
    if (!ctx || !out || n < 0) return fail(YG_BAD_ARG, "yg_vector_create: bad argument");
    auto *v = new yg_vector_t();
    v->ctx = ctx;
    v->n = n;
    yg_status s = dev_alloc_t(ctx, &v->d, n > 0 ? n : 1);
    if (s != YG_OK) { delete v; return s; }
    cudaMemsetAsync(v->d, 0, sizeof(double) * (n > 0 ? n : 1), ctx->stream);
    *out = v;
    return YG_OK;
}

extern "C" yg_status yg_vector_destroy(yg_vector v) {
    if (!v) return YG_OK;
    dev_free(v->ctx, v->d);
    delete v;
    return YG_OK;
}

extern "C" int64_t yg_vector_size(yg_vector v) { return v ? v->n : -1; }

extern "C" yg_status yg_vector_upload(yg_vector v, const double *host, int64_t n) {
    if (!v || (!host && n) || n != v->n) return fail(YG_BAD_ARG, "yg_vector_upload: size %lld != %lld", (long long)n, v ? (long long)v->n : -1LL);
    YG_CUDA(cudaMemcpyAsync(v->d, host, sizeof(double) * n, cudaMemcpyHostToDevice, v->ctx->stream));
    YG_CUDA(cudaStreamSynchronize(v->ctx->stream));
    return YG_OK;
}

extern "C" yg_status yg_vector_download(yg_vector v, double *host, int64_t n) {
    if (!v || (!host && n) || n != v->n) return fail(YG_BAD_ARG, "yg_vector_download: size mismatch");
    YG_CUDA(cudaMemcpyAsync(host, v->d, sizeof(double) * n, cudaMemcpyDeviceToHost, v->ctx->stream));
    YG_CUDA(cudaStreamSynchronize(v->ctx->stream));
    return YG_OK;
}

extern "C" yg_status yg_vector_fill(yg_vector v, double value) {
    if (!v) return fail(YG_BAD_ARG, "NULL vector");
    k_fill<<<stream_grid(v->ctx, v->n), kThreads, 0, v->ctx->stream>>>(v->d, v->n, value);
    YG_LAUNCHED(v->ctx);
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

extern "C" yg_status yg_vector_copy(yg_vector dst, yg_vector src) {
    if (!dst || !src || dst->n != src->n) return fail(YG_BAD_ARG, "yg_vector_copy: size mismatch");
    YG_CUDA(cudaMemcpyAsync(dst->d, src->d, sizeof(double) * src->n, cudaMemcpyDeviceToDevice, src->ctx->stream));
    return YG_OK;
}

extern "C" yg_status yg_vector_dot(yg_vector a, yg_vector b, double *out) {
    if (!a || !b || !out || a->n != b->n) return fail(YG_BAD_ARG, "yg_vector_dot: size mismatch");
    return vector_dot(a->ctx, a->d, b->d, a->n, out);
}

extern "C" yg_status yg_vector_axpy(double alpha, yg_vector x, yg_vector y) {
    if (!x || !y || x->n != y->n) return fail(YG_BAD_ARG, "yg_vector_axpy: size mismatch");
    k_axpy<<<stream_grid(x->ctx, x->n), kThreads, 0, x->ctx->stream>>>(alpha, x->d, y->d, x->n);
    YG_LAUNCHED(x->ctx);
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

// ================================================================ matrices

extern "C" yg_status yg_matrix_from_triplets(yg_context ctx, int32_t block, const uint64_t *rows,
                                             const uint64_t *cols, const double *vals, uint64_t n,
                                             yg_matrix *out) {
    if (!ctx || !out || block < 1 || block > 8 || (n && (!rows || !cols || !vals)))
        return fail(YG_BAD_ARG, "yg_matrix_from_triplets: bad argument");
    *out = nullptr;
    if (n == 0) return fail(YG_BAD_ARG, "yg_matrix_from_triplets: empty triplet list (the reference does not support empty matrices)");
    const int64_t B = block, B2 = B * B;
    uint64_t maxr = 0, maxc = 0;
    for (uint64_t i = 0; i < n; ++i) { maxr = std::max(maxr, rows[i]); maxc = std::max(maxc, cols[i]); }
    int64_t nbrows = (int64_t)(maxr / B) + 1, nbcols = (int64_t)(maxc / B) + 1;
    // Order: CSR sorts (row, col, value) so duplicates are summed in ascending
    // value order (sparse_csr.hpp:103-104); BCSR sorts (I, J, i, j) and keeps
    // the input order among duplicates.
    std::vector<uint64_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    if (block == 1) {
        std::sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
            if (rows[a] != rows[b]) return rows[a] < rows[b];
            if (cols[a] != cols[b]) return cols[a] < cols[b];
            return vals[a] < vals[b];
        });
    } else {
        std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
            uint64_t ka[4] = {rows[a] / B, cols[a] / B, rows[a] % B, cols[a] % B};
            uint64_t kb[4] = {rows[b] / B, cols[b] / B, rows[b] % B, cols[b] % B};
            for (int k = 0; k < 4; ++k) if (ka[k] != kb[k]) return ka[k] < kb[k];
            return false;
        });
    }
    std::vector<int64_t> rp(nbrows + 1, 0), col;
    std::vector<double> val;
    col.reserve(n);
    val.reserve(n * (block == 1 ? 1 : 1));
    int64_t curI = -1, curJ = -1;
    for (uint64_t t = 0; t < n; ++t) {
        uint64_t k = idx[t];
        int64_t I = rows[k] / B, J = cols[k] / B;
        if (I != curI || J != curJ) {
            col.push_back(J);
            val.resize(val.size() + B2, 0.0);
            rp[I + 1]++;
            curI = I; curJ = J;
        }
        val[(col.size() - 1) * B2 + (rows[k] % B) * B + (cols[k] % B)] += vals[k];
    }
    for (int64_t i = 0; i < nbrows; ++i) rp[i + 1] += rp[i];
    return upload_bcsr(ctx, block, nbrows, nbcols, rp, col, val.data(), out);
}

extern "C" yg_status yg_matrix_from_csr(yg_context ctx, int32_t block, int64_t nbrows, int64_t nbcols,
                                        const int64_t *brow_ptr, const int64_t *bcol, const double *vals,
                                        yg_matrix *out) {
    if (!ctx || !out || block < 1 || block > 8 || nbrows < 0 || !brow_ptr)
        return fail(YG_BAD_ARG, "yg_matrix_from_csr: bad argument");
    std::vector<int64_t> rp(brow_ptr, brow_ptr + nbrows + 1);
    if (rp[0] != 0) return fail(YG_BAD_ARG, "yg_matrix_from_csr: row pointer must start at 0");
    for (int64_t i = 0; i < nbrows; ++i)
        if (rp[i + 1] < rp[i]) return fail(YG_BAD_ARG, "yg_matrix_from_csr: row pointer decreases at row %lld", (long long)i);
    int64_t nnzb = rp[nbrows];
    std::vector<int64_t> col(bcol, bcol + nnzb);
    for (int64_t i = 0; i < nbrows; ++i)
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
            if (col[k] < 0 || col[k] >= nbcols) return fail(YG_BAD_ARG, "column %lld out of range in row %lld", (long long)col[k], (long long)i);
            if (k > rp[i] && col[k] <= col[k - 1]) return fail(YG_BAD_ARG, "columns not strictly increasing in row %lld", (long long)i);
        }
    return upload_bcsr(ctx, block, nbrows, nbcols, rp, col, vals, out);
}

extern "C" yg_status yg_matrix_destroy(yg_matrix A) {
    if (!A) return YG_OK;
    yg_context ctx = A->ctx;
    dev_free(ctx, A->d_rowptr);
    dev_free(ctx, A->d_col);
    dev_free(ctx, A->d_val);
    dev_free(ctx, A->d_val32);
    dev_free(ctx, A->d_corr32);
    dev_free(ctx, A->d_diag);
    for (int k = 0; k < 3; ++k) dev_free(ctx, A->d_ctiles[k]);
    for (void *p : {(void *)A->d_bcmask, (void *)A->d_bcg, (void *)A->d_bcq, (void *)A->d_bcvals, (void *)A->d_bcdofs})
        dev_free(ctx, p);
    delete A;
    return YG_OK;
}

extern "C" yg_status yg_matrix_sizes(yg_matrix A, int64_t *rows, int64_t *cols, int64_t *nnz, int32_t *block) {
    if (!A) return fail(YG_BAD_ARG, "NULL matrix");
    if (rows) *rows = A->rows();
    if (cols) *cols = A->cols();
    if (nnz) *nnz = A->nnzb * A->block * A->block;
    if (block) *block = A->block;
    return YG_OK;
}

extern "C" yg_status yg_matrix_get(yg_matrix A, int64_t *brow_ptr, int64_t *bcol, double *vals) {
    if (!A) return fail(YG_BAD_ARG, "NULL matrix");
    yg_context ctx = A->ctx;
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (brow_ptr) {
        std::vector<int32_t> t(A->nbrows + 1);
        YG_CUDA(cudaMemcpy(t.data(), A->d_rowptr, sizeof(int32_t) * (A->nbrows + 1), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i <= A->nbrows; ++i) brow_ptr[i] = t[i];
    }
    if (bcol) {
        std::vector<int32_t> t(A->nnzb);
        YG_CUDA(cudaMemcpy(t.data(), A->d_col, sizeof(int32_t) * A->nnzb, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < A->nnzb; ++i) bcol[i] = t[i];
    }
    if (vals) YG_CUDA(cudaMemcpy(vals, A->d_val, sizeof(double) * A->nnzb * A->block * A->block, cudaMemcpyDeviceToHost));
    return YG_OK;
}

extern "C" yg_status yg_matrix_make_fp32(yg_matrix A) {
    if (!A) return fail(YG_BAD_ARG, "NULL matrix");
    yg_context ctx = A->ctx;
    int64_t n = A->nnzb * A->block * A->block;
    if (!A->d_val32) YG_TRY(dev_alloc_t(ctx, &A->d_val32, n));
    k_to_fp32<<<stream_grid(ctx, n), kThreads, 0, ctx->stream>>>(A->d_val, A->d_val32, n);
    YG_LAUNCHED(ctx);
    const int grid = (int)std::min<int64_t>((A->nbrows + kThreads / 32 - 1) / (kThreads / 32), (int64_t)ctx->num_sms * 8);
    if (A->block <= 3 && A->nbrows == A->nbcols && grid > 0) {  // square, a block size the SpMV kernels take
        if (!A->d_corr32) YG_TRY(dev_alloc_t(ctx, &A->d_corr32, A->nbrows * A->block * A->block));
        switch (A->block) {
        case 1: k_fp32_correction<1><<<grid, kThreads, 0, ctx->stream>>>(A->nbrows, A->d_rowptr, A->d_val, A->d_corr32); break;
        case 2: k_fp32_correction<2><<<grid, kThreads, 0, ctx->stream>>>(A->nbrows, A->d_rowptr, A->d_val, A->d_corr32); break;
        default: k_fp32_correction<3><<<grid, kThreads, 0, ctx->stream>>>(A->nbrows, A->d_rowptr, A->d_val, A->d_corr32); break;
        }
        YG_LAUNCHED(ctx);
    }
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

extern "C" yg_status yg_spmv_ex(yg_matrix A, yg_vector x, yg_vector y, int32_t precision) {
    if (!A || !x || !y) return fail(YG_BAD_ARG, "yg_spmv: NULL argument");
    if (x->n != A->cols() || y->n != A->rows())
        return fail(YG_BAD_ARG, "yg_spmv: dimension mismatch (A %lldx%lld, x %lld, y %lld)", (long long)A->rows(),
                    (long long)A->cols(), (long long)x->n, (long long)y->n);
    if (precision != YG_PREC_FP64 && precision != YG_PREC_MIXED && precision != YG_SPMV_MIXED_CORRECTED)
        return fail(YG_BAD_ARG, "yg_spmv: precision %d is not an SpMV precision", (int)precision);
    const bool corrected = precision == YG_SPMV_MIXED_CORRECTED;
    if (corrected) precision = YG_PREC_MIXED;
    if (precision == YG_PREC_MIXED && !A->d_val32) YG_TRY(yg_matrix_make_fp32(A));
    if (corrected && !A->d_corr32) return fail(YG_UNSUPPORTED, "yg_spmv: the row-sum correction needs a square matrix");
    YG_TRY(spmv_autotune_device(A));
    YG_TRY(spmv_launch(A, x->d, y->d, precision, nullptr, nullptr, spmv_default_grid(A), nullptr,
                       corrected ? A->d_corr32 : nullptr));
    YG_CUDA(cudaStreamSynchronize(A->ctx->stream));
    return check_device_error(A->ctx);
}

extern "C" yg_status yg_spmv(yg_matrix A, yg_vector x, yg_vector y) { return yg_spmv_ex(A, x, y, YG_PREC_FP64); }

// Checks a (variant, lanes) choice for A and builds what it needs.
static yg_status spmv_choice_check(yg_matrix A, int32_t variant, int32_t lanes) {
    if (!A || variant < -1 || variant > 4 ||
        (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32))
        return fail(YG_BAD_ARG, "yg_matrix_set_spmv: bad variant/lanes");
    if ((variant == 1 || variant == 2 || variant == 4) && A->block != 2 && A->block != 3)
        return fail(YG_UNSUPPORTED, "staged SpMV needs 2x2 or 3x3 blocks");
    if (variant == 0 && lanes == 1) return fail(YG_BAD_ARG, "flat SpMV needs 2..32 lanes");
    if (variant == 3 || variant == 4) YG_TRY(spmv_prepare(A, variant, lanes));
    return YG_OK;
}

extern "C" yg_status yg_matrix_set_spmv_for(yg_matrix A, int32_t precision, int32_t variant, int32_t lanes) {
    if (variant < 0) return fail(YG_BAD_ARG, "yg_matrix_set_spmv_for: a variant (0..4), not the autotuner");
    YG_TRY(spmv_choice_check(A, variant, lanes));
    if (precision == YG_PREC_FP64) {
        A->variant = variant;
        A->lanes = lanes;
        A->tuned = true;
    } else {
        A->variant32 = variant;
        A->lanes32 = lanes;
        A->tuned32 = true;
    }
    return YG_OK;
}

extern "C" yg_status yg_matrix_set_spmv(yg_matrix A, int32_t variant, int32_t lanes) {
    YG_TRY(spmv_choice_check(A, variant, lanes));
    if (variant < 0) {  // re-run the device autotuner
        A->tuned = false;
        A->tuned32 = false;
        return spmv_autotune_device(A);
    }
    A->variant = variant;
    A->lanes = lanes;
    A->tuned = true;
    A->variant32 = variant;  // the same kernel for FP32 values
    A->lanes32 = lanes;
    A->tuned32 = true;
    return YG_OK;
}

extern "C" yg_status yg_matrix_get_spmv(yg_matrix A, int32_t *variant, int32_t *lanes) {
    if (!A) return fail(YG_BAD_ARG, "NULL matrix");
    if (variant) *variant = A->variant;
    if (lanes) *lanes = A->lanes;
    return YG_OK;
}

extern "C" yg_status yg_matrix_get_spmv_for(yg_matrix A, int32_t precision, int32_t *variant, int32_t *lanes) {
    if (!A) return fail(YG_BAD_ARG, "NULL matrix");
    const bool f32 = precision != YG_PREC_FP64;
    if (variant) *variant = f32 ? A->variant32 : A->variant;
    if (lanes) *lanes = f32 ? A->lanes32 : A->lanes;
    return YG_OK;
}

extern "C" yg_status yg_spmv_bench(yg_matrix A, yg_vector x, yg_vector y, int32_t precision, int32_t reps,
                                   double *ms_per_launch) {
    if (!A || !x || !y || reps < 1 || !ms_per_launch) return fail(YG_BAD_ARG, "yg_spmv_bench: bad argument");
    if (x->n != A->cols() || y->n != A->rows()) return fail(YG_BAD_ARG, "yg_spmv_bench: dimension mismatch");
    if (precision != YG_PREC_FP64 && precision != YG_PREC_MIXED && precision != YG_SPMV_MIXED_CORRECTED)
        return fail(YG_BAD_ARG, "yg_spmv_bench: precision %d is not an SpMV precision", (int)precision);
    const bool corrected = precision == YG_SPMV_MIXED_CORRECTED;
    if (corrected) precision = YG_PREC_MIXED;
    if (precision == YG_PREC_MIXED && !A->d_val32) YG_TRY(yg_matrix_make_fp32(A));
    const double *corr = corrected ? A->d_corr32 : nullptr;
    yg_context ctx = A->ctx;
    int grid = spmv_grid_for(A, precision);
    // the FP32-value form the mixed-precision solvers run: with 2x2/3x3 blocks x
    // is gathered from an FP32 node-padded copy
    float *x32 = nullptr;
    if (precision == YG_PREC_MIXED && (A->block == 2 || A->block == 3)) {
        const int xs = spmv_x32_stride(A->block);
        const int64_t m32 = (A->cols() / A->block + 1) * xs;
        YG_TRY(dev_alloc_t(ctx, &x32, m32));
        cudaMemsetAsync(x32, 0, sizeof(float) * m32, ctx->stream);
        k_to_x32<<<stream_grid(ctx, x->n), kThreads, 0, ctx->stream>>>(x->d, x32, x->n, A->block, xs);
        YG_LAUNCHED(ctx);
    }
    yg_status s = spmv_launch(A, x->d, y->d, precision, nullptr, nullptr, grid, x32, corr);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (s == YG_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        s = fail(YG_CUDA_ERROR, "yg_spmv_bench: events");
    float ms = 0;
    if (s == YG_OK) {
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < reps && s == YG_OK; ++r)
            s = spmv_launch(A, x->d, y->d, precision, nullptr, nullptr, grid, x32, corr);
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) s = fail(YG_CUDA_ERROR, "yg_spmv_bench: launch");
        cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, x32);
    if (s != YG_OK) return s;
    *ms_per_launch = ms / reps;
    return check_device_error(ctx);
}
