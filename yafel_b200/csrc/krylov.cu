// krylov.cu -- CG / PCG and BiCGSTAB on the GPU with fused iterations.
//
// Replaces cg_solve (solver/iterative/cg_solve.hpp:23-81), pcg_solve
// (pcg_solve.hpp:115-178) and bicgstab_solve (bicgstab_solve.hpp:207-283).
//
// One PCG iteration is three kernels on a persistent grid of G blocks:
//   1. q = A p fused with per-block partials of p.q                (spmv.cu)
//   2. every block reduces the G partials in the same order -> alpha;
//      x += alpha p, r -= alpha q, z = M^-1 r (Jacobi fused), partials of r.z, r.r
//   3. every block reduces those -> beta; p = z + beta p; block 0 records the
//      scalars and the convergence flag.
// Scalars live in device memory (KrylovScalars); r.z is double-buffered by
// iteration parity so no block reads a value another block of the same kernel
// is writing.  A run of iterations is captured once into a CUDA graph and
// replayed; kernels return immediately once the flag is set, and the host reads
// the flag once per replay.  All reductions have a fixed order, so a solve is
// bit-reproducible.  ILU(0) goes through the general path (z stored, apply by
// precond.cu, then a separate r.z reduction).
#include "internal.h"
#include "device_common.cuh"

#include <algorithm>
#include <cmath>
#include <chrono>

namespace yg {

yg_status precond_apply_dev(yg_precond M, const double *r, double *z);
bool precond_fusable(yg_precond M);
const double *precond_dinv(yg_precond M);
int stream_grid(yg_context ctx, int64_t n);

enum { FLAG_RUN = 0, FLAG_CONVERGED = 1, FLAG_BREAKDOWN = 2, FLAG_NAN = 3, FLAG_MAXITER = 4 };

// ------------------------------------------------------------------ kernels

// r = b - q; optional z = dinv*r; partials of r.z and r.r and b.b
__global__ void __launch_bounds__(kThreads)
k_residual_init(int64_t n, const double *__restrict__ b, const double *__restrict__ q, double *__restrict__ r,
                double *__restrict__ z, const double *__restrict__ dinv, double *__restrict__ partials) {
    __shared__ double sm[kThreads / 32 + 1];
    int64_t lo, hi;
    block_chunk(n, lo, hi);
    double srz = 0, srr = 0, sbb = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        double ri = b[i] - q[i];
        r[i] = ri;
        double zi = dinv ? dinv[i] * ri : ri;
        if (z) z[i] = zi;
        srz += ri * zi;
        srr += ri * ri;
        sbb += b[i] * b[i];
    }
    srz = block_sum<kThreads>(srz, sm);
    srr = block_sum<kThreads>(srr, sm);
    sbb = block_sum<kThreads>(sbb, sm);
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x + 0] = srz;
        partials[3 * blockIdx.x + 1] = srr;
        partials[3 * blockIdx.x + 2] = sbb;
    }
}

// partials of r.z (general preconditioner path)
__global__ void __launch_bounds__(kThreads)
k_dot2_partials(int64_t n, const double *__restrict__ r, const double *__restrict__ z, double *__restrict__ partials,
                const int32_t *__restrict__ flag, int off, int stride) {
    __shared__ double sm[kThreads / 32 + 1];
    if (flag && read_flag(flag)) return;
    int64_t lo, hi;
    block_chunk(n, lo, hi);
    double s = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += r[i] * z[i];
    s = block_sum<kThreads>(s, sm);
    if (threadIdx.x == 0) partials[(int64_t)stride * blockIdx.x + off] = s;
}

// Scalars after the initial residual: rz0, bb; flag set when r0.z0 == 0
// (the initial guess solves the system exactly, cg_solve.hpp:52-54).
__global__ void __launch_bounds__(kThreads)
k_cg_scalars_init(KrylovScalars *S, const double *__restrict__ partials, int np, int stride, double tol,
                  int64_t maxiter, int criterion) {
    __shared__ double sm[kThreads / 32 + 1];
    double rz = reduce_partials<kThreads>(partials, np, stride, 0, sm);
    double rr = reduce_partials<kThreads>(partials, np, stride, 1, sm);
    double bb = reduce_partials<kThreads>(partials, np, stride, 2, sm);
    if (threadIdx.x == 0) {
        S->rz[0] = rz;
        S->rz[1] = rz;
        S->rz0 = rz;
        S->rr = rr;
        S->bb = bb;
        S->tol = tol;
        S->iter = 0;
        S->maxiter = maxiter;
        S->criterion = criterion;
        S->flag = FLAG_RUN;
        if (rz == 0) S->flag = FLAG_CONVERGED;
        else if (criterion == YG_CRIT_RELRES && sqrt(rr) <= tol * sqrt(bb)) S->flag = FLAG_CONVERGED;
        if (maxiter <= 0 && S->flag == FLAG_RUN) S->flag = FLAG_MAXITER;
    }
}

// After a residual replacement: r.z and r.r of the true FP64 residual into both
// parity slots.
__global__ void __launch_bounds__(kThreads)
k_cg_scalars_replace(KrylovScalars *S, const double *__restrict__ partials, int np, int stride, int clear_flag) {
    __shared__ double sm[kThreads / 32 + 1];
    double rz = reduce_partials<kThreads>(partials, np, stride, 0, sm);
    double rr = reduce_partials<kThreads>(partials, np, stride, 1, sm);
    if (threadIdx.x == 0) {
        S->rz[0] = rz;
        S->rz[1] = rz;
        S->rr = rr;
        if (clear_flag) S->flag = 0;
    }
}

// Kernel 2 of the iteration.  JAC: z = dinv*r computed in registers (M is
// Jacobi or identity); otherwise only r.r partials (z comes from M later).
template <bool FUSED>
__global__ void __launch_bounds__(kThreads)
k_cg_update(int64_t n, const double *__restrict__ pq_partials, int np, KrylovScalars *S, int parity,
            double *__restrict__ x, double *__restrict__ r, const double *__restrict__ p,
            const double *__restrict__ q, const double *__restrict__ dinv, double *__restrict__ partials_out) {
    __shared__ double sm[kThreads / 32 + 1];
    if (read_flag(&S->flag)) return;
    const double pq = reduce_partials<kThreads>(pq_partials, np, 1, 0, sm);
    const double alpha = S->rz[parity] / pq;
    // no definiteness test: the reference runs CG on negative definite systems
    // too (test/test_cg_solve.cpp uses tridiag(1,-2,1)); only p.Ap = 0 breaks down
    if (pq == 0 || !isfinite(alpha)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) S->flag = isfinite(pq) ? FLAG_BREAKDOWN : FLAG_NAN;
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) S->iter_seen = S->iter;  // for k_cg_pupdate's iteration cap test
    int64_t lo, hi;
    block_chunk2(n, lo, hi);
    double srz = 0, srr = 0;
    // pairs of entries as 16-byte loads (the chunk starts on an even index)
    auto one = [&](int64_t i) {
        x[i] += p[i] * alpha;
        double ri = r[i] + (-alpha) * q[i];
        r[i] = ri;
        srr += ri * ri;
        if (FUSED) {
            double zi = dinv ? dinv[i] * ri : ri;
            srz += ri * zi;
        }
    };
    const int64_t v1 = hi >> 1;
#pragma unroll 2
    for (int64_t v = (lo >> 1) + threadIdx.x; v < v1; v += blockDim.x) {
        double2 xv = reinterpret_cast<const double2 *>(x)[v];
        const double2 pv = reinterpret_cast<const double2 *>(p)[v];
        double2 rv = reinterpret_cast<const double2 *>(r)[v];
        const double2 qv = reinterpret_cast<const double2 *>(q)[v];
        xv.x += pv.x * alpha;
        xv.y += pv.y * alpha;
        rv.x = rv.x + (-alpha) * qv.x;
        rv.y = rv.y + (-alpha) * qv.y;
        reinterpret_cast<double2 *>(x)[v] = xv;
        reinterpret_cast<double2 *>(r)[v] = rv;
        srr += rv.x * rv.x;
        srr += rv.y * rv.y;
        if (FUSED) {
            double2 zv = rv;
            if (dinv) {
                const double2 dv = reinterpret_cast<const double2 *>(dinv)[v];
                zv.x = dv.x * rv.x;
                zv.y = dv.y * rv.y;
            }
            srz += rv.x * zv.x;
            srz += rv.y * zv.y;
        }
    }
    if ((hi & 1) && hi > lo && threadIdx.x == 0) one(hi - 1);  // odd n: the last entry
    srr = block_sum<kThreads>(srr, sm);
    if (FUSED) srz = block_sum<kThreads>(srz, sm);
    if (threadIdx.x == 0) {
        partials_out[2 * blockIdx.x + 0] = srz;
        partials_out[2 * blockIdx.x + 1] = srr;
    }
}

// Kernel 3: beta, p = z + beta p, scalars and convergence (block 0).
// FP32 gather copy of the direction for the mixed-precision SpMV: entry i of a
// vector with `blk`-sized node blocks goes to p32[(i / blk) * xs + i % blk].
struct Dir32 {
    float *p32 = nullptr;
    int blk = 1, xs = 1;
    __device__ __forceinline__ void put(int64_t i, double v) const {
        if (!p32) return;
        if (blk == 1) p32[i] = (float)v;
        else p32[(i / blk) * xs + i % blk] = (float)v;
    }
};

template <bool FUSED>
__global__ void __launch_bounds__(kThreads)
k_cg_pupdate(int64_t n, const double *__restrict__ partials_in, int np, KrylovScalars *S, int parity,
             double *__restrict__ p, const double *__restrict__ r, const double *__restrict__ z,
             const double *__restrict__ dinv, Dir32 d32) {
    __shared__ double sm[kThreads / 32 + 1];
    if (read_flag(&S->flag)) return;
    const double rz_new = reduce_partials<kThreads>(partials_in, np, 2, 0, sm);
    const double rr = reduce_partials<kThreads>(partials_in, np, 2, 1, sm);
    const double rz_old = S->rz[parity];
    // convergence test before the direction update, as the reference does
    bool done = false;
    int flag = FLAG_RUN;
    if (S->criterion == YG_CRIT_REFERENCE) {
        if (rz_new / S->rz0 < S->tol) { done = true; flag = FLAG_CONVERGED; }
    } else {
        if (sqrt(rr) <= S->tol * sqrt(S->bb)) { done = true; flag = FLAG_CONVERGED; }
    }
    if (!isfinite(rz_new)) { done = true; flag = FLAG_NAN; }
    // the cap test reads the count the previous kernel recorded: S->iter itself is
    // incremented below by block 0 while other blocks may still be deciding
    const int64_t it = S->iter_seen;
    if (!done && it + 1 >= S->maxiter) { done = true; flag = FLAG_MAXITER; }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->rz[parity ^ 1] = rz_new;
        S->rr = rr;
        S->iter = it + 1;
        if (done) S->flag = flag;
    }
    if (done) return;
    const double beta = rz_new / rz_old;
    int64_t lo, hi;
    block_chunk2(n, lo, hi);
    const int64_t v1 = hi >> 1;
#pragma unroll 2
    for (int64_t v = (lo >> 1) + threadIdx.x; v < v1; v += blockDim.x) {
        const double2 rv = reinterpret_cast<const double2 *>(FUSED ? r : z)[v];
        double2 zv = rv;
        if (FUSED && dinv) {
            const double2 dv = reinterpret_cast<const double2 *>(dinv)[v];
            zv.x = dv.x * rv.x;
            zv.y = dv.y * rv.y;
        }
        double2 pv = reinterpret_cast<const double2 *>(p)[v];
        pv.x = zv.x + beta * pv.x;
        pv.y = zv.y + beta * pv.y;
        reinterpret_cast<double2 *>(p)[v] = pv;
        d32.put(2 * v, pv.x);
        d32.put(2 * v + 1, pv.y);
    }
    if ((hi & 1) && hi > lo && threadIdx.x == 0) {  // odd n: the last entry
        const int64_t i = hi - 1;
        double zi = FUSED ? (dinv ? dinv[i] * r[i] : r[i]) : z[i];
        const double pi = zi + beta * p[i];
        p[i] = pi;
        d32.put(i, pi);
    }
}

// p = z (start of the iteration); z is dinv*r or r in the fused path
__global__ void k_p_init(int64_t n, double *__restrict__ p, const double *__restrict__ r,
                         const double *__restrict__ z, const double *__restrict__ dinv, Dir32 d32) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double pi = z ? z[i] : (dinv ? dinv[i] * r[i] : r[i]);
        p[i] = pi;
        d32.put(i, pi);
    }
}

__global__ void k_sub(int64_t n, const double *__restrict__ b, const double *__restrict__ q, double *__restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - q[i];
}

__global__ void k_add(int64_t n, double *__restrict__ x, const double *__restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += d[i];
}

__global__ void k_copy(int64_t n, double *__restrict__ dst, const double *__restrict__ src) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// ------------------------------------------------------------------ host side

struct Work {
    yg_context ctx;
    int64_t n;
    double *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *t = nullptr, *s = nullptr, *v = nullptr,
           *rhat = nullptr, *ph = nullptr, *sh = nullptr, *d = nullptr;
    Dir32 d32;  // FP32 copy of p for the mixed-precision SpMV (p32 NULL otherwise)
    ~Work() {
        for (double *ptr : {r, p, q, z, t, s, v, rhat, ph, sh, d}) dev_free(ctx, ptr);
        dev_free(ctx, d32.p32);
    }
};

static yg_status alloc_vec(yg_context ctx, double **p, int64_t n) { return dev_alloc_t(ctx, p, n > 0 ? n : 1); }

// Read flag and iteration count of the scalars (one small D2H copy + sync).
static yg_status read_scalars(yg_context ctx, KrylovScalars *out) {
    YG_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_scalars, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, ctx->stream));
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    memcpy(out, ctx->h_pinned, sizeof(KrylovScalars));
    return YG_OK;
}

static yg_status true_relres(yg_matrix A, const double *b, const double *x, double *tmp, double *out) {
    yg_context ctx = A->ctx;
    int64_t n = A->rows();
    YG_TRY(spmv_launch(A, x, tmp, YG_PREC_FP64, nullptr, nullptr, spmv_default_grid(A)));
    k_sub<<<stream_grid(ctx, n), kThreads, 0, ctx->stream>>>(n, b, tmp, tmp);
    YG_LAUNCHED(ctx);
    double rr = 0, bb = 0;
    YG_TRY(vector_dot(ctx, tmp, tmp, n, &rr));
    YG_TRY(vector_dot(ctx, b, b, n, &bb));
    *out = bb > 0 ? sqrt(rr / bb) : sqrt(rr);
    return YG_OK;
}

static yg_status flag_to_status(int flag) {
    switch (flag) {
    case FLAG_CONVERGED: return YG_OK;
    case FLAG_BREAKDOWN: return YG_BREAKDOWN;
    case FLAG_NAN: return YG_NAN;
    case FLAG_MAXITER: return YG_NOT_CONVERGED;
    default: return YG_NOT_CONVERGED;
    }
}

// Captured graph of `m` iterations (m even so parities line up across replays).
struct IterGraph {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    int64_t kernels = 0;
    ~IterGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

template <typename F>
static yg_status capture(yg_context ctx, int m, F &&one_iteration, IterGraph &g) {
    int64_t before = ctx->launches;
    YG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    yg_status s = YG_OK;
    for (int it = 0; it < m && s == YG_OK; ++it) s = one_iteration(it & 1);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    g.kernels = ctx->launches - before;
    ctx->launches = before;
    if (s != YG_OK) { if (graph) cudaGraphDestroy(graph); return s; }
    if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "graph capture: %s", cudaGetErrorString(e));
    g.graph = graph;
    YG_CUDA(cudaGraphInstantiate(&g.exec, graph, 0));
    return YG_OK;
}

static int default_check_every(int64_t n, const yg_solve_opts *o) {
    int m = o && o->check_every > 0 ? o->check_every : (n < 200000 ? 16 : 32);
    if (m & 1) ++m;
    return m;
}

// Core PCG on (A, precision) with x updated in place.  The right-hand side is b.
// SpMV timing inside captured iterations: an event pair around each SpMV.
struct SpmvProfile {
    bool on = false;
    std::vector<cudaEvent_t> start, stop;
    double ms = 0;
    int64_t launches = 0;
    ~SpmvProfile() {
        for (auto e : start) cudaEventDestroy(e);
        for (auto e : stop) cudaEventDestroy(e);
    }
    yg_status init(int m) {
        if (!on) return YG_OK;
        start.resize(m);
        stop.resize(m);
        for (int i = 0; i < m; ++i) {
            YG_CUDA(cudaEventCreate(&start[i]));
            YG_CUDA(cudaEventCreate(&stop[i]));
        }
        return YG_OK;
    }
    // add the first `done` pairs of the last replay (later ones were no-ops)
    yg_status collect(int64_t done) {
        if (!on) return YG_OK;
        for (int64_t i = 0; i < done && i < (int64_t)start.size(); ++i) {
            float t = 0;
            YG_CUDA(cudaEventElapsedTime(&t, start[i], stop[i]));
            ms += t;
            ++launches;
        }
        return YG_OK;
    }
};

static yg_status pcg_core(yg_matrix A, yg_precond M, const double *b, double *x, int precision, int criterion,
                          double tol, int64_t maxiter, int check_every, Work &w, int64_t *iters, int *flag_out,
                          SpmvProfile *prof = nullptr, int64_t *replacements = nullptr) {
    yg_context ctx = A->ctx;
    const int64_t n = A->rows();
    // the update kernels stream pairs of entries as 16-byte loads
    if (((uintptr_t)b | (uintptr_t)x) & 15) return fail(YG_BAD_ARG, "solver vectors must be 16-byte aligned");
    const bool fused = !M || precond_fusable(M);
    const double *dinv = M ? precond_dinv(M) : nullptr;
    const int G = ctx->reduce_blocks;
    const int spmv_grid = std::min(spmv_grid_for(A, precision), kMaxReduceBlocks);
    double *P = ctx->d_partials;  // [0,G): p.q ; [2G,4G): r.z/r.r pairs ; [4G, 7G): init triples
    KrylovScalars *S = ctx->d_scalars;
    cudaStream_t st = ctx->stream;
    // the FP32 direction copy serves the FP32-value iteration SpMV only; so does
    // the row-sum correction of the FP32 values (the operator A32 x + C x_own)
    const bool f32 = precision == YG_PREC_MIXED || precision == YG_PREC_MIXED_IR;
    const Dir32 d32 = f32 ? w.d32 : Dir32{};
    const double *corr = f32 ? A->d_corr32 : nullptr;

    // r = b - A x ; z = M^-1 r ; p = z
    YG_TRY(spmv_launch(A, x, w.q, precision, nullptr, nullptr, spmv_grid, nullptr, corr));
    if (fused) {
        k_residual_init<<<G, kThreads, 0, st>>>(n, b, w.q, w.r, nullptr, dinv, P + 4 * G);
        YG_LAUNCHED(ctx);
        k_p_init<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, w.p, w.r, nullptr, dinv, d32);
        YG_LAUNCHED(ctx);
    } else {
        k_residual_init<<<G, kThreads, 0, st>>>(n, b, w.q, w.r, nullptr, nullptr, P + 4 * G);
        YG_LAUNCHED(ctx);
        YG_TRY(precond_apply_dev(M, w.r, w.z));
        k_dot2_partials<<<G, kThreads, 0, st>>>(n, w.r, w.z, P + 4 * G, nullptr, 0, 3);
        YG_LAUNCHED(ctx);
        k_p_init<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, w.p, w.r, w.z, nullptr, d32);
        YG_LAUNCHED(ctx);
    }
    k_cg_scalars_init<<<1, kThreads, 0, st>>>(S, P + 4 * G, G, 3, tol, maxiter, criterion);
    YG_LAUNCHED(ctx);
    YG_CUDA(cudaGetLastError());

    int slot = 0;
    auto one = [&](int parity) -> yg_status {
        if (prof && prof->on) YG_CUDA(cudaEventRecordWithFlags(prof->start[slot], st, cudaEventRecordExternal));
        YG_TRY(spmv_launch(A, w.p, w.q, precision, P, &S->flag, spmv_grid, d32.p32, corr));
        if (prof && prof->on) YG_CUDA(cudaEventRecordWithFlags(prof->stop[slot], st, cudaEventRecordExternal));
        ++slot;
        if (fused) {
            k_cg_update<true><<<G, kThreads, 0, st>>>(n, P, spmv_grid, S, parity, x, w.r, w.p, w.q, dinv, P + 2 * G);
            YG_LAUNCHED(ctx);
            k_cg_pupdate<true><<<G, kThreads, 0, st>>>(n, P + 2 * G, G, S, parity, w.p, w.r, nullptr, dinv, d32);
            YG_LAUNCHED(ctx);
        } else {
            k_cg_update<false><<<G, kThreads, 0, st>>>(n, P, spmv_grid, S, parity, x, w.r, w.p, w.q, nullptr, P + 2 * G);
            YG_LAUNCHED(ctx);
            YG_TRY(precond_apply_dev(M, w.r, w.z));
            k_dot2_partials<<<G, kThreads, 0, st>>>(n, w.r, w.z, P + 2 * G, &S->flag, 0, 2);
            YG_LAUNCHED(ctx);
            k_cg_pupdate<false><<<G, kThreads, 0, st>>>(n, P + 2 * G, G, S, parity, w.p, w.r, w.z, nullptr, d32);
            YG_LAUNCHED(ctx);
        }
        return YG_OK;
    };
    // Residual replacement: r = b - A x with the FP64 matrix, r.z and r.r of it into
    // the scalars (z stays implicit in the fused path).  It is the FP64
    // iterative-refinement step of the mixed-precision solve, and the final check
    // of every RELRES solve.
    auto replace = [&](int clear_flag) -> yg_status {
        YG_TRY(spmv_launch(A, x, w.q, YG_PREC_FP64, nullptr, nullptr, spmv_default_grid(A)));
        if (fused) {
            k_residual_init<<<G, kThreads, 0, st>>>(n, b, w.q, w.r, nullptr, dinv, P + 4 * G);
            YG_LAUNCHED(ctx);
        } else {
            k_residual_init<<<G, kThreads, 0, st>>>(n, b, w.q, w.r, nullptr, nullptr, P + 4 * G);
            YG_LAUNCHED(ctx);
            YG_TRY(precond_apply_dev(M, w.r, w.z));
            k_dot2_partials<<<G, kThreads, 0, st>>>(n, w.r, w.z, P + 4 * G, nullptr, 0, 3);
            YG_LAUNCHED(ctx);
        }
        k_cg_scalars_replace<<<1, kThreads, 0, st>>>(S, P + 4 * G, G, 3, clear_flag);
        YG_LAUNCHED(ctx);
        if (replacements) ++*replacements;
        return YG_OK;
    };
    const bool reliable = (precision == YG_PREC_MIXED);
    KrylovScalars hs;
    YG_TRY(read_scalars(ctx, &hs));
    if (hs.flag == FLAG_RUN || (hs.flag == FLAG_CONVERGED && criterion == YG_CRIT_RELRES && hs.iter > 0)) {
        IterGraph g;
        if (prof && prof->on && prof->start.empty()) YG_TRY(prof->init(check_every));
        YG_TRY(capture(ctx, check_every, one, g));
        double rr_last = hs.rr;  // r.r at the last replacement
        int false_stops = 0;
        for (;;) {
            int64_t before = hs.iter;
            YG_CUDA(cudaGraphLaunch(g.exec, st));
            ctx->launches += g.kernels;
            YG_TRY(read_scalars(ctx, &hs));
            if (prof) YG_TRY(prof->collect(hs.iter - before));
            if (hs.flag == FLAG_RUN) {
                // replace once the recursive residual fell 10x since the last time
                if (reliable && hs.rr < 1e-2 * rr_last) {
                    YG_TRY(replace(0));
                    YG_TRY(read_scalars(ctx, &hs));
                    rr_last = hs.rr;
                }
                continue;
            }
            if (hs.flag == FLAG_CONVERGED && criterion == YG_CRIT_RELRES) {
                // the recursive residual triggered the stop; the FP64 residual decides
                YG_TRY(replace(1));
                YG_TRY(read_scalars(ctx, &hs));
                rr_last = hs.rr;
                if (sqrt(hs.rr) <= tol * sqrt(hs.bb) || hs.iter >= maxiter || ++false_stops > 20) {
                    hs.flag = (sqrt(hs.rr) <= tol * sqrt(hs.bb)) ? FLAG_CONVERGED
                                                                  : (hs.iter >= maxiter ? FLAG_MAXITER : FLAG_CONVERGED);
                    break;
                }
                // continue from the true residual with a fresh direction p = M^-1 r
                if (fused) {
                    k_p_init<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, w.p, w.r, nullptr, dinv, d32);
                } else {
                    k_p_init<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, w.p, w.r, w.z, nullptr, d32);
                }
                YG_LAUNCHED(ctx);
                continue;
            }
            break;
        }
    }
    *iters = hs.iter;
    *flag_out = hs.flag;
    return YG_OK;
}

yg_status solve_cg(yg_matrix A, yg_precond M, yg_vector bv, yg_vector xv, const yg_solve_opts *opts,
                   yg_solve_stats *stats) {
    yg_context ctx = A->ctx;
    const int64_t n = A->rows();
    yg_solve_opts o = opts ? *opts : yg_solve_opts{YG_CRIT_REFERENCE, YG_PREC_FP64, 1e-14, 0, 0, 0};
    int64_t maxiter = o.maxiter > 0 ? o.maxiter : n;  // cg_solve.hpp:46
    int m = default_check_every(n, &o);
    Work w;
    w.ctx = ctx;
    w.n = n;
    YG_TRY(alloc_vec(ctx, &w.r, n));
    YG_TRY(alloc_vec(ctx, &w.p, n));
    YG_TRY(alloc_vec(ctx, &w.q, n));
    if (M && !precond_fusable(M)) YG_TRY(alloc_vec(ctx, &w.z, n));
    if (o.precision != YG_PREC_FP64 && (A->block == 2 || A->block == 3)) {
        // FP32 gather copy of p (node-padded) for the FP32-value TMA SpMV
        const int xs = spmv_x32_stride(A->block);
        const int64_t m32 = (n / A->block + 1) * xs;
        YG_TRY(dev_alloc_t(ctx, &w.d32.p32, m32));
        YG_CUDA(cudaMemsetAsync(w.d32.p32, 0, sizeof(float) * m32, ctx->stream));
        w.d32.blk = A->block;
        w.d32.xs = xs;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    yg_solve_stats st{};
    int flag = FLAG_RUN;
    int64_t its = 0;
    SpmvProfile prof;
    prof.on = o.profile != 0;
    if (o.precision == YG_PREC_FP64 || o.precision == YG_PREC_MIXED) {
        // FP64, or FP32 matrix values in the iteration with the residual replaced
        // by the FP64 true residual each time it fell 10x (refinement steps).
        if (o.precision == YG_PREC_MIXED && !A->d_val32) YG_TRY(yg_matrix_make_fp32(A));
        YG_TRY(spmv_autotune_device(A));  // the FP32-value kernel has its own tuning
        int64_t repl = 0;
        YG_TRY(pcg_core(A, M, bv->d, xv->d, o.precision, o.criterion, o.tol, maxiter, m, w, &its, &flag, &prof,
                        &repl));
        st.iterations = its;
        st.refinements = (int32_t)repl;
    } else {
        // YG_PREC_MIXED_IR: restarted FP64 iterative refinement around a PCG whose
        // SpMV reads FP32 values (FP64 vectors and accumulation).  Outer residuals
        // and the final check are FP64.
        if (!A->d_val32) YG_TRY(yg_matrix_make_fp32(A));
        YG_TRY(spmv_autotune_device(A));
        YG_TRY(alloc_vec(ctx, &w.d, n));
        YG_TRY(alloc_vec(ctx, &w.t, n));
        double bnorm = 0;
        YG_TRY(vector_dot(ctx, bv->d, bv->d, n, &bnorm));
        bnorm = sqrt(bnorm);
        const double tol = o.tol;
        flag = FLAG_MAXITER;
        for (int outer = 0; outer < 30; ++outer) {
            // t = b - A x (FP64)
            YG_TRY(spmv_launch(A, xv->d, w.q, YG_PREC_FP64, nullptr, nullptr, spmv_default_grid(A)));
            k_sub<<<stream_grid(ctx, n), kThreads, 0, ctx->stream>>>(n, bv->d, w.q, w.t);
            YG_LAUNCHED(ctx);
            double rr = 0;
            YG_TRY(vector_dot(ctx, w.t, w.t, n, &rr));
            double rel = bnorm > 0 ? sqrt(rr) / bnorm : sqrt(rr);
            if (rel <= tol) { flag = FLAG_CONVERGED; break; }
            if (!std::isfinite(rel)) { flag = FLAG_NAN; break; }
            if (st.iterations >= maxiter) { flag = FLAG_MAXITER; break; }
            // inner: A32 d = t to relative accuracy eta (FP32 values limit it to ~1e-6)
            double eta = std::max(1e-5, 0.3 * tol / std::max(rel, 1e-300));
            if (eta > 0.5) eta = 0.5;
            YG_CUDA(cudaMemsetAsync(w.d, 0, sizeof(double) * n, ctx->stream));
            int iflag = 0;
            int64_t iits = 0;
            YG_TRY(pcg_core(A, M, w.t, w.d, YG_PREC_MIXED_IR, YG_CRIT_RELRES, eta, maxiter - st.iterations, m, w, &iits, &iflag, &prof));
            st.iterations += iits;
            st.refinements += 1;
            k_add<<<stream_grid(ctx, n), kThreads, 0, ctx->stream>>>(n, xv->d, w.d);
            YG_LAUNCHED(ctx);
            if (iflag == FLAG_BREAKDOWN || iflag == FLAG_NAN) { flag = iflag; break; }
        }
    }
    cudaEventRecord(e1, ctx->stream);
    double rel = 0;
    YG_TRY(true_relres(A, bv->d, xv->d, w.q, &rel));
    float ms = 0;
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st.rel_residual = rel;
    st.device_ms = ms;
    st.spmv_ms = prof.ms;
    st.spmv_launches = prof.launches;
    yg_status s = flag_to_status(flag);
    if (o.criterion == YG_CRIT_RELRES && s == YG_OK && !(rel <= o.tol)) s = YG_NOT_CONVERGED;
    st.status = s;
    if (stats) *stats = st;
    return s;
}

}  // namespace yg

using namespace yg;

extern "C" yg_status yg_cg(yg_matrix A, yg_precond M, yg_vector b, yg_vector x, const yg_solve_opts *opts,
                           yg_solve_stats *stats) {
    if (!A || !b || !x) return fail(YG_BAD_ARG, "yg_cg: NULL argument");
    if (A->rows() != A->cols() || b->n != A->rows() || x->n != A->rows())
        return fail(YG_BAD_ARG, "yg_cg: dimension mismatch");
    if (M && M->A->rows() != A->rows()) return fail(YG_BAD_ARG, "yg_cg: preconditioner size mismatch");
    if (opts && opts->precision != YG_PREC_FP64 && opts->precision != YG_PREC_MIXED &&
        opts->precision != YG_PREC_MIXED_IR)
        return fail(YG_BAD_ARG, "yg_cg: precision %d is not a solver precision", (int)opts->precision);
    YG_TRY(spmv_autotune_device(A));
    yg_status s = solve_cg(A, M, b, x, opts, stats);
    if (s != YG_OK && s != YG_NOT_CONVERGED && s != YG_BREAKDOWN && s != YG_NAN) return s;
    if (s != YG_OK) set_error("yg_cg: %s", yg_status_string(s));
    return s;
}
