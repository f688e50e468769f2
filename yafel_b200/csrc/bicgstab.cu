// bicgstab.cu -- BiCGSTAB on the GPU (optionally right-preconditioned).
//
// Replaces bicgstab_solve (solver/iterative/bicgstab_solve.hpp:207-283).  One
// iteration is five kernels on a persistent grid:
//   a. reduce rhat.r (and r.r) -> rho, beta; convergence test;
//      p = r + beta p - beta omega v;  ph = M^-1 p
//   b. v = A ph fused with partials of rhat.v                    (spmv.cu)
//   c. alpha = rho / rhat.v;  s = r - alpha v;  sh = M^-1 s
//   d. t = A sh fused with partials of s.t and t.t               (spmv.cu)
//   e. omega = t.s / t.t (0 if t.t = 0); x += alpha ph + omega sh;
//      r = s - omega t; partials of rhat.r and r.r
// rho is double-buffered by iteration parity; alpha and omega are written by
// kernels (c) and (e) and read by (a) of the next iteration only.  The
// reference's criterion (true residual every max(N/100,1) iterations) is
// evaluated between graph replays at exactly those iterations.
#include "internal.h"
#include "device_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace yg {

int stream_grid(yg_context ctx, int64_t n);
bool precond_fusable(yg_precond M);
const double *precond_dinv(yg_precond M);
yg_status precond_apply_dev(yg_precond M, const double *r, double *z);

enum { BF_RUN = 0, BF_CONVERGED = 1, BF_BREAKDOWN = 2, BF_NAN = 3, BF_MAXITER = 4 };

// r = b - q, rhat = r, p = v = 0; partials of rhat.r, r.r, b.b
__global__ void __launch_bounds__(kThreads)
k_bicg_init(int64_t n, const double *__restrict__ b, const double *__restrict__ q, double *__restrict__ r,
            double *__restrict__ rhat, double *__restrict__ p, double *__restrict__ v, double *__restrict__ partials) {
    __shared__ double sm[kThreads / 32 + 1];
    int64_t lo, hi;
    block_chunk(n, lo, hi);
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        double ri = b[i] - q[i];
        r[i] = ri;
        rhat[i] = ri;
        p[i] = 0;
        v[i] = 0;
        s0 += ri * ri;
        s2 += b[i] * b[i];
    }
    s1 = s0;
    s0 = block_sum<kThreads>(s0, sm);
    s1 = block_sum<kThreads>(s1, sm);
    s2 = block_sum<kThreads>(s2, sm);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = s0;
        partials[2 * blockIdx.x + 1] = s1;
        partials[2 * kMaxReduceBlocks + blockIdx.x] = s2;
    }
}

__global__ void __launch_bounds__(kThreads)
k_bicg_scalars_init(KrylovScalars *S, const double *__restrict__ partials, int np, double tol, int64_t maxiter,
                    int criterion) {
    __shared__ double sm[kThreads / 32 + 1];
    double bb = reduce_partials<kThreads>(partials + 2 * kMaxReduceBlocks, np, 1, 0, sm);
    double rr = reduce_partials<kThreads>(partials, np, 2, 1, sm);
    if (threadIdx.x == 0) {
        S->rho[0] = 1.0;  // rho_old = alpha = w_old = 1 (bicgstab_solve.hpp:235-237)
        S->rho[1] = 1.0;
        S->alpha = 1.0;
        S->omega = 1.0;
        S->bb = bb;
        S->rr = rr;
        S->tol = tol;
        S->iter = 0;
        S->maxiter = maxiter;
        S->criterion = criterion;
        S->flag = BF_RUN;
        if (criterion == YG_CRIT_RELRES && sqrt(rr) <= tol * sqrt(bb)) S->flag = BF_CONVERGED;
        if (maxiter <= 0 && S->flag == BF_RUN) S->flag = BF_MAXITER;
    }
}

// (a): rho_new from partials (stride 2: rhat.r, r.r), convergence test, p update
__global__ void __launch_bounds__(kThreads)
k_bicg_p(int64_t n, const double *__restrict__ partials, int np, KrylovScalars *S, int parity, double *__restrict__ p,
         const double *__restrict__ r, const double *__restrict__ v, double *__restrict__ ph,
         const double *__restrict__ dinv) {
    __shared__ double sm[kThreads / 32 + 1];
    if (read_flag(&S->flag)) return;
    const double rho_new = reduce_partials<kThreads>(partials, np, 2, 0, sm);
    const double rr = reduce_partials<kThreads>(partials, np, 2, 1, sm);
    int flag = BF_RUN;
    if (S->criterion == YG_CRIT_RELRES && S->iter > 0 && sqrt(rr) <= S->tol * sqrt(S->bb)) flag = BF_CONVERGED;
    else if (!isfinite(rho_new) || !isfinite(rr)) flag = BF_NAN;
    else if (rho_new == 0) flag = BF_BREAKDOWN;
    else if (S->iter >= S->maxiter) flag = BF_MAXITER;
    if (flag != BF_RUN) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { S->flag = flag; S->rr = rr; }
        return;
    }
    const double rho_old = S->rho[parity];
    const double beta = (rho_new / rho_old) * (S->alpha / S->omega);
    if (blockIdx.x == 0 && threadIdx.x == 0) { S->rho[parity ^ 1] = rho_new; S->rr = rr; }
    const double wb = S->omega * beta;
    int64_t lo, hi;
    block_chunk(n, lo, hi);
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        double pi = r[i] + p[i] * beta - v[i] * wb;
        p[i] = pi;
        if (ph) ph[i] = dinv[i] * pi;
    }
}

// (c): alpha = rho / rhat.v ; s = r - alpha v ; sh = M^-1 s
__global__ void __launch_bounds__(kThreads)
k_bicg_s(int64_t n, const double *__restrict__ partials, int np, KrylovScalars *S, int parity,
         const double *__restrict__ r, const double *__restrict__ v, double *__restrict__ s, double *__restrict__ sh,
         const double *__restrict__ dinv) {
    __shared__ double sm[kThreads / 32 + 1];
    if (read_flag(&S->flag)) return;
    const double rv = reduce_partials<kThreads>(partials, np, 1, 0, sm);
    const double alpha = S->rho[parity ^ 1] / rv;
    if (!isfinite(alpha)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) S->flag = isfinite(rv) ? BF_BREAKDOWN : BF_NAN;
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) S->alpha = alpha;
    int64_t lo, hi;
    block_chunk(n, lo, hi);
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        double si = r[i] - v[i] * alpha;
        s[i] = si;
        if (sh) sh[i] = dinv[i] * si;
    }
}

// (e): omega, x and r updates, partials of rhat.r and r.r (stride 2)
__global__ void __launch_bounds__(kThreads)
k_bicg_x(int64_t n, const double *__restrict__ partials, int np, KrylovScalars *S, double *__restrict__ x,
         double *__restrict__ r, const double *__restrict__ rhat, const double *__restrict__ ph,
         const double *__restrict__ sh, const double *__restrict__ s, const double *__restrict__ t,
         double *__restrict__ partials_out) {
    __shared__ double sm[kThreads / 32 + 1];
    if (read_flag(&S->flag)) return;
    const double ts = reduce_partials<kThreads>(partials, np, 2, 0, sm);
    const double tt = reduce_partials<kThreads>(partials, np, 2, 1, sm);
    const double omega = (tt == 0) ? 0.0 : ts / tt;
    const double alpha = S->alpha;
    int64_t lo, hi;
    block_chunk(n, lo, hi);
    double s0 = 0, s1 = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        x[i] += ph[i] * alpha + sh[i] * omega;  // M^-1 p and M^-1 s (p and s without M)
        double ri = s[i] - t[i] * omega;
        r[i] = ri;
        s0 += rhat[i] * ri;
        s1 += ri * ri;
    }
    s0 = block_sum<kThreads>(s0, sm);
    s1 = block_sum<kThreads>(s1, sm);
    if (threadIdx.x == 0) {
        partials_out[2 * blockIdx.x] = s0;
        partials_out[2 * blockIdx.x + 1] = s1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->omega = omega;
        S->iter += 1;
    }
}

__global__ void k_axmb(int64_t n, const double *__restrict__ q, const double *__restrict__ b, double *__restrict__ u) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        u[i] = q[i] - b[i];
}

__global__ void k_copyv(int64_t n, const double *__restrict__ a, double *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

static yg_status read_s(yg_context ctx, KrylovScalars *out) {
    YG_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_scalars, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, ctx->stream));
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    memcpy(out, ctx->h_pinned, sizeof(KrylovScalars));
    return YG_OK;
}

struct BGraph {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    int64_t kernels = 0;
    int iters = 0;
    ~BGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

yg_status solve_bicgstab(yg_matrix A, yg_precond M, yg_vector bv, yg_vector xv, const yg_solve_opts *opts,
                         yg_solve_stats *stats) {
    yg_context ctx = A->ctx;
    const int64_t n = A->rows();
    yg_solve_opts o = opts ? *opts : yg_solve_opts{YG_CRIT_REFERENCE, YG_PREC_FP64, 1e-14, 0, 0, 0};
    if (o.precision != YG_PREC_FP64) return fail(YG_UNSUPPORTED, "BiCGSTAB supports FP64 only");
    if (M && !precond_fusable(M)) return fail(YG_UNSUPPORTED, "BiCGSTAB takes Jacobi or identity preconditioning");
    const double *dinv = precond_dinv(M);
    const int64_t maxiter = o.maxiter > 0 ? o.maxiter : 100 * n + 1000;
    const int G = ctx->reduce_blocks;
    // SpMV grid = partials count: up to 2G, so that r^.v (at [2G, 2G+SG)) and
    // s.t, t.t (at [4G, 4G+2SG)) stay inside their regions and below b.b
    const int SG = std::min(spmv_default_grid(A), 2 * G);
    cudaStream_t st = ctx->stream;
    double *P = ctx->d_partials;
    KrylovScalars *S = ctx->d_scalars;
    double *r = nullptr, *rhat = nullptr, *p = nullptr, *v = nullptr, *s = nullptr, *t = nullptr, *ph = nullptr,
           *sh = nullptr, *q = nullptr;
    auto cleanup = [&]() { for (double *ptr : {r, rhat, p, v, s, t, ph, sh, q}) dev_free(ctx, ptr); };
    yg_status ss;
#define TRYB(x) do { ss = (x); if (ss != YG_OK) { cleanup(); return ss; } } while (0)
    for (double **ptr : {&r, &rhat, &p, &v, &s, &t, &q}) TRYB(dev_alloc_t(ctx, ptr, n + 1));
    if (dinv) { TRYB(dev_alloc_t(ctx, &ph, n + 1)); TRYB(dev_alloc_t(ctx, &sh, n + 1)); }
    double *pin = dinv ? ph : p, *sin = dinv ? sh : s;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    yg_solve_stats stt{};
    int flag = BF_RUN;

    // The reference returns b itself when b.b < TOL (bicgstab_solve.hpp:229-233).
    double bb0 = 0;
    TRYB(vector_dot(ctx, bv->d, bv->d, n, &bb0));
    if (o.criterion == YG_CRIT_REFERENCE && bb0 < o.tol) {
        k_copyv<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, bv->d, xv->d);
        YG_LAUNCHED(ctx);
        flag = BF_CONVERGED;
    } else {
        // P layout: [0,2G) rhat.r/r.r ; [2G,3G) rhat.v ; [4G,6G) s.t/t.t ; b.b at 2*kMax
        auto init = [&](int64_t iters_left) -> yg_status {
            YG_TRY(spmv_launch(A, xv->d, q, YG_PREC_FP64, nullptr, nullptr, spmv_default_grid(A)));
            k_bicg_init<<<G, kThreads, 0, st>>>(n, bv->d, q, r, rhat, p, v, P);
            YG_LAUNCHED(ctx);
            k_bicg_scalars_init<<<1, kThreads, 0, st>>>(S, P, G, o.tol, iters_left, o.criterion);
            YG_LAUNCHED(ctx);
            return YG_OK;
        };
        TRYB(init(maxiter));
        auto one = [&](int parity) -> yg_status {
            k_bicg_p<<<G, kThreads, 0, st>>>(n, P, G, S, parity, p, r, v, ph, dinv);
            YG_LAUNCHED(ctx);
            YG_TRY(spmv_launch_ex(A, pin, v, YG_PREC_FP64, rhat, P + 2 * G, 1, &S->flag, SG));
            k_bicg_s<<<G, kThreads, 0, st>>>(n, P + 2 * G, SG, S, parity, r, v, s, sh, dinv);
            YG_LAUNCHED(ctx);
            YG_TRY(spmv_launch_ex(A, sin, t, YG_PREC_FP64, s, P + 4 * G, 2, &S->flag, SG));
            k_bicg_x<<<G, kThreads, 0, st>>>(n, P + 4 * G, SG, S, xv->d, r, rhat, pin, sin, s, t, P);
            YG_LAUNCHED(ctx);
            return YG_OK;
        };
        auto build = [&](int m, BGraph &g) -> yg_status {
            int64_t before = ctx->launches;
            YG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            yg_status s2 = YG_OK;
            for (int it = 0; it < m && s2 == YG_OK; ++it) s2 = one(it & 1);
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamEndCapture(st, &graph);
            g.kernels = ctx->launches - before;
            ctx->launches = before;
            if (s2 != YG_OK) { if (graph) cudaGraphDestroy(graph); return s2; }
            if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "capture: %s", cudaGetErrorString(e));
            g.graph = graph;
            g.iters = m;
            YG_CUDA(cudaGraphInstantiate(&g.exec, graph, 0));
            return YG_OK;
        };
        auto replay = [&](BGraph &g, int64_t &it) -> yg_status {
            YG_CUDA(cudaGraphLaunch(g.exec, st));
            ctx->launches += g.kernels;
            it += g.iters;
            return YG_OK;
        };
        KrylovScalars hs;
        TRYB(read_s(ctx, &hs));
        flag = hs.flag;
        if (flag == BF_RUN) {
            if (o.criterion == YG_CRIT_RELRES) {
                int m = o.check_every > 0 ? o.check_every : 16;
                if (m & 1) ++m;
                BGraph g;
                TRYB(build(m, g));
                int64_t total = 0;
                // The recursive residual triggers the stop; the FP64 true residual
                // decides.  If they drifted apart, or the iteration broke down
                // (rho or omega vanished), restart from the true residual with
                // r^ = r, at most 8 times (as the batched BiCGSTAB does).
                for (int restart = 0; restart < 8; ++restart) {
                    int64_t it = 0;
                    for (;;) {
                        TRYB(replay(g, it));
                        TRYB(read_s(ctx, &hs));
                        if (hs.flag != BF_RUN) break;
                    }
                    total += hs.iter;
                    flag = hs.flag;
                    if (flag != BF_CONVERGED && flag != BF_BREAKDOWN) break;
                    TRYB(spmv_launch(A, xv->d, q, YG_PREC_FP64, nullptr, nullptr, spmv_default_grid(A)));
                    k_axmb<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, q, bv->d, q);
                    YG_LAUNCHED(ctx);
                    double rr = 0;
                    TRYB(vector_dot(ctx, q, q, n, &rr));
                    if (std::sqrt(rr) <= o.tol * std::sqrt(bb0)) {
                        flag = BF_CONVERGED;
                        break;
                    }
                    if (total >= maxiter) { flag = BF_MAXITER; break; }
                    TRYB(init(maxiter - total));
                    TRYB(read_s(ctx, &hs));
                }
                hs.iter = total;
            } else {
                // true residual ||Ax-b||^2/||b||^2 after iterations k = 0, f, 2f, ...
                const int64_t freq = (n / 100 > 1) ? n / 100 : 1;
                BGraph g1, g32, gr;
                TRYB(build(1, g1));  // parity bookkeeping: graphs with odd counts alternate parity
                // Parity of the next iteration must be tracked: build both-parity singles.
                BGraph g1b;
                {
                    int64_t before = ctx->launches;
                    YG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                    yg_status s2 = one(1);
                    cudaGraph_t graph = nullptr;
                    cudaError_t e = cudaStreamEndCapture(st, &graph);
                    g1b.kernels = ctx->launches - before;
                    ctx->launches = before;
                    if (s2 != YG_OK || e != cudaSuccess) { cleanup(); return s2 != YG_OK ? s2 : fail(YG_CUDA_ERROR, "capture"); }
                    g1b.graph = graph;
                    g1b.iters = 1;
                    YG_CUDA(cudaGraphInstantiate(&g1b.exec, graph, 0));
                }
                TRYB(build(32, g32));
                int64_t it = 0;  // iterations done == k of the next iteration
                auto run_iters = [&](int64_t cnt) -> yg_status {
                    while (cnt > 0) {
                        if (cnt >= 32 && (it & 1) == 0) { YG_TRY(replay(g32, it)); cnt -= 32; }
                        else { YG_TRY(replay((it & 1) ? g1b : g1, it)); cnt -= 1; }
                    }
                    return YG_OK;
                };
                double res0 = bb0;
                for (;;) {
                    TRYB(run_iters(1));  // iteration k (k % freq == 0) followed by the check
                    TRYB(read_s(ctx, &hs));
                    if (hs.flag != BF_RUN) break;
                    TRYB(spmv_launch(A, xv->d, q, YG_PREC_FP64, nullptr, nullptr, spmv_default_grid(A)));
                    k_axmb<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, q, bv->d, q);
                    YG_LAUNCHED(ctx);
                    double res = 0;
                    TRYB(vector_dot(ctx, q, q, n, &res));
                    if (res / res0 < o.tol) { hs.flag = BF_CONVERGED; break; }
                    if (it >= maxiter) { hs.flag = BF_MAXITER; break; }
                    TRYB(run_iters(freq - 1));
                    TRYB(read_s(ctx, &hs));
                    if (hs.flag != BF_RUN) break;
                }
                flag = hs.flag;
            }
        }
        stt.iterations = hs.iter;
    }
    cudaEventRecord(e1, st);
    // final FP64 true residual
    TRYB(spmv_launch(A, xv->d, q, YG_PREC_FP64, nullptr, nullptr, spmv_default_grid(A)));
    k_axmb<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, q, bv->d, q);
    YG_LAUNCHED(ctx);
    double rr = 0;
    TRYB(vector_dot(ctx, q, q, n, &rr));
    float ms = 0;
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cleanup();
#undef TRYB
    stt.rel_residual = bb0 > 0 ? std::sqrt(rr / bb0) : std::sqrt(rr);
    stt.device_ms = ms;
    yg_status res = YG_NOT_CONVERGED;
    if (flag == BF_CONVERGED) res = YG_OK;
    else if (flag == BF_BREAKDOWN) res = YG_BREAKDOWN;
    else if (flag == BF_NAN) res = YG_NAN;
    if (o.criterion == YG_CRIT_RELRES && res == YG_OK && !(stt.rel_residual <= o.tol * 1.0000001)) res = YG_NOT_CONVERGED;
    stt.status = res;
    if (stats) *stats = stt;
    return res;
}

}  // namespace yg

using namespace yg;

extern "C" yg_status yg_bicgstab(yg_matrix A, yg_precond M, yg_vector b, yg_vector x, const yg_solve_opts *opts,
                                 yg_solve_stats *stats) {
    if (!A || !b || !x) return fail(YG_BAD_ARG, "yg_bicgstab: NULL argument");
    if (A->rows() != A->cols() || b->n != A->rows() || x->n != A->rows())
        return fail(YG_BAD_ARG, "yg_bicgstab: dimension mismatch");
    YG_TRY(spmv_autotune_device(A));
    yg_status s = solve_bicgstab(A, M, b, x, opts, stats);
    if (s != YG_OK && s != YG_UNSUPPORTED && s < YG_TIMEOUT) set_error("yg_bicgstab: %s", yg_status_string(s));
    return s;
}
