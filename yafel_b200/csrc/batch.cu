// batch.cu -- many independent systems solved together (batched / served PCG).
//
// No reference counterpart: the reference solves one system per call
// (pcg_solve.hpp:126-178).  Each system keeps its own matrix (CSR or BCSR with
// 2x2 / 3x3 blocks), right-hand side, iterate and work vectors; a device table
// of system descriptors and a table of work items (row ranges of one system)
// drive persistent-grid kernels that advance every active system by one Jacobi-
// PCG iteration:
//   SpMV (one launch per block size present) with per-item partials of p.Ap,
//   update   : every CTA of a system reduces that system's items in a fixed order
//              -> alpha_s; x, r update; Jacobi z; partials of r.z, r.r
//   pupdate  : -> beta_s; p update; the CTA of the system's first item records
//              the scalars and a stop reason.
// Converged systems drop out of the iteration kernels at once.  A block of m
// iterations plus a verification pass is captured into one CUDA graph and
// replayed; the verification pass recomputes b - A x in FP64 for systems whose
// recursive residual converged (stop) or, in mixed precision, fell 10x since
// the last replacement (replace), and for newly added systems (init).  Systems
// can be added and removed between replays (continuous batching): only the
// descriptor and item tables change, and kernels read their item counts from
// device memory, so the captured graph stays valid while the set of block
// sizes present does not change.
#include "internal.h"
#include "device_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace yg {
int stream_grid(yg_context ctx, int64_t n);
yg_status spmv_autotune_device(yg_matrix A);
}

enum BatchFlag : int32_t { BF_RUN = 0, BF_DONE = 1, BF_BREAK = 2, BF_NANF = 3, BF_MAXIT = 4, BF_INIT = 5, BF_EMPTY = 6 };
enum BatchStop : int32_t { BS_NONE = 0, BS_CONV = 1, BS_BREAK = 2, BS_NAN = 3, BS_MAXIT = 4 };

struct BatchSys {
    int32_t block, nbrows;
    const int32_t *rowptr, *col;
    const double *val;
    const float *val32;
    const double *b, *dinv;
    double *x, *r, *p, *q;
    int32_t item_begin, item_end;
    int32_t precision;  // YG_PREC_FP64 or YG_PREC_MIXED
    int32_t pad;
};

struct BatchScal {
    double rz[2];
    double bb, rr, rr_last, tol;
    int64_t iter, maxiter;
    int32_t flag, stop, replace, restart;
    int64_t replacements;
    double true_rr;  // r.r of the last FP64 true residual
};

struct BatchItem {
    int32_t sys, brow_begin, brow_end, pad;
};

struct yg_batch_t {
    yg_context ctx = nullptr;
    int32_t capacity = 0;
    std::vector<BatchSys> sys;          // host mirror
    std::vector<int32_t> used;          // slot in use
    std::vector<yg_matrix> mats;
    std::vector<yg_solve_opts> opts;
    BatchSys *d_sys = nullptr;
    BatchScal *d_scal = nullptr;
    BatchItem *d_items = nullptr;
    int32_t *d_ranges = nullptr;        // [4]: item offsets of block sizes 1,2,3 and the end
    double *d_part = nullptr;           // partials: 2 per item
    double *d_part2 = nullptr;
    int32_t max_items = 0, n_items = 0;
    int32_t group_rows[4] = {0, 0, 0, 0};  // rows per item per block size
    int32_t lanes[4] = {4, 4, 4, 4};
    unsigned groups_present = 0, graph_groups = 0;
    int m = 16;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    int64_t graph_kernels = 0;
    std::vector<BatchScal> h_scal;
};

namespace yg {

// ---------------------------------------------------------------- kernels

// Whether system state `sc` takes part in a kernel of the given kind, decided
// once per CTA: thread 0 reads the state (a peer CTA of the same system may
// change `stop` during update/pupdate) and broadcasts it, so every thread of the
// CTA takes the same branch around the block reductions.
enum { ACT_ITER = 0, ACT_VERIFY = 1, ACT_RESTART = 2 };
__device__ __forceinline__ bool cta_active(const BatchScal *sc, int kind, int *flag_sm) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const volatile BatchScal *v = sc;
        const int flag = v->flag, stop = v->stop, rep = v->replace, rst = v->restart;
        int a;
        if (kind == ACT_ITER) a = (flag == BF_RUN && stop == BS_NONE);
        else if (kind == ACT_VERIFY) a = (flag == BF_INIT) || (flag == BF_RUN && (stop == BS_CONV || rep));
        else a = rst != 0;
        *flag_sm = a;
    }
    __syncthreads();
    return *flag_sm != 0;
}

// Reduce the partials of system s (items [ib, ie), stride 2, offset off).
__device__ __forceinline__ double sys_reduce(const double *__restrict__ part, int ib, int ie, int off, double *sm) {
    double v = 0;
    for (int i = ib + threadIdx.x; i < ie; i += blockDim.x) v += part[2 * (int64_t)i + off];
    return block_sum_all<kThreads>(v, sm);
}

// MODE 0: iteration, q = A p (FP32 or FP64 values), partials of p.q.
// MODE 1: verification, q = A x with FP64 values for systems being initialised,
//         stopped on a converged recursive residual, or due a replacement.
template <int B, int L, int MODE>
__global__ void __launch_bounds__(kThreads)
k_batch_spmv(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
             const BatchScal *__restrict__ scal, double *__restrict__ part) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int act;
    constexpr int B2 = B * B;
    constexpr int GPB = kThreads / L;  // row groups per CTA
    const int g0 = ranges[B - 1], g1 = ranges[B];
    const int lane = threadIdx.x & 31, glane = lane % L;
    const int grp = threadIdx.x / L;
    for (int it = g0 + blockIdx.x; it < g1; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        if (!cta_active(&scal[s], MODE == 0 ? ACT_ITER : ACT_VERIFY, &act)) continue;
        const BatchSys d = sys[s];
        const double *xin = MODE == 0 ? d.p : d.x;
        const bool f32 = (MODE == 0 && d.precision == YG_PREC_MIXED);
        double dot = 0;
        for (int rb = item.brow_begin; rb < item.brow_end; rb += GPB) {
            const int r = rb + grp;
            double acc[B];
#pragma unroll
            for (int i = 0; i < B; ++i) acc[i] = 0;
            if (r < item.brow_end) {
                const int rs = d.rowptr[r], re = d.rowptr[r + 1];
                const int nv = (re - rs) * B2;
                int j = glane / B2, e = glane % B2;
                for (int k = glane; k < nv; k += L) {
                    const double v = f32 ? (double)d.val32[(int64_t)rs * B2 + k] : d.val[(int64_t)rs * B2 + k];
                    const int i = e / B, c = e - (e / B) * B;
                    const double xv = xin[(int64_t)B * d.col[rs + j] + c];
#pragma unroll
                    for (int ii = 0; ii < B; ++ii) acc[ii] = (ii == i) ? fma(v, xv, acc[ii]) : acc[ii];
                    e += L % B2;
                    j += L / B2;
                    if (e >= B2) { e -= B2; ++j; }
                }
            }
#pragma unroll
            for (int i = 0; i < B; ++i) {
#pragma unroll
                for (int o = L / 2; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
            }
            if (r < item.brow_end && glane == 0) {
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    d.q[(int64_t)B * r + i] = acc[i];
                    if (MODE == 0) dot = fma(acc[i], xin[(int64_t)B * r + i], dot);
                }
            }
        }
        if (MODE == 0) {
            dot = block_sum<kThreads>(dot, sm);
            if (threadIdx.x == 0) part[2 * (int64_t)it] = dot;
        }
    }
}

// alpha, x and r updates, Jacobi z, partials of r.z and r.r
__global__ void __launch_bounds__(kThreads)
k_batch_update(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
               BatchScal *__restrict__ scal, int parity, const double *__restrict__ part_in, double *__restrict__ part_out) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int act;
    const int n_items = ranges[3];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        BatchScal &sc = scal[s];
        if (!cta_active(&sc, ACT_ITER, &act)) continue;
        const BatchSys d = sys[s];
        const double pq = sys_reduce(part_in, d.item_begin, d.item_end, 0, sm);
        const double alpha = sc.rz[parity] / pq;
        if (pq == 0 || !isfinite(alpha)) {
            if (it == d.item_begin && threadIdx.x == 0) sc.stop = isfinite(pq) ? BS_BREAK : BS_NAN;
            continue;
        }
        // the iteration count changes here, not in pupdate, whose CTAs all read it
        if (it == d.item_begin && threadIdx.x == 0) sc.iter += 1;
        const int64_t lo = (int64_t)item.brow_begin * d.block, hi = (int64_t)item.brow_end * d.block;
        double srz = 0, srr = 0;
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            d.x[i] += d.p[i] * alpha;
            const double ri = d.r[i] + (-alpha) * d.q[i];
            d.r[i] = ri;
            srz += ri * (d.dinv[i] * ri);
            srr += ri * ri;
        }
        srz = block_sum<kThreads>(srz, sm);
        srr = block_sum<kThreads>(srr, sm);
        if (threadIdx.x == 0) {
            part_out[2 * (int64_t)it] = srz;
            part_out[2 * (int64_t)it + 1] = srr;
        }
    }
}

// beta and p update; the first item's CTA records the scalars and stop reason
__global__ void __launch_bounds__(kThreads)
k_batch_pupdate(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
                BatchScal *__restrict__ scal, int parity, const double *__restrict__ part) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int act;
    const int n_items = ranges[3];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        BatchScal &sc = scal[s];
        // a peer CTA of this system may set `stop` during this kernel; it only
        // does so when the decision below is also to stop, so skipping is consistent
        if (!cta_active(&sc, ACT_ITER, &act)) continue;
        const BatchSys d = sys[s];
        const double rz_new = sys_reduce(part, d.item_begin, d.item_end, 0, sm);
        const double rr = sys_reduce(part, d.item_begin, d.item_end, 1, sm);
        const double rz_old = sc.rz[parity];
        int stop = BS_NONE;
        if (sqrt(rr) <= sc.tol * sqrt(sc.bb)) stop = BS_CONV;
        else if (!isfinite(rz_new)) stop = BS_NAN;
        else if (sc.iter >= sc.maxiter) stop = BS_MAXIT;
        const bool rep = (stop == BS_NONE && d.precision == YG_PREC_MIXED && rr < 1e-2 * sc.rr_last);
        if (it == d.item_begin && threadIdx.x == 0) {
            sc.rz[parity ^ 1] = rz_new;
            sc.rr = rr;
            if (stop != BS_NONE) sc.stop = stop;
            if (rep) sc.replace = 1;
        }
        if (stop != BS_NONE) continue;
        const double beta = rz_new / rz_old;
        const int64_t lo = (int64_t)item.brow_begin * d.block, hi = (int64_t)item.brow_end * d.block;
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) d.p[i] = d.dinv[i] * d.r[i] + beta * d.p[i];
    }
}

// verification, step 2: r = b - q (q = A x from the MODE 1 SpMV), partials of r.z,
// r.r (and b.b for systems being initialised) for the systems under verification
__global__ void __launch_bounds__(kThreads)
k_batch_residual(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
                 const BatchScal *__restrict__ scal, double *__restrict__ part, double *__restrict__ part_bb) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int act;
    const int n_items = ranges[3];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        if (!cta_active(&scal[s], ACT_VERIFY, &act)) continue;
        const BatchSys d = sys[s];
        const int64_t lo = (int64_t)item.brow_begin * d.block, hi = (int64_t)item.brow_end * d.block;
        double srz = 0, srr = 0, sbb = 0;
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const double ri = d.b[i] - d.q[i];
            d.r[i] = ri;
            srz += ri * (d.dinv[i] * ri);
            srr += ri * ri;
            sbb += d.b[i] * d.b[i];
        }
        srz = block_sum<kThreads>(srz, sm);
        srr = block_sum<kThreads>(srr, sm);
        sbb = block_sum<kThreads>(sbb, sm);
        if (threadIdx.x == 0) {
            part[2 * (int64_t)it] = srz;
            part[2 * (int64_t)it + 1] = srr;
            part_bb[2 * (int64_t)it] = sbb;
        }
    }
}

// verification, step 3 (one thread per system): decisions
__global__ void k_batch_decide(int cap, const BatchSys *__restrict__ sys, BatchScal *__restrict__ scal,
                               const double *__restrict__ part, const double *__restrict__ part_bb) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= cap) return;
    BatchScal &sc = scal[s];
    sc.restart = 0;
    if (sc.flag == BF_RUN && (sc.stop == BS_BREAK || sc.stop == BS_NAN || sc.stop == BS_MAXIT)) {
        sc.flag = sc.stop == BS_BREAK ? BF_BREAK : (sc.stop == BS_NAN ? BF_NANF : BF_MAXIT);
        return;
    }
    const bool init = sc.flag == BF_INIT;
    const bool ver = sc.flag == BF_RUN && (sc.stop == BS_CONV || sc.replace);
    if (!init && !ver) return;
    const BatchSys d = sys[s];
    double rz = 0, rr = 0, bb = 0;
    for (int i = d.item_begin; i < d.item_end; ++i) {
        rz += part[2 * (int64_t)i];
        rr += part[2 * (int64_t)i + 1];
        bb += part_bb[2 * (int64_t)i];
    }
    if (init) sc.bb = bb;
    sc.true_rr = rr;
    sc.rr = rr;
    sc.rr_last = rr;
    sc.rz[0] = sc.rz[1] = rz;
    sc.replacements += (init ? 0 : 1);
    const bool conv = sqrt(rr) <= sc.tol * sqrt(sc.bb);
    if (init) {
        sc.flag = (conv || rz == 0) ? BF_DONE : BF_RUN;
        sc.stop = BS_NONE;
        sc.restart = conv ? 0 : 1;  // p = z
    } else if (sc.stop == BS_CONV) {
        if (conv) {
            sc.flag = BF_DONE;
        } else {
            sc.stop = BS_NONE;   // continue from the true residual with p = z
            sc.restart = 1;
            if (sc.iter >= sc.maxiter) sc.flag = BF_MAXIT;
        }
    }
    sc.replace = 0;
}

// verification, step 4: p = z for restarted systems
__global__ void __launch_bounds__(kThreads)
k_batch_restart(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
                const BatchScal *__restrict__ scal) {
    __shared__ int act;
    const int n_items = ranges[3];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        if (!cta_active(&scal[s], ACT_RESTART, &act)) continue;
        const BatchSys d = sys[s];
        const int64_t lo = (int64_t)item.brow_begin * d.block, hi = (int64_t)item.brow_end * d.block;
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) d.p[i] = d.dinv[i] * d.r[i];
    }
}

__global__ void k_batch_jacobi(int64_t nbrows, int B, const int32_t *__restrict__ diag, const double *__restrict__ val,
                               double *__restrict__ dinv) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nbrows * B; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = r / B, i = r % B;
        const int32_t dp = diag[I];
        const double a = dp >= 0 ? val[(int64_t)dp * B * B + i * B + i] : 0.0;
        dinv[r] = 1.0 / a;
    }
}

// ---------------------------------------------------------------- host

static int batch_grid(yg_context ctx) { return ctx->num_sms * 4; }

template <int B, int MODE>
static void launch_bspmv(yg_batch bt, int L) {
    yg_context ctx = bt->ctx;
    const int g = batch_grid(ctx);
    switch (L) {
    case 2: k_batch_spmv<B, 2, MODE><<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_part); break;
    case 4: k_batch_spmv<B, 4, MODE><<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_part); break;
    case 8: k_batch_spmv<B, 8, MODE><<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_part); break;
    case 16: k_batch_spmv<B, 16, MODE><<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_part); break;
    default: k_batch_spmv<B, 32, MODE><<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_part); break;
    }
    YG_LAUNCHED(ctx);
}

template <int MODE>
static void launch_bspmv_groups(yg_batch bt) {
    if (bt->groups_present & 1) launch_bspmv<1, MODE>(bt, bt->lanes[1]);
    if (bt->groups_present & 2) launch_bspmv<2, MODE>(bt, bt->lanes[2]);
    if (bt->groups_present & 4) launch_bspmv<3, MODE>(bt, bt->lanes[3]);
}

// the verification pass (also initialises newly added systems)
static void launch_verify(yg_batch bt) {
    yg_context ctx = bt->ctx;
    const int g = batch_grid(ctx);
    launch_bspmv_groups<1>(bt);
    k_batch_residual<<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_part,
                                                     bt->d_part2);
    YG_LAUNCHED(ctx);
    k_batch_decide<<<(bt->capacity + 127) / 128, 128, 0, ctx->stream>>>(bt->capacity, bt->d_sys, bt->d_scal, bt->d_part,
                                                                         bt->d_part2);
    YG_LAUNCHED(ctx);
    k_batch_restart<<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal);
    YG_LAUNCHED(ctx);
}

static void launch_iteration(yg_batch bt, int parity) {
    yg_context ctx = bt->ctx;
    const int g = batch_grid(ctx);
    launch_bspmv_groups<0>(bt);
    k_batch_update<<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, parity, bt->d_part,
                                                   bt->d_part2);
    YG_LAUNCHED(ctx);
    k_batch_pupdate<<<g, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, parity,
                                                    bt->d_part2);
    YG_LAUNCHED(ctx);
}

static void drop_graph(yg_batch bt) {
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    bt->exec = nullptr;
    bt->graph = nullptr;
}

// Rebuild the item table: systems grouped by block size, rows cut into items.
static yg_status rebuild_items(yg_batch bt) {
    yg_context ctx = bt->ctx;
    std::vector<BatchItem> items;
    int32_t ranges[4] = {0, 0, 0, 0};
    unsigned present = 0;
    for (int B = 1; B <= 3; ++B) {
        ranges[B - 1] = (int32_t)items.size();
        const int R = bt->group_rows[B];
        for (int s = 0; s < bt->capacity; ++s) {
            if (!bt->used[s] || bt->sys[s].block != B) continue;
            present |= 1u << (B - 1);
            bt->sys[s].item_begin = (int32_t)items.size();
            for (int r0 = 0; r0 < bt->sys[s].nbrows; r0 += R)
                items.push_back({s, r0, std::min(bt->sys[s].nbrows, r0 + R), 0});
            if (bt->sys[s].nbrows == 0) items.push_back({s, 0, 0, 0});
            bt->sys[s].item_end = (int32_t)items.size();
        }
    }
    // items were appended by block size, so group b is [ranges[b-1], ranges[b])
    {
        int32_t cnt[4] = {0, 0, 0, 0};
        for (auto &it : items) cnt[bt->sys[it.sys].block]++;
        ranges[0] = 0;
        ranges[1] = cnt[1];
        ranges[2] = cnt[1] + cnt[2];
        ranges[3] = cnt[1] + cnt[2] + cnt[3];
    }
    if ((int32_t)items.size() > bt->max_items) {
        dev_free(ctx, bt->d_items);
        dev_free(ctx, bt->d_part);
        dev_free(ctx, bt->d_part2);
        bt->d_items = nullptr;
        bt->d_part = bt->d_part2 = nullptr;
        int32_t cap = (int32_t)items.size() * 2 + 64;
        YG_TRY(dev_alloc_t(ctx, &bt->d_items, cap));
        YG_TRY(dev_alloc_t(ctx, &bt->d_part, 2 * (size_t)cap));
        YG_TRY(dev_alloc_t(ctx, &bt->d_part2, 2 * (size_t)cap));
        bt->max_items = cap;
        drop_graph(bt);  // the graph captured the old pointers
    }
    bt->n_items = (int32_t)items.size();
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (!items.empty())
        YG_CUDA(cudaMemcpy(bt->d_items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice));
    YG_CUDA(cudaMemcpy(bt->d_ranges, ranges, sizeof(ranges), cudaMemcpyHostToDevice));
    YG_CUDA(cudaMemcpy(bt->d_sys, bt->sys.data(), sizeof(BatchSys) * bt->capacity, cudaMemcpyHostToDevice));
    bt->groups_present = present;
    return YG_OK;
}

static yg_status capture_graph(yg_batch bt) {
    yg_context ctx = bt->ctx;
    drop_graph(bt);
    int64_t before = ctx->launches;
    YG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < bt->m; ++it) launch_iteration(bt, it & 1);
    launch_verify(bt);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    bt->graph_kernels = ctx->launches - before;
    ctx->launches = before;
    if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "batch graph capture: %s", cudaGetErrorString(e));
    bt->graph = g;
    YG_CUDA(cudaGraphInstantiate(&bt->exec, g, 0));
    bt->graph_groups = bt->groups_present;
    return YG_OK;
}

static void release_slot(yg_batch bt, int s) {
    yg_context ctx = bt->ctx;
    BatchSys &d = bt->sys[s];
    for (void *ptr : {(void *)d.r, (void *)d.p, (void *)d.q, (void *)d.dinv}) dev_free(ctx, ptr);
    d = BatchSys{};
    bt->used[s] = 0;
    bt->mats[s] = nullptr;
}

}  // namespace yg

using namespace yg;

extern "C" yg_status yg_batch_create(yg_context ctx, int32_t capacity, yg_batch *out) {
    if (!ctx || !out || capacity < 1) return fail(YG_BAD_ARG, "yg_batch_create: bad argument");
    auto *bt = new yg_batch_t();
    bt->ctx = ctx;
    bt->capacity = capacity;
    bt->sys.assign(capacity, BatchSys{});
    bt->used.assign(capacity, 0);
    bt->mats.assign(capacity, nullptr);
    bt->opts.assign(capacity, yg_solve_opts{});
    bt->h_scal.assign(capacity, BatchScal{});
    bt->group_rows[1] = 1024;
    bt->group_rows[2] = 512;
    bt->group_rows[3] = 256;
    bt->lanes[1] = 4;
    bt->lanes[2] = 8;
    bt->lanes[3] = 16;
    yg_status s;
    if ((s = dev_alloc_t(ctx, &bt->d_sys, capacity)) != YG_OK || (s = dev_alloc_t(ctx, &bt->d_scal, capacity)) != YG_OK ||
        (s = dev_alloc_t(ctx, &bt->d_ranges, 4)) != YG_OK) {
        yg_batch_destroy(bt);
        return s;
    }
    std::vector<BatchScal> init(capacity);
    for (auto &c : init) c.flag = BF_EMPTY;
    cudaMemcpy(bt->d_scal, init.data(), sizeof(BatchScal) * capacity, cudaMemcpyHostToDevice);
    cudaMemset(bt->d_ranges, 0, sizeof(int32_t) * 4);
    *out = bt;
    return YG_OK;
}

extern "C" yg_status yg_batch_destroy(yg_batch bt) {
    if (!bt) return YG_OK;
    cudaStreamSynchronize(bt->ctx->stream);
    drop_graph(bt);
    for (int s = 0; s < bt->capacity; ++s)
        if (bt->used[s]) release_slot(bt, s);
    for (void *p : {(void *)bt->d_sys, (void *)bt->d_scal, (void *)bt->d_items, (void *)bt->d_ranges, (void *)bt->d_part,
                    (void *)bt->d_part2})
        dev_free(bt->ctx, p);
    delete bt;
    return YG_OK;
}

extern "C" yg_status yg_batch_add(yg_batch bt, yg_matrix A, yg_vector b, yg_vector x, const yg_solve_opts *opts,
                                  int32_t *slot) {
    if (!bt || !A || !b || !x || !slot) return fail(YG_BAD_ARG, "yg_batch_add: NULL argument");
    if (A->ctx != bt->ctx || b->ctx != bt->ctx || x->ctx != bt->ctx) return fail(YG_BAD_ARG, "yg_batch_add: context mismatch");
    if (A->rows() != A->cols() || b->n != A->rows() || x->n != A->rows()) return fail(YG_BAD_ARG, "yg_batch_add: dimension mismatch");
    if (A->block < 1 || A->block > 3) return fail(YG_UNSUPPORTED, "yg_batch_add: block size %d", A->block);
    yg_solve_opts o = opts ? *opts : yg_solve_opts{YG_CRIT_RELRES, YG_PREC_FP64, 1e-10, 0, 0, 0};
    if (o.criterion != YG_CRIT_RELRES) return fail(YG_UNSUPPORTED, "batched solves stop on the relative residual");
    if (o.precision != YG_PREC_FP64 && o.precision != YG_PREC_MIXED) return fail(YG_UNSUPPORTED, "batched precision");
    int s = -1;
    for (int i = 0; i < bt->capacity; ++i)
        if (!bt->used[i]) { s = i; break; }
    if (s < 0) return fail(YG_OVER_BUDGET, "yg_batch_add: all %d slots in use", bt->capacity);
    yg_context ctx = bt->ctx;
    if (o.precision == YG_PREC_MIXED && !A->d_val32) YG_TRY(yg_matrix_make_fp32(A));
    BatchSys d{};
    d.block = A->block;
    d.nbrows = (int32_t)A->nbrows;
    d.rowptr = A->d_rowptr;
    d.col = A->d_col;
    d.val = A->d_val;
    d.val32 = A->d_val32;
    d.b = b->d;
    d.x = x->d;
    d.precision = o.precision;
    const int64_t n = A->rows();
    double *dinv = nullptr;
    yg_status st;
    if ((st = dev_alloc_t(ctx, &d.r, n + 1)) != YG_OK || (st = dev_alloc_t(ctx, &d.p, n + 1)) != YG_OK ||
        (st = dev_alloc_t(ctx, &d.q, n + 1)) != YG_OK || (st = dev_alloc_t(ctx, &dinv, n + 1)) != YG_OK) {
        for (void *ptr : {(void *)d.r, (void *)d.p, (void *)d.q, (void *)dinv}) dev_free(ctx, ptr);
        return st;
    }
    d.dinv = dinv;
    k_batch_jacobi<<<stream_grid(ctx, n), kThreads, 0, ctx->stream>>>(A->nbrows, A->block, A->d_diag, A->d_val, dinv);
    YG_LAUNCHED(ctx);
    BatchScal sc{};
    sc.flag = BF_INIT;
    sc.tol = o.tol;
    sc.maxiter = o.maxiter > 0 ? o.maxiter : n;
    bt->sys[s] = d;
    bt->used[s] = 1;
    bt->mats[s] = A;
    bt->opts[s] = o;
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    YG_CUDA(cudaMemcpy(bt->d_scal + s, &sc, sizeof(BatchScal), cudaMemcpyHostToDevice));
    YG_TRY(rebuild_items(bt));
    *slot = s;
    return YG_OK;
}

extern "C" yg_status yg_batch_remove(yg_batch bt, int32_t slot) {
    if (!bt || slot < 0 || slot >= bt->capacity || !bt->used[slot]) return fail(YG_BAD_ARG, "yg_batch_remove: bad slot");
    YG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
    release_slot(bt, slot);
    BatchScal sc{};
    sc.flag = BF_EMPTY;
    YG_CUDA(cudaMemcpy(bt->d_scal + slot, &sc, sizeof(BatchScal), cudaMemcpyHostToDevice));
    return rebuild_items(bt);
}

// Advance every active system by blocks of m iterations plus a verification
// pass, at most max_blocks blocks (0 = until none is active).  *n_active
// receives the number of systems still running.
extern "C" yg_status yg_batch_run(yg_batch bt, int32_t max_blocks, int32_t *n_active) {
    if (!bt) return fail(YG_BAD_ARG, "yg_batch_run: NULL batch");
    yg_context ctx = bt->ctx;
    if (!bt->exec || bt->graph_groups != bt->groups_present) YG_TRY(capture_graph(bt));
    launch_verify(bt);  // initialise systems added since the last run
    int active = 0;
    for (int blk = 0; max_blocks <= 0 || blk < max_blocks; ++blk) {
        YG_CUDA(cudaGraphLaunch(bt->exec, ctx->stream));
        ctx->launches += bt->graph_kernels;
        YG_CUDA(cudaMemcpyAsync(bt->h_scal.data(), bt->d_scal, sizeof(BatchScal) * bt->capacity, cudaMemcpyDeviceToHost,
                                ctx->stream));
        YG_CUDA(cudaStreamSynchronize(ctx->stream));
        active = 0;
        for (int s = 0; s < bt->capacity; ++s)
            if (bt->used[s] && (bt->h_scal[s].flag == BF_RUN || bt->h_scal[s].flag == BF_INIT)) ++active;
        if (active == 0) break;
    }
    if (n_active) *n_active = active;
    return check_device_error(ctx);
}

extern "C" yg_status yg_batch_stats(yg_batch bt, int32_t slot, yg_solve_stats *out) {
    if (!bt || slot < 0 || slot >= bt->capacity || !out) return fail(YG_BAD_ARG, "yg_batch_stats: bad argument");
    if (!bt->used[slot]) return fail(YG_BAD_ARG, "yg_batch_stats: empty slot");
    YG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
    BatchScal sc;
    YG_CUDA(cudaMemcpy(&sc, bt->d_scal + slot, sizeof(BatchScal), cudaMemcpyDeviceToHost));
    yg_solve_stats st{};
    st.iterations = sc.iter;
    st.rel_residual = sc.bb > 0 ? std::sqrt(sc.true_rr / sc.bb) : std::sqrt(sc.true_rr);
    st.refinements = (int32_t)sc.replacements;
    switch (sc.flag) {
    case BF_DONE: st.status = YG_OK; break;
    case BF_BREAK: st.status = YG_BREAKDOWN; break;
    case BF_NANF: st.status = YG_NAN; break;
    default: st.status = YG_NOT_CONVERGED; break;
    }
    *out = st;
    return YG_OK;
}

// Choose rows per item and lanes per row for each block size from the systems
// present, by timing the iteration SpMV of the whole batch (autotuned tiles).
extern "C" yg_status yg_batch_tune(yg_batch bt) {
    if (!bt) return fail(YG_BAD_ARG, "yg_batch_tune: NULL batch");
    yg_context ctx = bt->ctx;
    // initialise p from a verification pass so the SpMV reads defined data
    YG_TRY(rebuild_items(bt));
    launch_verify(bt);
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int B = 1; B <= 3; ++B) {
        if (!(bt->groups_present & (1u << (B - 1)))) continue;
        float best = 1e30f;
        int bestL = bt->lanes[B], bestR = bt->group_rows[B];
        for (int R : {256, 1024, 4096}) {
            bt->group_rows[B] = R;
            YG_TRY(rebuild_items(bt));
            for (int L : {2, 4, 8, 16, 32}) {
                auto launch = [&]() {
                    if (B == 1) launch_bspmv<1, 0>(bt, L);
                    else if (B == 2) launch_bspmv<2, 0>(bt, L);
                    else launch_bspmv<3, 0>(bt, L);
                };
                launch();
                cudaEventRecord(e0, ctx->stream);
                for (int r = 0; r < 3; ++r) launch();
                cudaEventRecord(e1, ctx->stream);
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) { best = ms; bestL = L; bestR = R; }
            }
        }
        bt->lanes[B] = bestL;
        bt->group_rows[B] = bestR;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    YG_TRY(rebuild_items(bt));
    drop_graph(bt);
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}
