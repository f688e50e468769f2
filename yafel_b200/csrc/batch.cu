// batch.cu -- many independent systems solved together (batched / served Krylov).
//
// No reference counterpart: the reference solves one system per call
// (pcg_solve.hpp:126-178, bicgstab_solve.hpp:19-95).  Each system keeps its own
// matrix (CSR or BCSR with 2x2 / 3x3 blocks), right-hand side, iterate and work
// vectors, and is solved either by Jacobi-PCG (symmetric positive definite
// systems) or by BiCGSTAB with right Jacobi preconditioning (non-symmetric
// ones).  A system's block rows are cut into tiles of whole rows holding at
// most TileCfg<B>::BLOCKS blocks, and runs of consecutive tiles form work items,
// grouped by (method, block size).  Persistent-grid kernels advance every
// active system by one iteration in five steps:
//   V1  BiCGSTAB: p = r + beta (p - omega v), ph = D^-1 p
//   S1  SpMV: PCG q = A p (partials of p.q -> alpha); BiCGSTAB v = A ph
//       (partials of r0.v -> alpha)
//   V2  PCG: x, r updates, z = D^-1 r, partials of r.z, r.r -> beta and the
//       stopping tests; BiCGSTAB: s = r - alpha v, sh = D^-1 s
//   S2  BiCGSTAB SpMV t = A sh (partials of t.s, t.t -> omega)
//   V3  PCG: p = z + beta p; BiCGSTAB: x += alpha ph + omega sh, r = s - omega t,
//       partials of r0.r, r.r -> beta and the stopping tests
// (V1 and S2 are launched only when BiCGSTAB systems are present).  Each SpMV
// CTA streams the tiles of its items through a shared-memory ring filled by
// bulk asynchronous copies (cp.async.bulk + mbarrier).  Every decision about a
// system is taken once, by the CTA that completes the system's last item of a
// kernel (a per-system ticket), so every CTA of the next kernel sees the same
// state.  Sums run in a fixed order over a fixed item decomposition: a system's
// result does not depend on which other systems share the batch.  Converged
// systems drop out of the kernels at once and out of the item table at the next
// compaction.  A block of m iterations plus a verification pass is captured into
// one CUDA graph and replayed; the verification pass recomputes b - A x in FP64
// for systems whose recursive residual converged or broke down (stop), whose
// mixed-precision residual fell 100x since the last replacement (replace), and
// for newly added systems (init).  Systems can be added and removed between
// replays (continuous batching): only the descriptor and item tables change,
// and kernels read their item ranges from device memory, so the captured graph
// stays valid while the set of (method, block size) groups present does not
// change.
#include "internal.h"
#include "device_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace yg {
int stream_grid(yg_context ctx, int64_t n);
}

enum BatchFlag : int32_t { BF_RUN = 0, BF_DONE = 1, BF_BREAK = 2, BF_NANF = 3, BF_MAXIT = 4, BF_INIT = 5, BF_EMPTY = 6 };
enum BatchStop : int32_t { BS_NONE = 0, BS_CONV = 1, BS_BREAK = 2, BS_NAN = 3, BS_MAXIT = 4 };
enum BatchMethod : int32_t { BM_CG = 0, BM_BICG = 1 };
constexpr int kBicgRestarts = 8;  // BiCGSTAB restarts after a breakdown before giving up

struct BatchSys {
    int32_t block, nbrows;
    const int32_t *rowptr, *col;
    const double *val;
    const float *val32;
    const double *b, *dinv;
    double *x, *r, *p, *q;        // q: SpMV output of PCG and of the verification (BiCGSTAB: q is t)
    double *r0, *v, *s, *t, *ph, *sh;  // BiCGSTAB only
    const int32_t *tiles;         // first block row of each tile, ntiles + 1 entries
    int32_t item_begin, item_end;
    int32_t precision;            // YG_PREC_FP64 or YG_PREC_MIXED
    int32_t ntiles;
    int32_t method, pad;
};

struct BatchScal {
    double rz[2];                 // PCG: r.z, double-buffered by iteration parity
    double bb, rr, rr_last, tol;
    double alpha, beta, omega, rho;
    int64_t iter, maxiter;
    int32_t flag, stop, replace, restart;
    int32_t ticket, fresh;        // items of the running kernel finished; BiCGSTAB p = r next
    int32_t restarts, pad;
    int64_t replacements;
    double true_rr;               // r.r of the last FP64 true residual
};

struct BatchItem {
    int32_t sys, tile_begin, tile_end, row_begin, row_end, pad;
};

constexpr int kGroups = 6;  // (method, block size): group = 3 * method + block - 1

struct yg_batch_t {
    yg_context ctx = nullptr;
    int32_t capacity = 0;
    std::vector<BatchSys> sys;          // host mirror
    std::vector<std::vector<int32_t>> tiles;  // host copy of each system's tiles
    std::vector<int32_t> used;          // slot in use
    std::vector<yg_matrix> mats;
    std::vector<yg_solve_opts> opts;
    BatchSys *d_sys = nullptr;
    BatchScal *d_scal = nullptr;
    BatchItem *d_items = nullptr;
    int32_t *d_ranges = nullptr;        // [8]: first item of each group, then the end
    double *d_part = nullptr;           // partials: 2 per item
    double *d_part2 = nullptr;
    int32_t max_items = 0, n_items = 0;
    int32_t tiles_per_item[4] = {0, 8, 8, 8};
    int32_t lanes[4] = {4, 4, 8, 16};
    unsigned groups_present = 0, graph_groups = 0;
    bool dirty = false;                 // item table out of date (systems added, removed or reset)
    int32_t live_items = 0;             // items of systems that may still iterate (host view)
    int m = 16;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    int64_t graph_kernels = 0;
    std::vector<BatchScal> h_scal;
};

namespace yg {

// ---------------------------------------------------------------- tiles

// Blocks per tile: the values and block columns of a full FP64 tile fill one
// shared-memory stage of about 18 KB.
template <int B> struct TileCfg;
template <> struct TileCfg<1> { static constexpr int BLOCKS = 1536; };
template <> struct TileCfg<2> { static constexpr int BLOCKS = 512; };
template <> struct TileCfg<3> { static constexpr int BLOCKS = 224; };

static int tile_blocks(int B) { return B == 1 ? TileCfg<1>::BLOCKS : (B == 2 ? TileCfg<2>::BLOCKS : TileCfg<3>::BLOCKS); }

template <int B>
struct Stage {
    static constexpr int NST = 3;
    static constexpr int VBYTES = TileCfg<B>::BLOCKS * B * B * 8 + 32;  // FP64 values + alignment slack
    static constexpr int CBYTES = TileCfg<B>::BLOCKS * 4 + 32;
    static constexpr int BYTES = VBYTES + CBYTES;
    static constexpr int SMEM = NST * BYTES + NST * 8;  // stages + mbarriers
};

// SpMV kinds
enum { SP_CG = 0, SP_VERIFY = 1, SP_BICG_V = 2, SP_BICG_T = 3 };

// ---------------------------------------------------------------- kernels

// Whether system state `sc` takes part in a kernel of the given kind, decided
// once per CTA: thread 0 reads the state and broadcasts it, so every thread of
// the CTA takes the same branch around the block reductions.
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

// After thread 0 published this item's partials: count the item in the system's
// ticket; returns (to every thread) whether this CTA finished the system's last
// item, in which case the ticket is reset and all partials are visible.
__device__ __forceinline__ bool last_of_system(BatchScal *sc, int n_items, int *flag_sm) {
    if (threadIdx.x == 0) {
        __threadfence();
        const int old = atomicAdd(&sc->ticket, 1);
        const int last = (old == n_items - 1);
        if (last) {
            sc->ticket = 0;
            __threadfence();
        }
        *flag_sm = last;
    }
    __syncthreads();
    return *flag_sm != 0;
}

// Fixed-order sum of partials [ib, ie) (stride 2, offset off), result in every thread.
__device__ __forceinline__ double sum_items(const double *part, int ib, int ie, int off, double *sm) {
    double v = 0;
    for (int i = ib + threadIdx.x; i < ie; i += blockDim.x) v += __ldcg(part + 2 * (int64_t)i + off);
    return block_sum_all<kThreads>(v, sm);
}

// Rows [r0, r1) of one tile: L lanes per block row; vals / cols point at the
// tile's first block (shared memory, or global memory for an oversized tile).
// out = A xin on those rows; dot1 += out.w (iteration kinds), dot2 += out.out (SP_BICG_T).
template <int B, int L, int KIND, typename VT>
__device__ __forceinline__ void tile_rows(const int32_t *__restrict__ rowptr, int r0, int r1, int b0, const VT *vals,
                                          const int32_t *cols, const double *__restrict__ xin, double *__restrict__ out,
                                          const double *__restrict__ w, double &dot1, double &dot2) {
    constexpr int B2 = B * B;
    constexpr int G = kThreads / L;
    const int lane = threadIdx.x & 31, glane = lane % L, grp = threadIdx.x / L;
    for (int rb = r0; rb < r1; rb += G) {
        const int r = rb + grp;
        double acc[B];
#pragma unroll
        for (int i = 0; i < B; ++i) acc[i] = 0;
        if (r < r1) {
            const int rs = rowptr[r] - b0, re = rowptr[r + 1] - b0;
            int j = rs + glane;
            for (; j + L < re; j += 2 * L) {
                const int c0 = cols[j], c1 = cols[j + L];
                double x0[B], x1[B];
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    x0[k] = __ldg(xin + (int64_t)B * c0 + k);
                    x1[k] = __ldg(xin + (int64_t)B * c1 + k);
                }
#pragma unroll
                for (int i = 0; i < B; ++i)
#pragma unroll
                    for (int k = 0; k < B; ++k) {
                        acc[i] = fma((double)vals[j * B2 + i * B + k], x0[k], acc[i]);
                        acc[i] = fma((double)vals[(j + L) * B2 + i * B + k], x1[k], acc[i]);
                    }
            }
            if (j < re) {
                const int c0 = cols[j];
#pragma unroll
                for (int i = 0; i < B; ++i)
#pragma unroll
                    for (int k = 0; k < B; ++k)
                        acc[i] = fma((double)vals[j * B2 + i * B + k], __ldg(xin + (int64_t)B * c0 + k), acc[i]);
            }
        }
#pragma unroll
        for (int i = 0; i < B; ++i)
#pragma unroll
            for (int o = L / 2; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
        if (r < r1 && glane == 0) {
#pragma unroll
            for (int i = 0; i < B; ++i) {
                out[(int64_t)B * r + i] = acc[i];
                if (KIND != SP_VERIFY) dot1 = fma(acc[i], w[(int64_t)B * r + i], dot1);
                if (KIND == SP_BICG_T) dot2 = fma(acc[i], acc[i], dot2);
            }
        }
    }
}

// CTA-wide bounded wait on a stage: thread 0 polls, the verdict is broadcast;
// the other threads then observe the completed phase themselves (acquire).
__device__ __forceinline__ bool stage_wait(uint64_t *bar, unsigned parity, int *flag_sm) {
    if (threadIdx.x == 0) {
        long long spins = 0;
        int ok = 1;
        while (!mbar_try_wait(bar, parity))
            if (++spins > kSpinLimit) { ok = 0; break; }
        *flag_sm = ok;
    }
    __syncthreads();
    const bool ok = *flag_sm != 0;
    if (ok && threadIdx.x != 0) mbar_try_wait(bar, parity);
    return ok;
}

// Thread 0 issues the bulk copies of tile t (values, then block columns) into
// stage seq % NST; an empty or oversized tile completes its phase with no
// transfer and is read from global memory instead.
template <int B>
__device__ __forceinline__ void issue_tile(unsigned char *smem_raw, uint64_t *bars, uint32_t seq,
                                           const int32_t *__restrict__ rowptr, const int32_t *__restrict__ tiles, int t,
                                           const char *vbase, int vsz, const int32_t *col, uint64_t pol) {
    using S = Stage<B>;
    constexpr int B2 = B * B;
    if (threadIdx.x != 0) return;
    const int st = seq % S::NST;
    const int b0 = rowptr[tiles[t]], b1 = rowptr[tiles[t + 1]];
    const int nb = b1 - b0;
    if (nb > 0 && nb <= TileCfg<B>::BLOCKS) {
        const int64_t vs = (int64_t)b0 * B2 * vsz, va = vs & ~(int64_t)15;
        const int64_t ve = (vs + (int64_t)nb * B2 * vsz + 15) & ~(int64_t)15;
        const int64_t cs = (int64_t)b0 * 4, ca = cs & ~(int64_t)15, ce = (cs + (int64_t)nb * 4 + 15) & ~(int64_t)15;
        unsigned char *dst = smem_raw + (size_t)st * S::BYTES;
        mbar_expect_tx(&bars[st], (unsigned)((ve - va) + (ce - ca)));
        bulk_g2s(dst, vbase + va, (unsigned)(ve - va), &bars[st], pol);
        bulk_g2s(dst + S::VBYTES, reinterpret_cast<const char *>(col) + ca, (unsigned)(ce - ca), &bars[st], pol);
    } else {
        mbar_expect_tx(&bars[st], 0);
    }
}

// The SpMV of one group of items (ranges[g], ranges[g + 1]):
//   SP_CG      q = A p, partials of p.q; last CTA: alpha = r.z / p.q
//   SP_VERIFY  q = A x with FP64 values (systems under verification)
//   SP_BICG_V  v = A ph, partials of r0.v; last CTA: alpha = rho / r0.v
//   SP_BICG_T  t = A sh, partials of t.s and t.t; last CTA: omega = t.s / t.t
// The iteration kinds read FP32 values for mixed-precision systems.  With
// commit == 0 (autotuning) the reductions are not taken.
template <int B, int L, int KIND>
__global__ void __launch_bounds__(kThreads)
k_batch_spmv(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, int g,
             const BatchSys *__restrict__ sys, BatchScal *__restrict__ scal, double *__restrict__ part, int parity,
             int commit, int32_t *__restrict__ err) {
    using S = Stage<B>;
    constexpr int B2 = B * B;
    constexpr int CAP = TileCfg<B>::BLOCKS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int flag_sm;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)S::NST * S::BYTES);
    if (threadIdx.x == 0)
        for (int k = 0; k < S::NST; ++k) mbar_init(&bars[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    const uint64_t pol = evict_first_policy();
    uint32_t seq_issue = 0, seq_wait = 0;  // tiles issued / consumed by this CTA
    bool timed_out = false;
    const int g0 = ranges[g], g1 = ranges[g + 1];
    for (int it = g0 + blockIdx.x; it < g1 && !timed_out; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        if (!cta_active(&scal[s], KIND == SP_VERIFY ? ACT_VERIFY : ACT_ITER, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const bool f32 = (KIND != SP_VERIFY && d.precision == YG_PREC_MIXED);
        const int vsz = f32 ? 4 : 8;
        const char *vbase = f32 ? reinterpret_cast<const char *>(d.val32) : reinterpret_cast<const char *>(d.val);
        const double *xin = KIND == SP_CG ? d.p : KIND == SP_VERIFY ? d.x : KIND == SP_BICG_V ? d.ph : d.sh;
        double *out = (KIND == SP_CG || KIND == SP_VERIFY) ? d.q : KIND == SP_BICG_V ? d.v : d.t;
        const double *w = KIND == SP_CG ? d.p : KIND == SP_BICG_V ? d.r0 : d.s;
        int t_issue = item.tile_begin;
        while (t_issue < item.tile_end && seq_issue - seq_wait < (uint32_t)(S::NST - 1))
            issue_tile<B>(smem_raw, bars, seq_issue++, d.rowptr, d.tiles, t_issue++, vbase, vsz, d.col, pol);
        double dot1 = 0, dot2 = 0;
        for (int t = item.tile_begin; t < item.tile_end; ++t) {
            if (t_issue < item.tile_end && seq_issue - seq_wait < (uint32_t)S::NST)
                issue_tile<B>(smem_raw, bars, seq_issue++, d.rowptr, d.tiles, t_issue++, vbase, vsz, d.col, pol);
            const int st = seq_wait % S::NST;
            if (!stage_wait(&bars[st], (seq_wait / S::NST) & 1u, &flag_sm)) {
                timed_out = true;
                break;
            }
            const int r0 = d.tiles[t], r1 = d.tiles[t + 1];
            const int b0 = d.rowptr[r0], nb = d.rowptr[r1] - b0;
            const unsigned char *stg = smem_raw + (size_t)st * S::BYTES;
            const int lv = (int)(((int64_t)b0 * B2 * vsz) & 15), lc = (int)(((int64_t)b0 * 4) & 15);
            const int32_t *cols = nb <= CAP ? reinterpret_cast<const int32_t *>(stg + S::VBYTES + lc) : d.col + b0;
            if (f32) {
                const float *v = nb <= CAP ? reinterpret_cast<const float *>(stg + lv) : d.val32 + (int64_t)b0 * B2;
                tile_rows<B, L, KIND, float>(d.rowptr, r0, r1, b0, v, cols, xin, out, w, dot1, dot2);
            } else {
                const double *v = nb <= CAP ? reinterpret_cast<const double *>(stg + lv) : d.val + (int64_t)b0 * B2;
                tile_rows<B, L, KIND, double>(d.rowptr, r0, r1, b0, v, cols, xin, out, w, dot1, dot2);
            }
            ++seq_wait;
            __syncthreads();  // the stage is free for the next issue
        }
        if (timed_out) break;
        if (KIND != SP_VERIFY && commit) {
            dot1 = block_sum<kThreads>(dot1, sm);
            if (KIND == SP_BICG_T) dot2 = block_sum<kThreads>(dot2, sm);
            if (threadIdx.x == 0) {
                part[2 * (int64_t)it] = dot1;
                if (KIND == SP_BICG_T) part[2 * (int64_t)it + 1] = dot2;
            }
            if (last_of_system(&scal[s], d.item_end - d.item_begin, &flag_sm)) {
                const double a = sum_items(part, d.item_begin, d.item_end, 0, sm);
                const double tt = KIND == SP_BICG_T ? sum_items(part, d.item_begin, d.item_end, 1, sm) : 0.0;
                if (threadIdx.x == 0) {
                    BatchScal &sc = scal[s];
                    if (KIND == SP_CG) {
                        const double alpha = sc.rz[parity] / a;
                        if (a == 0 || !isfinite(alpha)) sc.stop = isfinite(a) ? BS_BREAK : BS_NAN;
                        else sc.alpha = alpha;
                    } else if (KIND == SP_BICG_V) {
                        const double alpha = sc.rho / a;
                        sc.fresh = 0;
                        if (a == 0 || !isfinite(alpha)) sc.stop = isfinite(a) ? BS_CONV : BS_NAN;  // restart via verify
                        else sc.alpha = alpha;
                    } else {
                        sc.omega = tt > 0 ? a / tt : 0.0;
                    }
                }
            }
        }
    }
    if (timed_out && threadIdx.x == 0 && err) atomicExch(err, (int32_t)YG_TIMEOUT);
    // drain the copies still in flight before the CTA exits (bounded)
    if (threadIdx.x == 0) {
        while (seq_wait != seq_issue) {
            const int st = seq_wait % S::NST;
            long long spins = 0;
            while (!mbar_try_wait(&bars[st], (seq_wait / S::NST) & 1u) && ++spins <= kSpinLimit) {
            }
            ++seq_wait;
        }
    }
    __syncthreads();
}

// V1 (BiCGSTAB items only): p = r + beta (p - omega v) (p = r after a restart), ph = D^-1 p
__global__ void __launch_bounds__(kThreads)
k_batch_v1(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
           const BatchScal *__restrict__ scal) {
    __shared__ int flag_sm;
    const int i0 = ranges[3], i1 = ranges[kGroups];
    for (int it = i0 + blockIdx.x; it < i1; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        if (!cta_active(&scal[s], ACT_ITER, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const bool fresh = __ldcg(&scal[s].fresh) != 0;
        const double beta = __ldcg(&scal[s].beta), omega = __ldcg(&scal[s].omega);
        const int64_t lo = (int64_t)item.row_begin * d.block, hi = (int64_t)item.row_end * d.block;
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const double pi = fresh ? d.r[i] : d.r[i] + beta * (d.p[i] - omega * d.v[i]);
            d.p[i] = pi;
            d.ph[i] = d.dinv[i] * pi;
        }
    }
}

// V2: PCG x and r updates, Jacobi z, partials of r.z and r.r, the last CTA of a
// system takes its decisions (beta, convergence of the recursive residual, NaN,
// iteration cap, a due mixed-precision replacement); BiCGSTAB s = r - alpha v,
// sh = D^-1 s.
__global__ void __launch_bounds__(kThreads)
k_batch_v2(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
           BatchScal *__restrict__ scal, int parity, double *__restrict__ part) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int flag_sm;
    const int n_items = ranges[kGroups];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        BatchScal &sc = scal[s];
        if (!cta_active(&sc, ACT_ITER, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const double alpha = __ldcg(&sc.alpha);
        const int64_t lo = (int64_t)item.row_begin * d.block, hi = (int64_t)item.row_end * d.block;
        if (d.method == BM_BICG) {
            for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
                const double si = d.r[i] - alpha * d.v[i];
                d.s[i] = si;
                d.sh[i] = d.dinv[i] * si;
            }
            continue;
        }
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
            part[2 * (int64_t)it] = srz;
            part[2 * (int64_t)it + 1] = srr;
        }
        if (last_of_system(&sc, d.item_end - d.item_begin, &flag_sm)) {
            const double rz_new = sum_items(part, d.item_begin, d.item_end, 0, sm);
            const double rr = sum_items(part, d.item_begin, d.item_end, 1, sm);
            if (threadIdx.x == 0) {
                int stop = BS_NONE;
                if (sqrt(rr) <= sc.tol * sqrt(sc.bb)) stop = BS_CONV;
                else if (!isfinite(rz_new)) stop = BS_NAN;
                else if (sc.iter + 1 >= sc.maxiter) stop = BS_MAXIT;
                sc.beta = rz_new / sc.rz[parity];
                sc.rz[parity ^ 1] = rz_new;
                sc.rr = rr;
                sc.iter += 1;
                if (stop == BS_NONE && d.precision == YG_PREC_MIXED && rr < 1e-2 * sc.rr_last) sc.replace = 1;
                sc.stop = stop;
            }
        }
    }
}

// V3: PCG p = z + beta p; BiCGSTAB x += alpha ph + omega sh, r = s - omega t,
// partials of r0.r and r.r, the last CTA of a system takes its decisions (beta,
// convergence, NaN, cap, replacement; a breakdown asks the verification pass
// for a restart).
__global__ void __launch_bounds__(kThreads)
k_batch_v3(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
           BatchScal *__restrict__ scal, double *__restrict__ part) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int flag_sm;
    const int n_items = ranges[kGroups];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        BatchScal &sc = scal[s];
        if (!cta_active(&sc, ACT_ITER, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const int64_t lo = (int64_t)item.row_begin * d.block, hi = (int64_t)item.row_end * d.block;
        if (d.method == BM_CG) {
            const double beta = __ldcg(&sc.beta);
            for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) d.p[i] = d.dinv[i] * d.r[i] + beta * d.p[i];
            continue;
        }
        const double alpha = __ldcg(&sc.alpha), omega = __ldcg(&sc.omega);
        double srr0 = 0, srr = 0;
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            d.x[i] += alpha * d.ph[i] + omega * d.sh[i];
            const double ri = d.s[i] - omega * d.t[i];
            d.r[i] = ri;
            srr0 += d.r0[i] * ri;
            srr += ri * ri;
        }
        srr0 = block_sum<kThreads>(srr0, sm);
        srr = block_sum<kThreads>(srr, sm);
        if (threadIdx.x == 0) {
            part[2 * (int64_t)it] = srr0;
            part[2 * (int64_t)it + 1] = srr;
        }
        if (last_of_system(&sc, d.item_end - d.item_begin, &flag_sm)) {
            const double rho_new = sum_items(part, d.item_begin, d.item_end, 0, sm);
            const double rr = sum_items(part, d.item_begin, d.item_end, 1, sm);
            if (threadIdx.x == 0) {
                const double beta = (rho_new / sc.rho) * (alpha / omega);
                int stop = BS_NONE;
                if (sqrt(rr) <= sc.tol * sqrt(sc.bb)) stop = BS_CONV;
                else if (!isfinite(rr) || !isfinite(rho_new)) stop = BS_NAN;
                else if (sc.iter + 1 >= sc.maxiter) stop = BS_MAXIT;
                else if (rho_new == 0 || omega == 0 || !isfinite(beta)) stop = BS_CONV;  // restart via verify
                sc.beta = beta;
                sc.rho = rho_new;
                sc.rr = rr;
                sc.iter += 1;
                if (stop == BS_NONE && d.precision == YG_PREC_MIXED && rr < 1e-2 * sc.rr_last) sc.replace = 1;
                sc.stop = stop;
            }
        }
    }
}

// verification, step 2: r = b - q (q = A x from the verification SpMV), partials
// of r.z (PCG) or r0.r (BiCGSTAB; r.r for a system being initialised), r.r and
// b.b for the systems under verification
__global__ void __launch_bounds__(kThreads)
k_batch_residual(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
                 const BatchScal *__restrict__ scal, double *__restrict__ part, double *__restrict__ part_bb) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int flag_sm;
    const int n_items = ranges[kGroups];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        if (!cta_active(&scal[s], ACT_VERIFY, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const bool bicg = d.method == BM_BICG;
        const bool init = __ldcg(&scal[s].flag) == BF_INIT;
        const int64_t lo = (int64_t)item.row_begin * d.block, hi = (int64_t)item.row_end * d.block;
        double s1 = 0, srr = 0, sbb = 0;
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const double ri = d.b[i] - d.q[i];
            d.r[i] = ri;
            s1 += bicg ? (init ? ri : d.r0[i]) * ri : ri * (d.dinv[i] * ri);
            srr += ri * ri;
            sbb += d.b[i] * d.b[i];
        }
        s1 = block_sum<kThreads>(s1, sm);
        srr = block_sum<kThreads>(srr, sm);
        sbb = block_sum<kThreads>(sbb, sm);
        if (threadIdx.x == 0) {
            part[2 * (int64_t)it] = s1;
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
    sc.ticket = 0;
    if (sc.flag == BF_RUN && (sc.stop == BS_BREAK || sc.stop == BS_NAN || sc.stop == BS_MAXIT)) {
        sc.flag = sc.stop == BS_BREAK ? BF_BREAK : (sc.stop == BS_NAN ? BF_NANF : BF_MAXIT);
        return;
    }
    const bool init = sc.flag == BF_INIT;
    const bool ver = sc.flag == BF_RUN && (sc.stop == BS_CONV || sc.replace);
    if (!init && !ver) return;
    const BatchSys d = sys[s];
    const bool bicg = d.method == BM_BICG;
    double s1 = 0, rr = 0, bb = 0;
    for (int i = d.item_begin; i < d.item_end; ++i) {
        s1 += part[2 * (int64_t)i];
        rr += part[2 * (int64_t)i + 1];
        bb += part_bb[2 * (int64_t)i];
    }
    if (init) sc.bb = bb;
    sc.true_rr = rr;
    sc.rr = rr;
    sc.rr_last = rr;
    sc.replacements += (init ? 0 : 1);
    const bool conv = sqrt(rr) <= sc.tol * sqrt(sc.bb);
    // restart: PCG p = z (restart kernel); BiCGSTAB r0 = r (restart kernel), p = r (fresh)
    bool restart = false;
    if (init) {
        sc.flag = (conv || (!bicg && s1 == 0)) ? BF_DONE : BF_RUN;
        restart = !conv;
    } else if (sc.stop == BS_CONV) {
        if (conv) {
            sc.flag = BF_DONE;
        } else {
            restart = true;
            if (sc.iter >= sc.maxiter) sc.flag = BF_MAXIT;
            if (bicg && ++sc.restarts > kBicgRestarts) sc.flag = BF_BREAK;
        }
    }
    sc.stop = BS_NONE;
    if (bicg) {
        sc.rho = restart ? rr : s1;  // r0.r: r.r after r0 = r, else with the kept r0
        if (restart) sc.fresh = 1;
    } else {
        sc.rz[0] = sc.rz[1] = s1;
    }
    sc.restart = (restart && sc.flag == BF_RUN) ? 1 : 0;
    sc.replace = 0;
}

// verification, step 4: PCG p = z, BiCGSTAB r0 = r for restarted systems
__global__ void __launch_bounds__(kThreads)
k_batch_restart(const BatchItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
                const BatchScal *__restrict__ scal) {
    __shared__ int flag_sm;
    const int n_items = ranges[kGroups];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const int s = item.sys;
        if (!cta_active(&scal[s], ACT_RESTART, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const int64_t lo = (int64_t)item.row_begin * d.block, hi = (int64_t)item.row_end * d.block;
        if (d.method == BM_BICG)
            for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) d.r0[i] = d.r[i];
        else
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

// grid of the SpMV kernels: resident CTAs per SM (shared memory bound) x SMs
template <int B, int L, int KIND>
static int spmv_grid(yg_context ctx) {
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaFuncSetAttribute(k_batch_spmv<B, L, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, Stage<B>::SMEM);
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_spmv<B, L, KIND>, kThreads, Stage<B>::SMEM) !=
                cudaSuccess || n < 1)
            n = 1;
        per_sm = n;
    }
    return per_sm * ctx->num_sms;
}

template <int B, int L, int KIND>
static void launch_spmv_l(yg_batch bt, int g, int parity, int commit) {
    yg_context ctx = bt->ctx;
    k_batch_spmv<B, L, KIND><<<spmv_grid<B, L, KIND>(ctx), kThreads, Stage<B>::SMEM, ctx->stream>>>(
        bt->d_items, bt->d_ranges, g, bt->d_sys, bt->d_scal, bt->d_part, parity, commit, ctx->d_err);
    YG_LAUNCHED(ctx);
}

template <int B, int KIND>
static void launch_spmv_b(yg_batch bt, int L, int g, int parity, int commit) {
    switch (L) {
    case 2: launch_spmv_l<B, 2, KIND>(bt, g, parity, commit); break;
    case 4: launch_spmv_l<B, 4, KIND>(bt, g, parity, commit); break;
    case 8: launch_spmv_l<B, 8, KIND>(bt, g, parity, commit); break;
    case 16: launch_spmv_l<B, 16, KIND>(bt, g, parity, commit); break;
    default: launch_spmv_l<B, 32, KIND>(bt, g, parity, commit); break;
    }
}

template <int KIND>
static void launch_spmv_kind(yg_batch bt, int B, int L, int g, int parity, int commit) {
    if (B == 1) launch_spmv_b<1, KIND>(bt, L, g, parity, commit);
    else if (B == 2) launch_spmv_b<2, KIND>(bt, L, g, parity, commit);
    else launch_spmv_b<3, KIND>(bt, L, g, parity, commit);
}

// one SpMV launch for group g (method, block size) of the given kind
static void launch_spmv(yg_batch bt, int kind, int g, int parity, int commit, int L = 0) {
    const int B = g % 3 + 1;
    if (L == 0) L = bt->lanes[B];
    switch (kind) {
    case SP_CG: launch_spmv_kind<SP_CG>(bt, B, L, g, parity, commit); break;
    case SP_VERIFY: launch_spmv_kind<SP_VERIFY>(bt, B, L, g, parity, commit); break;
    case SP_BICG_V: launch_spmv_kind<SP_BICG_V>(bt, B, L, g, parity, commit); break;
    default: launch_spmv_kind<SP_BICG_T>(bt, B, L, g, parity, commit); break;
    }
}

// set the shared-memory attribute of every SpMV instantiation (outside capture)
template <int B, int KIND>
static void prepare_spmv_bk(yg_context ctx) {
    spmv_grid<B, 2, KIND>(ctx); spmv_grid<B, 4, KIND>(ctx); spmv_grid<B, 8, KIND>(ctx);
    spmv_grid<B, 16, KIND>(ctx); spmv_grid<B, 32, KIND>(ctx);
}
template <int B>
static void prepare_spmv_b(yg_context ctx) {
    prepare_spmv_bk<B, SP_CG>(ctx); prepare_spmv_bk<B, SP_VERIFY>(ctx);
    prepare_spmv_bk<B, SP_BICG_V>(ctx); prepare_spmv_bk<B, SP_BICG_T>(ctx);
}

static bool has(yg_batch bt, int g) { return (bt->groups_present >> g) & 1u; }
static bool has_bicg(yg_batch bt) { return (bt->groups_present >> 3) != 0; }

// the verification pass (also initialises newly added systems)
static void launch_verify(yg_batch bt) {
    yg_context ctx = bt->ctx;
    const int grid = batch_grid(ctx);
    for (int g = 0; g < kGroups; ++g)
        if (has(bt, g)) launch_spmv(bt, SP_VERIFY, g, 0, 1);
    k_batch_residual<<<grid, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_part,
                                                        bt->d_part2);
    YG_LAUNCHED(ctx);
    k_batch_decide<<<(bt->capacity + 127) / 128, 128, 0, ctx->stream>>>(bt->capacity, bt->d_sys, bt->d_scal, bt->d_part,
                                                                         bt->d_part2);
    YG_LAUNCHED(ctx);
    k_batch_restart<<<grid, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal);
    YG_LAUNCHED(ctx);
}

static void launch_iteration(yg_batch bt, int parity) {
    yg_context ctx = bt->ctx;
    const int grid = batch_grid(ctx);
    if (has_bicg(bt)) {
        k_batch_v1<<<grid, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal);
        YG_LAUNCHED(ctx);
    }
    for (int g = 0; g < kGroups; ++g)
        if (has(bt, g)) launch_spmv(bt, g < 3 ? SP_CG : SP_BICG_V, g, parity, 1);
    k_batch_v2<<<grid, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, parity,
                                                  bt->d_part2);
    YG_LAUNCHED(ctx);
    for (int g = 3; g < kGroups; ++g)
        if (has(bt, g)) launch_spmv(bt, SP_BICG_T, g, parity, 1);
    k_batch_v3<<<grid, kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_part2);
    YG_LAUNCHED(ctx);
}

static void drop_graph(yg_batch bt) {
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    bt->exec = nullptr;
    bt->graph = nullptr;
}

// Whether system s may still iterate, as the host last saw its flag.
static bool sys_live(yg_batch bt, int s) {
    const int f = bt->h_scal[s].flag;
    return bt->used[s] && (f == BF_RUN || f == BF_INIT);
}

// Rebuild the item table: systems grouped by (method, block size), tiles
// grouped into items.  Systems that finished are left out (their kernels' item
// loops stay short); the groups present count every system in the batch, so
// compaction never changes the set of SpMV launches that the captured graph
// holds.  A system's tiles are always grouped the same way for a given tuning,
// so its reductions add the same partials in the same order whatever else is in
// the table.
static yg_status rebuild_items(yg_batch bt) {
    yg_context ctx = bt->ctx;
    std::vector<BatchItem> items;
    int32_t ranges[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    unsigned present = 0;
    for (int g = 0; g < kGroups; ++g) {
        const int method = g / 3, B = g % 3 + 1;
        ranges[g] = (int32_t)items.size();
        const int T = std::max(1, bt->tiles_per_item[B]);
        for (int s = 0; s < bt->capacity; ++s) {
            if (!bt->used[s] || bt->sys[s].block != B || bt->sys[s].method != method) continue;
            present |= 1u << g;
            BatchSys &d = bt->sys[s];
            d.item_begin = (int32_t)items.size();
            if (!sys_live(bt, s)) {
                d.item_end = d.item_begin;
                continue;
            }
            const std::vector<int32_t> &tl = bt->tiles[s];
            for (int t0 = 0; t0 < d.ntiles; t0 += T) {
                const int t1 = std::min(d.ntiles, t0 + T);
                items.push_back({s, t0, t1, tl[t0], tl[t1], 0});
            }
            if (d.ntiles == 0) items.push_back({s, 0, 0, 0, 0, 0});
            d.item_end = (int32_t)items.size();
        }
    }
    ranges[kGroups] = (int32_t)items.size();
    ranges[kGroups + 1] = (int32_t)items.size();
    if ((int32_t)items.size() > bt->max_items) {
        YG_CUDA(cudaStreamSynchronize(ctx->stream));
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
    bt->live_items = bt->n_items;
    bt->dirty = false;
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
    // for a BiCGSTAB system q is t: freed once, as q
    for (void *ptr : {(void *)d.r, (void *)d.p, (void *)d.q, (void *)d.dinv, (void *)d.tiles, (void *)d.r0, (void *)d.v,
                      (void *)d.s, (void *)d.ph, (void *)d.sh})
        dev_free(ctx, ptr);
    d = BatchSys{};
    bt->tiles[s].clear();
    bt->used[s] = 0;
    bt->mats[s] = nullptr;
}

// Cut block rows into tiles of whole rows with at most `cap` blocks each (a row
// longer than cap forms a tile of its own, read from global memory).
static void make_tiles(const std::vector<int32_t> &rp, int cap, std::vector<int32_t> &tiles) {
    tiles.clear();
    const int n = (int)rp.size() - 1;
    tiles.push_back(0);
    int start = 0;
    for (int r = 0; r < n; ++r) {
        if (r > start && rp[r + 1] - rp[start] > cap) {
            tiles.push_back(r);
            start = r;
        }
    }
    if (n > 0) tiles.push_back(n);
}

}  // namespace yg

using namespace yg;

extern "C" yg_status yg_batch_create(yg_context ctx, int32_t capacity, yg_batch *out) {
    if (!ctx || !out || capacity < 1) return fail(YG_BAD_ARG, "yg_batch_create: bad argument");
    auto *bt = new yg_batch_t();
    bt->ctx = ctx;
    bt->capacity = capacity;
    bt->sys.assign(capacity, BatchSys{});
    bt->tiles.assign(capacity, std::vector<int32_t>());
    bt->used.assign(capacity, 0);
    bt->mats.assign(capacity, nullptr);
    bt->opts.assign(capacity, yg_solve_opts{});
    yg_status s;
    if ((s = dev_alloc_t(ctx, &bt->d_sys, capacity)) != YG_OK || (s = dev_alloc_t(ctx, &bt->d_scal, capacity)) != YG_OK ||
        (s = dev_alloc_t(ctx, &bt->d_ranges, 8)) != YG_OK) {
        yg_batch_destroy(bt);
        return s;
    }
    prepare_spmv_b<1>(ctx);
    prepare_spmv_b<2>(ctx);
    prepare_spmv_b<3>(ctx);
    std::vector<BatchScal> init(capacity);
    for (auto &c : init) c.flag = BF_EMPTY;
    bt->h_scal = init;
    cudaMemcpy(bt->d_scal, init.data(), sizeof(BatchScal) * capacity, cudaMemcpyHostToDevice);
    cudaMemset(bt->d_ranges, 0, sizeof(int32_t) * 8);
    YG_CUDA(cudaGetLastError());
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

extern "C" int64_t yg_batch_work_bytes(int64_t rows, int32_t method) {
    // work vectors (each with the 16-byte allocation padding) and the tile table
    const int64_t nvec = method == YG_METHOD_BICGSTAB ? 9 : 4;
    return nvec * (8 * (rows + 1) + 16) + 4 * (rows + 2) + 16;
}

extern "C" yg_status yg_batch_add(yg_batch bt, yg_matrix A, yg_vector b, yg_vector x, int32_t method,
                                  const yg_solve_opts *opts, int32_t *slot) {
    if (!bt || !A || !b || !x || !slot) return fail(YG_BAD_ARG, "yg_batch_add: NULL argument");
    if (A->ctx != bt->ctx || b->ctx != bt->ctx || x->ctx != bt->ctx) return fail(YG_BAD_ARG, "yg_batch_add: context mismatch");
    if (A->rows() != A->cols() || b->n != A->rows() || x->n != A->rows()) return fail(YG_BAD_ARG, "yg_batch_add: dimension mismatch");
    if (A->block < 1 || A->block > 3) return fail(YG_UNSUPPORTED, "yg_batch_add: block size %d", A->block);
    if (method != YG_METHOD_CG && method != YG_METHOD_BICGSTAB) return fail(YG_BAD_ARG, "yg_batch_add: method %d", method);
    yg_solve_opts o = opts ? *opts : yg_solve_opts{YG_CRIT_RELRES, YG_PREC_FP64, 1e-10, 0, 0, 0};
    if (o.criterion != YG_CRIT_RELRES) return fail(YG_UNSUPPORTED, "batched solves stop on the relative residual");
    if (o.precision != YG_PREC_FP64 && o.precision != YG_PREC_MIXED) return fail(YG_UNSUPPORTED, "batched precision");
    int s = -1;
    for (int i = 0; i < bt->capacity; ++i)
        if (!bt->used[i]) { s = i; break; }
    if (s < 0) return fail(YG_OVER_BUDGET, "yg_batch_add: all %d slots in use", bt->capacity);
    yg_context ctx = bt->ctx;
    if (o.precision == YG_PREC_MIXED && !A->d_val32) YG_TRY(yg_matrix_make_fp32(A));
    // tiles of whole rows, from the row pointer
    std::vector<int32_t> rp(A->nbrows + 1);
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    YG_CUDA(cudaMemcpy(rp.data(), A->d_rowptr, sizeof(int32_t) * rp.size(), cudaMemcpyDeviceToHost));
    std::vector<int32_t> tl;
    make_tiles(rp, tile_blocks(A->block), tl);
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
    d.method = method;
    d.ntiles = (int32_t)tl.size() - 1;
    const int64_t n = A->rows();
    double *dinv = nullptr;
    int32_t *dtiles = nullptr;
    yg_status st = YG_OK;
    auto alloc = [&](double **p) {
        if (st == YG_OK) st = dev_alloc_t(ctx, p, n + 1);
    };
    alloc(&d.r);
    alloc(&d.p);
    alloc(&dinv);
    if (method == YG_METHOD_BICGSTAB) {
        alloc(&d.r0);
        alloc(&d.v);
        alloc(&d.s);
        alloc(&d.t);
        alloc(&d.ph);
        alloc(&d.sh);
        d.q = d.t;
    } else {
        alloc(&d.q);
    }
    if (st == YG_OK) st = dev_alloc_t(ctx, &dtiles, tl.size());
    if (st != YG_OK) {
        for (void *ptr : {(void *)d.r, (void *)d.p, (void *)dinv, (void *)d.r0, (void *)d.v, (void *)d.s, (void *)d.ph,
                          (void *)d.sh, (void *)d.q, (void *)dtiles})
            dev_free(ctx, ptr);
        return st;
    }
    YG_CUDA(cudaMemcpy(dtiles, tl.data(), sizeof(int32_t) * tl.size(), cudaMemcpyHostToDevice));
    d.dinv = dinv;
    d.tiles = dtiles;
    k_batch_jacobi<<<stream_grid(ctx, n), kThreads, 0, ctx->stream>>>(A->nbrows, A->block, A->d_diag, A->d_val, dinv);
    YG_LAUNCHED(ctx);
    BatchScal sc{};
    sc.flag = BF_INIT;
    sc.tol = o.tol;
    sc.maxiter = o.maxiter > 0 ? o.maxiter : n;
    bt->sys[s] = d;
    bt->tiles[s] = std::move(tl);
    bt->used[s] = 1;
    bt->mats[s] = A;
    bt->opts[s] = o;
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    YG_CUDA(cudaMemcpy(bt->d_scal + s, &sc, sizeof(BatchScal), cudaMemcpyHostToDevice));
    bt->h_scal[s] = sc;
    bt->dirty = true;
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
    bt->h_scal[slot] = sc;
    bt->dirty = true;
    return YG_OK;
}

extern "C" yg_status yg_batch_reset(yg_batch bt, int32_t slot) {
    if (!bt || slot < -1 || slot >= bt->capacity || (slot >= 0 && !bt->used[slot]))
        return fail(YG_BAD_ARG, "yg_batch_reset: bad slot");
    YG_CUDA(cudaStreamSynchronize(bt->ctx->stream));
    const int s0 = slot < 0 ? 0 : slot, s1 = slot < 0 ? bt->capacity : slot + 1;
    for (int s = s0; s < s1; ++s) {
        if (!bt->used[s]) continue;
        const yg_solve_opts &o = bt->opts[s];
        BatchScal sc{};
        sc.flag = BF_INIT;
        sc.tol = o.tol;
        sc.maxiter = o.maxiter > 0 ? o.maxiter : (int64_t)bt->sys[s].nbrows * bt->sys[s].block;
        bt->h_scal[s] = sc;
    }
    YG_CUDA(cudaMemcpy(bt->d_scal + s0, bt->h_scal.data() + s0, sizeof(BatchScal) * (s1 - s0), cudaMemcpyHostToDevice));
    bt->dirty = true;
    return YG_OK;
}

// Launch one block of iterations (graph replay) and the copy of the system
// states to the host, without waiting.
static yg_status batch_launch(yg_batch bt) {
    yg_context ctx = bt->ctx;
    YG_CUDA(cudaGraphLaunch(bt->exec, ctx->stream));
    ctx->launches += bt->graph_kernels;
    YG_CUDA(cudaMemcpyAsync(bt->h_scal.data(), bt->d_scal, sizeof(BatchScal) * bt->capacity, cudaMemcpyDeviceToHost,
                            ctx->stream));
    return YG_OK;
}

// Wait for the launched block, count the systems still running and compact the
// item table once a quarter of it is idle.
static yg_status batch_collect(yg_batch bt, int *active_out) {
    yg_context ctx = bt->ctx;
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    YG_TRY(check_device_error(ctx));
    int active = 0;
    int32_t live = 0;
    for (int s = 0; s < bt->capacity; ++s)
        if (sys_live(bt, s)) {
            ++active;
            live += bt->sys[s].item_end - bt->sys[s].item_begin;
        }
    if (active > 0 && live < bt->live_items - bt->live_items / 4 && bt->live_items - live >= 64)
        YG_TRY(rebuild_items(bt));
    *active_out = active;
    return YG_OK;
}

static yg_status batch_prepare(yg_batch bt) {
    if (bt->dirty) YG_TRY(rebuild_items(bt));
    if (!bt->exec || bt->graph_groups != bt->groups_present) YG_TRY(capture_graph(bt));
    launch_verify(bt);  // initialise systems added since the last run
    return YG_OK;
}

// Advance every active system by blocks of m iterations plus a verification
// pass, at most max_blocks blocks (0 = until none is active).  *n_active
// receives the number of systems still running.
extern "C" yg_status yg_batch_run(yg_batch bt, int32_t max_blocks, int32_t *n_active) {
    if (!bt) return fail(YG_BAD_ARG, "yg_batch_run: NULL batch");
    YG_TRY(batch_prepare(bt));
    int active = 0;
    for (int blk = 0; max_blocks <= 0 || blk < max_blocks; ++blk) {
        YG_TRY(batch_launch(bt));
        YG_TRY(batch_collect(bt, &active));
        if (active == 0) break;
    }
    if (n_active) *n_active = active;
    return check_device_error(bt->ctx);
}

extern "C" yg_status yg_batch_launch(yg_batch bt) {
    if (!bt) return fail(YG_BAD_ARG, "yg_batch_launch: NULL batch");
    YG_TRY(batch_prepare(bt));
    return batch_launch(bt);
}

extern "C" yg_status yg_batch_wait(yg_batch bt, int32_t *n_active) {
    if (!bt) return fail(YG_BAD_ARG, "yg_batch_wait: NULL batch");
    int active = 0;
    YG_TRY(batch_collect(bt, &active));
    if (n_active) *n_active = active;
    return YG_OK;
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
    case BF_RUN: case BF_INIT: st.status = YG_RUNNING; break;
    default: st.status = YG_NOT_CONVERGED; break;
    }
    *out = st;
    return YG_OK;
}

// Choose tiles per item and lanes per block row for each block size from the
// systems present, by timing the iteration SpMV of the whole batch (without
// committing its reductions).
extern "C" yg_status yg_batch_tune(yg_batch bt) {
    if (!bt) return fail(YG_BAD_ARG, "yg_batch_tune: NULL batch");
    yg_context ctx = bt->ctx;
    // initialise p / ph from a verification pass so the SpMV reads defined data
    YG_TRY(rebuild_items(bt));
    launch_verify(bt);
    if (has_bicg(bt)) {
        k_batch_v1<<<batch_grid(ctx), kThreads, 0, ctx->stream>>>(bt->d_items, bt->d_ranges, bt->d_sys, bt->d_scal);
        YG_LAUNCHED(ctx);
    }
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    YG_TRY(check_device_error(ctx));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int B = 1; B <= 3; ++B) {
        const bool cg = has(bt, B - 1), bi = has(bt, 3 + B - 1);
        if (!cg && !bi) continue;
        float best = 1e30f;
        int bestL = bt->lanes[B], bestT = bt->tiles_per_item[B];
        for (int T : {2, 8, 32}) {
            bt->tiles_per_item[B] = T;
            YG_TRY(rebuild_items(bt));
            for (int L : {2, 4, 8, 16, 32}) {
                auto launch = [&]() {
                    if (cg) launch_spmv(bt, SP_CG, B - 1, 0, 0, L);
                    if (bi) launch_spmv(bt, SP_BICG_V, 3 + B - 1, 0, 0, L);
                };
                launch();
                cudaEventRecord(e0, ctx->stream);
                for (int r = 0; r < 3; ++r) launch();
                cudaEventRecord(e1, ctx->stream);
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) { best = ms; bestL = L; bestT = T; }
            }
        }
        bt->lanes[B] = bestL;
        bt->tiles_per_item[B] = bestT;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    YG_TRY(rebuild_items(bt));
    drop_graph(bt);
    YG_CUDA(cudaGetLastError());
    return check_device_error(ctx);
}

namespace yg {
// Host view of a slot after the last wait: whether it still iterates, and its
// stats (from the state copied back at the end of the block).
bool batch_slot_running(yg_batch bt, int32_t slot) { return sys_live(bt, slot); }

void batch_slot_stats(yg_batch bt, int32_t slot, yg_solve_stats *out) {
    const BatchScal &sc = bt->h_scal[slot];
    yg_solve_stats st{};
    st.iterations = sc.iter;
    st.rel_residual = sc.bb > 0 ? std::sqrt(sc.true_rr / sc.bb) : std::sqrt(sc.true_rr);
    st.refinements = (int32_t)sc.replacements;
    switch (sc.flag) {
    case BF_DONE: st.status = YG_OK; break;
    case BF_BREAK: st.status = YG_BREAKDOWN; break;
    case BF_NANF: st.status = YG_NAN; break;
    case BF_RUN: case BF_INIT: st.status = YG_RUNNING; break;
    default: st.status = YG_NOT_CONVERGED; break;
    }
    *out = st;
}
}  // namespace yg
