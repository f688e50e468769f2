// batch.cu -- many independent systems solved together (batched / served Krylov).
//
// No reference counterpart: the reference solves one system per call
// (pcg_solve.hpp:126-178, bicgstab_solve.hpp:19-95).  Each system keeps its own
// matrix (CSR or BCSR with 2x2 / 3x3 blocks), right-hand side, iterate and work
// vectors, and is solved either by Jacobi-PCG (symmetric positive definite
// systems) or by BiCGSTAB with right Jacobi preconditioning (non-symmetric
// ones).  Two work tables drive persistent-grid kernels over all systems:
//   matrix items: a system's block rows cut into tiles of whole rows (at most
//     WCfg<B>::CAP blocks each), runs of consecutive tiles forming an item that
//     one warp streams through its own shared-memory ring (bulk asynchronous
//     copies, cp.async.bulk + mbarrier) -- no CTA-wide barrier in the SpMV;
//   vector items: row chunks of about 4096 entries, one CTA each.
// Both are grouped by (method, block size).  One iteration is five steps:
//   V1  BiCGSTAB: p = r + beta (p - omega v), ph = D^-1 p
//   S1  SpMV: PCG q = A p (partials of p.q -> alpha); BiCGSTAB v = A ph
//       (partials of r0.v -> alpha)
//   V2  PCG: x, r updates, z = D^-1 r, partials of r.z, r.r -> beta and the
//       stopping tests; BiCGSTAB: s = r - alpha v, sh = D^-1 s
//   S2  BiCGSTAB SpMV t = A sh (partials of t.s, t.t -> omega)
//   V3  PCG: p = z + beta p; BiCGSTAB: x += alpha ph + omega sh, r = s - omega t,
//       partials of r0.r, r.r -> beta and the stopping tests
// (V1 and S2 are launched only when BiCGSTAB systems are present).  Every
// decision about a system is taken once, by the warp or CTA that completes the
// system's last item of a kernel (a per-system ticket; systems with more than
// kChunk matrix items sum their partials in two levels), so every CTA of the
// next kernel sees the same state.  A system whose matrix holds at least
// solo_bytes runs S1/S2 as its own launch of the single-system SpMV kernel
// followed by a one-warp decision kernel, both in the captured graph.  Sums run in a fixed order over a fixed item
// decomposition: a system's result does not depend on which other systems
// share the batch.  Converged systems drop out of the kernels at once and out
// of the work tables at the next compaction.  A block of m iterations plus a
// verification pass is captured into one CUDA graph and replayed; the
// verification pass recomputes b - A x in FP64 for systems whose recursive
// residual converged or broke down (stop), whose mixed-precision residual fell
// 100x since the last replacement (replace), and for newly added systems
// (init).  Systems can be added and removed between replays (continuous
// batching): only the descriptor and work tables change, and kernels read their
// ranges from device memory, so the captured graph stays valid while the set of
// (method, block size) groups present and of systems with their own SpMV launch
// does not change.
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
    const double *corr32;         // mixed precision: the FP32 values' row-sum correction (else NULL)
    const double *b, *dinv;
    double *x, *r, *p, *q;        // q: SpMV output of PCG and of the verification (BiCGSTAB: q is t)
    double *r0, *v, *s, *t, *ph, *sh;  // BiCGSTAB only
    const int32_t *tiles;         // first block row of each tile, ntiles + 1 entries
    int32_t mitem_begin, mitem_end;  // matrix items (SpMV)
    int32_t vitem_begin, vitem_end;  // vector items
    int32_t precision;            // YG_PREC_FP64 or YG_PREC_MIXED
    int32_t ntiles;
    int32_t method;
    int32_t solo;                 // 1: the iteration SpMV is the single-system kernel (large matrix)
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

struct BatchMItem {
    int32_t sys, tile_begin, tile_end;  // tiles [tile_begin, tile_end) of system sys
    int32_t row_begin, row_end;         // their block rows
    int32_t pad[3];
};
struct BatchVItem {
    int32_t sys, row_begin, row_end, pad;  // block rows
};

constexpr int kGroups = 6;  // (method, block size): group = 3 * method + block - 1
// d_ranges: [0, 8) first matrix item of each group then the end; [8, 16) the same for vector items
constexpr int kVR = 8;
// [16, 16 + kGroups): end of each group's matrix items that the iteration SpMV
// kernels take (the items of systems with their own SpMV follow, for the
// verification pass only)
constexpr int kRanges = 3 * kVR;
// A system whose FP64 matrix holds at least this many bytes runs its iteration
// SpMV as one launch of the single-system kernel (autotuned for its matrix, fused
// dot products) inside the batch's graph: at that size the launch is amortised
// and the single-system kernels stream closer to the HBM roofline than the
// shared batch kernels.
constexpr int64_t kSoloSpmvBytes = 128ll << 20;

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
    BatchMItem *d_mitems = nullptr;
    BatchVItem *d_vitems = nullptr;
    int32_t *d_ranges = nullptr;
    double *d_mpart = nullptr;          // SpMV partials: 2 per matrix item
    int32_t *d_cticket = nullptr;       // per matrix item: finished items of the chunk it starts (zero between kernels)
    double *d_vpart = nullptr;          // vector partials: 2 per vector item
    double *d_vpart2 = nullptr;         // b.b partials of the verification
    int32_t max_mitems = 0, max_vitems = 0, cticket_cap = 0;
    int32_t tiles_per_item[4] = {0, 4, 4, 4};
    int32_t lanes[4] = {4, 4, 8, 16};
    int32_t variant[4] = {1, 1, 1, 0};   // SpMV variant per block size: 0 staged, 1 direct
    unsigned groups_present = 0, graph_groups = 0;
    bool dirty = false;                 // work tables out of date (systems added, removed or reset)
    int32_t live_items = 0;             // vector items of systems that may still iterate (host view)
    int m = 16;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;         // recorded after each launched block
    bool in_flight = false;
    // live systems with their own SpMV launches (slot, matrix), and the list the
    // captured graph holds; partial sums of those launches
    std::vector<std::pair<int, yg_matrix>> solo, graph_solo;
    double *d_solo_part = nullptr;
    yg_status solo_err = YG_OK;         // first failed launch of those SpMVs while capturing
    int64_t solo_bytes = kSoloSpmvBytes;  // threshold for systems added from now on (0: none)
    cudaGraph_t graph = nullptr;
    int64_t graph_kernels = 0;
    std::vector<BatchScal> h_scal;
};

namespace yg {

// ---------------------------------------------------------------- configuration

// Per block size: blocks (and rows) per tile (CAP), stages of each warp's ring
// (NST) and warps per CTA.  A stage holds one FP64 tile's values, block columns
// and row pointers (4-10 KB).
template <int B> struct WCfg;
template <> struct WCfg<1> { static constexpr int CAP = 192, NST = 2, WARPS = 8; };
template <> struct WCfg<2> { static constexpr int CAP = 72, NST = 2, WARPS = 8; };
template <> struct WCfg<3> { static constexpr int CAP = 128, NST = 2, WARPS = 4; };

static int tile_cap(int B) { return B == 1 ? WCfg<1>::CAP : (B == 2 ? WCfg<2>::CAP : WCfg<3>::CAP); }

template <int B>
struct WStage {
    static constexpr int VB = WCfg<B>::CAP * B * B * 8 + 32;  // FP64 values + alignment slack
    static constexpr int CB = WCfg<B>::CAP * 4 + 32;
    static constexpr int RB = WCfg<B>::CAP * 4 + 48;  // row pointers of the tile's rows + 1
    static constexpr int HB = 32;                      // tile header (TileHdr)
    static constexpr int BYTES = VB + CB + RB + HB;
    static constexpr int WARP_BYTES = WCfg<B>::NST * BYTES;
    static constexpr int SMEM = WCfg<B>::WARPS * (WARP_BYTES + WCfg<B>::NST * 8);
};

// block rows per vector item: about 4096 entries
static int vitem_rows(int B) { return 4096 / B; }

// SpMV kinds
enum { SP_CG = 0, SP_VERIFY = 1, SP_BICG_V = 2, SP_BICG_T = 3 };

// ---------------------------------------------------------------- device helpers

enum { ACT_ITER = 0, ACT_VERIFY = 1, ACT_RESTART = 2 };
__device__ __forceinline__ int activity(const BatchScal *sc, int kind) {
    const volatile BatchScal *v = sc;
    const int flag = v->flag, stop = v->stop, rep = v->replace, rst = v->restart;
    if (kind == ACT_ITER) return flag == BF_RUN && stop == BS_NONE;
    if (kind == ACT_VERIFY) return (flag == BF_INIT) || (flag == BF_RUN && (stop == BS_CONV || rep));
    return rst != 0;
}

// Whether system state `sc` takes part in a kernel of the given kind, decided
// once per CTA: thread 0 reads the state and broadcasts it, so every thread of
// the CTA takes the same branch around the block reductions.
__device__ __forceinline__ bool cta_active(const BatchScal *sc, int kind, int *flag_sm) {
    __syncthreads();
    if (threadIdx.x == 0) *flag_sm = activity(sc, kind);
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

// The same for one warp and any ticket (lane 0 publishes, the verdict is
// broadcast).
__device__ __forceinline__ bool warp_last_of(int32_t *ticket, int n_items, int lane) {
    int last = 0;
    if (lane == 0) {
        __threadfence();
        const int old = atomicAdd(ticket, 1);
        last = (old == n_items - 1);
        if (last) {
            *ticket = 0;
            __threadfence();
        }
    }
    return __shfl_sync(0xffffffffu, last, 0) != 0;
}
__device__ __forceinline__ bool warp_last_of_system(BatchScal *sc, int n_items, int lane) {
    return warp_last_of(&sc->ticket, n_items, lane);
}

// Fixed-order sums of partials [ib, ie) (stride 2, offset off): by a CTA (result
// in every thread) or by a warp (xor butterfly; result in every lane).
__device__ __forceinline__ double sum_items(const double *part, int ib, int ie, int off, double *sm) {
    double v = 0;
    for (int i = ib + threadIdx.x; i < ie; i += blockDim.x) v += __ldcg(part + 2 * (int64_t)i + off);
    return block_sum_all<kThreads>(v, sm);
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum_items(const double *part, int ib, int ie, int off, int lane) {
    double v = 0;
    for (int i = ib + lane; i < ie; i += 32) v += __ldcg(part + 2 * (int64_t)i + off);
    return warp_sum(v);
}
// Sum of the partials of items ib, ib + step, ib + 2 step, ... (n of them).
__device__ __forceinline__ double warp_sum_strided(const double *part, int ib, int n, int step, int off, int lane) {
    double v = 0;
#pragma unroll 4
    for (int k = lane; k < n; k += 32) v += __ldcg(part + 2 * ((int64_t)ib + (int64_t)k * step) + off);
    return warp_sum(v);
}

// Matrix items per reduction chunk: a system with more items than this sums
// its item partials in two levels (chunks of kChunk items, then the chunk sums),
// so the warp that finishes a large system reads a few thousand partials
// instead of tens of thousands one after the other.
constexpr int kChunk = 32;
// Matrix items of one system at most (longer items beyond): enough for every
// warp of the grid to take a few, few enough that the per-item publication
// (fence, ticket, partial) stays small against the item's rows.
constexpr int kMaxItems = 16384;

// Rows [r0, r1) of one tile, by one warp with L lanes per block row; vals / cols
// point at the tile's first block and rowptr at row r0's pointer (shared
// memory, or global memory for an oversized tile).  out = A xin on those rows; dot1 += out.w (iteration kinds),
// dot2 += out.out (SP_BICG_T); the sums stay in the lanes that wrote the rows.
template <int B, int L, int KIND, typename VT>
__device__ __forceinline__ void tile_rows(const int32_t *rowptr, int r0, int r1, int b0, const VT *vals,
                                          const int32_t *cols, const double *__restrict__ xin, double *__restrict__ out,
                                          const double *__restrict__ w, double &dot1, double &dot2, int lane,
                                          const double *__restrict__ corr) {
    constexpr int B2 = B * B;
    constexpr int G = 32 / L;
    const int glane = lane % L, grp = lane / L;
    for (int rb = r0; rb < r1; rb += G) {
        const int r = rb + grp;
        double acc[B];
#pragma unroll
        for (int i = 0; i < B; ++i) acc[i] = 0;
        if (r < r1) {
            const int rs = rowptr[r - r0] - b0, re = rowptr[r - r0 + 1] - b0;
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
            if (corr) add_corr<B>(corr, xin, r, acc);
#pragma unroll
            for (int i = 0; i < B; ++i) {
                out[(int64_t)B * r + i] = acc[i];
                if (KIND != SP_VERIFY) dot1 = fma(acc[i], w[(int64_t)B * r + i], dot1);
                if (KIND == SP_BICG_T) dot2 = fma(acc[i], acc[i], dot2);
            }
        }
    }
}

// Header of a staged tile, written by the issuing lane.
struct TileHdr {
    int32_t item, r0, r1, b0, nb, last, pad0, pad1;
};

// The same with every lane on consecutive blocks of the tile (lanes == 1 in the
// tuning): 32 blocks per round, each lane's block product, a segmented
// inclusive warp scan by row (rows are contiguous runs of blocks), and the lane
// that ends a row's run writes the row (a row continuing into the next round
// carries its partial sum).  Rows without blocks are written as zero.
template <int B, int KIND, typename VT>
__device__ __forceinline__ void tile_rows_seg(const int32_t *rows, int r0, int r1, int b0, const VT *vals,
                                              const int32_t *cols, const double *__restrict__ xin,
                                              double *__restrict__ out, const double *__restrict__ w, double &dot1,
                                              double &dot2, int lane, const double *__restrict__ corr) {
    constexpr int B2 = B * B;
    const int nrows = r1 - r0;
    const int nb = rows[nrows] - b0;
    double carry[B];
#pragma unroll
    for (int i = 0; i < B; ++i) carry[i] = 0;
    int carry_row = -1;
    int rl = 0;  // local row of this lane's block (only grows)
    for (int base = 0; base < nb; base += 32) {
        const int j = base + lane;
        const bool valid = j < nb;
        double v[B];
#pragma unroll
        for (int i = 0; i < B; ++i) v[i] = 0;
        int myrow = 1 << 30;
        if (valid) {
            while (rows[rl + 1] - b0 <= j) ++rl;
            myrow = rl;
            const int c = cols[j];
            double x[B];
#pragma unroll
            for (int k = 0; k < B; ++k) x[k] = __ldg(xin + (int64_t)B * c + k);
#pragma unroll
            for (int i = 0; i < B; ++i)
#pragma unroll
                for (int k = 0; k < B; ++k) v[i] = fma((double)vals[j * B2 + i * B + k], x[k], v[i]);
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int ro = __shfl_up_sync(0xffffffffu, myrow, o);
#pragma unroll
            for (int i = 0; i < B; ++i) {
                const double vo = __shfl_up_sync(0xffffffffu, v[i], o);
                if (lane >= o && ro == myrow) v[i] += vo;
            }
        }
        const int next_row = __shfl_down_sync(0xffffffffu, myrow, 1);
        const bool seg_end = valid && (lane == 31 || next_row != myrow);
        // the run of this segment continues a row carried from the previous round
        if (seg_end && myrow == carry_row) {
#pragma unroll
            for (int i = 0; i < B; ++i) v[i] += carry[i];
        }
        const bool row_done = seg_end && (rows[myrow + 1] - b0 - 1 == j);
        if (row_done) {
            const int r = r0 + myrow;
            if (corr) add_corr<B>(corr, xin, r, v);
#pragma unroll
            for (int i = 0; i < B; ++i) {
                out[(int64_t)B * r + i] = v[i];
                if (KIND != SP_VERIFY) dot1 = fma(v[i], w[(int64_t)B * r + i], dot1);
                if (KIND == SP_BICG_T) dot2 = fma(v[i], v[i], dot2);
            }
        }
        // lane 31 ends the round: an unfinished row is carried
        const int last_open = __shfl_sync(0xffffffffu, (valid && !row_done) ? 1 : 0, 31);
        if (last_open) {
#pragma unroll
            for (int i = 0; i < B; ++i) carry[i] = __shfl_sync(0xffffffffu, v[i], 31);
            carry_row = __shfl_sync(0xffffffffu, myrow, 31);
        } else {
            carry_row = -1;
        }
    }
    // rows without blocks
    for (int k = lane; k < nrows; k += 32)
        if (rows[k + 1] == rows[k]) {
#pragma unroll
            for (int i = 0; i < B; ++i) out[(int64_t)B * (r0 + k) + i] = 0;
        }
}

// Lane 0 issues the bulk copies of tile t of a system (values, block columns,
// row pointers) into stage seq % NST of this warp's ring and writes the tile's
// header; an empty or oversized tile completes its phase with no transfer and
// is read from global memory instead.  t < 0 stands for an item without tiles.
template <int B>
__device__ __forceinline__ void issue_tile(unsigned char *ring, uint64_t *bars, uint32_t seq, int item, int last,
                                           const int32_t *__restrict__ rowptr, const int32_t *__restrict__ tiles, int t,
                                           const char *vbase, int vsz, const int32_t *col, uint64_t pol, int lane) {
    using S = WStage<B>;
    constexpr int B2 = B * B;
    if (lane != 0) return;
    const int st = seq % WCfg<B>::NST;
    unsigned char *dst = ring + (size_t)st * S::BYTES;
    TileHdr *h = reinterpret_cast<TileHdr *>(dst + S::VB + S::CB + S::RB);
    int r0 = 0, r1 = 0, b0 = 0, nb = 0;
    if (t >= 0) {
        r0 = tiles[t];
        r1 = tiles[t + 1];
        b0 = rowptr[r0];
        nb = rowptr[r1] - b0;
    }
    h->item = item;
    h->r0 = r0;
    h->r1 = r1;
    h->b0 = b0;
    h->nb = nb;
    h->last = last;
    if (nb > 0 && nb <= WCfg<B>::CAP) {
        const int64_t vs = (int64_t)b0 * B2 * vsz, va = vs & ~(int64_t)15;
        const int64_t ve = (vs + (int64_t)nb * B2 * vsz + 15) & ~(int64_t)15;
        const int64_t cs = (int64_t)b0 * 4, ca = cs & ~(int64_t)15, ce = (cs + (int64_t)nb * 4 + 15) & ~(int64_t)15;
        const int64_t ps = (int64_t)r0 * 4, pa = ps & ~(int64_t)15, pe = ((int64_t)r1 * 4 + 4 + 15) & ~(int64_t)15;
        mbar_expect_tx(&bars[st], (unsigned)((ve - va) + (ce - ca) + (pe - pa)));
        bulk_g2s(dst, vbase + va, (unsigned)(ve - va), &bars[st], pol);
        bulk_g2s(dst + S::VB, reinterpret_cast<const char *>(col) + ca, (unsigned)(ce - ca), &bars[st], pol);
        bulk_g2s(dst + S::VB + S::CB, reinterpret_cast<const char *>(rowptr) + pa, (unsigned)(pe - pa), &bars[st], pol);
    } else {
        mbar_expect_tx(&bars[st], 0);
    }
}

// Loads of one block's values (streamed: L1 no-allocate, L2 evict-first) and of
// the B entries of x it multiplies, with vector loads where the layout allows.
__device__ __forceinline__ double2 ld_stream2(const double *p, uint64_t pol) {
    double2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
        : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream_f(const float *p, uint64_t pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ld_stream_f4(const float *p, uint64_t pol) {
    float4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p), "l"(pol));
    return v;
}
template <int B2>
__device__ __forceinline__ void load_block(const double *p, double *v, uint64_t pol) {
    if (B2 == 4) {  // 32-byte blocks: 16-byte aligned
        const double2 a = ld_stream2(p, pol), b = ld_stream2(p + 2, pol);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
#pragma unroll
        for (int k = 0; k < B2; ++k) v[k] = ld_stream(p + k, pol);
    }
}
template <int B2>
__device__ __forceinline__ void load_block(const float *p, double *v, uint64_t pol) {
    if (B2 == 4) {  // 16-byte blocks: 16-byte aligned
        const float4 a = ld_stream_f4(p, pol);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else {
#pragma unroll
        for (int k = 0; k < B2; ++k) v[k] = ld_stream_f(p + k, pol);
    }
}
template <int B>
__device__ __forceinline__ void load_x(const double *p, double *x) {
    if (B == 2) {  // 16-byte aligned pairs
        const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
        x[0] = a.x; x[1] = a.y;
    } else {
#pragma unroll
        for (int k = 0; k < B; ++k) x[k] = __ldg(p + k);
    }
}

// Warp-wide bounded wait on a stage: lane 0 polls, the verdict is broadcast; the
// other lanes then observe the completed phase themselves (acquire).
__device__ __forceinline__ bool warp_stage_wait(uint64_t *bar, unsigned parity, int lane) {
    int ok = 1;
    if (lane == 0) {
        long long spins = 0;
        while (!mbar_try_wait(bar, parity))
            if (++spins > kSpinLimit) { ok = 0; break; }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (ok && lane != 0) mbar_try_wait(bar, parity);
    return ok != 0;
}

// ---------------------------------------------------------------- kernels

// End of a matrix item in a warp: publish its partials; the warp that
// completes the system's last item takes the reduction and the decision.
// The decision after an iteration SpMV of a system, from its dot products:
//   SP_CG      alpha = r.z / p.q
//   SP_BICG_V  alpha = rho / r0.v
//   SP_BICG_T  omega = t.s / t.t
template <int KIND>
__device__ __forceinline__ void decide_spmv(BatchScal &sc, double a, double tt, int parity) {
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

// Systems with more than kChunk items: the warp that finishes a chunk's last
// item sums the chunk (in item order) into the partial slot of the chunk's
// first item (cticket[first item] counts the chunk's finished items); the warp
// that finishes the last chunk sums the chunk sums in chunk order.
template <int KIND>
__device__ __forceinline__ void finish_item(const BatchSys *__restrict__ sys, BatchScal *__restrict__ scal,
                                            double *__restrict__ part, int32_t *__restrict__ cticket, int it, int s,
                                            int parity, double dot1, double dot2, int lane) {
    dot1 = warp_sum(dot1);
    if (KIND == SP_BICG_T) dot2 = warp_sum(dot2);
    if (lane == 0) {
        part[2 * (int64_t)it] = dot1;
        if (KIND == SP_BICG_T) part[2 * (int64_t)it + 1] = dot2;
    }
    const int ib = sys[s].mitem_begin, ie = sys[s].mitem_end;
    double a, tt = 0.0;
    if (ie - ib <= kChunk) {
        if (!warp_last_of_system(&scal[s], ie - ib, lane)) return;
        a = warp_sum_items(part, ib, ie, 0, lane);
        if (KIND == SP_BICG_T) tt = warp_sum_items(part, ib, ie, 1, lane);
    } else {
        const int cb = ib + (it - ib) / kChunk * kChunk, ce = min(ie, cb + kChunk);
        if (!warp_last_of(&cticket[cb], ce - cb, lane)) return;
        const double ca = warp_sum_items(part, cb, ce, 0, lane);
        const double ct = KIND == SP_BICG_T ? warp_sum_items(part, cb, ce, 1, lane) : 0.0;
        if (lane == 0) {
            part[2 * (int64_t)cb] = ca;
            if (KIND == SP_BICG_T) part[2 * (int64_t)cb + 1] = ct;
        }
        const int nch = (ie - ib + kChunk - 1) / kChunk;
        if (!warp_last_of_system(&scal[s], nch, lane)) return;
        a = warp_sum_strided(part, ib, nch, kChunk, 0, lane);
        if (KIND == SP_BICG_T) tt = warp_sum_strided(part, ib, nch, kChunk, 1, lane);
    }
    if (lane != 0) return;
    decide_spmv<KIND>(scal[s], a, tt, parity);
}

// A system with its own SpMV launch: one warp sums that launch's per-CTA
// partials (np of them; DOT 2 launches store pairs) in CTA order and takes the
// same decision as the last item of a batched SpMV.
template <int KIND>
__global__ void k_batch_solo_finish(BatchScal *__restrict__ scal, const double *__restrict__ part, int np, int s,
                                    int parity) {
    const int lane = threadIdx.x & 31;
    int act = lane == 0 ? activity(&scal[s], ACT_ITER) : 0;
    if (!__shfl_sync(0xffffffffu, act, 0)) return;
    double a = 0, tt = 0;
    for (int i = lane; i < np; i += 32) {
        if (KIND == SP_BICG_T) {
            a += __ldcg(part + 2 * i);
            tt += __ldcg(part + 2 * i + 1);
        } else {
            a += __ldcg(part + i);
        }
    }
    a = warp_sum(a);
    if (KIND == SP_BICG_T) tt = warp_sum(tt);
    if (lane == 0) decide_spmv<KIND>(scal[s], a, tt, parity);
}

// Direct-load SpMV of one group (no staging): each warp takes whole items; L
// lanes per block row, each lane loading up to U whole blocks (values with
// vector loads and an L2 evict-first hint, columns) and then the gathered x
// before using them; the next row group's bounds are loaded one step ahead.
// Same operations and reductions as k_batch_spmv.
template <int B, int L, int KIND, typename VT>
__device__ __forceinline__ void direct_rows(const int32_t *__restrict__ rowptr, int r0, int r1,
                                            const VT *__restrict__ val, const int32_t *__restrict__ col,
                                            const double *__restrict__ xin, double *__restrict__ out,
                                            const double *__restrict__ w, double &dot1, double &dot2, int lane,
                                            uint64_t pol, const double *__restrict__ corr) {
    constexpr int B2 = B * B;
    constexpr int G = 32 / L;
    constexpr int U = B == 1 ? 4 : (B == 2 ? 2 : 1);
    const int glane = lane % L, grp = lane / L;
    int r = r0 + grp;
    int rs = 0, re = 0;
    if (r < r1) { rs = __ldg(rowptr + r); re = __ldg(rowptr + r + 1); }
#pragma unroll 1
    for (int rb = r0; rb < r1; rb += G, r += G) {
        int rs_n = 0, re_n = 0;
        if (r + G < r1) { rs_n = __ldg(rowptr + r + G); re_n = __ldg(rowptr + r + G + 1); }
        double acc[B];
#pragma unroll
        for (int i = 0; i < B; ++i) acc[i] = 0;
#pragma unroll 1
        for (int j0 = rs + glane; j0 < re; j0 += U * L) {
            int c[U];
            double v[U][B2], x[U][B];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = j0 + u * L;
                c[u] = 0;
                if (j < re) {
                    c[u] = ld_stream_i(col + j, pol);
                    load_block<B2>(val + (int64_t)j * B2, v[u], pol);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (j0 + u * L < re) load_x<B>(xin + (int64_t)B * c[u], x[u]);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (j0 + u * L < re) {
#pragma unroll
                    for (int i = 0; i < B; ++i)
#pragma unroll
                        for (int k = 0; k < B; ++k) acc[i] = fma(v[u][i * B + k], x[u][k], acc[i]);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < B; ++i)
#pragma unroll
            for (int o = L / 2; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
        if (r < r1 && glane == 0) {
            if (corr) add_corr<B>(corr, xin, r, acc);
#pragma unroll
            for (int i = 0; i < B; ++i) {
                out[(int64_t)B * r + i] = acc[i];
                if (KIND != SP_VERIFY) dot1 = fma(acc[i], w[(int64_t)B * r + i], dot1);
                if (KIND == SP_BICG_T) dot2 = fma(acc[i], acc[i], dot2);
            }
        }
        rs = rs_n;
        re = re_n;
    }
}

// Each warp walks its items (grid stride), loading the next item's descriptor
// while it works on the current one.
template <int B, int L, int KIND>
__global__ void __launch_bounds__(256, 3)
k_batch_spmv_direct(const BatchMItem *__restrict__ items, const int32_t *__restrict__ ranges, int g,
                    const BatchSys *__restrict__ sys, BatchScal *__restrict__ scal, double *__restrict__ part,
                    int32_t *__restrict__ cticket, int parity, int commit) {
    const int lane = threadIdx.x & 31;
    const int W = gridDim.x * (blockDim.x >> 5);
    const int g1 = KIND == SP_VERIFY ? ranges[g + 1] : ranges[2 * kVR + g];
    const uint64_t pol = evict_first_policy();
    int it = ranges[g] + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int s_n = 0, r0_n = 0, r1_n = 0;  // the item to work on next
    if (it < g1) { s_n = items[it].sys; r0_n = items[it].row_begin; r1_n = items[it].row_end; }
    for (; it < g1; it += W) {
        const int s = s_n, r0 = r0_n, r1 = r1_n;
        if (it + W < g1) { s_n = items[it + W].sys; r0_n = items[it + W].row_begin; r1_n = items[it + W].row_end; }
        int act = lane == 0 ? activity(&scal[s], KIND == SP_VERIFY ? ACT_VERIFY : ACT_ITER) : 0;
        if (__shfl_sync(0xffffffffu, act, 0)) {
            const BatchSys &d = sys[s];
            const double *xin = KIND == SP_CG ? d.p : KIND == SP_VERIFY ? d.x : KIND == SP_BICG_V ? d.ph : d.sh;
            double *out = (KIND == SP_CG || KIND == SP_VERIFY) ? d.q : KIND == SP_BICG_V ? d.v : d.t;
            const double *w = KIND == SP_CG ? d.p : KIND == SP_BICG_V ? d.r0 : d.s;
            double dot1 = 0, dot2 = 0;
            if (KIND != SP_VERIFY && d.precision == YG_PREC_MIXED)
                direct_rows<B, L, KIND, float>(d.rowptr, r0, r1, d.val32, d.col, xin, out, w, dot1, dot2, lane, pol,
                                               d.corr32);
            else
                direct_rows<B, L, KIND, double>(d.rowptr, r0, r1, d.val, d.col, xin, out, w, dot1, dot2, lane, pol,
                                                nullptr);
            if (KIND != SP_VERIFY && commit)
                finish_item<KIND>(sys, scal, part, cticket, it, s, parity, dot1, dot2, lane);
        }
    }
}

// The SpMV of one group of matrix items (ranges[g], ranges[g + 1]); each warp
// takes whole items (g0 + warp id, then every W-th) and streams their tiles
// through its ring, the issuing lane running up to NST tiles ahead, across item
// boundaries:
//   SP_CG      q = A p, partials of p.q; last warp: alpha = r.z / p.q
//   SP_VERIFY  q = A x with FP64 values (systems under verification)
//   SP_BICG_V  v = A ph, partials of r0.v; last warp: alpha = rho / r0.v
//   SP_BICG_T  t = A sh, partials of t.s and t.t; last warp: omega = t.s / t.t
// The iteration kinds read FP32 values for mixed-precision systems.  With
// commit == 0 (autotuning) the reductions are not taken.  A system's state
// cannot change while one of its items is still to be processed (its reductions
// wait for all of them), so the activity test of an item read ahead holds.
template <int B, int L, int KIND>
__global__ void __launch_bounds__(WCfg<B>::WARPS * 32)
k_batch_spmv(const BatchMItem *__restrict__ items, const int32_t *__restrict__ ranges, int g,
             const BatchSys *__restrict__ sys, BatchScal *__restrict__ scal, double *__restrict__ part,
             int32_t *__restrict__ cticket, int parity, int commit, int32_t *__restrict__ err) {
    using S = WStage<B>;
    constexpr int B2 = B * B;
    constexpr int CAP = WCfg<B>::CAP, NST = WCfg<B>::NST, WARPS = WCfg<B>::WARPS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *ring = smem_raw + (size_t)wib * S::WARP_BYTES;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)WARPS * S::WARP_BYTES) + wib * NST;
    if (lane == 0)
        for (int k = 0; k < NST; ++k) mbar_init(&bars[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();
    const uint64_t pol = evict_first_policy();
    const int g1 = KIND == SP_VERIFY ? ranges[g + 1] : ranges[2 * kVR + g];
    const int W = gridDim.x * WARPS;
    const int act_kind = KIND == SP_VERIFY ? ACT_VERIFY : ACT_ITER;

    // issue cursor (uniform in the warp): item ii, its next tile ti < te
    int ii = ranges[g] + blockIdx.x * WARPS + wib - W;
    int ti = 0, te = 0;
    const int32_t *i_rowptr = nullptr, *i_tiles = nullptr, *i_col = nullptr;
    const char *i_vbase = nullptr;
    int i_vsz = 8;
    bool issue_done = false;
    auto next_item = [&]() {  // advance the issue cursor to the next active item
        for (;;) {
            ii += W;
            if (ii >= g1) {
                issue_done = true;
                return;
            }
            const BatchMItem item = items[ii];
            int act = lane == 0 ? activity(&scal[item.sys], act_kind) : 0;
            if (!__shfl_sync(0xffffffffu, act, 0)) continue;
            const BatchSys &d = sys[item.sys];
            const bool f32 = (KIND != SP_VERIFY && d.precision == YG_PREC_MIXED);
            i_rowptr = d.rowptr;
            i_tiles = d.tiles;
            i_col = d.col;
            i_vsz = f32 ? 4 : 8;
            i_vbase = f32 ? reinterpret_cast<const char *>(d.val32) : reinterpret_cast<const char *>(d.val);
            ti = item.tile_begin;
            te = item.tile_end;
            return;
        }
    };
    uint32_t seq_issue = 0, seq_wait = 0;  // tiles issued / consumed by this warp
    auto issue_next = [&]() {
        if (ti >= te) {  // an item without tiles: one empty tile closes it
            issue_tile<B>(ring, bars, seq_issue++, ii, 1, i_rowptr, i_tiles, -1, i_vbase, i_vsz, i_col, pol, lane);
            next_item();
            return;
        }
        const int last = ti + 1 == te;
        issue_tile<B>(ring, bars, seq_issue++, ii, last, i_rowptr, i_tiles, ti, i_vbase, i_vsz, i_col, pol, lane);
        if (++ti == te) next_item();
    };
    next_item();

    // consume cursor: the item of the last consumed tile and its operands
    int ci = -1, cs = 0;
    const double *xin = nullptr, *w = nullptr;
    double *out = nullptr;
    const int32_t *c_rowptr = nullptr, *c_col = nullptr;
    const double *c_val = nullptr;
    const float *c_val32 = nullptr;
    const double *c_corr = nullptr;
    bool c_f32 = false;
    double dot1 = 0, dot2 = 0;
    bool timed_out = false;
    for (;;) {
        while (!issue_done && seq_issue - seq_wait < (uint32_t)NST) issue_next();
        if (seq_wait == seq_issue) break;
        const int st = seq_wait % NST;
        if (!warp_stage_wait(&bars[st], (seq_wait / NST) & 1u, lane)) {
            timed_out = true;
            break;
        }
        const unsigned char *stg = ring + (size_t)st * S::BYTES;
        const TileHdr h = *reinterpret_cast<const TileHdr *>(stg + S::VB + S::CB + S::RB);
        if (h.item != ci) {
            ci = h.item;
            cs = items[ci].sys;
            const BatchSys &d = sys[cs];
            c_f32 = (KIND != SP_VERIFY && d.precision == YG_PREC_MIXED);
            c_rowptr = d.rowptr;
            c_col = d.col;
            c_val = d.val;
            c_val32 = d.val32;
            c_corr = c_f32 ? d.corr32 : nullptr;
            xin = KIND == SP_CG ? d.p : KIND == SP_VERIFY ? d.x : KIND == SP_BICG_V ? d.ph : d.sh;
            out = (KIND == SP_CG || KIND == SP_VERIFY) ? d.q : KIND == SP_BICG_V ? d.v : d.t;
            w = KIND == SP_CG ? d.p : KIND == SP_BICG_V ? d.r0 : d.s;
        }
        if (h.r1 > h.r0) {
            const int vsz = c_f32 ? 4 : 8;
            const int lv = (int)(((int64_t)h.b0 * B2 * vsz) & 15), lc = (int)(((int64_t)h.b0 * 4) & 15);
            const bool staged = h.nb > 0 && h.nb <= CAP;
            const int32_t *cols = staged ? reinterpret_cast<const int32_t *>(stg + S::VB + lc) : c_col + h.b0;
            const int32_t *rows = staged ? reinterpret_cast<const int32_t *>(stg + S::VB + S::CB + ((h.r0 * 4) & 15))
                                         : c_rowptr + h.r0;
            if (c_f32) {
                const float *v = staged ? reinterpret_cast<const float *>(stg + lv) : c_val32 + (int64_t)h.b0 * B2;
                if (L == 1)
                    tile_rows_seg<B, KIND, float>(rows, h.r0, h.r1, h.b0, v, cols, xin, out, w, dot1, dot2, lane, c_corr);
                else
                    tile_rows<B, L, KIND, float>(rows, h.r0, h.r1, h.b0, v, cols, xin, out, w, dot1, dot2, lane, c_corr);
            } else {
                const double *v = staged ? reinterpret_cast<const double *>(stg + lv) : c_val + (int64_t)h.b0 * B2;
                if (L == 1)
                    tile_rows_seg<B, KIND, double>(rows, h.r0, h.r1, h.b0, v, cols, xin, out, w, dot1, dot2, lane, nullptr);
                else
                    tile_rows<B, L, KIND, double>(rows, h.r0, h.r1, h.b0, v, cols, xin, out, w, dot1, dot2, lane, nullptr);
            }
        }
        ++seq_wait;
        __syncwarp();  // the stage is free for the next issue
        if (h.last) {
            if (KIND != SP_VERIFY && commit)
                finish_item<KIND>(sys, scal, part, cticket, ci, cs, parity, dot1, dot2, lane);
            dot1 = dot2 = 0;
        }
    }
    if (timed_out && lane == 0 && err) atomicExch(err, (int32_t)YG_TIMEOUT);
    // drain the copies still in flight before the warp exits (bounded)
    if (lane == 0) {
        while (seq_wait != seq_issue) {
            const int st = seq_wait % NST;
            long long spins = 0;
            while (!mbar_try_wait(&bars[st], (seq_wait / NST) & 1u) && ++spins <= kSpinLimit) {
            }
            ++seq_wait;
        }
    }
    __syncwarp();
}

// Vector kernels take kU elements per thread per step, loads first, so each
// thread keeps kU independent loads of every operand in flight.
constexpr int kU = 4;

// V1 (BiCGSTAB vector items only): p = r + beta (p - omega v) (p = r after a restart), ph = D^-1 p
__global__ void __launch_bounds__(kThreads)
k_batch_v1(const BatchVItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
           const BatchScal *__restrict__ scal) {
    __shared__ int flag_sm;
    const int i0 = ranges[kVR + 3], i1 = ranges[kVR + kGroups];
    for (int it = i0 + blockIdx.x; it < i1; it += gridDim.x) {
        const BatchVItem item = items[it];
        const int s = item.sys;
        if (!cta_active(&scal[s], ACT_ITER, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const bool fresh = __ldcg(&scal[s].fresh) != 0;
        const double beta = __ldcg(&scal[s].beta), omega = __ldcg(&scal[s].omega);
        const int64_t lo = (int64_t)item.row_begin * d.block, hi = (int64_t)item.row_end * d.block;
        double *__restrict__ p = d.p, *__restrict__ ph = d.ph;
        const double *__restrict__ r = d.r, *__restrict__ v = d.v, *__restrict__ dinv = d.dinv;
        for (int64_t i0 = lo + threadIdx.x; i0 < hi; i0 += kU * kThreads) {
            double pv[kU], rv[kU], vv[kU], dv[kU];
#pragma unroll
            for (int k = 0; k < kU; ++k) {
                const int64_t i = i0 + k * kThreads;
                if (i < hi) { rv[k] = r[i]; dv[k] = dinv[i]; pv[k] = fresh ? 0.0 : p[i]; vv[k] = fresh ? 0.0 : v[i]; }
            }
#pragma unroll
            for (int k = 0; k < kU; ++k) {
                const int64_t i = i0 + k * kThreads;
                if (i < hi) {
                    const double pi = fresh ? rv[k] : rv[k] + beta * (pv[k] - omega * vv[k]);
                    p[i] = pi;
                    ph[i] = dv[k] * pi;
                }
            }
        }
    }
}

// V2: PCG x and r updates, Jacobi z, partials of r.z and r.r, the last CTA of a
// system takes its decisions (beta, convergence of the recursive residual, NaN,
// iteration cap, a due mixed-precision replacement); BiCGSTAB s = r - alpha v,
// sh = D^-1 s.
__global__ void __launch_bounds__(kThreads)
k_batch_v2(const BatchVItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
           BatchScal *__restrict__ scal, int parity, double *__restrict__ part) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int flag_sm;
    const int n_items = ranges[kVR + kGroups];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchVItem item = items[it];
        const int s = item.sys;
        BatchScal &sc = scal[s];
        if (!cta_active(&sc, ACT_ITER, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const double alpha = __ldcg(&sc.alpha);
        const int64_t lo = (int64_t)item.row_begin * d.block, hi = (int64_t)item.row_end * d.block;
        if (d.method == BM_BICG) {
            double *__restrict__ sv = d.s, *__restrict__ sh = d.sh;
            const double *__restrict__ r = d.r, *__restrict__ v = d.v, *__restrict__ dinv = d.dinv;
            for (int64_t i0 = lo + threadIdx.x; i0 < hi; i0 += kU * kThreads) {
                double rv[kU], vv[kU], dv[kU];
#pragma unroll
                for (int k = 0; k < kU; ++k) {
                    const int64_t i = i0 + k * kThreads;
                    if (i < hi) { rv[k] = r[i]; vv[k] = v[i]; dv[k] = dinv[i]; }
                }
#pragma unroll
                for (int k = 0; k < kU; ++k) {
                    const int64_t i = i0 + k * kThreads;
                    if (i < hi) {
                        const double si = rv[k] - alpha * vv[k];
                        sv[i] = si;
                        sh[i] = dv[k] * si;
                    }
                }
            }
            continue;
        }
        double srz = 0, srr = 0;
        {
            double *__restrict__ x = d.x, *__restrict__ r = d.r;
            const double *__restrict__ p = d.p, *__restrict__ q = d.q, *__restrict__ dinv = d.dinv;
            for (int64_t i0 = lo + threadIdx.x; i0 < hi; i0 += kU * kThreads) {
                double pv[kU], qv[kU], rv[kU], xv[kU], dv[kU];
#pragma unroll
                for (int k = 0; k < kU; ++k) {
                    const int64_t i = i0 + k * kThreads;
                    if (i < hi) { pv[k] = p[i]; qv[k] = q[i]; rv[k] = r[i]; xv[k] = x[i]; dv[k] = dinv[i]; }
                }
#pragma unroll
                for (int k = 0; k < kU; ++k) {
                    const int64_t i = i0 + k * kThreads;
                    if (i < hi) {
                        x[i] = xv[k] + pv[k] * alpha;
                        const double ri = rv[k] + (-alpha) * qv[k];
                        r[i] = ri;
                        srz += ri * (dv[k] * ri);
                        srr += ri * ri;
                    }
                }
            }
        }
        srz = block_sum<kThreads>(srz, sm);
        srr = block_sum<kThreads>(srr, sm);
        if (threadIdx.x == 0) {
            part[2 * (int64_t)it] = srz;
            part[2 * (int64_t)it + 1] = srr;
        }
        if (last_of_system(&sc, d.vitem_end - d.vitem_begin, &flag_sm)) {
            const double rz_new = sum_items(part, d.vitem_begin, d.vitem_end, 0, sm);
            const double rr = sum_items(part, d.vitem_begin, d.vitem_end, 1, sm);
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
k_batch_v3(const BatchVItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
           BatchScal *__restrict__ scal, double *__restrict__ part) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int flag_sm;
    const int n_items = ranges[kVR + kGroups];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchVItem item = items[it];
        const int s = item.sys;
        BatchScal &sc = scal[s];
        if (!cta_active(&sc, ACT_ITER, &flag_sm)) continue;
        const BatchSys d = sys[s];
        const int64_t lo = (int64_t)item.row_begin * d.block, hi = (int64_t)item.row_end * d.block;
        if (d.method == BM_CG) {
            const double beta = __ldcg(&sc.beta);
            double *__restrict__ p = d.p;
            const double *__restrict__ r = d.r, *__restrict__ dinv = d.dinv;
            for (int64_t i0 = lo + threadIdx.x; i0 < hi; i0 += kU * kThreads) {
                double pv[kU], rv[kU], dv[kU];
#pragma unroll
                for (int k = 0; k < kU; ++k) {
                    const int64_t i = i0 + k * kThreads;
                    if (i < hi) { pv[k] = p[i]; rv[k] = r[i]; dv[k] = dinv[i]; }
                }
#pragma unroll
                for (int k = 0; k < kU; ++k) {
                    const int64_t i = i0 + k * kThreads;
                    if (i < hi) p[i] = dv[k] * rv[k] + beta * pv[k];
                }
            }
            continue;
        }
        const double alpha = __ldcg(&sc.alpha), omega = __ldcg(&sc.omega);
        double srr0 = 0, srr = 0;
        {
            double *__restrict__ x = d.x, *__restrict__ r = d.r;
            const double *__restrict__ ph = d.ph, *__restrict__ sh = d.sh, *__restrict__ sv = d.s,
                                      *__restrict__ tv = d.t, *__restrict__ r0 = d.r0;
            for (int64_t i0 = lo + threadIdx.x; i0 < hi; i0 += kU * kThreads) {
                double a[kU], b[kU], c[kU], e[kU], f[kU], g[kU];
#pragma unroll
                for (int k = 0; k < kU; ++k) {
                    const int64_t i = i0 + k * kThreads;
                    if (i < hi) { a[k] = x[i]; b[k] = ph[i]; c[k] = sh[i]; e[k] = sv[i]; f[k] = tv[i]; g[k] = r0[i]; }
                }
#pragma unroll
                for (int k = 0; k < kU; ++k) {
                    const int64_t i = i0 + k * kThreads;
                    if (i < hi) {
                        x[i] = a[k] + (alpha * b[k] + omega * c[k]);
                        const double ri = e[k] - omega * f[k];
                        r[i] = ri;
                        srr0 += g[k] * ri;
                        srr += ri * ri;
                    }
                }
            }
        }
        srr0 = block_sum<kThreads>(srr0, sm);
        srr = block_sum<kThreads>(srr, sm);
        if (threadIdx.x == 0) {
            part[2 * (int64_t)it] = srr0;
            part[2 * (int64_t)it + 1] = srr;
        }
        if (last_of_system(&sc, d.vitem_end - d.vitem_begin, &flag_sm)) {
            const double rho_new = sum_items(part, d.vitem_begin, d.vitem_end, 0, sm);
            const double rr = sum_items(part, d.vitem_begin, d.vitem_end, 1, sm);
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
k_batch_residual(const BatchVItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
                 const BatchScal *__restrict__ scal, double *__restrict__ part, double *__restrict__ part_bb) {
    __shared__ double sm[kThreads / 32 + 1];
    __shared__ int flag_sm;
    const int n_items = ranges[kVR + kGroups];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchVItem item = items[it];
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
    for (int i = d.vitem_begin; i < d.vitem_end; ++i) {
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
k_batch_restart(const BatchVItem *__restrict__ items, const int32_t *__restrict__ ranges, const BatchSys *__restrict__ sys,
                const BatchScal *__restrict__ scal) {
    __shared__ int flag_sm;
    const int n_items = ranges[kVR + kGroups];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchVItem item = items[it];
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
        cudaFuncSetAttribute(k_batch_spmv<B, L, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, WStage<B>::SMEM);
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_spmv<B, L, KIND>, WCfg<B>::WARPS * 32,
                                                          WStage<B>::SMEM) != cudaSuccess || n < 1)
            n = 1;
        per_sm = n;
    }
    return per_sm * ctx->num_sms;
}

template <int B, int L, int KIND>
static int direct_grid(yg_context ctx) {
    static int per_sm = 0;
    if (per_sm == 0) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_spmv_direct<B, L, KIND>, 256, 0) != cudaSuccess ||
            n < 1)
            n = 1;
        per_sm = n;
    }
    return per_sm * ctx->num_sms;
}

template <int B, int L, int KIND>
static void launch_spmv_l(yg_batch bt, int variant, int g, int parity, int commit) {
    yg_context ctx = bt->ctx;
    if (variant == 1) {
        k_batch_spmv_direct<B, L, KIND><<<direct_grid<B, L, KIND>(ctx), 256, 0, ctx->stream>>>(
            bt->d_mitems, bt->d_ranges, g, bt->d_sys, bt->d_scal, bt->d_mpart, bt->d_cticket, parity, commit);
    } else {
        k_batch_spmv<B, L, KIND><<<spmv_grid<B, L, KIND>(ctx), WCfg<B>::WARPS * 32, WStage<B>::SMEM, ctx->stream>>>(
            bt->d_mitems, bt->d_ranges, g, bt->d_sys, bt->d_scal, bt->d_mpart, bt->d_cticket, parity, commit,
            ctx->d_err);
    }
    YG_LAUNCHED(ctx);
}

template <int B, int KIND>
static void launch_spmv_b(yg_batch bt, int V, int L, int g, int parity, int commit) {
    switch (L) {
    case 1: launch_spmv_l<B, 1, KIND>(bt, V, g, parity, commit); break;
    case 2: launch_spmv_l<B, 2, KIND>(bt, V, g, parity, commit); break;
    case 4: launch_spmv_l<B, 4, KIND>(bt, V, g, parity, commit); break;
    case 8: launch_spmv_l<B, 8, KIND>(bt, V, g, parity, commit); break;
    case 16: launch_spmv_l<B, 16, KIND>(bt, V, g, parity, commit); break;
    default: launch_spmv_l<B, 32, KIND>(bt, V, g, parity, commit); break;
    }
}

template <int KIND>
static void launch_spmv_kind(yg_batch bt, int B, int V, int L, int g, int parity, int commit) {
    if (B == 1) launch_spmv_b<1, KIND>(bt, V, L, g, parity, commit);
    else if (B == 2) launch_spmv_b<2, KIND>(bt, V, L, g, parity, commit);
    else launch_spmv_b<3, KIND>(bt, V, L, g, parity, commit);
}

// one SpMV launch for group g (method, block size) of the given kind; variant
// 0 stages tiles in shared memory, 1 loads directly
static void launch_spmv(yg_batch bt, int kind, int g, int parity, int commit, int L = 0, int V = -1) {
    const int B = g % 3 + 1;
    if (L == 0) L = bt->lanes[B];
    if (V < 0) V = bt->variant[B];
    switch (kind) {
    case SP_CG: launch_spmv_kind<SP_CG>(bt, B, V, L, g, parity, commit); break;
    case SP_VERIFY: launch_spmv_kind<SP_VERIFY>(bt, B, V, L, g, parity, commit); break;
    case SP_BICG_V: launch_spmv_kind<SP_BICG_V>(bt, B, V, L, g, parity, commit); break;
    default: launch_spmv_kind<SP_BICG_T>(bt, B, V, L, g, parity, commit); break;
    }
}

// set the shared-memory attribute of every SpMV instantiation (outside capture)
template <int B, int KIND>
static void prepare_spmv_bk(yg_context ctx) {
    spmv_grid<B, 1, KIND>(ctx); direct_grid<B, 1, KIND>(ctx);
    spmv_grid<B, 2, KIND>(ctx); spmv_grid<B, 4, KIND>(ctx); spmv_grid<B, 8, KIND>(ctx);
    spmv_grid<B, 16, KIND>(ctx); spmv_grid<B, 32, KIND>(ctx);
    direct_grid<B, 2, KIND>(ctx); direct_grid<B, 4, KIND>(ctx); direct_grid<B, 8, KIND>(ctx);
    direct_grid<B, 16, KIND>(ctx); direct_grid<B, 32, KIND>(ctx);
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
    k_batch_residual<<<grid, kThreads, 0, ctx->stream>>>(bt->d_vitems, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_vpart,
                                                        bt->d_vpart2);
    YG_LAUNCHED(ctx);
    k_batch_decide<<<(bt->capacity + 127) / 128, 128, 0, ctx->stream>>>(bt->capacity, bt->d_sys, bt->d_scal, bt->d_vpart,
                                                                         bt->d_vpart2);
    YG_LAUNCHED(ctx);
    k_batch_restart<<<grid, kThreads, 0, ctx->stream>>>(bt->d_vitems, bt->d_ranges, bt->d_sys, bt->d_scal);
    YG_LAUNCHED(ctx);
}

// The iteration SpMV of each system that has its own launch (kind SP_CG or
// SP_BICG_V for the first SpMV of an iteration, SP_BICG_T for the second), each
// followed by its one-warp decision.  The SpMV kernel skips a system whose flag
// says it is not running; the decision also skips a stopped one.
static void launch_solo(yg_batch bt, int kind, int parity) {
    yg_context ctx = bt->ctx;
    for (const auto &e : bt->solo) {
        const int s = e.first;
        yg_matrix A = e.second;
        const BatchSys &d = bt->sys[s];
        const bool bicg = d.method == BM_BICG;
        if ((kind == SP_BICG_T || kind == SP_BICG_V) != bicg) continue;
        const int prec = d.precision == YG_PREC_MIXED ? YG_PREC_MIXED : YG_PREC_FP64;
        const int grid = std::min(spmv_grid_for(A, prec), kMaxReduceBlocks);  // the launch's CTAs = partials
        const int32_t *flag = &bt->d_scal[s].flag;
        const int64_t l0 = A->ctx->launches;
        yg_status st;
        const double *corr = prec == YG_PREC_MIXED ? A->d_corr32 : nullptr;
        if (kind == SP_CG) {
            st = spmv_launch_ex(A, d.p, d.q, prec, d.p, bt->d_solo_part, 1, flag, grid, ctx->stream, nullptr, corr);
            k_batch_solo_finish<SP_CG><<<1, 32, 0, ctx->stream>>>(bt->d_scal, bt->d_solo_part, grid, s, parity);
        } else if (kind == SP_BICG_V) {
            st = spmv_launch_ex(A, d.ph, d.v, prec, d.r0, bt->d_solo_part, 1, flag, grid, ctx->stream, nullptr, corr);
            k_batch_solo_finish<SP_BICG_V><<<1, 32, 0, ctx->stream>>>(bt->d_scal, bt->d_solo_part, grid, s, parity);
        } else {
            st = spmv_launch_ex(A, d.sh, d.t, prec, d.s, bt->d_solo_part, 2, flag, grid, ctx->stream, nullptr, corr);
            k_batch_solo_finish<SP_BICG_T><<<1, 32, 0, ctx->stream>>>(bt->d_scal, bt->d_solo_part, grid, s, parity);
        }
        if (st != YG_OK && bt->solo_err == YG_OK) bt->solo_err = st;
        // count the SpMV on this context (A may belong to another one), and the decision
        const int64_t dl = A->ctx->launches - l0;
        A->ctx->launches -= dl;
        ctx->launches += dl + 1;
    }
}

static void launch_iteration(yg_batch bt, int parity) {
    yg_context ctx = bt->ctx;
    const int grid = batch_grid(ctx);
    if (has_bicg(bt)) {
        k_batch_v1<<<grid, kThreads, 0, ctx->stream>>>(bt->d_vitems, bt->d_ranges, bt->d_sys, bt->d_scal);
        YG_LAUNCHED(ctx);
    }
    for (int g = 0; g < kGroups; ++g)
        if (has(bt, g)) launch_spmv(bt, g < 3 ? SP_CG : SP_BICG_V, g, parity, 1);
    launch_solo(bt, SP_CG, parity);
    launch_solo(bt, SP_BICG_V, parity);
    k_batch_v2<<<grid, kThreads, 0, ctx->stream>>>(bt->d_vitems, bt->d_ranges, bt->d_sys, bt->d_scal, parity,
                                                  bt->d_vpart);
    YG_LAUNCHED(ctx);
    for (int g = 3; g < kGroups; ++g)
        if (has(bt, g)) launch_spmv(bt, SP_BICG_T, g, parity, 1);
    launch_solo(bt, SP_BICG_T, parity);
    k_batch_v3<<<grid, kThreads, 0, ctx->stream>>>(bt->d_vitems, bt->d_ranges, bt->d_sys, bt->d_scal, bt->d_vpart);
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

template <typename T>
static yg_status grow(yg_context ctx, T **p, int32_t *cap, size_t need, double **part, double **part2) {
    if ((int64_t)need <= *cap) return YG_OK;
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    dev_free(ctx, *p);
    dev_free(ctx, *part);
    if (part2) dev_free(ctx, *part2);
    *p = nullptr;
    *part = nullptr;
    if (part2) *part2 = nullptr;
    const int32_t c = (int32_t)need * 2 + 64;
    YG_TRY(dev_alloc_t(ctx, p, c));
    YG_TRY(dev_alloc_t(ctx, part, 2 * (size_t)c));
    if (part2) YG_TRY(dev_alloc_t(ctx, part2, 2 * (size_t)c));
    *cap = c;
    return YG_OK;
}

// Rebuild the work tables: systems grouped by (method, block size); matrix
// items of tiles_per_item tiles, vector items of vitem_rows block rows.
// Systems that finished are left out (their kernels' item loops stay short);
// the groups present count every system in the batch, so compaction never
// changes the set of SpMV launches that the captured graph holds.  A system's
// items are always cut the same way for a given tuning, so its reductions add
// the same partials in the same order whatever else is in the tables.
static yg_status rebuild_items(yg_batch bt) {
    yg_context ctx = bt->ctx;
    std::vector<BatchMItem> mitems;
    std::vector<BatchVItem> vitems;
    int32_t ranges[kRanges] = {0};
    unsigned present = 0;
    std::vector<std::pair<int, yg_matrix>> solo;
    for (int g = 0; g < kGroups; ++g) {
        const int method = g / 3, B = g % 3 + 1;
        ranges[g] = (int32_t)mitems.size();
        ranges[kVR + g] = (int32_t)vitems.size();
        const int T = std::max(1, bt->tiles_per_item[B]), VR = vitem_rows(B);
        // systems of the group with batched iteration SpMVs first, then those with their own
        for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) ranges[2 * kVR + g] = (int32_t)mitems.size();
        for (int s = 0; s < bt->capacity; ++s) {
            if (!bt->used[s] || bt->sys[s].block != B || bt->sys[s].method != method) continue;
            if (bt->sys[s].solo != pass) continue;
            if (pass == 1 && sys_live(bt, s)) solo.push_back({s, bt->mats[s]});
            present |= 1u << g;
            BatchSys &d = bt->sys[s];
            d.mitem_begin = (int32_t)mitems.size();
            d.vitem_begin = (int32_t)vitems.size();
            if (sys_live(bt, s)) {
                const std::vector<int32_t> &tl = bt->tiles[s];
                // a large system takes longer items: at most kMaxItems of them
                const int Ts = std::max(T, (d.ntiles + kMaxItems - 1) / kMaxItems);
                for (int t0 = 0; t0 < d.ntiles; t0 += Ts) {
                    const int t1 = std::min(d.ntiles, t0 + Ts);
                    mitems.push_back({s, t0, t1, tl[t0], tl[t1], {0, 0, 0}});
                }
                if (d.ntiles == 0) mitems.push_back({s, 0, 0, 0, 0, {0, 0, 0}});
                for (int r0 = 0; r0 < d.nbrows; r0 += VR) vitems.push_back({s, r0, std::min(d.nbrows, r0 + VR), 0});
                if (d.nbrows == 0) vitems.push_back({s, 0, 0, 0});
            }
            d.mitem_end = (int32_t)mitems.size();
            d.vitem_end = (int32_t)vitems.size();
        }
        }
    }
    ranges[kGroups] = ranges[kGroups + 1] = (int32_t)mitems.size();
    ranges[kVR + kGroups] = ranges[kVR + kGroups + 1] = (int32_t)vitems.size();
    const bool regrow = (int64_t)mitems.size() > bt->max_mitems || (int64_t)vitems.size() > bt->max_vitems;
    YG_TRY(grow(ctx, &bt->d_mitems, &bt->max_mitems, mitems.size(), &bt->d_mpart, (double **)nullptr));
    if (bt->cticket_cap < bt->max_mitems) {  // grew: the stream is idle (grow synchronised it)
        dev_free(ctx, bt->d_cticket);
        bt->d_cticket = nullptr;
        bt->cticket_cap = 0;
        YG_TRY(dev_alloc_t(ctx, &bt->d_cticket, bt->max_mitems));
        YG_CUDA(cudaMemsetAsync(bt->d_cticket, 0, sizeof(int32_t) * bt->max_mitems, ctx->stream));
        bt->cticket_cap = bt->max_mitems;
    }
    YG_TRY(grow(ctx, &bt->d_vitems, &bt->max_vitems, vitems.size(), &bt->d_vpart, &bt->d_vpart2));
    if (regrow) drop_graph(bt);  // the graph captured the old pointers
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (!mitems.empty())
        YG_CUDA(cudaMemcpy(bt->d_mitems, mitems.data(), sizeof(BatchMItem) * mitems.size(), cudaMemcpyHostToDevice));
    if (!vitems.empty())
        YG_CUDA(cudaMemcpy(bt->d_vitems, vitems.data(), sizeof(BatchVItem) * vitems.size(), cudaMemcpyHostToDevice));
    YG_CUDA(cudaMemcpy(bt->d_ranges, ranges, sizeof(ranges), cudaMemcpyHostToDevice));
    YG_CUDA(cudaMemcpy(bt->d_sys, bt->sys.data(), sizeof(BatchSys) * bt->capacity, cudaMemcpyHostToDevice));
    bt->groups_present = present;
    bt->solo = solo;
    bt->live_items = (int32_t)vitems.size();
    bt->dirty = false;
    return YG_OK;
}

static yg_status capture_graph(yg_batch bt) {
    yg_context ctx = bt->ctx;
    drop_graph(bt);
    int64_t before = ctx->launches;
    bt->solo_err = YG_OK;
    YG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < bt->m; ++it) launch_iteration(bt, it & 1);
    launch_verify(bt);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    bt->graph_kernels = ctx->launches - before;
    ctx->launches = before;
    if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "batch graph capture: %s", cudaGetErrorString(e));
    if (bt->solo_err != YG_OK) {
        cudaGraphDestroy(g);
        return bt->solo_err;
    }
    bt->graph = g;
    YG_CUDA(cudaGraphInstantiate(&bt->exec, g, 0));
    bt->graph_groups = bt->groups_present;
    bt->graph_solo = bt->solo;
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

// Cut block rows into tiles of whole rows with at most `cap` blocks and `cap`
// rows each (a row longer than cap forms a tile of its own, read from global
// memory).
static void make_tiles(const std::vector<int32_t> &rp, int cap, std::vector<int32_t> &tiles) {
    tiles.clear();
    const int n = (int)rp.size() - 1;
    tiles.push_back(0);
    int start = 0;
    for (int r = 0; r < n; ++r) {
        if (r > start && (rp[r + 1] - rp[start] > cap || r - start >= cap)) {
            tiles.push_back(r);
            start = r;
        }
    }
    if (n > 0) tiles.push_back(n);
}

// Host view of a slot after the last wait: whether it still iterates, and its
// stats (from the state copied back at the end of the block).
bool batch_slot_running(yg_batch bt, int32_t slot) { return sys_live(bt, slot); }

static void stats_of(const BatchScal &sc, yg_solve_stats *out) {
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

void batch_slot_stats(yg_batch bt, int32_t slot, yg_solve_stats *out) { stats_of(bt->h_scal[slot], out); }

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
        (s = dev_alloc_t(ctx, &bt->d_ranges, kRanges)) != YG_OK ||
        (s = dev_alloc_t(ctx, &bt->d_solo_part, 2 * kMaxReduceBlocks)) != YG_OK) {
        yg_batch_destroy(bt);
        return s;
    }
    prepare_spmv_b<1>(ctx);
    prepare_spmv_b<2>(ctx);
    prepare_spmv_b<3>(ctx);
    if (cudaEventCreateWithFlags(&bt->done, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        bt->done = nullptr;
        yg_batch_destroy(bt);
        return fail(YG_CUDA_ERROR, "yg_batch_create: event creation failed");
    }
    std::vector<BatchScal> init(capacity);
    for (auto &c : init) c.flag = BF_EMPTY;
    bt->h_scal = init;
    cudaMemcpy(bt->d_scal, init.data(), sizeof(BatchScal) * capacity, cudaMemcpyHostToDevice);
    cudaMemset(bt->d_ranges, 0, sizeof(int32_t) * kRanges);
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
    for (void *p : {(void *)bt->d_sys, (void *)bt->d_scal, (void *)bt->d_mitems, (void *)bt->d_vitems, (void *)bt->d_ranges,
                    (void *)bt->d_mpart, (void *)bt->d_cticket, (void *)bt->d_vpart, (void *)bt->d_vpart2,
                    (void *)bt->d_solo_part})
        dev_free(bt->ctx, p);
    if (bt->done) cudaEventDestroy(bt->done);
    delete bt;
    return YG_OK;
}

extern "C" yg_status yg_batch_set_solo_bytes(yg_batch bt, int64_t bytes) {
    if (!bt) return fail(YG_BAD_ARG, "yg_batch_set_solo_bytes: NULL batch");
    bt->solo_bytes = bytes < 0 ? 0 : bytes;
    return YG_OK;
}

extern "C" yg_status yg_batch_ready(yg_batch bt, int32_t *ready) {
    if (!bt || !ready) return fail(YG_BAD_ARG, "yg_batch_ready: NULL argument");
    *ready = 1;
    if (!bt->in_flight) return YG_OK;
    const cudaError_t e = cudaEventQuery(bt->done);
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        *ready = 0;
        return YG_OK;
    }
    if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "yg_batch_ready: %s", cudaGetErrorString(e));
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
    for (yg_context c : {A->ctx, b->ctx, x->ctx})
        if (c->device != bt->ctx->device)
            return fail(YG_BAD_ARG, "yg_batch_add: the system lives on device %d, the batch on device %d", c->device,
                        bt->ctx->device);
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
    // Objects built on another context of the device (its own stream, so their
    // assembly overlaps a running block): their pending work completes first.
    for (yg_context c : {A->ctx, b->ctx, x->ctx})
        if (c != ctx) YG_CUDA(cudaStreamSynchronize(c->stream));
    // tiles of whole rows, from the row pointer
    std::vector<int32_t> rp(A->nbrows + 1);
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    YG_CUDA(cudaMemcpy(rp.data(), A->d_rowptr, sizeof(int32_t) * rp.size(), cudaMemcpyDeviceToHost));
    std::vector<int32_t> tl;
    make_tiles(rp, tile_cap(A->block), tl);
    BatchSys d{};
    d.block = A->block;
    d.nbrows = (int32_t)A->nbrows;
    d.rowptr = A->d_rowptr;
    d.col = A->d_col;
    d.val = A->d_val;
    d.val32 = A->d_val32;
    d.corr32 = o.precision == YG_PREC_MIXED ? A->d_corr32 : nullptr;
    d.b = b->d;
    d.x = x->d;
    d.precision = o.precision;
    d.method = method;
    d.ntiles = (int32_t)tl.size() - 1;
    d.solo = bt->solo_bytes > 0 && A->nnzb * (int64_t)A->block * A->block * 8 >= bt->solo_bytes;
    if (d.solo) YG_TRY(spmv_autotune_device(A));  // its own SpMV: tune it now, outside any capture
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
    YG_CUDA(cudaEventRecord(bt->done, ctx->stream));
    bt->in_flight = true;
    return YG_OK;
}

// Wait for the launched block, count the systems still running and compact the
// work tables once a quarter of the vector items is idle.
static yg_status batch_collect(yg_batch bt, int *active_out) {
    yg_context ctx = bt->ctx;
    YG_CUDA(cudaStreamSynchronize(ctx->stream));
    bt->in_flight = false;
    YG_TRY(check_device_error(ctx));
    int active = 0;
    int32_t live = 0;
    for (int s = 0; s < bt->capacity; ++s)
        if (sys_live(bt, s)) {
            ++active;
            live += bt->sys[s].vitem_end - bt->sys[s].vitem_begin;
        }
    if (active > 0 && live < bt->live_items - bt->live_items / 4 && bt->live_items - live >= 16)
        YG_TRY(rebuild_items(bt));
    *active_out = active;
    return YG_OK;
}

static yg_status batch_prepare(yg_batch bt) {
    if (bt->dirty) YG_TRY(rebuild_items(bt));
    if (!bt->exec || bt->graph_groups != bt->groups_present || bt->graph_solo != bt->solo) YG_TRY(capture_graph(bt));
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
    stats_of(sc, out);
    return YG_OK;
}

// Choose the SpMV variant, tiles per matrix item and lanes per block row for each block size from
// the systems present, by timing the iteration SpMV of the whole batch (without
// committing its reductions).
extern "C" yg_status yg_batch_tune(yg_batch bt) {
    if (!bt) return fail(YG_BAD_ARG, "yg_batch_tune: NULL batch");
    yg_context ctx = bt->ctx;
    // initialise p / ph from a verification pass so the SpMV reads defined data
    YG_TRY(rebuild_items(bt));
    launch_verify(bt);
    if (has_bicg(bt)) {
        k_batch_v1<<<batch_grid(ctx), kThreads, 0, ctx->stream>>>(bt->d_vitems, bt->d_ranges, bt->d_sys, bt->d_scal);
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
        int bestL = bt->lanes[B], bestT = bt->tiles_per_item[B], bestV = bt->variant[B];
        for (int T : {1, 4, 16}) {
            bt->tiles_per_item[B] = T;
            YG_TRY(rebuild_items(bt));
            for (int V : {0, 1})
                for (int L : {1, 2, 4, 8, 16, 32}) {
                    auto launch = [&]() {
                        if (cg) launch_spmv(bt, SP_CG, B - 1, 0, 0, L, V);
                        if (bi) launch_spmv(bt, SP_BICG_V, 3 + B - 1, 0, 0, L, V);
                    };
                    launch();
                    cudaEventRecord(e0, ctx->stream);
                    for (int r = 0; r < 3; ++r) launch();
                    cudaEventRecord(e1, ctx->stream);
                    cudaEventSynchronize(e1);
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (ms < best) { best = ms; bestL = L; bestT = T; bestV = V; }
                }
        }
        bt->lanes[B] = bestL;
        bt->tiles_per_item[B] = bestT;
        bt->variant[B] = bestV;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    YG_TRY(rebuild_items(bt));
    drop_graph(bt);
    YG_CUDA(cudaGetLastError());
    return check_device_error(ctx);
}

extern "C" yg_status yg_batch_get_tuning(yg_batch bt, int32_t *out) {
    if (!bt || !out) return fail(YG_BAD_ARG, "yg_batch_get_tuning: NULL argument");
    for (int B = 1; B <= 3; ++B) {
        out[3 * (B - 1)] = bt->variant[B];
        out[3 * (B - 1) + 1] = bt->lanes[B];
        out[3 * (B - 1) + 2] = bt->tiles_per_item[B];
    }
    return YG_OK;
}

extern "C" yg_status yg_batch_set_tuning(yg_batch bt, int32_t block, int32_t variant, int32_t lanes, int32_t tiles) {
    if (!bt || block < 1 || block > 3 || (variant != 0 && variant != 1) || tiles < 1 ||
        (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32))
        return fail(YG_BAD_ARG, "yg_batch_set_tuning: bad argument");
    bt->variant[block] = variant;
    bt->lanes[block] = lanes;
    bt->tiles_per_item[block] = tiles;
    bt->dirty = true;
    drop_graph(bt);
    return YG_OK;
}
