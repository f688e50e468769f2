// spmv.cu -- block-CSR / CSR sparse matrix-vector product, FP64 or FP32 values
// with FP64 accumulation, optionally fused with the dot product x.(Ax).
//
// Replaces csr_spmv (include/old_handmade_linalg/csr_spmv.hpp:25-56) and
// bcsr_spmv (bcsr_spmv.hpp:23-62).  Layout: int32 block-row pointer, int32
// block columns, values row-major inside each BxB block (the reference's
// sparse_bcsr layout, sparse_bcsr.hpp:227-229); block size 1 is plain CSR.
//
// Mapping: a group of L lanes owns one block row.  The lanes walk the row's
// value range flat and coalesced (lane l reads values l, l+L, ...), so every
// warp-wide load of the value stream touches consecutive bytes; each lane maps
// its value index to (block j, row i, column c) incrementally and gathers
// x[B*col[j]+c] through the read-only path.  The B partial row sums are reduced
// across the L lanes with a fixed xor-butterfly, so results are bit-identical
// from run to run.  The value stream carries an L2 evict-first hint so the
// gathered vector stays in L2.
#include "internal.h"
#include "device_common.cuh"

#include <type_traits>
#include <atomic>

// cudaFuncSetAttribute sets a kernel's shared-memory limit on the current device
// only: each launcher keeps one bit per device (0..63) it has been set on.  Two
// threads that both see the bit clear both set the same value.
static bool smem_attr_due(const std::atomic<uint64_t> &done, int device) {
    return device < 0 || device >= 64 || !(done.load(std::memory_order_acquire) & (1ull << device));
}
static void smem_attr_done(std::atomic<uint64_t> &done, int device) {
    if (device >= 0 && device < 64) done.fetch_or(1ull << device, std::memory_order_release);
}

namespace yg {

// DOT = 0: y = A x.  DOT = 1: also per-block sums of w.y.  DOT = 2: per-block
// sums of w.y and y.y (partials[2b], partials[2b+1]).
template <int B, int L, typename VT, int DOT>
__global__ void __launch_bounds__(kThreads, B == 1 ? 8 : 1)
k_bcsr_spmv(int64_t nbrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
            const VT *__restrict__ val, const double *__restrict__ x, double *__restrict__ y,
            const double *__restrict__ w, double *__restrict__ partials, const int32_t *__restrict__ flag, const double *__restrict__ corr) {
    __shared__ double sm[kThreads / 32 + 1];
    if (flag && read_flag(flag)) return;
    constexpr int B2 = B * B;
    constexpr int GPW = 32 / L;  // row groups per warp
    const uint64_t pol = evict_first_policy();
    const int lane = threadIdx.x & 31;
    const int glane = lane % L;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    double dot = 0, yy = 0;
    if constexpr (B == 1) {
        // Scalar rows: a lane issues the loads of up to U of its entries before
        // the first gather, and the next step's row bounds are fetched one step
        // ahead, so a step costs one value/column round trip and one gather round
        // trip instead of one per U/4 entries.  The accumulation order (the lane's
        // entries left to right, then the butterfly) is that of the loop below.
        constexpr int U = 8;
        const int64_t step = nwarps * GPW;
        int64_t r = warp * GPW + lane / L;
        int rs = 0, re = 0;
        if (r < nbrows) { rs = __ldg(rowptr + r); re = __ldg(rowptr + r + 1); }
        for (int64_t rb = warp * GPW; rb < nbrows; rb += step, r += step) {
            int rs_n = 0, re_n = 0;
            if (r + step < nbrows) { rs_n = __ldg(rowptr + r + step); re_n = __ldg(rowptr + r + step + 1); }
            double acc = 0;
            for (int k0 = rs + glane; k0 < re; k0 += L * U) {
                double v[U];
                int c[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int k = k0 + u * L;
                    v[u] = 0;
                    c[u] = 0;
                    if (k < re) {
                        v[u] = ld_stream(val + k, pol);
                        c[u] = ld_stream_i(col + k, pol);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (k0 + u * L < re) acc = fma(v[u], __ldg(x + c[u]), acc);
            }
#pragma unroll
            for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (r < nbrows && glane == 0) {
                if (corr) acc = fma(corr[r], x[r], acc);
                y[r] = acc;
                if (DOT >= 1) dot = fma(acc, w[r], dot);
                if (DOT == 2) yy = fma(acc, acc, yy);
            }
            rs = rs_n;
            re = re_n;
        }
    } else
    for (int64_t rb = warp * GPW; rb < nbrows; rb += nwarps * GPW) {
        const int64_t r = rb + lane / L;
        double acc[B];
#pragma unroll
        for (int i = 0; i < B; ++i) acc[i] = 0;
        if (r < nbrows) {
            const int rs = __ldg(rowptr + r), re = __ldg(rowptr + r + 1);
            const VT *vrow = val + (int64_t)rs * B2;
            const int32_t *crow = col + rs;
            const int nv = (re - rs) * B2;
            int j = glane / B2, e = glane % B2;
#pragma unroll 4
            for (int k = glane; k < nv; k += L) {
                const double v = ld_stream(vrow + k, pol);
                const int i = e / B, c = e - (e / B) * B;
                const double xv = __ldg(x + (int64_t)B * __ldg(crow + j) + c);
                if (B == 1) {
                    acc[0] = fma(v, xv, acc[0]);
                } else {
#pragma unroll
                    for (int ii = 0; ii < B; ++ii) acc[ii] = (ii == i) ? fma(v, xv, acc[ii]) : acc[ii];
                }
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
        if (r < nbrows && glane == 0) {
            if (corr) add_corr<B>(corr, x, r, acc);
#pragma unroll
            for (int i = 0; i < B; ++i) {
                y[B * r + i] = acc[i];
                if (DOT >= 1) dot = fma(acc[i], w[B * r + i], dot);
                if (DOT == 2) yy = fma(acc[i], acc[i], yy);
            }
        }
    }
    if (DOT == 1) {
        dot = block_sum<kThreads>(dot, sm);
        if (threadIdx.x == 0) partials[blockIdx.x] = dot;
    } else if (DOT == 2) {
        dot = block_sum<kThreads>(dot, sm);
        yy = block_sum<kThreads>(yy, sm);
        if (threadIdx.x == 0) { partials[2 * blockIdx.x] = dot; partials[2 * blockIdx.x + 1] = yy; }
    }
}

// ---------------------------------------------------------------------------
// Staged variant for B = 2, 3.  Each warp owns a sequence of block rows (grid
// stride) cut into chunks of at most CH blocks.  A chunk's value bytes and its
// block-column indices are copied into a per-warp shared-memory stage with
// 16-byte cp.async copies (L2 evict-first); NST stages form a ring, so NST-1
// chunks are in flight while one is consumed.  Consuming, lane l owns whole
// blocks l, l+32, ... of the chunk: B*B shared loads of values, one shared load
// of the column, B loads of x from L2, B*B FMAs.  Copies start at the 16-byte
// boundary at or below the data and end at the one at or above it (device
// allocations carry 16 bytes of padding); the consumer skips the lead bytes.
template <int B, typename VT>
struct Staged {
    static constexpr int CH = 64;                                      // blocks per chunk
    static constexpr int VBYTES = CH * B * B * (int)sizeof(VT) + 32;   // value bytes per stage
    static constexpr int CBYTES = CH * 4 + 32;                         // column bytes per stage
    static constexpr int STAGE = VBYTES + CBYTES;
    static constexpr int NST = 3;                                      // ring depth
    static constexpr int WARPS = 4;
    static constexpr int SMEM = WARPS * NST * STAGE;
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, uint64_t pol) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "l"(pol));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Chunk cursor of one warp: row r (grid stride `stride`), block offset b0.
struct ChunkCursor {
    int64_t r;
    int b0, rs, re;
    __device__ void load(const int32_t *__restrict__ rowptr, int64_t nbrows) {
        rs = re = 0;
        if (r < nbrows) { rs = __ldg(rowptr + r); re = __ldg(rowptr + r + 1); }
    }
    __device__ void advance(const int32_t *__restrict__ rowptr, int64_t nbrows, int64_t stride, int ch) {
        b0 += ch;
        if (b0 >= re - rs) {
            r += stride;
            b0 = 0;
            load(rowptr, nbrows);
        }
    }
};

template <int B, typename VT, int DOT>
__global__ void __launch_bounds__(Staged<B, VT>::WARPS * 32)
k_bcsr_spmv_staged(int64_t nbrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                   const VT *__restrict__ val, const double *__restrict__ x, double *__restrict__ y,
                   const double *__restrict__ w, double *__restrict__ partials, const int32_t *__restrict__ flag, const double *__restrict__ corr) {
    using S = Staged<B, VT>;
    constexpr int B2 = B * B;
    constexpr int BB = B2 * (int)sizeof(VT);  // value bytes per block
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[S::WARPS + 1];
    __shared__ int leads[S::WARPS][S::NST][2];
    if (flag && read_flag(flag)) return;
    const uint64_t pol = evict_first_policy();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *ring = smem_raw + (size_t)wib * S::NST * S::STAGE;
    const int64_t stride = (int64_t)gridDim.x * S::WARPS;
    const char *vbytes = reinterpret_cast<const char *>(val);
    const char *cbytes = reinterpret_cast<const char *>(col);

    auto issue = [&](const ChunkCursor &c, int st) {
        int lv = 0, lc = 0;
        if (c.r < nbrows && c.re > c.rs) {
            const int nb = min(S::CH, c.re - c.rs - c.b0);
            const int64_t first = (int64_t)(c.rs + c.b0);
            const int64_t vs = first * BB, va = vs & ~(int64_t)15, ve = (vs + (int64_t)nb * BB + 15) & ~(int64_t)15;
            const int64_t cs = first * 4, ca = cs & ~(int64_t)15, ce = (cs + (int64_t)nb * 4 + 15) & ~(int64_t)15;
            lv = (int)(vs - va);
            lc = (int)(cs - ca);
            unsigned char *dst = ring + st * S::STAGE;
            for (int64_t off = (int64_t)lane * 16; off < ve - va; off += 32 * 16) cp_async16(dst + off, vbytes + va + off, pol);
            for (int64_t off = (int64_t)lane * 16; off < ce - ca; off += 32 * 16)
                cp_async16(dst + S::VBYTES + off, cbytes + ca + off, pol);
        }
        if (lane == 0) { leads[wib][st][0] = lv; leads[wib][st][1] = lc; }
        cp_async_commit();
    };

    ChunkCursor ci{(int64_t)blockIdx.x * S::WARPS + wib, 0, 0, 0};
    ci.load(rowptr, nbrows);
    ChunkCursor cc = ci;
#pragma unroll
    for (int k = 0; k < S::NST - 1; ++k) {
        issue(ci, k);
        if (ci.r < nbrows) ci.advance(rowptr, nbrows, stride, S::CH);
    }
    double dot = 0, yy = 0;
    double acc[B];
#pragma unroll
    for (int i = 0; i < B; ++i) acc[i] = 0;
    int st = 0;
    while (cc.r < nbrows) {
        issue(ci, (st + S::NST - 1) % S::NST);
        if (ci.r < nbrows) ci.advance(rowptr, nbrows, stride, S::CH);
        cp_async_wait<S::NST - 1>();
        __syncwarp();
        const int nb = max(0, min(S::CH, cc.re - cc.rs - cc.b0));
        const unsigned char *stg = ring + st * S::STAGE;
        const VT *blk = reinterpret_cast<const VT *>(stg + leads[wib][st][0]);
        const int32_t *cix = reinterpret_cast<const int32_t *>(stg + S::VBYTES + leads[wib][st][1]);
        for (int j = lane; j < nb; j += 32) {
            const int c = cix[j];
            double xv[B];
#pragma unroll
            for (int k = 0; k < B; ++k) xv[k] = __ldg(x + (int64_t)B * c + k);
#pragma unroll
            for (int i = 0; i < B; ++i)
#pragma unroll
                for (int k = 0; k < B; ++k) acc[i] = fma((double)blk[j * B2 + i * B + k], xv[k], acc[i]);
        }
        __syncwarp();
        if (cc.b0 + S::CH >= cc.re - cc.rs) {  // row complete
#pragma unroll
            for (int i = 0; i < B; ++i) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
            }
            if (lane == 0) {
                if (corr) add_corr<B>(corr, x, cc.r, acc);
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    y[B * cc.r + i] = acc[i];
                    if (DOT >= 1) dot = fma(acc[i], w[B * cc.r + i], dot);
                    if (DOT == 2) yy = fma(acc[i], acc[i], yy);
                }
            }
#pragma unroll
            for (int i = 0; i < B; ++i) acc[i] = 0;
        }
        cc.advance(rowptr, nbrows, stride, S::CH);
        st = (st + 1) % S::NST;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (DOT) {
        // lane 0 of each warp holds the warp's sum; fixed-order block sum
        if (lane == 0) red[wib] = dot;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0;
            for (int i = 0; i < S::WARPS; ++i) sum += red[i];
            if (DOT == 1) partials[blockIdx.x] = sum;
            else partials[2 * blockIdx.x] = sum;
        }
        if (DOT == 2) {
            __syncthreads();
            if (lane == 0) red[wib] = yy;
            __syncthreads();
            if (threadIdx.x == 0) {
                double sum = 0;
                for (int i = 0; i < S::WARPS; ++i) sum += red[i];
                partials[2 * blockIdx.x + 1] = sum;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// TMA variant for B = 2, 3 (variant 2).  Same chunking and lane-per-block
// consumption as the staged variant, but each chunk is fetched by one lane with
// two bulk asynchronous copies (cp.async.bulk: values, then block columns) that
// complete on a per-stage mbarrier, so the copy costs two instructions instead
// of one 16-byte cp.async per lane and line.  Lanes take two blocks at a time
// with independent accumulators.  Waits on an mbarrier are bounded: after
// kSpinLimit polls the kernel records YG_TIMEOUT in `err` and stops.

template <int B, typename VT, int CH_, int NST_, int WARPS_>
struct TmaCfg {
    static constexpr int CH = CH_, NST = NST_, WARPS = WARPS_;
    static constexpr int VBYTES = CH * B * B * (int)sizeof(VT) + 32;
    static constexpr int CBYTES = CH * 4 + 32;
    static constexpr int STAGE = VBYTES + CBYTES;
    static constexpr int SMEM = WARPS * NST * STAGE + WARPS * NST * 8;  // stages + mbarriers
};

// XF: gather x from the FP32 node-padded copy x32 (one 16-byte load for a 3x3
// block, one 8-byte load for a 2x2 block) instead of B FP64 loads from x.
template <int B, bool XF>
__device__ __forceinline__ void gather_x(const double *__restrict__ x, const float *__restrict__ x32, int c,
                                         double (&xo)[B]) {
    if constexpr (XF && B == 3) {
        const float4 v = __ldg(reinterpret_cast<const float4 *>(x32) + c);
        xo[0] = v.x;
        xo[1] = v.y;
        xo[2] = v.z;
    } else if constexpr (XF && B == 2) {
        const float2 v = __ldg(reinterpret_cast<const float2 *>(x32) + c);
        xo[0] = v.x;
        xo[1] = v.y;
    } else {
#pragma unroll
        for (int k = 0; k < B; ++k) xo[k] = __ldg(x + (int64_t)B * c + k);
    }
}

// Transposed butterfly of B (2 or 3) sums over the warp: returns, in every lane,
// the full sum of component comp_of_lane(lane) = lane / (32 / Bp), Bp = 2 or 4.
template <int B>
__device__ __forceinline__ double reduce_rows_t(const double (&a)[B], int lane) {
    if constexpr (B == 2) {
        const bool up = lane & 16;
        double k = up ? a[1] : a[0];
        k += __shfl_xor_sync(0xffffffffu, up ? a[0] : a[1], 16);
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
        return k;
    } else {
        const bool up = lane & 16, mid = lane & 8;
        // step 1: the lower half keeps sums 0 and 1, the upper half sums 2 and 3 (3 is 0)
        double s0 = up ? a[2] : a[0];
        double s1 = up ? 0.0 : a[1];
        const double t0 = up ? a[0] : a[2];
        const double t1 = up ? a[1] : 0.0;
        s0 += __shfl_xor_sync(0xffffffffu, t0, 16);
        s1 += __shfl_xor_sync(0xffffffffu, t1, 16);
        // step 2: lanes with bit 3 keep the second of the two
        double k = mid ? s1 : s0;
        k += __shfl_xor_sync(0xffffffffu, mid ? s0 : s1, 8);
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
        return k;
    }
}

template <int B, typename VT, int DOT, typename C, bool XF>
__global__ void __launch_bounds__(C::WARPS * 32)
k_bcsr_spmv_tma(int64_t nbrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                const VT *__restrict__ val, const double *__restrict__ x, const float *__restrict__ x32,
                double *__restrict__ y, const double *__restrict__ w, double *__restrict__ partials,
                const int32_t *__restrict__ flag, const double *__restrict__ corr, int32_t *__restrict__ err) {
    constexpr int B2 = B * B;
    constexpr int BB = B2 * (int)sizeof(VT);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[C::WARPS + 1];
    __shared__ int leads[C::WARPS][C::NST][2];
    if (flag && read_flag(flag)) return;
    const uint64_t pol = evict_first_policy();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *ring = smem_raw + (size_t)wib * C::NST * C::STAGE;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)C::WARPS * C::NST * C::STAGE) + wib * C::NST;
    if (lane == 0)
        for (int k = 0; k < C::NST; ++k) mbar_init(&bars[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();
    const int64_t stride = (int64_t)gridDim.x * C::WARPS;
    const char *vbytes = reinterpret_cast<const char *>(val);
    const char *cbytes = reinterpret_cast<const char *>(col);

    // lane 0 issues both copies of chunk c into stage st
    auto issue = [&](const ChunkCursor &c, int st) {
        if (lane == 0) {
            int lv = 0, lc = 0;
            if (c.r < nbrows && c.re > c.rs) {
                const int nb = min(C::CH, c.re - c.rs - c.b0);
                const int64_t first = (int64_t)(c.rs + c.b0);
                const int64_t vs = first * BB, va = vs & ~(int64_t)15, ve = (vs + (int64_t)nb * BB + 15) & ~(int64_t)15;
                const int64_t cs = first * 4, ca = cs & ~(int64_t)15, ce = (cs + (int64_t)nb * 4 + 15) & ~(int64_t)15;
                lv = (int)(vs - va);
                lc = (int)(cs - ca);
                unsigned char *dst = ring + st * C::STAGE;
                mbar_expect_tx(&bars[st], (unsigned)((ve - va) + (ce - ca)));
                bulk_g2s(dst, vbytes + va, (unsigned)(ve - va), &bars[st], pol);
                bulk_g2s(dst + C::VBYTES, cbytes + ca, (unsigned)(ce - ca), &bars[st], pol);
            } else {
                mbar_expect_tx(&bars[st], 0);  // completes the phase with no transfer
            }
            leads[wib][st][0] = lv;
            leads[wib][st][1] = lc;
        }
    };

    ChunkCursor ci{(int64_t)blockIdx.x * C::WARPS + wib, 0, 0, 0};
    ci.load(rowptr, nbrows);
    ChunkCursor cc = ci;
#pragma unroll
    for (int k = 0; k < C::NST - 1; ++k) {
        issue(ci, k);
        if (ci.r < nbrows) ci.advance(rowptr, nbrows, stride, C::CH);
    }
    double dot = 0, yy = 0;
    double acc[B], acc2[B];
#pragma unroll
    for (int i = 0; i < B; ++i) acc[i] = acc2[i] = 0;
    double cv = 0, xo = 0;  // with corr: lane l < B*B holds corr_r[l], lane l < B holds x_r[l]
    constexpr int GL = B == 2 ? 16 : 8;  // lanes per reduced component
    const int comp = lane / GL;
    const bool writer = (lane % GL) == 0 && comp < B;
    int st = 0;
    unsigned phase = 0;  // bit k: parity of stage k's next completion
    bool timed_out = false;
    while (cc.r < nbrows) {
        issue(ci, (st + C::NST - 1) % C::NST);
        if (ci.r < nbrows) ci.advance(rowptr, nbrows, stride, C::CH);
        // bounded wait for stage st: lane 0 polls, the verdict is broadcast so the
        // warp leaves together; the other lanes then observe the completed phase
        // themselves (acquire) before reading the stage
        int ok = 1;
        if (lane == 0) {
            long long spins = 0;
            while (!mbar_try_wait(&bars[st], (phase >> st) & 1u))
                if (++spins > kSpinLimit) { ok = 0; break; }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) { timed_out = true; break; }
        if (lane != 0) mbar_try_wait(&bars[st], (phase >> st) & 1u);
        phase ^= (1u << st);
        __syncwarp();
        const int nb = max(0, min(C::CH, cc.re - cc.rs - cc.b0));
        if (corr && cc.b0 == 0) {  // first chunk of the row: its correction, used when the row completes
            if (lane < B2) cv = corr[cc.r * B2 + lane];
            if (lane < B) xo = x[B * cc.r + lane];
        }
        const unsigned char *stg = ring + st * C::STAGE;
        const VT *blk = reinterpret_cast<const VT *>(stg + leads[wib][st][0]);
        const int32_t *cix = reinterpret_cast<const int32_t *>(stg + C::VBYTES + leads[wib][st][1]);
        int j = lane;
        for (; j + 32 < nb; j += 64) {
            const int c0 = cix[j], c1 = cix[j + 32];
            double x0[B], x1[B];
            gather_x<B, XF>(x, x32, c0, x0);
            gather_x<B, XF>(x, x32, c1, x1);
#pragma unroll
            for (int i = 0; i < B; ++i)
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    acc[i] = fma((double)blk[j * B2 + i * B + k], x0[k], acc[i]);
                    acc2[i] = fma((double)blk[(j + 32) * B2 + i * B + k], x1[k], acc2[i]);
                }
        }
        if (j < nb) {
            const int c0 = cix[j];
            double x0[B];
            gather_x<B, XF>(x, x32, c0, x0);
#pragma unroll
            for (int i = 0; i < B; ++i)
#pragma unroll
                for (int k = 0; k < B; ++k) acc[i] = fma((double)blk[j * B2 + i * B + k], x0[k], acc[i]);
        }
        __syncwarp();
        if (cc.b0 + C::CH >= cc.re - cc.rs) {  // row complete
#pragma unroll
            for (int i = 0; i < B; ++i) acc[i] += acc2[i];
            // transposed butterfly: lane l ends with the row's sum l / GL, and the
            // first lane of each of the B groups writes that component
            double sr = reduce_rows_t<B>(acc, lane);
            if (corr) {
                // lane B*i+k holds corr_r[i][k]; row i's term sums lanes B*i .. B*i+B-1 in order
                const double pr = cv * __shfl_sync(0xffffffffu, xo, lane % B);
                double t = pr;
#pragma unroll
                for (int k = 1; k < B; ++k) t += __shfl_down_sync(0xffffffffu, pr, k);
                sr += __shfl_sync(0xffffffffu, t, B * (comp < B ? comp : 0));
            }
            if (writer) {
                const int64_t yi = B * cc.r + comp;
                y[yi] = sr;
                if (DOT >= 1) dot = fma(sr, w[yi], dot);
                if (DOT == 2) yy = fma(sr, sr, yy);
            }
#pragma unroll
            for (int i = 0; i < B; ++i) acc[i] = acc2[i] = 0;
        }
        cc.advance(rowptr, nbrows, stride, C::CH);
        st = (st + 1) % C::NST;
    }
    if (timed_out && lane == 0 && err) atomicExch(err, (int32_t)YG_TIMEOUT);
    // drain the copies still in flight into this warp's stages before the CTA
    // exits (also after a timeout, again with a bound)
    if (lane == 0) {
        for (int k = 0; k < C::NST - 1; ++k) {
            const int s2 = (st + k) % C::NST;
            long long spins = 0;
            while (!mbar_try_wait(&bars[s2], (phase >> s2) & 1u) && ++spins <= kSpinLimit) {
            }
            phase ^= (1u << s2);
        }
    }
    __syncwarp();
    if (DOT) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dot += __shfl_xor_sync(0xffffffffu, dot, o);
            if (DOT == 2) yy += __shfl_xor_sync(0xffffffffu, yy, o);
        }
        if (lane == 0) red[wib] = dot;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0;
            for (int i = 0; i < C::WARPS; ++i) sum += red[i];
            if (DOT == 1) partials[blockIdx.x] = sum;
            else partials[2 * blockIdx.x] = sum;
        }
        if (DOT == 2) {
            __syncthreads();
            if (lane == 0) red[wib] = yy;
            __syncthreads();
            if (threadIdx.x == 0) {
                double sum = 0;
                for (int i = 0; i < C::WARPS; ++i) sum += red[i];
                partials[2 * blockIdx.x + 1] = sum;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Row-tile variant for CSR (block size 1, variant 3).  Long scalar rows (3D
// order-2 elements: 27-125 entries) leave the flat kernel latency bound: each
// warp's row costs a row-pointer load, then the value and column loads, then
// the gathers of x, one after the other.  Here the rows are cut once into
// tiles of whole consecutive rows holding at most CAP entries (a table of tile
// starts, built on the device from the row pointers).  Each warp streams its
// tiles (grid stride) through a ring of NST shared-memory stages: one lane
// fetches a tile's values, columns and row pointers with three bulk
// asynchronous copies completing on the stage's mbarrier, running NST-1 tiles
// ahead, with the tile bounds of the next 32 tiles prefetched by the whole
// warp.  Consuming a tile, the lanes first form all its products v_k x[c_k]
// (up to U independent gathers per lane in flight) into a per-warp buffer,
// then lane r sums row r's products in entry order.  So each row is summed
// left to right, the order of the reference's csr_spmv loop, and the result
// does not depend on the launch shape.  Waits are bounded as in the TMA
// variant above.
template <typename VT, int CAP_, int NST_, int WARPS_>
struct CsrCfg {
    static constexpr int CAP = CAP_, NST = NST_, WARPS = WARPS_;
    static constexpr int U = CAP / 32 < 16 ? CAP / 32 : 16;  // products per lane per round
    static constexpr int VB = (CAP * (int)sizeof(VT) + 32 + 15) & ~15;
    static constexpr int CB = (CAP * 4 + 32 + 15) & ~15;
    static constexpr int RB = ((CAP + 1) * 4 + 32 + 15) & ~15;
    static constexpr int STAGE = VB + CB + RB;
    static constexpr int PB = CAP * 8;
    static constexpr int WARP_BYTES = NST * STAGE + PB;
    static constexpr int SMEM = WARPS * WARP_BYTES + WARPS * NST * 8;
};

template <typename VT, int DOT, typename C>
__global__ void __launch_bounds__(C::WARPS * 32)
k_csr_spmv_tiles(int64_t ntiles, const int32_t *__restrict__ tiles, const int32_t *__restrict__ rowptr,
                 const int32_t *__restrict__ col, const VT *__restrict__ val, const double *__restrict__ x,
                 double *__restrict__ y, const double *__restrict__ w, double *__restrict__ partials,
                 const int32_t *__restrict__ flag, const double *__restrict__ corr, int32_t *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[C::WARPS + 1];
    __shared__ int hdr[C::WARPS][C::NST][4];  // r0, r1, e0, e1 of the tile in each stage
    if (flag && read_flag(flag)) return;
    constexpr int VS = (int)sizeof(VT);
    const uint64_t pol = evict_first_policy();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *ring = smem_raw + (size_t)wib * C::WARP_BYTES;
    double *prod = reinterpret_cast<double *>(ring + (size_t)C::NST * C::STAGE);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)C::WARPS * C::WARP_BYTES) + wib * C::NST;
    if (lane == 0)
        for (int k = 0; k < C::NST; ++k) mbar_init(&bars[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();
    const int64_t stride = (int64_t)gridDim.x * C::WARPS;
    const char *vbytes = reinterpret_cast<const char *>(val);
    const char *cbytes = reinterpret_cast<const char *>(col);
    const char *rbytes = reinterpret_cast<const char *>(rowptr);

    // tile bounds of the next 32 tiles of this warp, lane k holding tile tb + k*stride
    int64_t t_issue = (int64_t)blockIdx.x * C::WARPS + wib;
    int64_t tb = t_issue;
    int nb_used = 32;
    int d_r0 = 0, d_r1 = 0, d_e0 = 0, d_e1 = 0;
    auto issue = [&](int st) {
        if (nb_used == 32) {
            tb = t_issue;
            const int64_t t = tb + (int64_t)lane * stride;
            d_r0 = d_r1 = d_e0 = d_e1 = 0;
            if (t < ntiles) {
                d_r0 = __ldg(tiles + t);
                d_r1 = __ldg(tiles + t + 1);
                d_e0 = __ldg(rowptr + d_r0);
                d_e1 = __ldg(rowptr + d_r1);
            }
            nb_used = 0;
        }
        const int r0 = __shfl_sync(0xffffffffu, d_r0, nb_used), r1 = __shfl_sync(0xffffffffu, d_r1, nb_used);
        const int e0 = __shfl_sync(0xffffffffu, d_e0, nb_used), e1 = __shfl_sync(0xffffffffu, d_e1, nb_used);
        ++nb_used;
        t_issue += stride;
        if (lane == 0) {
            hdr[wib][st][0] = r0;
            hdr[wib][st][1] = r1;
            hdr[wib][st][2] = e0;
            hdr[wib][st][3] = e1;
            if (r1 > r0) {
                const int64_t vs = (int64_t)e0 * VS, va = vs & ~(int64_t)15, ve = ((int64_t)e1 * VS + 15) & ~(int64_t)15;
                const int64_t cs = (int64_t)e0 * 4, ca = cs & ~(int64_t)15, ce = ((int64_t)e1 * 4 + 15) & ~(int64_t)15;
                const int64_t rs = (int64_t)r0 * 4, ra = rs & ~(int64_t)15, re = ((int64_t)(r1 + 1) * 4 + 15) & ~(int64_t)15;
                unsigned char *dst = ring + (size_t)st * C::STAGE;
                mbar_expect_tx(&bars[st], (unsigned)((ve - va) + (ce - ca) + (re - ra)));
                bulk_g2s(dst, vbytes + va, (unsigned)(ve - va), &bars[st], pol);
                bulk_g2s(dst + C::VB, cbytes + ca, (unsigned)(ce - ca), &bars[st], pol);
                bulk_g2s(dst + C::VB + C::CB, rbytes + ra, (unsigned)(re - ra), &bars[st], pol);
            } else {
                mbar_expect_tx(&bars[st], 0);  // completes the phase with no transfer
            }
        }
    };

#pragma unroll
    for (int k = 0; k < C::NST - 1; ++k) issue(k);
    double dot = 0, yy = 0;
    int st = 0;
    unsigned phase = 0;  // bit k: parity of stage k's next completion
    bool timed_out = false;
    for (int64_t t = (int64_t)blockIdx.x * C::WARPS + wib; t < ntiles; t += stride) {
        issue((st + C::NST - 1) % C::NST);
        int ok = 1;
        if (lane == 0) {
            long long spins = 0;
            while (!mbar_try_wait(&bars[st], (phase >> st) & 1u))
                if (++spins > kSpinLimit) { ok = 0; break; }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) { timed_out = true; break; }
        if (lane != 0) mbar_try_wait(&bars[st], (phase >> st) & 1u);
        phase ^= (1u << st);
        __syncwarp();
        const int r0 = hdr[wib][st][0], r1 = hdr[wib][st][1], e0 = hdr[wib][st][2], e1 = hdr[wib][st][3];
        const int E = e1 - e0, R = r1 - r0;
        const unsigned char *stg = ring + (size_t)st * C::STAGE;
        const VT *v = reinterpret_cast<const VT *>(stg + (((int64_t)e0 * VS) & 15));
        const int32_t *c = reinterpret_cast<const int32_t *>(stg + C::VB + (((int64_t)e0 * 4) & 15));
        const int32_t *rp = reinterpret_cast<const int32_t *>(stg + C::VB + C::CB + (((int64_t)r0 * 4) & 15));
        for (int k0 = 0; k0 < E; k0 += 32 * C::U) {
            double pv[C::U];
#pragma unroll
            for (int u = 0; u < C::U; ++u) {
                const int k = k0 + u * 32 + lane;
                pv[u] = 0;
                if (k < E) pv[u] = (double)v[k] * __ldg(x + c[k]);
            }
#pragma unroll
            for (int u = 0; u < C::U; ++u) {
                const int k = k0 + u * 32 + lane;
                if (k < E) prod[k] = pv[u];
            }
        }
        __syncwarp();
        for (int r = lane; r < R; r += 32) {
            const int a = rp[r] - e0, b = rp[r + 1] - e0;
            double sum = 0;
            for (int k = a; k < b; ++k) sum += prod[k];
            if (corr) sum = fma(corr[r0 + r], x[r0 + r], sum);
            y[r0 + r] = sum;
            if (DOT >= 1) dot = fma(sum, w[r0 + r], dot);
            if (DOT == 2) yy = fma(sum, sum, yy);
        }
        __syncwarp();  // the stage and the product buffer are free again
        st = (st + 1) % C::NST;
    }
    if (timed_out && lane == 0 && err) atomicExch(err, (int32_t)YG_TIMEOUT);
    // drain the copies still in flight into this warp's stages (bounded): NST-1
    // after the loop, all NST after a timeout (the failed stage included)
    if (lane == 0) {
        const int outstanding = timed_out ? C::NST : C::NST - 1;
        for (int k = 0; k < outstanding; ++k) {
            const int s2 = (st + k) % C::NST;
            long long spins = 0;
            while (!mbar_try_wait(&bars[s2], (phase >> s2) & 1u) && ++spins <= kSpinLimit) {
            }
            phase ^= (1u << s2);
        }
    }
    __syncwarp();
    if (DOT) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dot += __shfl_xor_sync(0xffffffffu, dot, o);
            if (DOT == 2) yy += __shfl_xor_sync(0xffffffffu, yy, o);
        }
        if (lane == 0) red[wib] = dot;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0;
            for (int i = 0; i < C::WARPS; ++i) sum += red[i];
            if (DOT == 1) partials[blockIdx.x] = sum;
            else partials[2 * blockIdx.x] = sum;
        }
        if (DOT == 2) {
            __syncthreads();
            if (lane == 0) red[wib] = yy;
            __syncthreads();
            if (threadIdx.x == 0) {
                double sum = 0;
                for (int i = 0; i < C::WARPS; ++i) sum += red[i];
                partials[2 * blockIdx.x + 1] = sum;
            }
        }
    }
}

// Row-tile configurations (tile entries, ring depth, warps per CTA), selected by
// the `lanes` field of a variant-3 matrix; each fills one SM's shared memory.
template <typename VT> using CsrL1 = CsrCfg<VT, 512, 3, 6>;
template <typename VT> using CsrL2 = CsrCfg<VT, 512, 2, 8>;
template <typename VT> using CsrL4 = CsrCfg<VT, 256, 3, 12>;
template <typename VT> using CsrL8 = CsrCfg<VT, 1024, 2, 4>;

// tile-table index of a configuration: capacity 256 << k entries
static int csr_table(int lanes) { return lanes == 4 ? 0 : lanes == 8 ? 2 : 1; }
static bool csr_lanes_ok(int lanes) { return lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8; }

__global__ void k_row_extent(int64_t n, const int32_t *__restrict__ rowptr, int32_t *__restrict__ out) {
    int lo = INT32_MAX, hi = 0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int len = rowptr[r + 1] - rowptr[r];
        lo = min(lo, len);
        hi = max(hi, len);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(out, lo);
        atomicMax(out + 1, hi);
    }
}

// tiles[t] = first row whose first entry is at or after t*per (t = 0..nt; the
// last is n): the rows starting in [t*per, (t+1)*per) form tile t, whose entries
// then span at most per - 1 + (longest row) positions.
__global__ void k_row_tiles(int64_t n, int64_t nt, int64_t per, const int32_t *__restrict__ rowptr,
                            int32_t *__restrict__ tiles) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t <= nt; t += (int64_t)gridDim.x * blockDim.x) {
        if (t == nt) { tiles[t] = (int32_t)n; continue; }
        const int64_t target = t * per;
        int64_t lo = 0, hi = n;  // first r in [0, n] with rowptr[r] >= target
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (rowptr[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        tiles[t] = (int32_t)lo;
    }
}

// Smallest and largest number of entries (blocks) per row of A, measured once.
static yg_status row_extent(yg_matrix A) {
    if (A->row_min >= 0) return YG_OK;
    yg_context ctx = A->ctx;
    cudaStreamCaptureStatus cs;
    YG_CUDA(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return fail(YG_BAD_ARG, "row extents cannot be measured during stream capture");
    int32_t *d = nullptr;
    YG_TRY(dev_alloc_t(ctx, &d, 2));
    const int32_t init[2] = {INT32_MAX, 0};
    int32_t h[2];
    cudaMemcpyAsync(d, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream);
    int blocks = (int)std::min<int64_t>((A->nbrows + kThreads - 1) / kThreads, (int64_t)ctx->num_sms * 4);
    if (blocks < 1) blocks = 1;
    k_row_extent<<<blocks, kThreads, 0, ctx->stream>>>(A->nbrows, A->d_rowptr, d);
    YG_LAUNCHED(ctx);
    cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, d);
    if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "row extent: %s", cudaGetErrorString(e));
    A->row_min = h[0];
    A->row_max = h[1];
    return YG_OK;
}

// Row tiles of capacity 256 << k for A (block size 1).  Needs every row to hold
// at least one and at most `cap` entries.
static yg_status csr_tiles_build(yg_matrix A, int k) {
    if (A->block != 1 || A->nbrows < 1) return fail(YG_UNSUPPORTED, "row-tile SpMV needs a non-empty CSR matrix");
    if (A->d_ctiles[k]) return YG_OK;
    yg_context ctx = A->ctx;
    cudaStreamCaptureStatus cs;
    YG_CUDA(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return fail(YG_BAD_ARG, "row tiles cannot be built during stream capture");
    YG_TRY(row_extent(A));
    const int cap = 256 << k;
    if (A->row_min < 1 || A->row_max > cap)
        return fail(YG_UNSUPPORTED, "row-tile SpMV needs 1..%d entries per row (rows hold %d..%d)", cap, A->row_min,
                    A->row_max);
    const int64_t per = cap - A->row_max + 1;
    const int64_t nt = (A->nnzb + per - 1) / per;
    YG_TRY(dev_alloc_t(ctx, &A->d_ctiles[k], nt + 1));
    int blocks = (int)std::min<int64_t>((nt + kThreads) / kThreads, (int64_t)ctx->num_sms * 4);
    k_row_tiles<<<blocks, kThreads, 0, ctx->stream>>>(A->nbrows, nt, per, A->d_rowptr, A->d_ctiles[k]);
    YG_LAUNCHED(ctx);
    YG_CUDA(cudaGetLastError());
    A->nctiles[k] = nt;
    return YG_OK;
}

static int rows_capacity_of(int lanes) { return lanes <= 2 ? 128 : 64; }

yg_status spmv_prepare(yg_matrix A, int variant, int lanes) {
    if (variant == 4) {  // whole rows: every block row must fit one stage
        if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8)
            return fail(YG_BAD_ARG, "whole-row SpMV configurations are lanes 1, 2, 4, 8");
        if (A->block != 2 && A->block != 3) return fail(YG_UNSUPPORTED, "whole-row SpMV needs 2x2 or 3x3 blocks");
        if (A->nbrows >= INT32_MAX) return fail(YG_UNSUPPORTED, "whole-row SpMV needs fewer than 2^31 block rows");
        YG_TRY(row_extent(A));
        if (A->row_max > rows_capacity_of(lanes))
            return fail(YG_UNSUPPORTED, "whole-row SpMV (lanes %d) holds rows of up to %d blocks; the longest has %d",
                        lanes, rows_capacity_of(lanes), A->row_max);
        return YG_OK;
    }
    if (variant != 3) return YG_OK;
    if (!csr_lanes_ok(lanes)) return fail(YG_BAD_ARG, "row-tile SpMV configurations are lanes 1, 2, 4, 8");
    return csr_tiles_build(A, csr_table(lanes));
}

template <typename VT, int DOT, typename C>
static yg_status launch_csr_cfg(yg_matrix A, int k, const VT *val, const double *x, double *y, const double *w,
                                double *partials, const int32_t *flag, const double *corr, int grid, cudaStream_t st) {
    static std::atomic<uint64_t> attr{0};
    if (smem_attr_due(attr, A->ctx->device)) {
        cudaFuncSetAttribute(k_csr_spmv_tiles<VT, DOT, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
        smem_attr_done(attr, A->ctx->device);
    }
    k_csr_spmv_tiles<VT, DOT, C><<<grid, C::WARPS * 32, C::SMEM, st>>>(A->nctiles[k], A->d_ctiles[k], A->d_rowptr,
                                                                       A->d_col, val, x, y, w, partials, flag, corr,
                                                                       A->ctx->d_err);
    YG_LAUNCHED(A->ctx);
    return YG_OK;
}

template <typename VT, int DOT>
static yg_status launch_csr(yg_matrix A, int lanes, const VT *val, const double *x, double *y, const double *w,
                            double *partials, const int32_t *flag, const double *corr, int grid, cudaStream_t st) {
    const int k = csr_table(lanes);
    if (A->block != 1 || !csr_lanes_ok(lanes) || !A->d_ctiles[k])
        return fail(YG_BAD_ARG, "row-tile SpMV launched without its row tiles (block %d, lanes %d)", A->block, lanes);
    switch (lanes) {
    case 1: return launch_csr_cfg<VT, DOT, CsrL1<VT>>(A, k, val, x, y, w, partials, flag, corr, grid, st);
    case 2: return launch_csr_cfg<VT, DOT, CsrL2<VT>>(A, k, val, x, y, w, partials, flag, corr, grid, st);
    case 4: return launch_csr_cfg<VT, DOT, CsrL4<VT>>(A, k, val, x, y, w, partials, flag, corr, grid, st);
    default: return launch_csr_cfg<VT, DOT, CsrL8<VT>>(A, k, val, x, y, w, partials, flag, corr, grid, st);
    }
}

template <typename VT>
static void csr_shape_v(int lanes, int *smem, int *wp) {
    switch (lanes) {
    case 1: *smem = CsrL1<VT>::SMEM; *wp = CsrL1<VT>::WARPS; break;
    case 2: *smem = CsrL2<VT>::SMEM; *wp = CsrL2<VT>::WARPS; break;
    case 4: *smem = CsrL4<VT>::SMEM; *wp = CsrL4<VT>::WARPS; break;
    default: *smem = CsrL8<VT>::SMEM; *wp = CsrL8<VT>::WARPS; break;
    }
}

template <int B, typename VT, int DOT, typename C, bool XF>
static yg_status launch_tma_xf(yg_matrix A, const VT *val, const double *x, const float *x32, double *y,
                               const double *w, double *partials, const int32_t *flag, const double *corr, int grid, cudaStream_t st) {
    static std::atomic<uint64_t> attr{0};
    if (smem_attr_due(attr, A->ctx->device)) {
        cudaFuncSetAttribute(k_bcsr_spmv_tma<B, VT, DOT, C, XF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             C::SMEM);
        smem_attr_done(attr, A->ctx->device);
    }
    k_bcsr_spmv_tma<B, VT, DOT, C, XF><<<grid, C::WARPS * 32, C::SMEM, st>>>(
        A->nbrows, A->d_rowptr, A->d_col, val, x, x32, y, w, partials, flag, corr, A->ctx->d_err);
    YG_LAUNCHED(A->ctx);
    return YG_OK;
}

// FP32 gathers only with FP32 values (the mixed-precision iteration SpMV).
template <int B, typename VT, int DOT, typename C>
static yg_status launch_tma_cfg(yg_matrix A, const VT *val, const double *x, const float *x32, double *y,
                                const double *w, double *partials, const int32_t *flag, const double *corr, int grid, cudaStream_t st) {
    if constexpr (std::is_same<VT, float>::value) {
        if (x32) return launch_tma_xf<B, VT, DOT, C, true>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    }
    return launch_tma_xf<B, VT, DOT, C, false>(A, val, x, nullptr, y, w, partials, flag, corr, grid, st);
}

// TMA configurations (chunk blocks, ring depth, warps per CTA) the autotuner
// tries, selected by the `lanes` field of a variant-2 matrix.
template <int B, typename VT> using TmaL32 = TmaCfg<B, VT, 64, 3, 4>;
template <int B, typename VT> using TmaL1 = TmaCfg<B, VT, 32, 4, 8>;
template <int B, typename VT> using TmaL2 = TmaCfg<B, VT, 32, 3, 8>;
template <int B, typename VT> using TmaL4 = TmaCfg<B, VT, 32, 2, 8>;
template <int B, typename VT> using TmaL8 = TmaCfg<B, VT, 32, 3, 12>;
template <int B, typename VT> using TmaL16 = TmaCfg<B, VT, 48, 3, 8>;

template <int B, typename VT, int DOT>
static yg_status launch_tma(yg_matrix A, int lanes, const VT *val, const double *x, const float *x32, double *y,
                            const double *w, double *partials, const int32_t *flag, const double *corr, int grid, cudaStream_t st) {
    switch (lanes) {
    case 1: return launch_tma_cfg<B, VT, DOT, TmaL1<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    case 2: return launch_tma_cfg<B, VT, DOT, TmaL2<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    case 4: return launch_tma_cfg<B, VT, DOT, TmaL4<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    case 8: return launch_tma_cfg<B, VT, DOT, TmaL8<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    case 16: return launch_tma_cfg<B, VT, DOT, TmaL16<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    default: return launch_tma_cfg<B, VT, DOT, TmaL32<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    }
}

template <typename C>
static void shape_of(int *smem, int *warps) {
    *smem = C::SMEM;
    *warps = C::WARPS;
}
template <int B, typename VT>
static void tma_shape_bv(int lanes, int *smem, int *wp) {
    switch (lanes) {
    case 1: shape_of<TmaL1<B, VT>>(smem, wp); break;
    case 2: shape_of<TmaL2<B, VT>>(smem, wp); break;
    case 4: shape_of<TmaL4<B, VT>>(smem, wp); break;
    case 8: shape_of<TmaL8<B, VT>>(smem, wp); break;
    case 16: shape_of<TmaL16<B, VT>>(smem, wp); break;
    default: shape_of<TmaL32<B, VT>>(smem, wp); break;
    }
}

// ---------------------------------------------------------------------------
// Whole-row variant for B = 2, 3 (variant 4).  The chunked TMA variant above
// spends most of its instructions outside the block products: per chunk the
// copy issue, a cursor with two row-pointer loads, the stage offsets through
// shared memory, a lane-divergent tail, and per row a 5-step butterfly of B
// sums.  With FP32 values that bookkeeping, not HBM, sets its speed.  Here
// every block row fits one stage (the matrix's longest row is at most CH
// blocks), so a row costs one copy pair, one bounded wait and one reduction:
// * the warp's next 32 rows' bounds are loaded at once, lane k holding row
//   r + k*stride, and handed out by shuffles;
// * stage offsets are recomputed from the row's first block, not stored;
// * each lane issues the x gathers of all its blocks (lane + 32u) before its
//   products, accumulating even and odd u in separate sums;
// * the B row sums are reduced by a transposed butterfly (the halves of the
//   warp first exchange different sums, then one sum per lane is reduced), so
//   sum i ends in lanes 32i/Bp .. (the lane groups of the padded B), whose
//   first lane writes y[B r + i] (and its dot terms).
// The summation order is fixed (lane order, then the butterfly), so results are
// reproducible.  Waits are bounded as in the variants above.
template <int B, typename VT, int CH_, int NST_, int WARPS_>
struct RowCfg {
    static constexpr int CH = CH_, NST = NST_, WARPS = WARPS_, U = CH / 32;
    static constexpr int VBYTES = (CH * B * B * (int)sizeof(VT) + 32 + 15) & ~15;
    static constexpr int CBYTES = (CH * 4 + 32 + 15) & ~15;
    static constexpr int STAGE = VBYTES + CBYTES;
    static constexpr int SMEM = WARPS * NST * STAGE + WARPS * NST * 8;  // stages + mbarriers
    static_assert(CH % 32 == 0, "whole 32-block groups per stage");
};

template <int B, typename VT, int DOT, typename C, bool XF>
__global__ void __launch_bounds__(C::WARPS * 32)
k_bcsr_spmv_rows(int32_t nbrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                 const VT *__restrict__ val, const double *__restrict__ x, const float *__restrict__ x32,
                 double *__restrict__ y, const double *__restrict__ w, double *__restrict__ partials,
                 const int32_t *__restrict__ flag, const double *__restrict__ corr, int32_t *__restrict__ err) {
    constexpr int B2 = B * B;
    constexpr int BB = B2 * (int)sizeof(VT);
    constexpr int GL = B == 2 ? 16 : 8;  // lanes per reduced component
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[C::WARPS + 1];
    __shared__ int hdr[C::WARPS][C::NST][2];  // first block and block count of the row in each stage
    if (flag && read_flag(flag)) return;
    const uint64_t pol = evict_first_policy();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *ring = smem_raw + (size_t)wib * C::NST * C::STAGE;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)C::WARPS * C::NST * C::STAGE) + wib * C::NST;
    if (lane == 0)
        for (int k = 0; k < C::NST; ++k) mbar_init(&bars[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();
    const int stride = gridDim.x * C::WARPS;
    const char *vbytes = reinterpret_cast<const char *>(val);
    const char *cbytes = reinterpret_cast<const char *>(col);

    // bounds of the warp's next 32 rows to issue: lane k holds row pf_base + k*stride
    int64_t pf_base = (int64_t)blockIdx.x * C::WARPS + wib;
    int pf_used = 32, pf_rs = 0, pf_re = 0;
    // lane 0 issues the copies of the next row into stage st (an empty copy past the end)
    auto issue = [&](int st) {
        if (pf_used == 32) {
            const int64_t r = pf_base + (int64_t)lane * stride;
            pf_rs = pf_re = 0;
            if (r < nbrows) {
                pf_rs = __ldg(rowptr + r);
                pf_re = __ldg(rowptr + r + 1);
            }
            pf_used = 0;
        }
        const int rs = __shfl_sync(0xffffffffu, pf_rs, pf_used), re = __shfl_sync(0xffffffffu, pf_re, pf_used);
        if (++pf_used == 32) pf_base += 32 * (int64_t)stride;
        if (lane == 0) {
            hdr[wib][st][0] = rs;
            hdr[wib][st][1] = re - rs;
            if (re > rs) {
                const int64_t vs = (int64_t)rs * BB, va = vs & ~(int64_t)15, ve = ((int64_t)re * BB + 15) & ~(int64_t)15;
                const int64_t cs = (int64_t)rs * 4, ca = cs & ~(int64_t)15, ce = ((int64_t)re * 4 + 15) & ~(int64_t)15;
                unsigned char *dst = ring + st * C::STAGE;
                mbar_expect_tx(&bars[st], (unsigned)((ve - va) + (ce - ca)));
                bulk_g2s(dst, vbytes + va, (unsigned)(ve - va), &bars[st], pol);
                bulk_g2s(dst + C::VBYTES, cbytes + ca, (unsigned)(ce - ca), &bars[st], pol);
            } else {
                mbar_expect_tx(&bars[st], 0);  // completes the phase with no transfer
            }
        }
    };

#pragma unroll
    for (int k = 0; k < C::NST - 1; ++k) issue(k);
    double dot = 0, yy = 0;
    int st = 0;
    unsigned phase = 0;  // bit k: parity of stage k's next completion
    bool timed_out = false;
    const int comp = lane / GL;               // the sum this lane holds after the reduction
    const bool writer = (lane % GL) == 0 && comp < B;
    for (int64_t r = (int64_t)blockIdx.x * C::WARPS + wib; r < nbrows; r += stride) {
        issue((st + C::NST - 1) % C::NST);
        // the writer lanes fetch the row's correction and own x early (used at the end)
        double cr[B], xr[B];
        if (corr && writer) {
#pragma unroll
            for (int k = 0; k < B; ++k) {
                cr[k] = corr[(r * B + comp) * B + k];
                xr[k] = x[r * B + k];
            }
        }
        int ok = 1;
        if (lane == 0) {
            long long spins = 0;
            while (!mbar_try_wait(&bars[st], (phase >> st) & 1u))
                if (++spins > kSpinLimit) { ok = 0; break; }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) { timed_out = true; break; }
        if (lane != 0) mbar_try_wait(&bars[st], (phase >> st) & 1u);
        phase ^= (1u << st);
        __syncwarp();
        const int rs = hdr[wib][st][0], nb = hdr[wib][st][1];
        const unsigned char *stg = ring + st * C::STAGE;
        const VT *blk = reinterpret_cast<const VT *>(stg + (((unsigned)rs * (unsigned)BB) & 15u));
        const int32_t *cix = reinterpret_cast<const int32_t *>(stg + C::VBYTES + (((unsigned)rs * 4u) & 15u));
        double xv[C::U][B];
#pragma unroll
        for (int u = 0; u < C::U; ++u) {
            if (32 * u < nb) {  // warp-uniform
                const int j = lane + 32 * u;
                if (j < nb) {
                    gather_x<B, XF>(x, x32, cix[j], xv[u]);
                } else {
#pragma unroll
                    for (int k = 0; k < B; ++k) xv[u][k] = 0;
                }
            }
        }
        double acc[B], acc2[B];
#pragma unroll
        for (int i = 0; i < B; ++i) acc[i] = acc2[i] = 0;
#pragma unroll
        for (int u = 0; u < C::U; ++u) {
            if (32 * u < nb) {
                const int j = lane + 32 * u;
                if (j < nb) {
#pragma unroll
                    for (int i = 0; i < B; ++i)
#pragma unroll
                        for (int k = 0; k < B; ++k) {
                            if (u & 1) acc2[i] = fma((double)blk[j * B2 + i * B + k], xv[u][k], acc2[i]);
                            else acc[i] = fma((double)blk[j * B2 + i * B + k], xv[u][k], acc[i]);
                        }
                }
            }
        }
        __syncwarp();  // the stage is free again
#pragma unroll
        for (int i = 0; i < B; ++i) acc[i] += acc2[i];
        double s = reduce_rows_t<B>(acc, lane);
        if (writer) {
            if (corr) {
                double t = cr[0] * xr[0];
#pragma unroll
                for (int k = 1; k < B; ++k) t = fma(cr[k], xr[k], t);
                s += t;
            }
            const int64_t yi = r * B + comp;
            y[yi] = s;
            if (DOT >= 1) dot = fma(s, w[yi], dot);
            if (DOT == 2) yy = fma(s, s, yy);
        }
        st = (st + 1) % C::NST;
    }
    if (timed_out && lane == 0 && err) atomicExch(err, (int32_t)YG_TIMEOUT);
    // drain the copies still in flight into this warp's stages (bounded): NST-1
    // after the loop, all NST after a timeout (the failed stage included)
    if (lane == 0) {
        const int outstanding = timed_out ? C::NST : C::NST - 1;
        for (int k = 0; k < outstanding; ++k) {
            const int s2 = (st + k) % C::NST;
            long long spins = 0;
            while (!mbar_try_wait(&bars[s2], (phase >> s2) & 1u) && ++spins <= kSpinLimit) {
            }
            phase ^= (1u << s2);
        }
    }
    __syncwarp();
    if (DOT) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dot += __shfl_xor_sync(0xffffffffu, dot, o);
            if (DOT == 2) yy += __shfl_xor_sync(0xffffffffu, yy, o);
        }
        if (lane == 0) red[wib] = dot;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0;
            for (int i = 0; i < C::WARPS; ++i) sum += red[i];
            if (DOT == 1) partials[blockIdx.x] = sum;
            else partials[2 * blockIdx.x] = sum;
        }
        if (DOT == 2) {
            __syncthreads();
            if (lane == 0) red[wib] = yy;
            __syncthreads();
            if (threadIdx.x == 0) {
                double sum = 0;
                for (int i = 0; i < C::WARPS; ++i) sum += red[i];
                partials[2 * blockIdx.x + 1] = sum;
            }
        }
    }
}

// Whole-row configurations (longest row in blocks, ring depth, warps per CTA),
// selected by the `lanes` field of a variant-4 matrix.
template <int B, typename VT> using RowL1 = RowCfg<B, VT, 128, 2, 4>;
template <int B, typename VT> using RowL2 = RowCfg<B, VT, 128, 3, 4>;
template <int B, typename VT> using RowL4 = RowCfg<B, VT, 64, 2, 8>;
template <int B, typename VT> using RowL8 = RowCfg<B, VT, 64, 3, 8>;
static bool rows_lanes_ok(int lanes) { return lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8; }

template <int B, typename VT, int DOT, typename C, bool XF>
static yg_status launch_rows_xf(yg_matrix A, const VT *val, const double *x, const float *x32, double *y,
                                const double *w, double *partials, const int32_t *flag, const double *corr, int grid,
                                cudaStream_t st) {
    static std::atomic<uint64_t> attr{0};
    if (smem_attr_due(attr, A->ctx->device)) {
        cudaFuncSetAttribute(k_bcsr_spmv_rows<B, VT, DOT, C, XF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             C::SMEM);
        smem_attr_done(attr, A->ctx->device);
    }
    k_bcsr_spmv_rows<B, VT, DOT, C, XF><<<grid, C::WARPS * 32, C::SMEM, st>>>(
        (int32_t)A->nbrows, A->d_rowptr, A->d_col, val, x, x32, y, w, partials, flag, corr, A->ctx->d_err);
    YG_LAUNCHED(A->ctx);
    return YG_OK;
}

template <int B, typename VT, int DOT, typename C>
static yg_status launch_rows_cfg(yg_matrix A, const VT *val, const double *x, const float *x32, double *y,
                                 const double *w, double *partials, const int32_t *flag, const double *corr, int grid,
                                 cudaStream_t st) {
    if constexpr (std::is_same<VT, float>::value) {
        if (x32) return launch_rows_xf<B, VT, DOT, C, true>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    }
    return launch_rows_xf<B, VT, DOT, C, false>(A, val, x, nullptr, y, w, partials, flag, corr, grid, st);
}

template <int B, typename VT, int DOT>
static yg_status launch_rows(yg_matrix A, int lanes, const VT *val, const double *x, const float *x32, double *y,
                             const double *w, double *partials, const int32_t *flag, const double *corr, int grid,
                             cudaStream_t st) {
    if (!rows_lanes_ok(lanes) || A->row_max < 0 || A->row_max > rows_capacity_of(lanes))
        return fail(YG_BAD_ARG, "whole-row SpMV launched on rows it does not hold (lanes %d, longest row %d)", lanes,
                    A->row_max);
    switch (lanes) {
    case 1: return launch_rows_cfg<B, VT, DOT, RowL1<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    case 2: return launch_rows_cfg<B, VT, DOT, RowL2<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    case 4: return launch_rows_cfg<B, VT, DOT, RowL4<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    default: return launch_rows_cfg<B, VT, DOT, RowL8<B, VT>>(A, val, x, x32, y, w, partials, flag, corr, grid, st);
    }
}

template <int B, typename VT>
static void rows_shape_bv(int lanes, int *smem, int *wp) {
    switch (lanes) {
    case 1: shape_of<RowL1<B, VT>>(smem, wp); break;
    case 2: shape_of<RowL2<B, VT>>(smem, wp); break;
    case 4: shape_of<RowL4<B, VT>>(smem, wp); break;
    default: shape_of<RowL8<B, VT>>(smem, wp); break;
    }
}

// CTAs per SM and warps per CTA of a TMA configuration (for the grid size): as
// many CTAs as the shared memory holds, at most 64 warps and 8 CTAs per SM (the
// Krylov kernels reserve 8 partial sums per SM for the SpMV).
static void tma_shape(yg_matrix A, int lanes, bool f32, int *ctas_per_sm, int *warps) {
    int smem = 0, wp = 1;
    if (A->block == 3) {
        if (f32) tma_shape_bv<3, float>(lanes, &smem, &wp);
        else tma_shape_bv<3, double>(lanes, &smem, &wp);
    } else {
        if (f32) tma_shape_bv<2, float>(lanes, &smem, &wp);
        else tma_shape_bv<2, double>(lanes, &smem, &wp);
    }
    int per = (220 * 1024) / (smem + 1024);
    if (per * wp > 64) per = 64 / wp;
    if (per > 8) per = 8;
    *ctas_per_sm = per < 1 ? 1 : per;
    *warps = wp;
}

template <int B, typename VT, int DOT>
static yg_status launch_staged(yg_matrix A, const VT *val, const double *x, double *y, const double *w,
                               double *partials, const int32_t *flag, const double *corr, int grid, cudaStream_t st) {
    using S = Staged<B, VT>;
    static std::atomic<uint64_t> attr{0};
    if (smem_attr_due(attr, A->ctx->device)) {
        cudaFuncSetAttribute(k_bcsr_spmv_staged<B, VT, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM);
        smem_attr_done(attr, A->ctx->device);
    }
    k_bcsr_spmv_staged<B, VT, DOT><<<grid, S::WARPS * 32, S::SMEM, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y,
                                                                        w, partials, flag, corr);
    YG_LAUNCHED(A->ctx);
    return YG_OK;
}

template <int B, typename VT, int DOT>
static yg_status launch_l(yg_matrix A, int lanes, const VT *val, const double *x, double *y, const double *w,
                          double *partials, const int32_t *flag, const double *corr, int grid, cudaStream_t st) {
    switch (lanes) {
    case 2: k_bcsr_spmv<B, 2, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag, corr); break;
    case 4: k_bcsr_spmv<B, 4, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag, corr); break;
    case 8: k_bcsr_spmv<B, 8, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag, corr); break;
    case 16: k_bcsr_spmv<B, 16, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag, corr); break;
    default: k_bcsr_spmv<B, 32, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag, corr); break;
    }
    YG_LAUNCHED(A->ctx);
    return YG_OK;
}

template <typename VT, int DOT>
static yg_status launch_b(yg_matrix A, int variant, int lanes, const VT *val, const double *x, const float *x32,
                          double *y, const double *w, double *partials, const int32_t *flag, const double *corr, int grid,
                          cudaStream_t st) {
    if (variant == 3) return launch_csr<VT, DOT>(A, lanes, val, x, y, w, partials, flag, corr, grid, st);
    if (variant == 4 && A->block == 3)
        return launch_rows<3, VT, DOT>(A, lanes, val, x, x32, y, w, partials, flag, corr, grid, st);
    if (variant == 4 && A->block == 2)
        return launch_rows<2, VT, DOT>(A, lanes, val, x, x32, y, w, partials, flag, corr, grid, st);
    if (variant == 2 && A->block == 3)
        return launch_tma<3, VT, DOT>(A, lanes, val, x, x32, y, w, partials, flag, corr, grid, st);
    if (variant == 2 && A->block == 2)
        return launch_tma<2, VT, DOT>(A, lanes, val, x, x32, y, w, partials, flag, corr, grid, st);
    if (variant == 1 && A->block == 3) return launch_staged<3, VT, DOT>(A, val, x, y, w, partials, flag, corr, grid, st);
    if (variant == 1 && A->block == 2) return launch_staged<2, VT, DOT>(A, val, x, y, w, partials, flag, corr, grid, st);
    switch (A->block) {
    case 1: return launch_l<1, VT, DOT>(A, lanes, val, x, y, w, partials, flag, corr, grid, st);
    case 2: return launch_l<2, VT, DOT>(A, lanes, val, x, y, w, partials, flag, corr, grid, st);
    case 3: return launch_l<3, VT, DOT>(A, lanes, val, x, y, w, partials, flag, corr, grid, st);
    default: return fail(YG_UNSUPPORTED, "SpMV block size %d not supported (1, 2, 3)", A->block);
    }
}

template <typename VT>
static yg_status launch_v(yg_matrix A, int variant, int lanes, const VT *val, const double *x, const float *x32,
                          double *y, const double *w, double *partials, int dot_mode, const int32_t *flag, const double *corr, int grid,
                          cudaStream_t st) {
    if (dot_mode == 0) return launch_b<VT, 0>(A, variant, lanes, val, x, x32, y, w, partials, flag, corr, grid, st);
    if (dot_mode == 1) return launch_b<VT, 1>(A, variant, lanes, val, x, x32, y, w, partials, flag, corr, grid, st);
    return launch_b<VT, 2>(A, variant, lanes, val, x, x32, y, w, partials, flag, corr, grid, st);
}

// The kernel choice for a precision: FP32-value SpMVs have their own tuning.
static void choice(yg_matrix A, int precision, int *variant, int *lanes) {
    const bool f32 = precision == YG_PREC_MIXED || precision == YG_PREC_MIXED_IR;
    if (f32 && A->variant32 >= 0) {
        *variant = A->variant32;
        *lanes = A->lanes32;
    } else {
        *variant = A->variant;
        *lanes = A->lanes;
    }
}

// y = A x.  With `partials`: per-block sums of w.y (dot_mode 1; w defaults to
// x) or of w.y and y.y (dot_mode 2).  The grid is persistent: `grid` blocks
// stride over the block rows.
yg_status spmv_launch_ex(yg_matrix A, const double *x, double *y, int precision, const double *w, double *partials,
                         int dot_mode, const int32_t *flag, int grid, cudaStream_t stream, const float *x32,
                         const double *corr) {
    cudaStream_t st = stream ? stream : A->ctx->stream;
    if (grid > kMaxReduceBlocks) grid = kMaxReduceBlocks;
    if (!partials) dot_mode = 0;
    if (!w) w = x;
    yg_status s;
    int variant, lanes;
    choice(A, precision, &variant, &lanes);
    if (precision == YG_PREC_MIXED || precision == YG_PREC_MIXED_IR) {
        if (!A->d_val32) return fail(YG_BAD_ARG, "mixed-precision SpMV without FP32 values");
        s = launch_v<float>(A, variant, lanes, A->d_val32, x, x32, y, w, partials, dot_mode, flag, corr, grid, st);
    } else {
        s = launch_v<double>(A, variant, lanes, A->d_val, x, nullptr, y, w, partials, dot_mode, flag, nullptr, grid, st);
    }
    if (s != YG_OK) return s;
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

yg_status spmv_launch(yg_matrix A, const double *x, double *y, int precision, double *partials,
                      const int32_t *flag, int grid, const float *x32, const double *corr) {
    return spmv_launch_ex(A, x, y, precision, x, partials, partials ? 1 : 0, flag, grid, nullptr, x32, corr);
}

// Resident blocks per SM of the flat kernel (the heaviest, DOT = 2, form) for a
// block size, lane count and value type; at most 8.
template <int B, typename VT>
static int flat_occupancy(int lanes) {
    static int cache[6] = {0, 0, 0, 0, 0, 0};
    const int li = lanes == 2 ? 0 : lanes == 4 ? 1 : lanes == 8 ? 2 : lanes == 16 ? 3 : 4;
    if (!cache[li]) {
        int n = 0;
        cudaError_t e;
        switch (lanes) {
        case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bcsr_spmv<B, 2, VT, 2>, kThreads, 0); break;
        case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bcsr_spmv<B, 4, VT, 2>, kThreads, 0); break;
        case 8: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bcsr_spmv<B, 8, VT, 2>, kThreads, 0); break;
        case 16: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bcsr_spmv<B, 16, VT, 2>, kThreads, 0); break;
        default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bcsr_spmv<B, 32, VT, 2>, kThreads, 0); break;
        }
        if (e != cudaSuccess) cudaGetLastError();
        cache[li] = (e != cudaSuccess || n < 1) ? 1 : (n > 8 ? 8 : n);
    }
    return cache[li];
}
static int flat_blocks_per_sm(int block, int lanes, bool f32) {
    if (block == 1) return f32 ? flat_occupancy<1, float>(lanes) : flat_occupancy<1, double>(lanes);
    if (block == 2) return f32 ? flat_occupancy<2, float>(lanes) : flat_occupancy<2, double>(lanes);
    return f32 ? flat_occupancy<3, float>(lanes) : flat_occupancy<3, double>(lanes);
}

int spmv_default_grid(yg_matrix A) { return spmv_grid_for(A, YG_PREC_FP64); }

int spmv_grid_for(yg_matrix A, int precision) {
    int variant, lanes;
    choice(A, precision, &variant, &lanes);
    const bool f32 = precision == YG_PREC_MIXED || precision == YG_PREC_MIXED_IR;
    if (variant == 3) {  // row tiles: as many CTAs as the shared memory holds, a warp per tile
        int smem = 0, wp = 1;
        if (f32) csr_shape_v<float>(lanes, &smem, &wp);
        else csr_shape_v<double>(lanes, &smem, &wp);
        int per = (220 * 1024) / (smem + 1024);
        if (per * wp > 64) per = 64 / wp;
        if (per > 8) per = 8;
        if (per < 1) per = 1;
        const int64_t nt = A->nctiles[csr_table(lanes)];
        int64_t need = (nt + wp - 1) / wp;
        int64_t g = (int64_t)A->ctx->num_sms * per;
        if (need < g) g = need;
        return (int)(g < 1 ? 1 : g);
    }
    if (variant == 4) {  // whole rows: as many CTAs as the shared memory holds, a warp per row
        int smem = 0, wp = 1;
        if (A->block == 3) {
            if (f32) rows_shape_bv<3, float>(lanes, &smem, &wp);
            else rows_shape_bv<3, double>(lanes, &smem, &wp);
        } else {
            if (f32) rows_shape_bv<2, float>(lanes, &smem, &wp);
            else rows_shape_bv<2, double>(lanes, &smem, &wp);
        }
        int per = (220 * 1024) / (smem + 1024);
        if (per * wp > 64) per = 64 / wp;
        if (per > 8) per = 8;
        if (per < 1) per = 1;
        int64_t need = (A->nbrows + wp - 1) / wp;
        int64_t g = (int64_t)A->ctx->num_sms * per;
        if (need < g) g = need;
        return (int)(g < 1 ? 1 : g);
    }
    if (variant == 2) {  // TMA: as many CTAs as fit, a warp per row
        int per, wp;
        tma_shape(A, lanes, f32, &per, &wp);
        int64_t need = (A->nbrows + wp - 1) / wp;
        int64_t g = (int64_t)A->ctx->num_sms * per;
        if (need < g) g = need;
        return (int)(g < 1 ? 1 : g);
    }
    if (variant == 1) {  // staged: 3 blocks of 4 warps per SM, a warp per row
        int64_t need = (A->nbrows + 3) / 4;
        int64_t g = (int64_t)A->ctx->num_sms * 3;
        if (need < g) g = need;
        return (int)(g < 1 ? 1 : g);
    }
    // as many blocks as are resident at once (one wave: a grid-stride loop over
    // equal shares would otherwise run a second, thinner wave), at most 8 of 256
    // threads per SM, and no more row groups than rows.
    int64_t groups_per_block = kThreads / lanes;
    int64_t need = (A->nbrows + groups_per_block - 1) / groups_per_block;
    int64_t g = (int64_t)A->ctx->num_sms * flat_blocks_per_sm(A->block, lanes, f32);
    if (need < g) g = need;
    if (g < 1) g = 1;
    if (g > kMaxReduceBlocks) g = kMaxReduceBlocks;
    return (int)g;
}

// Lanes per block row from the mean number of values per row: enough lanes
// that each loads a handful of values, at most a warp.  (Static guess; the
// device autotuner below replaces it on first use.)
void spmv_autotune(yg_matrix A) {
    double per_row = A->nbrows ? (double)A->nnzb * A->block * A->block / (double)A->nbrows : 1.0;
    int L = 2;
    while (L < 32 && per_row > 4.0 * L) L *= 2;
    A->lanes = L;
    A->variant = 0;
}

// Device autotuner: time each candidate (flat with 8/16/32 lanes, staged for
// 2x2 and 3x3 blocks) on this matrix with CUDA events and keep the fastest.
// Must not run during stream capture.
// Tuning results are cached per (rows, blocks, block size): a re-assembled
// matrix of the same pattern reuses the choice without timing again.
struct TuneKey {
    int64_t nbrows, nnzb;
    int block, f32;
    bool operator==(const TuneKey &o) const {
        return nbrows == o.nbrows && nnzb == o.nnzb && block == o.block && f32 == o.f32;
    }
};
static std::vector<std::pair<TuneKey, std::pair<int, int>>> g_tune_cache;

// Time every candidate for one precision on this matrix; returns the fastest.
static yg_status tune_precision(yg_matrix A, int precision, double *x, const float *x32, double *y,
                                int *best_variant, int *best_lanes) {
    yg_context ctx = A->ctx;
    struct Cand { int variant, lanes; };
    std::vector<Cand> cands;
    double per_row = A->nbrows ? (double)A->nnzb * A->block * A->block / (double)A->nbrows : 1.0;
    for (int L : {2, 4, 8, 16, 32})
        if (L <= 4 * per_row + 4) cands.push_back({0, L});
    if (A->block == 2 || A->block == 3) {
        cands.push_back({1, 32});
        for (int L : {32, 1, 2, 4, 8, 16}) cands.push_back({2, L});  // TMA configurations
        for (int L : {1, 2, 4, 8})  // whole-row configurations, where the longest row fits a stage
            if (spmv_prepare(A, 4, L) == YG_OK) cands.push_back({4, L});
    }
    const bool f32 = precision != YG_PREC_FP64;
    const double *corr = f32 ? A->d_corr32 : nullptr;
    int *pv = f32 ? &A->variant32 : &A->variant, *pl = f32 ? &A->lanes32 : &A->lanes;
    const int save_v = *pv, save_l = *pl;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    Cand bestc = {A->variant, A->lanes};
    yg_status s = YG_OK;
    const int reps = 3;
    for (const Cand &c : cands) {
        *pv = c.variant;
        *pl = c.lanes;
        const int grid = spmv_grid_for(A, precision);
        if ((s = spmv_launch(A, x, y, precision, nullptr, nullptr, grid, x32, corr)) != YG_OK) break;  // warm-up
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < reps; ++r) spmv_launch(A, x, y, precision, nullptr, nullptr, grid, x32, corr);
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; bestc = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *pv = save_v;
    *pl = save_l;
    *best_variant = bestc.variant;
    *best_lanes = bestc.lanes;
    return s;
}

// Device autotuner: time each candidate (flat with 2..32 lanes, cp.async
// staged and six TMA configurations for 2x2 and 3x3 blocks; the row-tile variant
// is taken only when set explicitly: on the assembled CSR matrices measured it
// stayed below the flat kernel) on this matrix with
// CUDA events and keep the fastest, separately for FP64 values and, when the
// matrix has them, FP32 values.  Must not run during stream capture.  Results
// are cached per (rows, blocks, block size, precision): a re-assembled matrix of
// the same pattern reuses the choice without timing again.
yg_status spmv_autotune_device(yg_matrix A) {
    const bool need64 = !A->tuned, need32 = A->d_val32 && !A->tuned32;
    if (!need64 && !need32) return YG_OK;
    yg_context ctx = A->ctx;
    cudaStreamCaptureStatus cs;
    YG_CUDA(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return YG_OK;
    double *x = nullptr, *y = nullptr;
    float *x32 = nullptr;  // FP32 gather copy: the mixed-precision solvers pass one to the TMA kernels
    bool allocated = false;
    for (int f32 = 0; f32 <= 1; ++f32) {
        if (f32 ? !need32 : !need64) continue;
        const TuneKey key{A->nbrows, A->nnzb, A->block, f32};
        bool hit = false;
        for (const auto &kv : g_tune_cache)
            if (kv.first == key && spmv_prepare(A, kv.second.first, kv.second.second) == YG_OK) {
                (f32 ? A->variant32 : A->variant) = kv.second.first;
                (f32 ? A->lanes32 : A->lanes) = kv.second.second;
                hit = true;
                break;
            }
        if (!hit) {
            if (!allocated) {
                const int64_t n = A->rows(), m = A->cols();
                const int64_t m32 = (m / A->block + 1) * spmv_x32_stride(A->block);
                YG_TRY(dev_alloc_t(ctx, &x, m + 1));
                yg_status s = dev_alloc_t(ctx, &y, n + 1);
                if (s == YG_OK) s = dev_alloc_t(ctx, &x32, m32);
                if (s != YG_OK) { dev_free(ctx, x); dev_free(ctx, y); return s; }
                cudaMemsetAsync(x, 0, sizeof(double) * (m + 1), ctx->stream);
                cudaMemsetAsync(x32, 0, sizeof(float) * m32, ctx->stream);
                allocated = true;
            }
            int v = 0, l = 32;
            yg_status s = tune_precision(A, f32 ? YG_PREC_MIXED : YG_PREC_FP64, x, f32 ? x32 : nullptr, y, &v, &l);
            if (s != YG_OK) {
                dev_free(ctx, x);
                dev_free(ctx, y);
                dev_free(ctx, x32);
                return s;
            }
            (f32 ? A->variant32 : A->variant) = v;
            (f32 ? A->lanes32 : A->lanes) = l;
            g_tune_cache.push_back({key, {v, l}});
        }
        (f32 ? A->tuned32 : A->tuned) = true;
    }
    if (allocated) {
        dev_free(ctx, x);
        dev_free(ctx, y);
        dev_free(ctx, x32);
    }
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

}  // namespace yg
