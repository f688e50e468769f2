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

namespace yg {

// DOT = 0: y = A x.  DOT = 1: also per-block sums of w.y.  DOT = 2: per-block
// sums of w.y and y.y (partials[2b], partials[2b+1]).
template <int B, int L, typename VT, int DOT>
__global__ void __launch_bounds__(kThreads)
k_bcsr_spmv(int64_t nbrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
            const VT *__restrict__ val, const double *__restrict__ x, double *__restrict__ y,
            const double *__restrict__ w, double *__restrict__ partials, const int32_t *__restrict__ flag) {
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
// Staged variant for B = 2, 3.  Each warp owns a sequence of block rows; the
// row's value bytes are copied into a per-warp shared-memory stage with 16-byte
// cp.async copies (L2 evict-first), double-buffered so the next chunk is in
// flight while the current one is consumed.  Then lane l owns whole blocks
// l, l+32, ... of the chunk: it reads the block's B*B values from shared memory,
// one column index and B entries of x, so each value costs one shared load and
// one FMA.  A chunk holds up to CH blocks; longer rows are processed in chunks.
// Copies start at the 16-byte boundary below the chunk and end at the one above
// it (allocations carry 16 bytes of padding), and the consumer skips the lead.
template <int B, typename VT>
struct Staged {
    static constexpr int CH = 64;                                     // blocks per chunk
    static constexpr int STAGE = CH * B * B * (int)sizeof(VT) + 32;   // bytes per stage
    static constexpr int WARPS = 8;
    static constexpr int SMEM = WARPS * 2 * STAGE;
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, uint64_t pol) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "l"(pol));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <int B, typename VT, int DOT>
__global__ void __launch_bounds__(Staged<B, VT>::WARPS * 32)
k_bcsr_spmv_staged(int64_t nbrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                   const VT *__restrict__ val, const double *__restrict__ x, double *__restrict__ y,
                   const double *__restrict__ w, double *__restrict__ partials, const int32_t *__restrict__ flag) {
    using S = Staged<B, VT>;
    constexpr int B2 = B * B;
    constexpr int BB = B2 * (int)sizeof(VT);  // bytes per block
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[S::WARPS + 1];
    if (flag && read_flag(flag)) return;
    const uint64_t pol = evict_first_policy();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *stage0 = smem_raw + (size_t)wib * 2 * S::STAGE;
    const int64_t warp = (int64_t)blockIdx.x * S::WARPS + wib;
    const int64_t nwarps = (int64_t)gridDim.x * S::WARPS;
    const char *vbytes = reinterpret_cast<const char *>(val);

    // chunk cursor: row r, block offset b0 within the row
    int64_t r = warp;
    int b0 = 0;
    int rs = 0, re = 0;
    if (r < nbrows) { rs = __ldg(rowptr + r); re = __ldg(rowptr + r + 1); }
    // issue the copy of chunk (r, b0) into stage st; returns the lead bytes
    auto issue = [&](int64_t rr, int bb0, int rrs, int rre, int st) -> int {
        int lead = 0;
        if (rr < nbrows && rre > rrs) {
            const int nb = min(S::CH, rre - rrs - bb0);
            const int64_t start = (int64_t)(rrs + bb0) * BB;
            const int64_t a0 = start & ~(int64_t)15;
            const int64_t a1 = (start + (int64_t)nb * BB + 15) & ~(int64_t)15;
            lead = (int)(start - a0);
            unsigned char *dst = stage0 + st * S::STAGE;
            for (int64_t off = (int64_t)lane * 16; off < a1 - a0; off += 32 * 16) cp_async16(dst + off, vbytes + a0 + off, pol);
        }
        cp_async_commit();
        return lead;
    };
    double dot = 0, yy = 0;
    double acc[B];
#pragma unroll
    for (int i = 0; i < B; ++i) acc[i] = 0;
    int st = 0;
    int lead_cur = issue(r, b0, rs, re, 0);
    while (r < nbrows) {
        // next chunk cursor
        int64_t rn = r;
        int bn = b0 + S::CH, rsn = rs, ren = re;
        if (bn >= re - rs) {
            rn = r + nwarps;
            bn = 0;
            rsn = ren = 0;
            if (rn < nbrows) { rsn = __ldg(rowptr + rn); ren = __ldg(rowptr + rn + 1); }
        }
        const int lead_next = issue(rn, bn, rsn, ren, st ^ 1);
        cp_async_wait1();
        __syncwarp();
        // consume chunk (r, b0) from stage st
        const int nb = max(0, min(S::CH, re - rs - b0));
        const VT *blk = reinterpret_cast<const VT *>(stage0 + st * S::STAGE + lead_cur);
        for (int j = lane; j < nb; j += 32) {
            const int c = __ldg(col + rs + b0 + j);
            double xv[B];
#pragma unroll
            for (int k = 0; k < B; ++k) xv[k] = __ldg(x + (int64_t)B * c + k);
#pragma unroll
            for (int i = 0; i < B; ++i)
#pragma unroll
                for (int k = 0; k < B; ++k) acc[i] = fma((double)blk[j * B2 + i * B + k], xv[k], acc[i]);
        }
        __syncwarp();
        if (b0 + S::CH >= re - rs) {  // row complete
#pragma unroll
            for (int i = 0; i < B; ++i) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
            }
            if (lane == 0) {
#pragma unroll
                for (int i = 0; i < B; ++i) {
                    y[B * r + i] = acc[i];
                    if (DOT >= 1) dot = fma(acc[i], w[B * r + i], dot);
                    if (DOT == 2) yy = fma(acc[i], acc[i], yy);
                }
            }
#pragma unroll
            for (int i = 0; i < B; ++i) acc[i] = 0;
        }
        r = rn;
        b0 = bn;
        rs = rsn;
        re = ren;
        lead_cur = lead_next;
        st ^= 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (DOT) {
        // lane 0 of each warp holds the warp's sum; fixed-order block sum
        if (lane == 0) red[wib] = dot;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0;
            for (int i = 0; i < S::WARPS; ++i) s += red[i];
            if (DOT == 1) partials[blockIdx.x] = s;
            else partials[2 * blockIdx.x] = s;
        }
        if (DOT == 2) {
            __syncthreads();
            if (lane == 0) red[wib] = yy;
            __syncthreads();
            if (threadIdx.x == 0) {
                double s = 0;
                for (int i = 0; i < S::WARPS; ++i) s += red[i];
                partials[2 * blockIdx.x + 1] = s;
            }
        }
    }
}

template <int B, typename VT, int DOT>
static yg_status launch_staged(yg_matrix A, const VT *val, const double *x, double *y, const double *w,
                               double *partials, const int32_t *flag, int grid, cudaStream_t st) {
    using S = Staged<B, VT>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_bcsr_spmv_staged<B, VT, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM);
        attr = true;
    }
    k_bcsr_spmv_staged<B, VT, DOT><<<grid, S::WARPS * 32, S::SMEM, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y,
                                                                        w, partials, flag);
    YG_LAUNCHED(A->ctx);
    return YG_OK;
}

template <int B, typename VT, int DOT>
static yg_status launch_l(yg_matrix A, const VT *val, const double *x, double *y, const double *w, double *partials,
                          const int32_t *flag, int grid, cudaStream_t st) {
    switch (A->lanes) {
    case 2: k_bcsr_spmv<B, 2, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag); break;
    case 4: k_bcsr_spmv<B, 4, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag); break;
    case 8: k_bcsr_spmv<B, 8, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag); break;
    case 16: k_bcsr_spmv<B, 16, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag); break;
    default: k_bcsr_spmv<B, 32, VT, DOT><<<grid, kThreads, 0, st>>>(A->nbrows, A->d_rowptr, A->d_col, val, x, y, w, partials, flag); break;
    }
    YG_LAUNCHED(A->ctx);
    return YG_OK;
}

template <typename VT, int DOT>
static yg_status launch_b(yg_matrix A, const VT *val, const double *x, double *y, const double *w, double *partials,
                          const int32_t *flag, int grid, cudaStream_t st) {
    if (A->variant == 1 && A->block == 3) return launch_staged<3, VT, DOT>(A, val, x, y, w, partials, flag, grid, st);
    if (A->variant == 1 && A->block == 2) return launch_staged<2, VT, DOT>(A, val, x, y, w, partials, flag, grid, st);
    switch (A->block) {
    case 1: return launch_l<1, VT, DOT>(A, val, x, y, w, partials, flag, grid, st);
    case 2: return launch_l<2, VT, DOT>(A, val, x, y, w, partials, flag, grid, st);
    case 3: return launch_l<3, VT, DOT>(A, val, x, y, w, partials, flag, grid, st);
    default: return fail(YG_UNSUPPORTED, "SpMV block size %d not supported (1, 2, 3)", A->block);
    }
}

template <typename VT>
static yg_status launch_v(yg_matrix A, const VT *val, const double *x, double *y, const double *w, double *partials,
                          int dot_mode, const int32_t *flag, int grid, cudaStream_t st) {
    if (dot_mode == 0) return launch_b<VT, 0>(A, val, x, y, w, partials, flag, grid, st);
    if (dot_mode == 1) return launch_b<VT, 1>(A, val, x, y, w, partials, flag, grid, st);
    return launch_b<VT, 2>(A, val, x, y, w, partials, flag, grid, st);
}

// y = A x.  With `partials`: per-block sums of w.y (dot_mode 1; w defaults to
// x) or of w.y and y.y (dot_mode 2).  The grid is persistent: `grid` blocks
// stride over the block rows.
yg_status spmv_launch_ex(yg_matrix A, const double *x, double *y, int precision, const double *w, double *partials,
                         int dot_mode, const int32_t *flag, int grid) {
    cudaStream_t st = A->ctx->stream;
    if (grid > kMaxReduceBlocks) grid = kMaxReduceBlocks;
    if (!partials) dot_mode = 0;
    if (!w) w = x;
    yg_status s;
    if (precision == YG_PREC_MIXED) {
        if (!A->d_val32) return fail(YG_BAD_ARG, "mixed-precision SpMV without FP32 values");
        s = launch_v<float>(A, A->d_val32, x, y, w, partials, dot_mode, flag, grid, st);
    } else {
        s = launch_v<double>(A, A->d_val, x, y, w, partials, dot_mode, flag, grid, st);
    }
    if (s != YG_OK) return s;
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

yg_status spmv_launch(yg_matrix A, const double *x, double *y, int precision, double *partials,
                      const int32_t *flag, int grid) {
    return spmv_launch_ex(A, x, y, precision, x, partials, partials ? 1 : 0, flag, grid);
}

int spmv_default_grid(yg_matrix A) {
    if (A->variant == 1) {  // staged: 2 blocks of 8 warps per SM, a warp per row
        int64_t need = (A->nbrows + 7) / 8;
        int64_t g = (int64_t)A->ctx->num_sms * 2;
        if (need < g) g = need;
        return (int)(g < 1 ? 1 : g);
    }
    // enough resident warps to keep HBM busy: 8 blocks of 256 threads per SM,
    // but no more row groups than rows.
    int64_t groups_per_block = kThreads / A->lanes;
    int64_t need = (A->nbrows + groups_per_block - 1) / groups_per_block;
    int64_t g = (int64_t)A->ctx->num_sms * 8;
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
    int block;
    bool operator==(const TuneKey &o) const { return nbrows == o.nbrows && nnzb == o.nnzb && block == o.block; }
};
static std::vector<std::pair<TuneKey, std::pair<int, int>>> g_tune_cache;

yg_status spmv_autotune_device(yg_matrix A) {
    if (A->tuned) return YG_OK;
    const TuneKey key{A->nbrows, A->nnzb, A->block};
    for (const auto &kv : g_tune_cache)
        if (kv.first == key) {
            A->variant = kv.second.first;
            A->lanes = kv.second.second;
            A->tuned = true;
            return YG_OK;
        }
    yg_context ctx = A->ctx;
    cudaStreamCaptureStatus cs;
    YG_CUDA(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return YG_OK;
    const int64_t n = A->rows(), m = A->cols();
    double *x = nullptr, *y = nullptr;
    YG_TRY(dev_alloc_t(ctx, &x, m + 1));
    yg_status s = dev_alloc_t(ctx, &y, n + 1);
    if (s != YG_OK) { dev_free(ctx, x); return s; }
    cudaMemsetAsync(x, 0, sizeof(double) * (m + 1), ctx->stream);
    struct Cand { int variant, lanes; };
    std::vector<Cand> cands;
    double per_row = A->nbrows ? (double)A->nnzb * A->block * A->block / (double)A->nbrows : 1.0;
    for (int L : {2, 4, 8, 16, 32})
        if (L <= 4 * per_row + 4) cands.push_back({0, L});
    if (A->block == 2 || A->block == 3) cands.push_back({1, 32});
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    Cand bestc = {A->variant, A->lanes};
    const int reps = 3;
    for (const Cand &c : cands) {
        A->variant = c.variant;
        A->lanes = c.lanes;
        int grid = spmv_default_grid(A);
        if ((s = spmv_launch(A, x, y, YG_PREC_FP64, nullptr, nullptr, grid)) != YG_OK) break;  // warm-up
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < reps; ++r) spmv_launch(A, x, y, YG_PREC_FP64, nullptr, nullptr, grid);
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; bestc = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    A->variant = bestc.variant;
    A->lanes = bestc.lanes;
    A->tuned = true;
    if (s == YG_OK) g_tune_cache.push_back({key, {bestc.variant, bestc.lanes}});
    dev_free(ctx, x);
    dev_free(ctx, y);
    if (s != YG_OK) return s;
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

}  // namespace yg
