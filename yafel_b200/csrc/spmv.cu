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
// that each loads a handful of values, at most a warp.
void spmv_autotune(yg_matrix A) {
    double per_row = A->nbrows ? (double)A->nnzb * A->block * A->block / (double)A->nbrows : 1.0;
    int L = 2;
    while (L < 32 && per_row > 4.0 * L) L *= 2;
    A->lanes = L;
}

}  // namespace yg
