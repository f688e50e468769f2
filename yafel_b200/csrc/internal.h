// internal.h -- shared definitions of libyafel_b200 (not part of the C ABI).
#pragma once

#include "../../include/yafel_gpu.h"

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <unordered_map>
#include <map>

namespace yg {

void set_error(const char *fmt, ...);
yg_status fail(yg_status s, const char *fmt, ...);

#define YG_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return yg::fail(e_ == cudaErrorMemoryAllocation ? YG_OUT_OF_MEMORY : YG_CUDA_ERROR, \
                            "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),       \
                            __FILE__, __LINE__);                                          \
    } while (0)

#define YG_TRY(expr)                                \
    do {                                            \
        yg_status s_ = (expr);                      \
        if (s_ != YG_OK) return s_;                 \
    } while (0)

// Launch bookkeeping: every kernel launch goes through this so the context can
// report how many of its kernels ran.
#define YG_LAUNCHED(ctx) ((ctx)->launches++)

constexpr int kThreads = 256;         // threads per block for streaming kernels
constexpr int kMaxReduceBlocks = 4096;  // upper bound of partial sums per reduction

}  // namespace yg

// Solver scalars kept on the device so that a whole iteration (and a captured
// sequence of iterations) never waits on the host.
struct KrylovScalars {
    double rz[2];     // r.z of the current iteration, double-buffered by parity
    double rz0;       // r0.z0 (reference criterion)
    double bb;        // b.b
    double tol;       // criterion tolerance
    double rr;        // last r.r
    double rho[2], alpha, omega;  // BiCGSTAB recurrences (parity-buffered rho)
    int64_t iter;     // completed iterations
    int64_t maxiter;
    int32_t flag;     // 0 running, 1 converged, 2 breakdown, 3 nan, 4 iteration cap
    int32_t criterion;
    int32_t check_freq;  // BiCGSTAB reference criterion: true-residual check period
    int32_t pad;
    int64_t iter_seen;   // CG: iter as the update kernel saw it (read by the next kernel,
                         // which increments iter: no block reads a value another block writes)
};

struct yg_context_t {
    int device = 0;
    int num_sms = 148;
    size_t smem_optin = 227 * 1024;  // largest dynamic shared memory a block may opt in to
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    uint64_t in_use = 0;
    int64_t launches = 0;
    std::unordered_map<void *, size_t> allocs;
    // freed blocks kept for reuse (exact size), each with an event recorded on the
    // stream at its release: a reuse waits for the work that used it before
    struct CachedBlock {
        void *p;
        cudaEvent_t ev;
    };
    std::multimap<size_t, CachedBlock> cache;
    size_t cached_bytes = 0;
    // reduction scratch (device) and pinned host mailbox
    double *d_partials = nullptr;   // 8 * kMaxReduceBlocks doubles
    double *h_pinned = nullptr;     // 64 doubles of pinned host memory
    KrylovScalars *d_scalars = nullptr;
    int32_t *d_err = nullptr;       // device-side error word (bounded waits that expired)
    int reduce_blocks = 592;        // persistent grid for fused Krylov kernels
};

struct yg_vector_t {
    yg_context ctx = nullptr;
    int64_t n = 0;
    double *d = nullptr;
};

struct DofmapDevice;

struct yg_matrix_t {
    yg_context ctx = nullptr;
    int32_t block = 1;
    int64_t nbrows = 0, nbcols = 0, nnzb = 0;
    int32_t *d_rowptr = nullptr;  // nbrows+1
    int32_t *d_col = nullptr;     // nnzb
    double *d_val = nullptr;      // nnzb*block*block (row-major blocks)
    float *d_val32 = nullptr;     // optional FP32 copy
    // with the FP32 copy: per block row, the FP64 sum over its blocks of
    // (A_ij - fl32(A_ij)) (B*B per block row, row-major), so that the
    // mixed-precision solvers' operator A32 x + C x_own keeps A's block row sums
    double *d_corr32 = nullptr;
    int32_t *d_diag = nullptr;    // position of the diagonal block in each block row, -1 if absent
    int lanes = 32;               // SpMV lanes per block row (flat variant)
    int variant = 0;              // SpMV variant: 0 flat lane-strided, 1 cp.async staged, 2 TMA bulk staged (B = 2, 3),
                                  // 3 TMA row tiles (B = 1), 4 TMA whole rows (B = 2, 3)
    int variant32 = -1, lanes32 = 32;  // choice for FP32 values (-1: as for FP64)
    bool tuned32 = false;
    bool tuned = false;
    const void *owner = nullptr;  // dofmap whose pattern this is (assembly re-use)
    int32_t owner_format = -1;
    // Dirichlet scratch, kept between calls: row/column mask, prescribed values
    // g, K g, and the staged dof / value lists (bc_cap entries)
    uint8_t *d_bcmask = nullptr;
    double *d_bcg = nullptr, *d_bcq = nullptr, *d_bcvals = nullptr;
    int64_t *d_bcdofs = nullptr;
    int64_t bc_cap = 0;
    // Row tiles of the tiled CSR SpMV (variant 3): table k holds the first row
    // of each tile of at most (256 << k) entries, then the row count
    int32_t *d_ctiles[3] = {nullptr, nullptr, nullptr};
    int64_t nctiles[3] = {0, 0, 0};
    int32_t row_min = -1, row_max = -1;  // entries per row, -1 until measured
    int64_t rows() const { return nbrows * block; }
    int64_t cols() const { return nbcols * block; }
};

struct yg_precond_t {
    yg_matrix A = nullptr;
    yg_context ctx = nullptr;  // A's context: destroy must not touch A, which may already be gone
    int32_t kind = 0;
    double *d_dinv = nullptr;     // Jacobi: 1/a_ii (scalar diagonal)
    int64_t zero_pivots = 0;
    // ILU(0): factor values on A's pattern (scalar CSR view) + level schedules
    double *d_lu = nullptr;
    int32_t *d_lower_levels = nullptr, *d_upper_levels = nullptr;  // row lists grouped by level
    std::vector<int32_t> lower_level_ptr, upper_level_ptr;
    int32_t *d_csr_rowptr = nullptr, *d_csr_col = nullptr, *d_csr_diag = nullptr;  // scalar view
    int32_t *d_lower_ptr = nullptr, *d_upper_ptr = nullptr;  // level pointers for the persistent sweeps
    uint32_t *d_bar = nullptr;                              // their grid barrier (count, generation)
    int64_t n = 0, nnz = 0;
    double *d_tmp = nullptr;
};

namespace yg {

yg_status dev_alloc(yg_context ctx, void **p, size_t bytes);
void dev_free(yg_context ctx, void *p);
template <typename T>
yg_status dev_alloc_t(yg_context ctx, T **p, size_t count) {
    return dev_alloc(ctx, reinterpret_cast<void **>(p), count * sizeof(T) + 16);
}

// ---- kernels-side entry points (implemented in .cu files) ----
// x32 (optional, FP32-value precisions only): the same vector rounded to FP32 in
// the node-padded layout of spmv_x32_stride(); the TMA kernels then gather it
// with one vector load per block instead of B scalar FP64 loads.
// corr (optional, FP32-value precisions only): the matrix's d_corr32; each
// block row r then gets y_r += corr_r x_r (FP64), the corrected FP32 operator
// of the mixed-precision solvers.
yg_status spmv_launch(yg_matrix A, const double *x, double *y, int precision, double *partials_dot,
                      const int32_t *flag, int grid, const float *x32 = nullptr, const double *corr = nullptr);
yg_status spmv_launch_ex(yg_matrix A, const double *x, double *y, int precision, const double *w, double *partials,
                         int dot_mode, const int32_t *flag, int grid, cudaStream_t stream = nullptr,
                         const float *x32 = nullptr, const double *corr = nullptr);
// Floats per block row of an FP32 gather copy: 4 for 3x3 blocks (16-byte rows),
// else the block size.
inline int spmv_x32_stride(int block) { return block == 3 ? 4 : block; }
int spmv_default_grid(yg_matrix A);
int spmv_grid_for(yg_matrix A, int precision);
void spmv_autotune(yg_matrix A);
yg_status spmv_autotune_device(yg_matrix A);
// Builds what SpMV variant/lanes needs before its first launch (the row tiles of
// variant 3); YG_UNSUPPORTED when the matrix cannot use it.  Not during capture.
yg_status spmv_prepare(yg_matrix A, int variant, int lanes);
yg_status vector_dot(yg_context ctx, const double *a, const double *b, int64_t n, double *out);
yg_status check_device_error(yg_context ctx);
yg_status matrix_build_diag(yg_matrix A);
void flush_alloc_cache(yg_context ctx);
// batch engine, host side (batch.cu)
bool batch_slot_running(yg_batch bt, int32_t slot);
void batch_slot_stats(yg_batch bt, int32_t slot, yg_solve_stats *out);
yg_status matrix_from_device_pattern(yg_matrix A);

}  // namespace yg
