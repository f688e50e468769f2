// device_common.cuh -- device helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

// Deterministic block reduction: fixed xor-butterfly inside each warp, then the
// warp sums added in warp order by thread 0.  Result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sm) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NT / 32; ++i) s += sm[i];
    }
    __syncthreads();
    return s;
}

// Same, with the result broadcast to every thread (sm needs NT/32+1 slots).
template <int NT>
__device__ __forceinline__ double block_sum_all(double v, double *sm) {
    double s = block_sum<NT>(v, sm);
    if (threadIdx.x == 0) sm[NT / 32] = s;
    __syncthreads();
    s = sm[NT / 32];
    __syncthreads();
    return s;
}

// Sum of `np` per-block partials (stride `stride`, offset `off`), computed
// identically by every block so that all blocks agree on the bits.
template <int NT>
__device__ __forceinline__ double reduce_partials(const double *__restrict__ partials, int np, int stride, int off,
                                                  double *sm) {
    double s = 0;
    for (int i = threadIdx.x; i < np; i += NT) s += partials[(int64_t)i * stride + off];
    return block_sum_all<NT>(s, sm);
}

// Streaming loads for matrix values: read once per SpMV, so they bypass L1 and
// carry an L2 evict-first policy, which keeps the gathered vector resident.
__device__ __forceinline__ uint64_t evict_first_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ double ld_stream(const double *p, uint64_t pol) {
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_stream(const float *p, uint64_t pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return (double)v;
}
__device__ __forceinline__ int ld_stream_i(const int *p, uint64_t pol) {
    int v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

// Contiguous chunk [lo, hi) of n items owned by block b of g.
__device__ __forceinline__ void block_chunk(int64_t n, int64_t &lo, int64_t &hi) {
    int64_t per = (n + gridDim.x - 1) / gridDim.x;
    lo = (int64_t)blockIdx.x * per;
    hi = lo + per;
    if (hi > n) hi = n;
    if (lo > n) lo = n;
}

// Corrected FP32 operator: s += corr_r x_r, row i of the block row's FP64
// correction (corr, B*B per block row: the sum over the row's blocks of
// A - fl32(A)) times the row's own entries of x (FP64).
template <int B>
__device__ __forceinline__ void add_corr(const double *__restrict__ corr, const double *__restrict__ x, int64_t r,
                                         double (&s)[B]) {
    double xr[B];
#pragma unroll
    for (int k = 0; k < B; ++k) xr[k] = x[(int64_t)B * r + k];
#pragma unroll
    for (int i = 0; i < B; ++i) {
        const double *c = corr + ((int64_t)B * r + i) * B;
        double t = c[0] * xr[0];
#pragma unroll
        for (int k = 1; k < B; ++k) t = fma(c[k], xr[k], t);
        s[i] += t;
    }
}

// As block_chunk, with chunk starts on even indices (16-byte aligned doubles) so
// that a block can stream its chunk as double2.
__device__ __forceinline__ void block_chunk2(int64_t n, int64_t &lo, int64_t &hi) {
    int64_t per = (n + gridDim.x - 1) / gridDim.x;
    per += per & 1;
    lo = (int64_t)blockIdx.x * per;
    hi = lo + per;
    if (hi > n) hi = n;
    if (lo > n) lo = n;
}

__device__ __forceinline__ int read_flag(const int32_t *flag) {
    return *reinterpret_cast<const volatile int32_t *>(flag);
}

// ---- mbarrier + bulk asynchronous copy (cp.async.bulk) helpers

// Bound on the polls of one mbarrier wait; a kernel that reaches it records
// YG_TIMEOUT and stops instead of spinning on.
constexpr long long kSpinLimit = 1ll << 26;

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar, uint64_t pol) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(d),
        "l"(src), "r"(bytes), "r"(b), "l"(pol)
        : "memory");
}
