// static_scratch.cu -- a dot product that allocates nothing.
//
// yg_vector_dot keeps its per-block partial sums in memory that yg_context_create
// allocated.  Some callers cannot allocate device memory at the point where they
// need a reduction, or cannot create a context at all:
//   * a host framework that has reserved the device's memory for its own pool
//     (a served solver that admits systems against a fixed HBM budget, say):
//     a cudaMalloc there either fails or grows past the budget it accounts for;
//   * a latency-bound loop between solver steps, where cudaMalloc / cudaFree
//     would synchronise the device and stall the streams of other work.
// yg_dot_static_scratch serves them: it takes plain device pointers and a
// stream, and its partial sums live in a fixed array of this library's device
// code (one copy per device), so a call allocates nothing.
#include "internal.h"
#include "device_common.cuh"

#include <mutex>

namespace {

using yg::kThreads;

// Each block reduces one fixed chunk of values, so the number of partial sums
// is ceil(n / kChunk) and the result does not depend on the device's SM count.
constexpr int kChunk = kThreads * 32;        // 8192 values per block
constexpr int kSlots = 8192;                 // partial sums: 64 KiB of doubles
constexpr int64_t kMaxN = (int64_t)kSlots * kChunk;  // 67,108,864 values
constexpr int kMaxDevices = 64;

// The scratch.  Nothing in it has to start at zero: every call writes each
// partial sum it later reads, in stream order.
static __device__ __align__(256) double g_dot_scratch[kSlots];

std::mutex g_addr_mu;
double *g_addr[kMaxDevices] = {};

__global__ void __launch_bounds__(kThreads) k_chunk_dot(const double *__restrict__ a, const double *__restrict__ b,
                                                        int64_t n, double *__restrict__ partials) {
    __shared__ double sm[kThreads / 32];
    const int64_t lo = (int64_t)blockIdx.x * kChunk;
    const int64_t hi = lo + kChunk < n ? lo + kChunk : n;
    double s = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += kThreads) s += a[i] * b[i];
    s = block_sum<kThreads>(s, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_chunk_sum(const double *__restrict__ partials, int np,
                                                        double *__restrict__ out) {
    __shared__ double sm[kThreads / 32];
    double s = 0;
    for (int i = threadIdx.x; i < np; i += kThreads) s += partials[i];
    s = block_sum<kThreads>(s, sm);
    if (threadIdx.x == 0) out[0] = s;
}

// Device address of the scratch on the current device, looked up once per
// device with cudaGetSymbolAddress and cached for the life of the process.
yg_status scratch_address(double **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return yg::fail(YG_CUDA_ERROR, "yg_dot_static_scratch: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return yg::fail(YG_UNSUPPORTED, "yg_dot_static_scratch: device %d is beyond the %d this library tracks", dev,
                        kMaxDevices);
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[dev]) {
        double *ptr = nullptr;
        e = cudaGetSymbolAddress((void **)&ptr, g_dot_scratch);
        if (e != cudaSuccess || !ptr)
            return yg::fail(YG_CUDA_ERROR, "yg_dot_static_scratch: cudaGetSymbolAddress on device %d: %s", dev,
                            cudaGetErrorString(e));
        g_addr[dev] = ptr;
    }
    *out = g_addr[dev];
    return YG_OK;
}

}  // namespace

extern "C" yg_status yg_dot_static_scratch(const double *x, const double *y, int64_t n, double *out, void *stream) {
    if (!out || n < 0 || (n > 0 && (!x || !y)))
        return yg::fail(YG_BAD_ARG, "yg_dot_static_scratch: NULL pointer or negative length");
    if (n > kMaxN)
        return yg::fail(YG_BAD_ARG,
                        "yg_dot_static_scratch: n = %lld exceeds the static scratch limit of %lld values "
                        "(%d partial sums of %d values); use yg_vector_dot",
                        (long long)n, (long long)kMaxN, kSlots, kChunk);
    double *partials = nullptr;
    YG_TRY(scratch_address(&partials));
    cudaStream_t st = (cudaStream_t)stream;
    const int g = (int)((n + kChunk - 1) / kChunk);
    if (g > 0) k_chunk_dot<<<g, kThreads, 0, st>>>(x, y, n, partials);
    k_chunk_sum<<<1, kThreads, 0, st>>>(partials, g, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return yg::fail(YG_CUDA_ERROR, "yg_dot_static_scratch: launch: %s", cudaGetErrorString(e));
    return YG_OK;
}
