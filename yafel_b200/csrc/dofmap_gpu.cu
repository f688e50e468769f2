// dofmap_gpu.cu -- the CG DoF numbering of p > 1 meshes on the GPU.
//
// Replaces DoFManager::make_raw_dofs + recombine_all_duplicates
// (src/utils/DoFManager.cpp:176-229, 340-414) for large meshes.  The steps and
// their arithmetic are those of the host numbering (host_fe.cpp), so the result
// is bit-identical to it whenever the host uses its stable radix sort (more than
// kReferenceOrderMaxRawNodes raw nodes, no simplex/tensor mix at p >= 3):
//   1. raw nodes: a warp per cell places the element's local nodes with
//      interpolate_from_corners (DoFManager.cpp:296-338), in the host's operation
//      order with rounded (never fused) multiplies and adds;
//   2. bounding box -> snap s = 1e-6 * largest extent; integer keys
//      round(x * (1/s)) per coordinate, packed (z, y, x) into 64 bits;
//   3. a stable LSD radix sort of (key, raw index), 8-bit digits: per-tile digit
//      histograms, one exclusive scan over (digit, tile), and a scatter in
//      which each warp ranks equal digits with __match_any_sync, so equal keys
//      keep raw order;
//   4. merge: a sorted entry starts a node unless it lies within 1e-6 of the
//      previous one; a scan of the starts numbers the nodes; each raw node gets
//      its node number and each node the coordinates of its first raw node.
// The numbering and coordinates are copied back to the host dofmap (the
// element colouring and the host API read them) and kept on the device.
// generate_box builds a structured quadrilateral or hexahedron box on the
// device, so that a box's DoFManager needs no mesh from the host.
#include "internal.h"
#include "host_fe.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

namespace yg {

int stream_grid(yg_context ctx, int64_t n);

namespace {

constexpr int kSortThreads = 256, kSortRounds = 16, kTile = kSortThreads * kSortRounds;

// interpolate_from_corners with the host's evaluation order and no contraction
__device__ double corner_map(int ct, const double *xl, const double *c, int k) {
    const double x0 = xl[0], x1 = xl[1], x2 = xl[2];
    auto mul = [](double a, double b) { return __dmul_rn(a, b); };
    auto add = [](double a, double b) { return __dadd_rn(a, b); };
    auto sub = [](double a, double b) { return __dsub_rn(a, b); };
    switch (ct) {
    case 1:  // Tri3
        return add(add(mul(sub(sub(1.0, x0), x1), c[k]), mul(x0, c[3 + k])), mul(x1, c[6 + k]));
    case 2:  // Tet4
        return add(add(add(mul(sub(sub(sub(1.0, x0), x1), x2), c[k]), mul(x0, c[3 + k])), mul(x1, c[6 + k])),
                   mul(x2, c[9 + k]));
    case 3: {  // Quad4
        const double m0 = sub(1.0, x0), p0 = add(1.0, x0), m1 = sub(1.0, x1), p1 = add(1.0, x1);
        double s = mul(mul(m0, m1), c[k]);
        s = add(s, mul(mul(p0, m1), c[3 + k]));
        s = add(s, mul(mul(p0, p1), c[6 + k]));
        s = add(s, mul(mul(m0, p1), c[9 + k]));
        return mul(1.0 / 4.0, s);
    }
    case 4: {  // Hex8
        const double m0 = sub(1.0, x0), p0 = add(1.0, x0), m1 = sub(1.0, x1), p1 = add(1.0, x1),
                     m2 = sub(1.0, x2), p2 = add(1.0, x2);
        double s = mul(mul(mul(m0, m1), m2), c[k]);
        s = add(s, mul(mul(mul(p0, m1), m2), c[3 + k]));
        s = add(s, mul(mul(mul(p0, p1), m2), c[6 + k]));
        s = add(s, mul(mul(mul(m0, p1), m2), c[9 + k]));
        s = add(s, mul(mul(mul(m0, m1), p2), c[12 + k]));
        s = add(s, mul(mul(mul(p0, m1), p2), c[15 + k]));
        s = add(s, mul(mul(mul(p0, p1), p2), c[18 + k]));
        s = add(s, mul(mul(mul(m0, p1), p2), c[21 + k]));
        return mul(1.0 / 8.0, s);
    }
    default: return 0.0;
    }
}

// 1. raw nodes: one warp per cell, lanes over its local nodes
__global__ void k_raw_nodes(int32_t ncells, const int32_t *__restrict__ coff, const int32_t *__restrict__ cnodes,
                            const int32_t *__restrict__ ctype, const double *__restrict__ xyz,
                            const int32_t *__restrict__ roff, const int32_t *__restrict__ tab_of_cell,
                            const double *__restrict__ tabs, const int32_t *__restrict__ tab_start,
                            double *__restrict__ raw) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c < ncells; c += nwarps) {
        const int tb = tab_of_cell[c];
        if (tb < 0) continue;
        double corners[24];
        const int nc = min(coff[c + 1] - coff[c], 8);
        for (int i = 0; i < 24; ++i) corners[i] = 0;
        for (int i = 0; i < nc; ++i)
            for (int k = 0; k < 3; ++k) corners[3 * i + k] = xyz[3 * (int64_t)cnodes[coff[c] + i] + k];
        const int nl = roff[c + 1] - roff[c];
        const double *L = tabs + 3 * (int64_t)tab_start[tb];
        for (int a = lane; a < nl; a += 32)
            for (int k = 0; k < 3; ++k) raw[3 * ((int64_t)roff[c] + a) + k] = corner_map(ctype[c], L + 3 * a, corners, k);
    }
}

// 2a. per-block min/max of each coordinate (then reduced on the host)
__global__ void k_bbox(int64_t n, const double *__restrict__ raw, double *__restrict__ out) {
    __shared__ double sm[6][kSortThreads];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k) {
            lo[k] = fmin(lo[k], raw[3 * i + k]);
            hi[k] = fmax(hi[k], raw[3 * i + k]);
        }
    for (int k = 0; k < 3; ++k) { sm[k][threadIdx.x] = lo[k]; sm[3 + k][threadIdx.x] = hi[k]; }
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int k = 0; k < 3; ++k) {
                sm[k][threadIdx.x] = fmin(sm[k][threadIdx.x], sm[k][threadIdx.x + o]);
                sm[3 + k][threadIdx.x] = fmax(sm[3 + k][threadIdx.x], sm[3 + k][threadIdx.x + o]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) out[6 * blockIdx.x + threadIdx.x] = sm[threadIdx.x][0];
}

__device__ __forceinline__ long long snap_key(double x, double inv) { return __double2ll_rn(round(__dmul_rn(x, inv))); }

// 2b. per-block min/max of the integer keys
__global__ void k_key_range(int64_t n, const double *__restrict__ raw, double inv, long long *__restrict__ out) {
    __shared__ long long sm[6][kSortThreads];
    long long lo[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, hi[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k) {
            const long long v = snap_key(raw[3 * i + k], inv);
            lo[k] = min(lo[k], v);
            hi[k] = max(hi[k], v);
        }
    for (int k = 0; k < 3; ++k) { sm[k][threadIdx.x] = lo[k]; sm[3 + k][threadIdx.x] = hi[k]; }
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int k = 0; k < 3; ++k) {
                sm[k][threadIdx.x] = min(sm[k][threadIdx.x], sm[k][threadIdx.x + o]);
                sm[3 + k][threadIdx.x] = max(sm[3 + k][threadIdx.x], sm[3 + k][threadIdx.x + o]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) out[6 * blockIdx.x + threadIdx.x] = sm[threadIdx.x][0];
}

// 2c. packed keys (z, y, x) and the identity permutation
__global__ void k_pack_keys(int64_t n, const double *__restrict__ raw, double inv, long long k0, long long k1,
                            long long k2, int b0, int b1, uint64_t *__restrict__ keys, int32_t *__restrict__ idx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t x = (uint64_t)(snap_key(raw[3 * i], inv) - k0);
        const uint64_t y = (uint64_t)(snap_key(raw[3 * i + 1], inv) - k1);
        const uint64_t z = (uint64_t)(snap_key(raw[3 * i + 2], inv) - k2);
        keys[i] = (z << (b0 + b1)) | (y << b0) | x;
        idx[i] = (int32_t)i;
    }
}

// 3a. digit histogram of each tile, stored digit-major: hist[d * ntiles + tile]
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(int64_t n, const uint64_t *__restrict__ keys, int shift,
                                                             int64_t ntiles, int32_t *__restrict__ hist) {
    __shared__ int32_t cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t t0 = blockIdx.x * (int64_t)kTile;
    for (int r = 0; r < kSortRounds; ++r) {
        const int64_t i = t0 + (int64_t)r * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255], 1);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// 3b. stable scatter: items in order (round, warp, lane); equal digits ranked
// within a warp by __match_any_sync, across warps by the per-round counts
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(int64_t n, const uint64_t *__restrict__ kin,
                                                                const int32_t *__restrict__ vin, int shift,
                                                                int64_t ntiles, const int64_t *__restrict__ offs,
                                                                uint64_t *__restrict__ kout, int32_t *__restrict__ vout) {
    constexpr int W = kSortThreads / 32;
    __shared__ int64_t base[256];
    __shared__ int32_t wcnt[W][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    base[threadIdx.x] = offs[(int64_t)threadIdx.x * ntiles + blockIdx.x];
    const int64_t t0 = blockIdx.x * (int64_t)kTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < kSortRounds; ++r) {
        const int64_t i = t0 + (int64_t)r * kSortThreads + threadIdx.x;
        const bool valid = i < n;
        const uint64_t key = valid ? kin[i] : 0;
        const int d = valid ? (int)((key >> shift) & 255) : 256;  // 256: no item
        for (int k = lane; k < 256; k += 32) wcnt[w][k] = 0;
        __syncthreads();
        const unsigned same = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(same & lt);
        if (valid && rank == 0) wcnt[w][d] = __popc(same);
        __syncthreads();
        if (valid) {
            int64_t pos = base[d] + rank;
            for (int v = 0; v < w; ++v) pos += wcnt[v][d];
            kout[pos] = key;
            vout[pos] = vin[i];
        }
        __syncthreads();
        int32_t add = 0;
        for (int v = 0; v < W; ++v) add += wcnt[v][threadIdx.x];
        base[threadIdx.x] += add;
        __syncthreads();
    }
}

// exclusive scan of int32 counts into int64 offsets (two levels; the second
// level is small enough for one block)
__global__ void __launch_bounds__(1024) k_scan_a(const int32_t *__restrict__ in, int64_t n, int64_t *__restrict__ out,
                                                 int64_t *__restrict__ sums) {
    __shared__ int64_t sm[1024];
    const int64_t i = blockIdx.x * (int64_t)1024 + threadIdx.x;
    const int64_t v = i < n ? in[i] : 0;
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int64_t t = threadIdx.x >= o ? sm[threadIdx.x - o] : 0;
        __syncthreads();
        sm[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) out[i] = sm[threadIdx.x] - v;
    if (threadIdx.x == 1023) sums[blockIdx.x] = sm[1023];
}
__global__ void __launch_bounds__(1024) k_scan_b(int64_t *__restrict__ sums, int64_t nb) {
    __shared__ int64_t sm[1024];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t s = 0; s < nb; s += 1024) {
        const int64_t i = s + threadIdx.x;
        const int64_t v = i < nb ? sums[i] : 0;
        sm[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int64_t t = threadIdx.x >= o ? sm[threadIdx.x - o] : 0;
            __syncthreads();
            sm[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nb) sums[i] = carry + sm[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += sm[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = carry;
}
__global__ void k_scan_c(int64_t *__restrict__ out, int64_t n, const int64_t *__restrict__ sums) {
    const int64_t i = blockIdx.x * (int64_t)1024 + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

// 4a. start flags of the sorted sequence
__global__ void k_merge_flags(int64_t n, const int32_t *__restrict__ idx, const double *__restrict__ raw,
                              int32_t *__restrict__ flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t f = 1;
        if (i > 0) {
            const double *a = raw + 3 * (int64_t)idx[i], *b = raw + 3 * (int64_t)idx[i - 1];
            double s2 = 0;
            for (int k = 0; k < 3; ++k) {
                const double d = __dsub_rn(a[k], b[k]);
                s2 = __dadd_rn(s2, __dmul_rn(d, d));
            }
            if (__dsqrt_rn(s2) < 1.0e-6) f = 0;
        }
        flag[i] = f;
    }
}

// 4b. node numbers of the raw nodes and coordinates of the merged nodes
__global__ void k_merge_scatter(int64_t n, const int32_t *__restrict__ idx, const int32_t *__restrict__ flag,
                                const int64_t *__restrict__ excl, const double *__restrict__ raw,
                                int32_t *__restrict__ elements, double *__restrict__ nodes) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = excl[i] + flag[i] - 1;
        const int32_t r = idx[i];
        elements[r] = (int32_t)g;
        if (flag[i])
            for (int k = 0; k < 3; ++k) nodes[3 * g + k] = raw[3 * (int64_t)r + k];
    }
}

struct Scratch {
    yg_context ctx;
    std::vector<void *> held;
    template <typename T>
    yg_status get(T **p, size_t n) {
        YG_TRY(dev_alloc_t(ctx, p, n));
        held.push_back(*p);
        return YG_OK;
    }
    ~Scratch() {
        for (void *p : held) dev_free(ctx, p);
    }
};

yg_status scan_counts(yg_context ctx, Scratch &S, const int32_t *in, int64_t n, int64_t *out) {
    const int64_t nb = std::max<int64_t>(1, (n + 1023) / 1024);
    int64_t *sums = nullptr;
    YG_TRY(S.get(&sums, nb + 1));
    k_scan_a<<<nb, 1024, 0, ctx->stream>>>(in, n, out, sums);
    YG_LAUNCHED(ctx);
    k_scan_b<<<1, 1024, 0, ctx->stream>>>(sums, nb);
    YG_LAUNCHED(ctx);
    k_scan_c<<<nb, 1024, 0, ctx->stream>>>(out, n, sums);
    YG_LAUNCHED(ctx);
    YG_CUDA(cudaMemcpyAsync(out + n, sums + nb, sizeof(int64_t), cudaMemcpyDeviceToDevice, ctx->stream));
    return YG_OK;
}

// Structured box: node (i, j, k) at (i dx, j dy, k dz), the last one of each
// direction at exactly (lx, ly, lz) (numpy.linspace's values); nodes x fastest.
__global__ void k_box_nodes(int64_t nnodes, int nx, int ny, int nz, double dx, double dy, double dz, double lx,
                            double ly, double lz, double *__restrict__ xyz) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nnodes; v += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % (nx + 1)), j = (int)((v / (nx + 1)) % (ny + 1)), k = (int)(v / ((int64_t)(nx + 1) * (ny + 1)));
        xyz[3 * v + 0] = i == nx ? lx : __dmul_rn((double)i, dx);
        xyz[3 * v + 1] = j == ny ? ly : __dmul_rn((double)j, dy);
        xyz[3 * v + 2] = nz == 0 ? 0.0 : (k == nz ? lz : __dmul_rn((double)k, dz));
    }
}

// Cells of the box: Quad4 (nz = 0) or Hex8, in counter-clockwise corner order
// (bottom face first) or x-fastest tensor order; offsets and types alongside.
__global__ void k_box_cells(int64_t ncells, int nx, int ny, int nz, int ccw, int32_t *__restrict__ cn,
                            int32_t *__restrict__ off, int32_t *__restrict__ type) {
    const int nc = nz == 0 ? 4 : 8;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells; c += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = nz == 0 ? 0 : (int)(c / ((int64_t)nx * ny));
        const int32_t sx = 1, sy = nx + 1, sz = (nx + 1) * (ny + 1);
        const int32_t n0 = k * sz + j * sy + i * sx;
        int32_t *o = cn + c * nc;
        if (ccw) {
            o[0] = n0; o[1] = n0 + sx; o[2] = n0 + sx + sy; o[3] = n0 + sy;
            if (nc == 8) { o[4] = n0 + sz; o[5] = n0 + sz + sx; o[6] = n0 + sz + sx + sy; o[7] = n0 + sz + sy; }
        } else {
            o[0] = n0; o[1] = n0 + sx; o[2] = n0 + sy; o[3] = n0 + sx + sy;
            if (nc == 8) { o[4] = n0 + sz; o[5] = n0 + sz + sx; o[6] = n0 + sz + sy; o[7] = n0 + sz + sx + sy; }
        }
        off[c] = (int32_t)(c * nc);
        type[c] = nc == 4 ? 3 : 4;
        if (c == ncells - 1) off[ncells] = (int32_t)(ncells * nc);
    }
}

}  // namespace

// The box mesh on the device (into caller-held arrays sized for it).
yg_status generate_box(yg_context ctx, int dim, int nx, int ny, int nz, double lx, double ly, double lz, bool ccw,
                       double *xyz, int32_t *cell_nodes, int32_t *cell_offsets, int32_t *cell_types) {
    const int64_t nnodes = (int64_t)(nx + 1) * (ny + 1) * (dim == 3 ? nz + 1 : 1);
    const int64_t ncells = (int64_t)nx * ny * (dim == 3 ? nz : 1);
    k_box_nodes<<<stream_grid(ctx, nnodes), kThreads, 0, ctx->stream>>>(
        nnodes, nx, ny, dim == 3 ? nz : 0, lx / nx, ly / ny, dim == 3 ? lz / nz : 0.0, lx, ly, lz, xyz);
    YG_LAUNCHED(ctx);
    k_box_cells<<<stream_grid(ctx, ncells), kThreads, 0, ctx->stream>>>(ncells, nx, ny, dim == 3 ? nz : 0, ccw ? 1 : 0,
                                                                       cell_nodes, cell_offsets, cell_types);
    YG_LAUNCHED(ctx);
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

yg_status number_on_device(yg_context ctx, const double *xyz, int32_t n_nodes, const int32_t *cell_nodes,
                           const int32_t *cell_offsets, const int32_t *cell_types, int32_t n_cells,
                           const RawLayout &lay, int64_t N, HostDofmap &d, double **d_nodes_out,
                           int32_t **d_elements_out, bool device_mesh) {
    *d_nodes_out = nullptr;
    *d_elements_out = nullptr;
    cudaStream_t st = ctx->stream;
    Scratch S{ctx, {}};
    // tables of the element types present, and each cell's table
    std::vector<double> tabs;
    std::vector<int32_t> tab_start, tab_of_cell(n_cells, -1);
    int tab_id[3][4];
    for (int t = 0; t < 3; ++t)
        for (int k = 0; k < 4; ++k) {
            tab_id[t][k] = -1;
            if (lay.nloc[t][k]) {
                tab_id[t][k] = (int)tab_start.size();
                tab_start.push_back((int32_t)(tabs.size() / 3));
                tabs.insert(tabs.end(), lay.loc[t][k].begin(), lay.loc[t][k].end());
            }
        }
    for (int32_t c = 0; c < n_cells; ++c)
        if (d.topology[c] != TOPO_NONE) tab_of_cell[c] = tab_id[d.topology[c]][d.topo_dim[c]];
    const double *dxyz;
    const int32_t *dcoff, *dcn, *dct;
    double *dtabs, *raw, *dnodes = nullptr;
    int32_t *droff, *dtoc, *dts, *delem = nullptr;
    if (device_mesh) {  // the mesh arrays are already on the device
        dxyz = xyz;
        dcoff = cell_offsets;
        dcn = cell_nodes;
        dct = cell_types;
    } else {
        const int64_t ncn = cell_offsets[n_cells];
        double *ux;
        int32_t *uo, *un, *ut;
        YG_TRY(S.get(&ux, 3 * (size_t)n_nodes + 1));
        YG_TRY(S.get(&uo, (size_t)n_cells + 1));
        YG_TRY(S.get(&un, (size_t)ncn + 1));
        YG_TRY(S.get(&ut, (size_t)n_cells + 1));
        YG_CUDA(cudaMemcpyAsync(ux, xyz, sizeof(double) * 3 * n_nodes, cudaMemcpyHostToDevice, st));
        YG_CUDA(cudaMemcpyAsync(uo, cell_offsets, sizeof(int32_t) * (n_cells + 1), cudaMemcpyHostToDevice, st));
        YG_CUDA(cudaMemcpyAsync(un, cell_nodes, sizeof(int32_t) * ncn, cudaMemcpyHostToDevice, st));
        YG_CUDA(cudaMemcpyAsync(ut, cell_types, sizeof(int32_t) * n_cells, cudaMemcpyHostToDevice, st));
        dxyz = ux;
        dcoff = uo;
        dcn = un;
        dct = ut;
    }
    YG_TRY(S.get(&droff, (size_t)n_cells + 1));
    YG_TRY(S.get(&dtoc, (size_t)n_cells + 1));
    YG_TRY(S.get(&dts, tab_start.size() + 1));
    YG_TRY(S.get(&dtabs, tabs.size() + 1));
    YG_TRY(S.get(&raw, 3 * (size_t)N));
    YG_CUDA(cudaMemcpyAsync(droff, d.offsets.data(), sizeof(int32_t) * (n_cells + 1), cudaMemcpyHostToDevice, st));
    YG_CUDA(cudaMemcpyAsync(dtoc, tab_of_cell.data(), sizeof(int32_t) * n_cells, cudaMemcpyHostToDevice, st));
    YG_CUDA(cudaMemcpyAsync(dts, tab_start.data(), sizeof(int32_t) * tab_start.size(), cudaMemcpyHostToDevice, st));
    YG_CUDA(cudaMemcpyAsync(dtabs, tabs.data(), sizeof(double) * tabs.size(), cudaMemcpyHostToDevice, st));
    const int grid = ctx->num_sms * 8;
    k_raw_nodes<<<grid, 256, 0, st>>>(n_cells, dcoff, dcn, dct, dxyz, droff, dtoc, dtabs, dts, raw);
    YG_LAUNCHED(ctx);
    // bounding box and snap
    const int rb = std::min<int64_t>(ctx->num_sms * 4, std::max<int64_t>(1, (N + kSortThreads - 1) / kSortThreads));
    double *dbox;
    long long *dkr;
    YG_TRY(S.get(&dbox, 6 * (size_t)rb));
    YG_TRY(S.get(&dkr, 6 * (size_t)rb));
    k_bbox<<<rb, kSortThreads, 0, st>>>(N, raw, dbox);
    YG_LAUNCHED(ctx);
    std::vector<double> hbox(6 * (size_t)rb);
    YG_CUDA(cudaMemcpyAsync(hbox.data(), dbox, sizeof(double) * hbox.size(), cudaMemcpyDeviceToHost, st));
    YG_CUDA(cudaStreamSynchronize(st));
    double bmin[3], bmax[3];
    for (int k = 0; k < 3; ++k) {
        bmin[k] = hbox[k];
        bmax[k] = hbox[3 + k];
        for (int b = 1; b < rb; ++b) {
            bmin[k] = std::min(bmin[k], hbox[6 * b + k]);
            bmax[k] = std::max(bmax[k], hbox[6 * b + 3 + k]);
        }
    }
    const double max_dim = std::max(bmax[0] - bmin[0], std::max(bmax[1] - bmin[1], bmax[2] - bmin[2]));
    const double snapv = max_dim * 1.0e-6;
    if (!(snapv > 0)) return fail(YG_UNSUPPORTED, "device numbering: degenerate bounding box");
    const double inv = 1.0 / snapv;
    k_key_range<<<rb, kSortThreads, 0, st>>>(N, raw, inv, dkr);
    YG_LAUNCHED(ctx);
    std::vector<long long> hkr(6 * (size_t)rb);
    YG_CUDA(cudaMemcpyAsync(hkr.data(), dkr, sizeof(long long) * hkr.size(), cudaMemcpyDeviceToHost, st));
    YG_CUDA(cudaStreamSynchronize(st));
    long long kmin[3], kmax[3];
    int bits[3];
    for (int k = 0; k < 3; ++k) {
        kmin[k] = hkr[k];
        kmax[k] = hkr[3 + k];
        for (int b = 1; b < rb; ++b) {
            kmin[k] = std::min(kmin[k], hkr[6 * b + k]);
            kmax[k] = std::max(kmax[k], hkr[6 * b + 3 + k]);
        }
        const uint64_t span = (uint64_t)(kmax[k] - kmin[k]);
        bits[k] = 0;
        while (bits[k] < 63 && (span >> bits[k]) != 0) ++bits[k];
    }
    const int nbits = bits[0] + bits[1] + bits[2];
    if (nbits > 64) return fail(YG_UNSUPPORTED, "device numbering: keys need %d bits", nbits);
    // keys and the radix sort
    uint64_t *ka, *kb;
    int32_t *va, *vb, *hist;
    int64_t *offs;
    const int64_t ntiles = (N + kTile - 1) / kTile;
    YG_TRY(S.get(&ka, (size_t)N));
    YG_TRY(S.get(&kb, (size_t)N));
    YG_TRY(S.get(&va, (size_t)N));
    YG_TRY(S.get(&vb, (size_t)N));
    YG_TRY(S.get(&hist, 256 * (size_t)ntiles));
    YG_TRY(S.get(&offs, 256 * (size_t)ntiles + 1));
    k_pack_keys<<<stream_grid(ctx, N), kThreads, 0, st>>>(N, raw, inv, kmin[0], kmin[1], kmin[2], bits[0], bits[1],
                                                         ka, va);
    YG_LAUNCHED(ctx);
    for (int shift = 0; shift < nbits; shift += 8) {
        k_radix_hist<<<ntiles, kSortThreads, 0, st>>>(N, ka, shift, ntiles, hist);
        YG_LAUNCHED(ctx);
        YG_TRY(scan_counts(ctx, S, hist, 256 * ntiles, offs));
        k_radix_scatter<<<ntiles, kSortThreads, 0, st>>>(N, ka, va, shift, ntiles, offs, kb, vb);
        YG_LAUNCHED(ctx);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    // merge
    int32_t *flag;
    int64_t *excl;
    YG_TRY(S.get(&flag, (size_t)N));
    YG_TRY(S.get(&excl, (size_t)N + 1));
    k_merge_flags<<<stream_grid(ctx, N), kThreads, 0, st>>>(N, va, raw, flag);
    YG_LAUNCHED(ctx);
    YG_TRY(scan_counts(ctx, S, flag, N, excl));
    int64_t ngroups = 0;
    YG_CUDA(cudaMemcpyAsync(&ngroups, excl + N, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    YG_CUDA(cudaStreamSynchronize(st));
    YG_TRY(dev_alloc_t(ctx, &dnodes, 3 * (size_t)ngroups + 1));
    yg_status s = dev_alloc_t(ctx, &delem, (size_t)N + 1);
    if (s != YG_OK) { dev_free(ctx, dnodes); return s; }
    k_merge_scatter<<<stream_grid(ctx, N), kThreads, 0, st>>>(N, va, flag, excl, raw, delem, dnodes);
    YG_LAUNCHED(ctx);
    d.nodes.resize(3 * (size_t)ngroups);
    d.elements.resize((size_t)N);
    cudaError_t e = cudaMemcpyAsync(d.nodes.data(), dnodes, sizeof(double) * 3 * ngroups, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d.elements.data(), delem, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        dev_free(ctx, dnodes);
        dev_free(ctx, delem);
        return fail(YG_CUDA_ERROR, "device numbering: %s", cudaGetErrorString(e));
    }
    *d_nodes_out = dnodes;
    *d_elements_out = delem;
    return YG_OK;
}

}  // namespace yg
