// assembly.cu -- DoF map handle, sparsity pattern, element assembly and
// Dirichlet conditions on the GPU.
//
// Replaces CGAssembly<Physics> (include/assembly/CGAssembly.hpp:27-186),
// Element::update (include/element/Element.hpp:109-149), the Physics callbacks
// of apps/BasicPoisson/main.cpp:25-61, apps/BasicLinearElasticity/main.cpp:41-113
// and apps/supg_learning/supg_advection.hpp:19-132, and DirichletBC::apply
// (src/boundary_conditions/DirichletBC.cpp:27-89).
//
// Pattern: the node graph (node -> nodes of its incident cells) is built on the
// GPU: incidence counts and lists, then a warp per node gathers the candidate
// columns into shared memory, bitonic-sorts and de-duplicates them (a count
// pass, an exclusive scan, a fill pass).  The matrix is that graph with
// dof_per_node x dof_per_node blocks (BCSR) or its scalar expansion (CSR); both
// equal the reference's pattern, which holds every (nen*dpn)^2 element entry
// (CGAssembly.hpp:149-156).
//
// Values: cells are coloured on the host so that cells of one colour share no
// node; one launch per colour, one CTA per cell.  The CTA computes the Jacobian,
// jxw and physical gradients of every quadrature point into shared memory, then
// each thread owns node pairs (A,B) of the element matrix, accumulates their
// dpn x dpn blocks over the quadrature points in registers and adds them into
// the global values (binary search of the column in the row).  No floating-point
// atomics: colours in ascending order fix the summation order, so assembly is
// deterministic.
#include "internal.h"
#include "device_common.cuh"
#include "host_fe.h"

#include <algorithm>
#include <cmath>
#include <memory>

namespace yg {
int stream_grid(yg_context ctx, int64_t n);
}

struct ElementGroup {
    int topology = 0;
    yg::ElementTable tab;
    double *d_tab = nullptr;        // N (nq*nen) | dN (nq*nen*dim) | w (nq)
    int32_t *d_order = nullptr;     // cells sorted by colour
    std::vector<int32_t> color_ptr; // colour c -> [color_ptr[c], color_ptr[c+1])
};

struct yg_dofmap_t {
    yg_context ctx = nullptr;
    yg::HostDofmap host;
    double *d_nodes = nullptr;
    int32_t *d_offsets = nullptr;
    int32_t *d_elements = nullptr;
    // node graph for one simulation dimension
    int pattern_nsd = -1;
    int32_t *d_nrowptr = nullptr;
    int32_t *d_ncol = nullptr;
    int64_t nnz_nodes = 0;
    std::vector<ElementGroup> groups;
};

namespace yg {

// ------------------------------------------------------------------ scan

__global__ void __launch_bounds__(1024) k_scan_blocks(const int32_t *__restrict__ in, int64_t n, int64_t *__restrict__ out,
                                                      int64_t *__restrict__ block_sums) {
    __shared__ int64_t sm[1024];
    int64_t i = blockIdx.x * (int64_t)1024 + threadIdx.x;
    int64_t v = i < n ? in[i] : 0;
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int64_t t = threadIdx.x >= o ? sm[threadIdx.x - o] : 0;
        __syncthreads();
        sm[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) out[i] = sm[threadIdx.x] - v;  // exclusive
    if (threadIdx.x == 1023) block_sums[blockIdx.x] = sm[1023];
}

__global__ void k_scan_sums(int64_t *__restrict__ sums, int64_t nb) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int64_t acc = 0;
        for (int64_t b = 0; b < nb; ++b) { int64_t t = sums[b]; sums[b] = acc; acc += t; }
        sums[nb] = acc;
    }
}

__global__ void k_scan_add(int64_t *__restrict__ out, int64_t n, const int64_t *__restrict__ sums) {
    int64_t i = blockIdx.x * (int64_t)1024 + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

// exclusive scan of n int32 counts into n+1 int64 offsets (last = total)
static yg_status exclusive_scan(yg_context ctx, const int32_t *in, int64_t n, int64_t *out, int64_t *total) {
    int64_t nb = (n + 1023) / 1024;
    if (nb < 1) nb = 1;
    int64_t *sums = nullptr;
    YG_TRY(dev_alloc_t(ctx, &sums, nb + 1));
    k_scan_blocks<<<nb, 1024, 0, ctx->stream>>>(in, n, out, sums);
    YG_LAUNCHED(ctx);
    k_scan_sums<<<1, 32, 0, ctx->stream>>>(sums, nb);
    YG_LAUNCHED(ctx);
    k_scan_add<<<nb, 1024, 0, ctx->stream>>>(out, n, sums);
    YG_LAUNCHED(ctx);
    cudaMemcpyAsync(out + n, sums + nb, sizeof(int64_t), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(total, sums + nb, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, sums);
    if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "scan: %s", cudaGetErrorString(e));
    return YG_OK;
}

// ------------------------------------------------------------------ pattern

__global__ void k_incidence_count(int32_t ncells, const int32_t *__restrict__ off, const int32_t *__restrict__ el,
                                  const int8_t *__restrict__ include, int32_t *__restrict__ cnt) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells; c += (int64_t)gridDim.x * blockDim.x) {
        if (!include[c]) continue;
        for (int i = off[c]; i < off[c + 1]; ++i) atomicAdd(&cnt[el[i]], 1);
    }
}

__global__ void k_incidence_fill(int32_t ncells, const int32_t *__restrict__ off, const int32_t *__restrict__ el,
                                 const int8_t *__restrict__ include, const int64_t *__restrict__ ptr,
                                 int32_t *__restrict__ cursor, int32_t *__restrict__ adj) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells; c += (int64_t)gridDim.x * blockDim.x) {
        if (!include[c]) continue;
        for (int i = off[c]; i < off[c + 1]; ++i) {
            int32_t n = el[i];
            int32_t k = atomicAdd(&cursor[n], 1);
            adj[ptr[n] + k] = (int32_t)c;
        }
    }
}

constexpr int kRowCap = 1024;        // candidate columns per node row
constexpr int kRowWarps = 4;         // warps per block in the row kernels

// Gather, sort and de-duplicate the neighbour nodes of `node` into buf (shared
// memory, kRowCap ints).  Returns the number of unique neighbours (or -1 if the
// candidate list overflows the buffer).
__device__ int row_unique(int node, const int64_t *__restrict__ aptr, const int32_t *__restrict__ adj,
                          const int32_t *__restrict__ off, const int32_t *__restrict__ el, int32_t *buf) {
    const int lane = threadIdx.x & 31;
    int cnt = 0;
    for (int64_t a = aptr[node]; a < aptr[node + 1]; ++a) {
        int c = adj[a];
        int b = off[c], e = off[c + 1];
        if (cnt + (e - b) > kRowCap) return -1;
        for (int i = b + lane; i < e; i += 32) buf[cnt + i - b] = el[i];
        cnt += e - b;
    }
    int P = 32;
    while (P < cnt) P <<= 1;
    for (int i = cnt + lane; i < P; i += 32) buf[i] = INT32_MAX;
    __syncwarp();
    // bitonic sort of P entries by one warp
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += 32) {
                int ixj = i ^ j;
                if (ixj > i) {
                    int a = buf[i], b = buf[ixj];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) { buf[i] = b; buf[ixj] = a; }
                }
            }
            __syncwarp();
        }
    }
    // unique count
    int u = 0;
    for (int i0 = 0; i0 < cnt; i0 += 32) {
        int i = i0 + lane;
        bool keep = i < cnt && (i == 0 || buf[i] != buf[i - 1]);
        u += __popc(__ballot_sync(0xffffffffu, keep));
    }
    return u;
}

__global__ void __launch_bounds__(kRowWarps * 32)
k_row_count(int32_t nnodes, const int64_t *__restrict__ aptr, const int32_t *__restrict__ adj,
            const int32_t *__restrict__ off, const int32_t *__restrict__ el, int32_t *__restrict__ rowcnt,
            int32_t *__restrict__ overflow) {
    __shared__ int32_t sbuf[kRowWarps][kRowCap];
    const int w = threadIdx.x >> 5;
    for (int64_t node = blockIdx.x * (int64_t)kRowWarps + w; node < nnodes; node += (int64_t)gridDim.x * kRowWarps) {
        int u = row_unique((int)node, aptr, adj, off, el, sbuf[w]);
        if ((threadIdx.x & 31) == 0) {
            rowcnt[node] = u < 0 ? 0 : u;
            if (u < 0) atomicExch(overflow, 1);
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kRowWarps * 32)
k_row_fill(int32_t nnodes, const int64_t *__restrict__ aptr, const int32_t *__restrict__ adj,
           const int32_t *__restrict__ off, const int32_t *__restrict__ el, const int64_t *__restrict__ rowptr64,
           int32_t *__restrict__ rowptr, int32_t *__restrict__ col) {
    __shared__ int32_t sbuf[kRowWarps][kRowCap];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t node = blockIdx.x * (int64_t)kRowWarps + w; node < nnodes; node += (int64_t)gridDim.x * kRowWarps) {
        int32_t *buf = sbuf[w];
        int u = row_unique((int)node, aptr, adj, off, el, buf);
        int cnt = 0;
        for (int64_t a = aptr[node]; a < aptr[node + 1]; ++a) cnt += off[adj[a] + 1] - off[adj[a]];
        int64_t base = rowptr64[node];
        if (lane == 0) rowptr[node] = (int32_t)base;
        int written = 0;
        for (int i0 = 0; i0 < cnt && u >= 0; i0 += 32) {
            int i = i0 + lane;
            bool keep = i < cnt && (i == 0 || buf[i] != buf[i - 1]);
            unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep) col[base + written + __popc(m & ((1u << lane) - 1))] = buf[i];
            written += __popc(m);
        }
        __syncwarp();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) rowptr[nnodes] = (int32_t)rowptr64[nnodes];
}

// Scalar CSR (and row pointer) from the node graph and dof_per_node.
__global__ void k_expand_pattern(int64_t nnodes, int D, const int32_t *__restrict__ nrp, const int32_t *__restrict__ ncol,
                                 int32_t *__restrict__ rp, int32_t *__restrict__ col) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nnodes * D; r += (int64_t)gridDim.x * blockDim.x) {
        int64_t I = r / D, i = r % D;
        int32_t len = nrp[I + 1] - nrp[I];
        int32_t pos = nrp[I] * D * D + (int32_t)i * len * D;
        rp[r] = pos;
        for (int32_t k = nrp[I]; k < nrp[I + 1]; ++k)
            for (int j = 0; j < D; ++j) col[pos++] = ncol[k] * D + j;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) rp[nnodes * D] = nrp[nnodes] * D * D;
}

// ------------------------------------------------------------------ element kernels

struct PhysParams {
    double p[8];
    double Kd[9];     // SUPG diffusion tensor
    double U[3];      // SUPG velocity
    double Uhat[3];   // SUPG scaled velocity for the residual
};

__device__ __forceinline__ int find_col(const int32_t *__restrict__ col, int lo, int hi, int c) {
    --hi;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int v = __ldg(col + mid);
        if (v == c) return mid;
        if (v < c) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

// Address of scalar entry (i,k) of node block (nA -> position pos in the node row).
__device__ __forceinline__ int64_t entry_addr(int format, int D, const int32_t *__restrict__ nrp, int nA, int pos, int i,
                                              int k) {
    if (format == YG_FORMAT_BCSR) return (int64_t)pos * D * D + i * D + k;
    int32_t rs = nrp[nA], len = nrp[nA + 1] - rs;
    return (int64_t)rs * D * D + (int64_t)i * len * D + (int64_t)(pos - rs) * D + k;
}

template <int NSD, int DPN, int PHYS>
__global__ void __launch_bounds__(128)
k_assemble(const int32_t *__restrict__ order, int ncell, const int32_t *__restrict__ off,
           const int32_t *__restrict__ el, const double *__restrict__ nodes, const double *__restrict__ tab, int nen,
           int nq, int tdim, PhysParams prm, const int32_t *__restrict__ nrp, const int32_t *__restrict__ ncol,
           double *__restrict__ val, int format, double *__restrict__ residual, int want_K, int want_R) {
    extern __shared__ double sm[];
    double *xe = sm;                       // nen*3
    double *G = xe + 3 * nen;              // nq*nen*NSD
    double *jxw = G + (size_t)nq * nen * NSD;  // nq
    double *Ji = jxw + nq;                 // nq*9
    int32_t *gn = reinterpret_cast<int32_t *>(Ji + 9 * nq);  // nen
    const double *tN = tab;
    const double *tdN = tab + (size_t)nq * nen;
    const double *tw = tdN + (size_t)nq * nen * tdim;
    constexpr bool SYM = (PHYS != YG_SUPG);

    for (int t = blockIdx.x; t < ncell; t += gridDim.x) {
        const int c = order[t];
        const int base = off[c];
        for (int a = threadIdx.x; a < nen; a += blockDim.x) {
            int n = el[base + a];
            gn[a] = n;
            xe[3 * a + 0] = nodes[3 * (int64_t)n + 0];
            xe[3 * a + 1] = nodes[3 * (int64_t)n + 1];
            xe[3 * a + 2] = nodes[3 * (int64_t)n + 2];
        }
        __syncthreads();
        // Element::update: Jacobian, det, inverse per quadrature point
        for (int q = threadIdx.x; q < nq; q += blockDim.x) {
            double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int A = 0; A < nen; ++A) {
                const double *d = tdN + ((size_t)q * nen + A) * tdim;
#pragma unroll
                for (int i = 0; i < NSD; ++i)
#pragma unroll
                    for (int j = 0; j < NSD; ++j) J[i][j] += xe[3 * A + i] * d[j];
            }
            double det, inv[3][3];
            if (NSD == 1) {
                det = J[0][0];
                inv[0][0] = 1.0 / J[0][0];
            } else if (NSD == 2) {
                det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
                double di = 1.0 / det;
                inv[0][0] = J[1][1] * di; inv[1][1] = J[0][0] * di;
                inv[0][1] = -J[0][1] * di; inv[1][0] = -J[1][0] * di;
            } else {
                det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[2][0] * J[1][2]) +
                      J[0][2] * (J[1][0] * J[2][1] - J[2][0] * J[1][1]);
                double di = 1.0 / det;
                inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * di;
                inv[0][1] = -(J[0][1] * J[2][2] - J[2][1] * J[0][2]) * di;
                inv[0][2] = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * di;
                inv[1][0] = -(J[1][0] * J[2][2] - J[2][0] * J[1][2]) * di;
                inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * di;
                inv[1][2] = -(J[0][0] * J[1][2] - J[1][0] * J[0][2]) * di;
                inv[2][0] = (J[1][0] * J[2][1] - J[2][0] * J[1][1]) * di;
                inv[2][1] = -(J[0][0] * J[2][1] - J[2][0] * J[0][1]) * di;
                inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * di;
            }
            jxw[q] = det * tw[q];
#pragma unroll
            for (int i = 0; i < NSD; ++i)
#pragma unroll
                for (int j = 0; j < NSD; ++j) Ji[9 * q + 3 * i + j] = inv[i][j];
        }
        __syncthreads();
        // physical gradients dN/dx_d = sum_j Jinv(j,d) dN/dxi_j
        for (int idx = threadIdx.x; idx < nq * nen; idx += blockDim.x) {
            const int q = idx / nen;
            const double *d = tdN + (size_t)idx * tdim;
#pragma unroll
            for (int dd = 0; dd < NSD; ++dd) {
                double s = 0;
#pragma unroll
                for (int j = 0; j < NSD; ++j) s += Ji[9 * q + 3 * j + dd] * d[j];
                G[(size_t)idx * NSD + dd] = s;
            }
        }
        __syncthreads();
        if (want_K) {
            const int npairs = SYM ? nen * (nen + 1) / 2 : nen * nen;
            for (int pr = threadIdx.x; pr < npairs; pr += blockDim.x) {
                int A, B;
                if (SYM) {  // pr -> (A <= B), row-major over the upper triangle
                    A = 0;
                    int rem = pr;
                    while (rem >= nen - A) { rem -= nen - A; ++A; }
                    B = A + rem;
                } else {
                    A = pr / nen;
                    B = pr % nen;
                }
                double K[DPN][DPN];
#pragma unroll
                for (int i = 0; i < DPN; ++i)
#pragma unroll
                    for (int k = 0; k < DPN; ++k) K[i][k] = 0;
                for (int q = 0; q < nq; ++q) {
                    const double *gA = G + ((size_t)q * nen + A) * NSD;
                    const double *gB = G + ((size_t)q * nen + B) * NSD;
                    const double w = jxw[q];
                    if (PHYS == YG_POISSON) {
                        double dt = 0;
#pragma unroll
                        for (int d = 0; d < NSD; ++d) dt += gA[d] * gB[d];
                        K[0][0] += prm.p[0] * (dt * w);
                    } else if (PHYS == YG_ELASTICITY) {
                        double a[NSD], b[NSD], dt = 0;
#pragma unroll
                        for (int d = 0; d < NSD; ++d) { a[d] = gA[d]; b[d] = gB[d]; dt += a[d] * b[d]; }
                        const double sw = prm.p[0] * w, lam = prm.p[1], mu = prm.p[2];
#pragma unroll
                        for (int i = 0; i < NSD; ++i)
#pragma unroll
                            for (int k = 0; k < NSD; ++k)
                                K[i][k] += sw * (lam * a[i] * b[k] + mu * ((i == k ? dt : 0.0) + a[k] * b[i]));
                    } else {  // SUPG: advection summed NSD times, as the reference does
                        const double NA = tN[(size_t)q * nen + A];
                        double s = 0;
#pragma unroll
                        for (int ac = 0; ac < NSD; ++ac)
#pragma unroll
                            for (int bc = 0; bc < NSD; ++bc)
                                s += NA * prm.U[bc] * gB[bc] + gA[ac] * gB[bc] * prm.Kd[3 * ac + bc];
                        K[0][0] += s * w;
                    }
                }
                const int nA = gn[A], nB = gn[B];
                int rs = __ldg(nrp + nA), re = __ldg(nrp + nA + 1);
                int pos = find_col(ncol, rs, re, nB);
                if (pos >= 0) {
#pragma unroll
                    for (int i = 0; i < DPN; ++i)
#pragma unroll
                        for (int k = 0; k < DPN; ++k) val[entry_addr(format, DPN, nrp, nA, pos, i, k)] += K[i][k];
                }
                if (SYM && A != B) {
                    rs = __ldg(nrp + nB);
                    re = __ldg(nrp + nB + 1);
                    pos = find_col(ncol, rs, re, nA);
                    if (pos >= 0) {
#pragma unroll
                        for (int i = 0; i < DPN; ++i)
#pragma unroll
                            for (int k = 0; k < DPN; ++k) val[entry_addr(format, DPN, nrp, nB, pos, k, i)] += K[i][k];
                    }
                }
            }
        }
        if (want_R) {
            for (int a = threadIdx.x; a < nen * DPN; a += blockDim.x) {
                const int A = a / DPN, comp = a % DPN;
                double R = 0;
                for (int q = 0; q < nq; ++q) {
                    const double NA = tN[(size_t)q * nen + A];
                    if (PHYS == YG_POISSON) {
                        R += (prm.p[1] * jxw[q]) * NA;
                    } else if (PHYS == YG_ELASTICITY) {
                        R += prm.p[3 + comp] * NA * jxw[q];
                    } else {
                        const double *gA = G + ((size_t)q * nen + A) * NSD;
#pragma unroll
                        for (int ac = 0; ac < NSD; ++ac) R -= (NA * prm.p[3] + prm.Uhat[ac] * gA[ac]) * jxw[q];
                    }
                }
                residual[(int64_t)gn[A] * DPN + comp] += R;
            }
        }
        __syncthreads();
    }
}

static size_t assemble_smem(int nen, int nq, int nsd) {
    return sizeof(double) * (3 * nen + (size_t)nq * nen * nsd + nq + 9 * nq) + sizeof(int32_t) * nen + 16;
}

template <int NSD, int DPN, int PHYS>
static yg_status launch_assemble(yg_context ctx, const ElementGroup &g, yg_dofmap d, const PhysParams &prm, double *val,
                                 int format, double *residual, int want_K, int want_R) {
    const int nen = g.tab.nen, nq = g.tab.nq;
    size_t smem = assemble_smem(nen, nq, NSD);
    auto kern = k_assemble<NSD, DPN, PHYS>;
    if (smem > ctx->smem_optin)
        return fail(YG_UNSUPPORTED, "CGAssembly: element (nen %d, nq %d) needs %zu B of shared memory, the device "
                    "allows %zu", nen, nq, smem, ctx->smem_optin);
    if (smem > 48 * 1024) YG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (size_t c = 0; c + 1 < g.color_ptr.size(); ++c) {
        int n = g.color_ptr[c + 1] - g.color_ptr[c];
        if (n == 0) continue;
        int grid = std::min(n, ctx->num_sms * 16);
        kern<<<grid, 128, smem, ctx->stream>>>(g.d_order + g.color_ptr[c], n, d->d_offsets, d->d_elements, d->d_nodes,
                                               g.d_tab, nen, nq, g.tab.dim, prm, d->d_nrowptr, d->d_ncol, val, format,
                                               residual, want_K, want_R);
        YG_LAUNCHED(ctx);
    }
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

template <int NSD>
static yg_status dispatch_physics(yg_context ctx, const ElementGroup &g, yg_dofmap d, int kind, int dpn,
                                  const PhysParams &prm, double *val, int format, double *residual, int wK, int wR) {
    if (kind == YG_POISSON && dpn == 1) return launch_assemble<NSD, 1, YG_POISSON>(ctx, g, d, prm, val, format, residual, wK, wR);
    if (kind == YG_SUPG && dpn == 1) return launch_assemble<NSD, 1, YG_SUPG>(ctx, g, d, prm, val, format, residual, wK, wR);
    if (kind == YG_ELASTICITY && dpn == NSD) return launch_assemble<NSD, NSD, YG_ELASTICITY>(ctx, g, d, prm, val, format, residual, wK, wR);
    return fail(YG_BAD_ARG, "physics %d needs dof_per_node %d (got %d)", kind, kind == YG_ELASTICITY ? NSD : 1, dpn);
}

// Node graph + element groups for simulation dimension nsd.
static yg_status build_pattern(yg_dofmap d, int nsd) {
    if (d->pattern_nsd == nsd) return YG_OK;
    yg_context ctx = d->ctx;
    dev_free(ctx, d->d_nrowptr);
    dev_free(ctx, d->d_ncol);
    for (auto &g : d->groups) { dev_free(ctx, g.d_tab); dev_free(ctx, g.d_order); }
    d->groups.clear();
    d->d_nrowptr = d->d_ncol = nullptr;
    const HostDofmap &h = d->host;
    const int32_t nc = h.n_cells(), nn = h.n_nodes();
    // element groups (one per topology present) with colourings
    for (int topo : {TOPO_TENSOR, TOPO_SIMPLEX}) {
        bool present = false;
        for (int32_t c = 0; c < nc && !present; ++c) present = (h.topo_dim[c] == nsd && h.topology[c] == topo);
        if (!present) continue;
        ElementGroup g;
        g.topology = topo;
        if (!make_element_table(topo, nsd, h.poly_order, g.tab))
            return fail(YG_UNSUPPORTED, "element (topology %d, dim %d, order %d) not supported", topo, nsd, h.poly_order);
        std::vector<int32_t> order;
        int ncol = color_cells(h, nsd, topo, order, g.color_ptr);
        if (ncol < 0) return fail(YG_UNSUPPORTED, "element colouring needs more than 64 colours");
        std::vector<double> tab;
        tab.insert(tab.end(), g.tab.N.begin(), g.tab.N.end());
        tab.insert(tab.end(), g.tab.dN.begin(), g.tab.dN.end());
        tab.insert(tab.end(), g.tab.qw.begin(), g.tab.qw.end());
        YG_TRY(dev_alloc_t(ctx, &g.d_tab, tab.size()));
        YG_TRY(dev_alloc_t(ctx, &g.d_order, order.size() + 1));
        YG_CUDA(cudaMemcpy(g.d_tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
        YG_CUDA(cudaMemcpy(g.d_order, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice));
        d->groups.push_back(std::move(g));
    }
    // incidence lists of the included cells
    std::vector<int8_t> include(nc);
    for (int32_t c = 0; c < nc; ++c) include[c] = (h.topo_dim[c] == nsd && h.topology[c] != TOPO_NONE);
    int8_t *d_inc = nullptr;
    int32_t *d_cnt = nullptr, *d_cursor = nullptr, *d_adj = nullptr, *d_rowcnt = nullptr, *d_flag = nullptr;
    int64_t *d_aptr = nullptr, *d_rp64 = nullptr;
    auto cleanup = [&]() {
        dev_free(ctx, d_inc); dev_free(ctx, d_cnt); dev_free(ctx, d_cursor); dev_free(ctx, d_adj);
        dev_free(ctx, d_rowcnt); dev_free(ctx, d_flag); dev_free(ctx, d_aptr); dev_free(ctx, d_rp64);
    };
    yg_status s;
#define TRYC(x) do { s = (x); if (s != YG_OK) { cleanup(); return s; } } while (0)
    TRYC(dev_alloc_t(ctx, &d_inc, nc + 1));
    TRYC(dev_alloc_t(ctx, &d_cnt, nn + 1));
    TRYC(dev_alloc_t(ctx, &d_cursor, nn + 1));
    TRYC(dev_alloc_t(ctx, &d_aptr, nn + 1));
    TRYC(dev_alloc_t(ctx, &d_flag, 1));
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(d_inc, include.data(), nc, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (nn + 1), st);
    cudaMemsetAsync(d_cursor, 0, sizeof(int32_t) * (nn + 1), st);
    cudaMemsetAsync(d_flag, 0, sizeof(int32_t), st);
    k_incidence_count<<<stream_grid(ctx, nc), kThreads, 0, st>>>(nc, d->d_offsets, d->d_elements, d_inc, d_cnt);
    YG_LAUNCHED(ctx);
    int64_t total = 0;
    TRYC(exclusive_scan(ctx, d_cnt, nn, d_aptr, &total));
    TRYC(dev_alloc_t(ctx, &d_adj, total + 1));
    k_incidence_fill<<<stream_grid(ctx, nc), kThreads, 0, st>>>(nc, d->d_offsets, d->d_elements, d_inc, d_aptr,
                                                               d_cursor, d_adj);
    YG_LAUNCHED(ctx);
    // rows of the node graph
    TRYC(dev_alloc_t(ctx, &d_rowcnt, nn + 1));
    TRYC(dev_alloc_t(ctx, &d_rp64, nn + 1));
    int rgrid = (int)std::min<int64_t>((nn + kRowWarps - 1) / kRowWarps, (int64_t)ctx->num_sms * 16);
    if (rgrid < 1) rgrid = 1;
    k_row_count<<<rgrid, kRowWarps * 32, 0, st>>>(nn, d_aptr, d_adj, d->d_offsets, d->d_elements, d_rowcnt, d_flag);
    YG_LAUNCHED(ctx);
    int overflow = 0;
    cudaMemcpyAsync(&overflow, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    int64_t nnz = 0;
    TRYC(exclusive_scan(ctx, d_rowcnt, nn, d_rp64, &nnz));
    if (overflow) { cleanup(); return fail(YG_UNSUPPORTED, "a node touches more than %d element nodes", kRowCap); }
    if (nnz >= INT32_MAX) { cleanup(); return fail(YG_UNSUPPORTED, "node graph too large for 32-bit offsets"); }
    TRYC(dev_alloc_t(ctx, &d->d_nrowptr, nn + 1));
    TRYC(dev_alloc_t(ctx, &d->d_ncol, nnz + 1));
    k_row_fill<<<rgrid, kRowWarps * 32, 0, st>>>(nn, d_aptr, d_adj, d->d_offsets, d->d_elements, d_rp64, d->d_nrowptr,
                                                 d->d_ncol);
    YG_LAUNCHED(ctx);
    cudaError_t e = cudaStreamSynchronize(st);
    cleanup();
#undef TRYC
    if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "pattern build: %s", cudaGetErrorString(e));
    d->nnz_nodes = nnz;
    d->pattern_nsd = nsd;
    return YG_OK;
}

static yg_status new_matrix_from_pattern(yg_dofmap d, int format, yg_matrix *out) {
    yg_context ctx = d->ctx;
    const int D = d->host.dof_per_node;
    const int64_t nn = d->host.n_nodes();
    auto *A = new yg_matrix_t();
    A->ctx = ctx;
    A->owner = d;
    A->owner_format = format;
    yg_status s = YG_OK;
    if (format == YG_FORMAT_BCSR) {
        A->block = D;
        A->nbrows = A->nbcols = nn;
        A->nnzb = d->nnz_nodes;
        if ((s = dev_alloc_t(ctx, &A->d_rowptr, nn + 1)) == YG_OK && (s = dev_alloc_t(ctx, &A->d_col, A->nnzb + 1)) == YG_OK) {
            cudaMemcpyAsync(A->d_rowptr, d->d_nrowptr, sizeof(int32_t) * (nn + 1), cudaMemcpyDeviceToDevice, ctx->stream);
            cudaMemcpyAsync(A->d_col, d->d_ncol, sizeof(int32_t) * A->nnzb, cudaMemcpyDeviceToDevice, ctx->stream);
        }
    } else {
        A->block = 1;
        A->nbrows = A->nbcols = nn * D;
        A->nnzb = d->nnz_nodes * D * D;
        if (A->nnzb >= INT32_MAX) s = fail(YG_UNSUPPORTED, "scalar CSR too large for 32-bit offsets; use BCSR");
        if (s == YG_OK && (s = dev_alloc_t(ctx, &A->d_rowptr, nn * D + 1)) == YG_OK &&
            (s = dev_alloc_t(ctx, &A->d_col, A->nnzb + 1)) == YG_OK) {
            k_expand_pattern<<<stream_grid(ctx, nn * D), kThreads, 0, ctx->stream>>>(nn, D, d->d_nrowptr, d->d_ncol,
                                                                                    A->d_rowptr, A->d_col);
            YG_LAUNCHED(ctx);
        }
    }
    if (s == YG_OK) s = dev_alloc_t(ctx, &A->d_val, A->nnzb * A->block * A->block);
    if (s == YG_OK) s = matrix_build_diag(A);
    if (s != YG_OK) { yg_matrix_destroy(A); return s; }
    spmv_autotune(A);
    *out = A;
    return YG_OK;
}

// ------------------------------------------------------------------ Dirichlet

__global__ void k_bc_scatter(int64_t nbc, const int64_t *__restrict__ dofs, const double *__restrict__ vals,
                             uint8_t *__restrict__ mask, double *__restrict__ g) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nbc; i += (int64_t)gridDim.x * blockDim.x) {
        mask[dofs[i]] = 1;
        g[dofs[i]] = vals[i];
    }
}

__global__ void k_sub_inplace(int64_t n, double *__restrict__ rhs, const double *__restrict__ q) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        rhs[i] -= q[i];
}

// Zero BC rows and columns, unit diagonal and rhs_r = g_r on BC rows
// (DirichletBC.cpp:137-149).  One thread per scalar row.
// Zero the rows and columns of the Dirichlet dofs (mask) and put 1 on their
// diagonal with rhs = g there (DirichletBC.cpp:58-89).  One warp per block row,
// lanes over its blocks (coalesced column reads); only masked entries are written.
__global__ void k_bc_zero(int64_t nbrows, int B, const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                          double *__restrict__ val, const uint8_t *__restrict__ mask, const double *__restrict__ g,
                          double *__restrict__ rhs) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t I = warp; I < nbrows; I += nwarps) {
        int mr = 0;  // bit i: scalar row I*B+i is a Dirichlet row
        for (int i = 0; i < B; ++i) mr |= mask[I * B + i] ? (1 << i) : 0;
        const int32_t k0 = rp[I], k1 = rp[I + 1];
        for (int32_t k = k0 + lane; k < k1; k += 32) {
            const int64_t J = col[k];
            int mc = 0;
            for (int j = 0; j < B; ++j) mc |= mask[J * B + j] ? (1 << j) : 0;
            if (!mr && !mc) continue;
            for (int i = 0; i < B; ++i)
                for (int j = 0; j < B; ++j) {
                    if (!((mr >> i) & 1) && !((mc >> j) & 1)) continue;
                    const int64_t r = I * B + i, c = J * B + j;
                    double *v = &val[(int64_t)k * B * B + i * B + j];
                    if (r == c) {
                        rhs[r] = g[c];
                        *v = 1;
                    } else {
                        *v = 0;
                    }
                }
        }
    }
}

const HostDofmap &dofmap_host(yg_dofmap d) { return d->host; }

yg_status number_on_device(yg_context ctx, const double *xyz, int32_t n_nodes, const int32_t *cell_nodes,
                           const int32_t *cell_offsets, const int32_t *cell_types, int32_t n_cells,
                           const RawLayout &lay, int64_t N, HostDofmap &d, double **d_nodes_out,
                           int32_t **d_elements_out, bool device_mesh);  // dofmap_gpu.cu
yg_status generate_box(yg_context ctx, int dim, int nx, int ny, int nz, double lx, double ly, double lz, bool ccw,
                       double *xyz, int32_t *cell_nodes, int32_t *cell_offsets, int32_t *cell_types);

}  // namespace yg

using namespace yg;

// ================================================================ C ABI

// Copies a host numbering to the device (when there is a context) and hands
// the dofmap out; on failure the dofmap is destroyed.
static yg_status upload_dofmap(yg_dofmap d, yg_dofmap *out) {
    yg_context ctx = d->ctx;
    const HostDofmap &h = d->host;
    if (!ctx) {  // host-only numbering (no device copy); assembly needs a context
        *out = d;
        return YG_OK;
    }
    yg_status s;
    if ((s = dev_alloc_t(ctx, &d->d_nodes, h.nodes.size() + 1)) != YG_OK ||
        (s = dev_alloc_t(ctx, &d->d_offsets, h.offsets.size() + 1)) != YG_OK ||
        (s = dev_alloc_t(ctx, &d->d_elements, h.elements.size() + 1)) != YG_OK) {
        yg_dofmap_destroy(d);
        return s;
    }
    cudaError_t e = cudaMemcpy(d->d_nodes, h.nodes.data(), sizeof(double) * h.nodes.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d->d_offsets, h.offsets.data(), sizeof(int32_t) * h.offsets.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d->d_elements, h.elements.data(), sizeof(int32_t) * h.elements.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { yg_dofmap_destroy(d); return fail(YG_CUDA_ERROR, "dofmap upload: %s", cudaGetErrorString(e)); }
    *out = d;
    return YG_OK;
}

static int cell_corner_count(int32_t ct) {
    switch (ct) {
    case CELL_LINE2: return 2;
    case CELL_TRI3: return 3;
    case CELL_TET4: return 4;
    case CELL_QUAD4: return 4;
    case CELL_HEX8: return 8;
    default: return -1;
    }
}

static yg_status check_mesh(const double *nodes_xyz, int32_t n_nodes, const int32_t *cell_nodes,
                            const int32_t *cell_offsets, const int32_t *cell_types, int32_t n_cells, int32_t poly_order,
                            int32_t dof_per_node) {
    if (n_nodes < 0 || n_cells < 0 || (n_nodes && !nodes_xyz) || (n_cells && (!cell_offsets || !cell_types)))
        return fail(YG_BAD_ARG, "yg_dofmap_create: bad argument");
    if (dof_per_node < 1 || dof_per_node > 3) return fail(YG_BAD_ARG, "dof_per_node must be 1..3");
    for (int32_t c = 0; c < n_cells; ++c) {
        if (cell_offsets[c + 1] < cell_offsets[c]) return fail(YG_BAD_ARG, "cell offsets decrease at cell %d", c);
        for (int32_t i = cell_offsets[c]; i < cell_offsets[c + 1]; ++i)
            if (cell_nodes[i] < 0 || cell_nodes[i] >= n_nodes) return fail(YG_BAD_ARG, "cell %d references node %d", c, cell_nodes[i]);
        const int nc = cell_corner_count(cell_types[c]);
        if (poly_order > 1 && nc > 0 && cell_offsets[c + 1] - cell_offsets[c] < nc)
            return fail(YG_BAD_ARG, "cell %d has %d corners, its type needs %d", c, cell_offsets[c + 1] - cell_offsets[c], nc);
    }
    return YG_OK;
}

// The numbering on the device: the host lays out the raw nodes (element types,
// offsets, local node tables) and the device does the rest (dofmap_gpu.cu).
// YG_UNSUPPORTED when the host must number instead: a mesh the reference's own
// comparison sort must order (unless forced: then the stable order is kept),
// or keys wider than 64 bits.
static yg_status try_number_on_device(yg_dofmap d, const double *xyz, int32_t n_nodes, const int32_t *cell_nodes,
                                      const int32_t *cell_offsets, const int32_t *cell_types, int32_t n_cells,
                                      int32_t p, int32_t dpn, bool forced) {
    HostDofmap &h = d->host;
    h.dof_per_node = dpn;
    h.poly_order = p;
    h.offsets.assign(n_cells + 1, 0);
    h.topology.resize(n_cells);
    h.topo_dim.resize(n_cells);
    h.porder.assign(n_cells, (int8_t)p);
    for (int32_t c = 0; c < n_cells; ++c) {
        int t, td;
        cell_element_type(cell_types[c], t, td);
        h.topology[c] = (int8_t)t;
        h.topo_dim[c] = (int8_t)td;
    }
    RawLayout lay;
    const int64_t N = raw_node_layout(n_cells, p, h, lay);
    if (N == 0 || (!forced && raw_mix_needs_reference_order(h, N))) return YG_UNSUPPORTED;
    yg_context ctx = d->ctx;
    YG_TRY(number_on_device(ctx, xyz, n_nodes, cell_nodes, cell_offsets, cell_types, n_cells, lay, N, h, &d->d_nodes,
                            &d->d_elements, false));
    YG_TRY(dev_alloc_t(ctx, &d->d_offsets, h.offsets.size() + 1));
    YG_CUDA(cudaMemcpy(d->d_offsets, h.offsets.data(), sizeof(int32_t) * h.offsets.size(), cudaMemcpyHostToDevice));
    return YG_OK;
}

extern "C" yg_status yg_dofmap_create(yg_context ctx, const double *nodes_xyz, int32_t n_nodes,
                                      const int32_t *cell_nodes, const int32_t *cell_offsets,
                                      const int32_t *cell_types, int32_t n_cells, int32_t poly_order,
                                      int32_t dof_per_node, yg_dofmap *out) {
    if (!out) return fail(YG_BAD_ARG, "yg_dofmap_create: bad argument");
    *out = nullptr;
    yg_status cs = check_mesh(nodes_xyz, n_nodes, cell_nodes, cell_offsets, cell_types, n_cells, poly_order, dof_per_node);
    if (cs != YG_OK) return cs;
    auto *d = new yg_dofmap_t();
    d->ctx = ctx;
    // large p > 1 meshes are numbered on the device (identical result, see dofmap_gpu.cu)
    if (ctx && poly_order > 1) {
        yg_status s = try_number_on_device(d, nodes_xyz, n_nodes, cell_nodes, cell_offsets, cell_types, n_cells,
                                           poly_order, dof_per_node, false);
        if (s == YG_OK) { *out = d; return YG_OK; }
        if (s != YG_UNSUPPORTED) { yg_dofmap_destroy(d); return s; }
        d->host = HostDofmap();
    }
    if (!build_dofmap(nodes_xyz, n_nodes, cell_nodes, cell_offsets, cell_types, n_cells, poly_order, dof_per_node, d->host)) {
        delete d;
        return fail(YG_BAD_ARG, "DoFManager: Invalid polynomial order");
    }
    return upload_dofmap(d, out);
}

extern "C" yg_status yg_dofmap_create_on_device(yg_context ctx, const double *nodes_xyz, int32_t n_nodes,
                                                const int32_t *cell_nodes, const int32_t *cell_offsets,
                                                const int32_t *cell_types, int32_t n_cells, int32_t poly_order,
                                                int32_t dof_per_node, yg_dofmap *out) {
    if (!ctx) return fail(YG_BAD_ARG, "yg_dofmap_create_on_device: needs a context");
    if (poly_order < 2) return yg_dofmap_create(ctx, nodes_xyz, n_nodes, cell_nodes, cell_offsets, cell_types, n_cells,
                                                poly_order, dof_per_node, out);
    yg_status s = check_mesh(nodes_xyz, n_nodes, cell_nodes, cell_offsets, cell_types, n_cells, poly_order, dof_per_node);
    if (s != YG_OK) return s;
    *out = nullptr;
    auto *d = new yg_dofmap_t();
    d->ctx = ctx;
    s = try_number_on_device(d, nodes_xyz, n_nodes, cell_nodes, cell_offsets, cell_types, n_cells, poly_order,
                             dof_per_node, true);
    if (s != YG_OK) { yg_dofmap_destroy(d); return s; }
    *out = d;
    return YG_OK;
}

extern "C" yg_status yg_dofmap_create_from_numbering(yg_context ctx, const double *dof_nodes_xyz, int32_t n_dof_nodes,
                                                     const int32_t *element_offsets, const int32_t *elements,
                                                     const int32_t *cell_types, int32_t n_cells, int32_t poly_order,
                                                     int32_t dof_per_node, yg_dofmap *out) {
    if (!out || n_dof_nodes < 0 || n_cells < 0 || (n_dof_nodes && !dof_nodes_xyz) ||
        (n_cells && (!element_offsets || !elements || !cell_types)))
        return fail(YG_BAD_ARG, "yg_dofmap_create_from_numbering: bad argument");
    if (dof_per_node < 1 || dof_per_node > 3) return fail(YG_BAD_ARG, "dof_per_node must be 1..3");
    if (poly_order < 1) return fail(YG_BAD_ARG, "DoFManager: Invalid polynomial order");
    *out = nullptr;
    auto *d = new yg_dofmap_t();
    d->ctx = ctx;
    HostDofmap &h = d->host;
    h.dof_per_node = dof_per_node;
    h.poly_order = poly_order;
    h.nodes.assign(dof_nodes_xyz, dof_nodes_xyz + 3 * (int64_t)n_dof_nodes);
    h.offsets.assign(element_offsets, element_offsets + n_cells + 1);
    h.elements.assign(elements, elements + (n_cells ? element_offsets[n_cells] : 0));
    h.topology.resize(n_cells);
    h.topo_dim.resize(n_cells);
    h.porder.assign(n_cells, (int8_t)poly_order);
    for (int32_t c = 0; c < n_cells; ++c) {
        int t, td;
        cell_element_type(cell_types[c], t, td);
        h.topology[c] = (int8_t)t;
        h.topo_dim[c] = (int8_t)td;
        const int32_t cnt = element_offsets[c + 1] - element_offsets[c];
        int nen = 0;
        if (t != TOPO_NONE) {
            ElementTable T;
            if (poly_order == 1) nen = cell_corner_count(cell_types[c]);
            else if (make_element_table(t, td, poly_order, T)) nen = T.nen;
            else { delete d; return fail(YG_UNSUPPORTED, "element (topology %d, dim %d, order %d) not supported", t, td, poly_order); }
        }
        if (cnt < 0 || cnt != nen) {
            delete d;
            return fail(YG_BAD_ARG, "element %d lists %d nodes, its type has %d", c, cnt, nen);
        }
        for (int32_t i = element_offsets[c]; i < element_offsets[c + 1]; ++i)
            if (elements[i] < 0 || elements[i] >= n_dof_nodes) {
                delete d;
                return fail(YG_BAD_ARG, "element %d references node %d", c, elements[i]);
            }
    }
    return upload_dofmap(d, out);
}

extern "C" yg_status yg_dofmap_create_box(yg_context ctx, int32_t dim, int32_t nx, int32_t ny, int32_t nz, double lx,
                                          double ly, double lz, int32_t poly_order, int32_t dof_per_node,
                                          yg_dofmap *out) {
    if (!ctx || !out || (dim != 2 && dim != 3) || nx < 1 || ny < 1 || (dim == 3 && nz < 1) || !(lx > 0) || !(ly > 0) ||
        (dim == 3 && !(lz > 0)))
        return fail(YG_BAD_ARG, "yg_dofmap_create_box: bad argument");
    if (dof_per_node < 1 || dof_per_node > 3) return fail(YG_BAD_ARG, "dof_per_node must be 1..3");
    if (poly_order < 1) return fail(YG_BAD_ARG, "DoFManager: Invalid polynomial order");
    *out = nullptr;
    const int64_t nnodes = (int64_t)(nx + 1) * (ny + 1) * (dim == 3 ? nz + 1 : 1);
    const int64_t ncells = (int64_t)nx * ny * (dim == 3 ? nz : 1);
    const int nc = dim == 3 ? 8 : 4;
    if (nnodes > INT32_MAX || ncells * nc > INT32_MAX) return fail(YG_BAD_ARG, "yg_dofmap_create_box: box too large");
    auto *d = new yg_dofmap_t();
    d->ctx = ctx;
    HostDofmap &h = d->host;
    h.dof_per_node = dof_per_node;
    h.poly_order = poly_order;
    h.offsets.resize(ncells + 1);
    for (int64_t c = 0; c <= ncells; ++c) h.offsets[c] = (int32_t)(c * nc);
    h.topology.assign(ncells, (int8_t)TOPO_TENSOR);
    h.topo_dim.assign(ncells, (int8_t)dim);
    h.porder.assign(ncells, (int8_t)poly_order);
    double *xyz = nullptr;
    int32_t *cn = nullptr, *co = nullptr, *ct = nullptr;
    auto done = [&](yg_status s) {
        dev_free(ctx, xyz);
        dev_free(ctx, cn);
        dev_free(ctx, co);
        dev_free(ctx, ct);
        if (s != YG_OK) yg_dofmap_destroy(d);
        else *out = d;
        return s;
    };
    yg_status s;
    if ((s = dev_alloc_t(ctx, &xyz, 3 * nnodes + 1)) != YG_OK || (s = dev_alloc_t(ctx, &cn, ncells * nc + 1)) != YG_OK ||
        (s = dev_alloc_t(ctx, &co, ncells + 1)) != YG_OK || (s = dev_alloc_t(ctx, &ct, ncells + 1)) != YG_OK)
        return done(s);
    // p = 1 keeps the mesh numbering, whose cells must be in the element's
    // x-fastest order; p > 1 places nodes with the counter-clockwise corner maps
    if ((s = generate_box(ctx, dim, nx, ny, nz, lx, ly, lz, poly_order > 1, xyz, cn, co, ct)) != YG_OK) return done(s);
    if (poly_order == 1) {  // DoFManager.cpp:153-160: the mesh itself
        h.nodes.resize(3 * nnodes);
        h.elements.resize(ncells * nc);
        cudaError_t e = cudaMemcpyAsync(h.nodes.data(), xyz, sizeof(double) * 3 * nnodes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h.elements.data(), cn, sizeof(int32_t) * ncells * nc, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return done(fail(YG_CUDA_ERROR, "yg_dofmap_create_box: %s", cudaGetErrorString(e)));
        d->d_nodes = xyz;
        d->d_elements = cn;
        xyz = nullptr;
        cn = nullptr;
    } else {
        RawLayout lay;
        const int64_t N = raw_node_layout((int32_t)ncells, poly_order, h, lay);
        if ((s = number_on_device(ctx, xyz, (int32_t)nnodes, cn, co, ct, (int32_t)ncells, lay, N, h, &d->d_nodes,
                                  &d->d_elements, true)) != YG_OK)
            return done(s);
    }
    if ((s = dev_alloc_t(ctx, &d->d_offsets, h.offsets.size() + 1)) != YG_OK) return done(s);
    cudaError_t e = cudaMemcpy(d->d_offsets, h.offsets.data(), sizeof(int32_t) * h.offsets.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return done(fail(YG_CUDA_ERROR, "yg_dofmap_create_box: %s", cudaGetErrorString(e)));
    return done(YG_OK);
}

extern "C" yg_status yg_element_table(int32_t topology, int32_t dim, int32_t poly_order, int32_t *nen, int32_t *nq,
                                      double *local_nodes_xyz, double *qp_xyz, double *qw, double *N, double *dN) {
    if (!nen || !nq || dim < 1 || dim > 3 || poly_order < 1) return fail(YG_BAD_ARG, "yg_element_table: bad argument");
    ElementTable T;
    if (!make_element_table(topology, dim, poly_order, T))
        return fail(YG_UNSUPPORTED, "element (topology %d, dim %d, order %d) not supported", topology, dim, poly_order);
    *nen = T.nen;
    *nq = T.nq;
    if (local_nodes_xyz) std::copy(T.local_nodes.begin(), T.local_nodes.end(), local_nodes_xyz);
    if (qp_xyz) std::copy(T.qpts.begin(), T.qpts.end(), qp_xyz);
    if (qw) std::copy(T.qw.begin(), T.qw.end(), qw);
    if (N) std::copy(T.N.begin(), T.N.end(), N);
    if (dN) std::copy(T.dN.begin(), T.dN.end(), dN);
    return YG_OK;
}

extern "C" yg_status yg_dofmap_destroy(yg_dofmap d) {
    if (!d) return YG_OK;
    yg_context ctx = d->ctx;
    if (!ctx) { delete d; return YG_OK; }
    dev_free(ctx, d->d_nodes);
    dev_free(ctx, d->d_offsets);
    dev_free(ctx, d->d_elements);
    dev_free(ctx, d->d_nrowptr);
    dev_free(ctx, d->d_ncol);
    for (auto &g : d->groups) { dev_free(ctx, g.d_tab); dev_free(ctx, g.d_order); }
    delete d;
    return YG_OK;
}

extern "C" yg_status yg_dofmap_sizes(yg_dofmap d, int32_t *n_dof_nodes, int32_t *n_cells, int64_t *n_element_nodes,
                                     int64_t *n_dofs) {
    if (!d) return fail(YG_BAD_ARG, "NULL dofmap");
    if (n_dof_nodes) *n_dof_nodes = d->host.n_nodes();
    if (n_cells) *n_cells = d->host.n_cells();
    if (n_element_nodes) *n_element_nodes = (int64_t)d->host.elements.size();
    if (n_dofs) *n_dofs = (int64_t)d->host.n_nodes() * d->host.dof_per_node;
    return YG_OK;
}

extern "C" yg_status yg_dofmap_get(yg_dofmap d, double *dof_nodes_xyz, int32_t *element_offsets, int32_t *elements,
                                   int8_t *topology, int8_t *topo_dim, int8_t *poly_order) {
    if (!d) return fail(YG_BAD_ARG, "NULL dofmap");
    const HostDofmap &h = d->host;
    if (dof_nodes_xyz) std::copy(h.nodes.begin(), h.nodes.end(), dof_nodes_xyz);
    if (element_offsets) std::copy(h.offsets.begin(), h.offsets.end(), element_offsets);
    if (elements) std::copy(h.elements.begin(), h.elements.end(), elements);
    if (topology) std::copy(h.topology.begin(), h.topology.end(), topology);
    if (topo_dim) std::copy(h.topo_dim.begin(), h.topo_dim.end(), topo_dim);
    if (poly_order) std::copy(h.porder.begin(), h.porder.end(), poly_order);
    return YG_OK;
}

extern "C" yg_status yg_assemble(yg_dofmap d, const yg_physics *physics, uint32_t requirements, int32_t format,
                                 yg_matrix *K, yg_vector residual) {
    if (!d || !physics) return fail(YG_BAD_ARG, "yg_assemble: NULL argument");
    const int nsd = physics->nsd;
    if (nsd < 1 || nsd > 3) return fail(YG_BAD_ARG, "physics nsd must be 1..3");
    if (format != YG_FORMAT_CSR && format != YG_FORMAT_BCSR) return fail(YG_BAD_ARG, "unknown format %d", format);
    const bool wantK = requirements & YG_REQ_TANGENT, wantR = requirements & YG_REQ_RESIDUAL;
    if (wantK && !K) return fail(YG_BAD_ARG, "tangent requested without a matrix slot");
    const int64_t ndofs = (int64_t)d->host.n_nodes() * d->host.dof_per_node;
    if (wantR && (!residual || residual->n != ndofs)) return fail(YG_BAD_ARG, "residual vector must have %lld entries", (long long)ndofs);
    const int dpn = d->host.dof_per_node;
    const int kind = physics->kind;
    if (kind == YG_ELASTICITY ? dpn != nsd : dpn != 1)
        return fail(YG_BAD_ARG, "physics %d needs dof_per_node %d (got %d)", kind, kind == YG_ELASTICITY ? nsd : 1, dpn);
    yg_context ctx = d->ctx;
    if (!ctx) return fail(YG_BAD_ARG, "yg_assemble: dofmap was created without a context");
    YG_TRY(build_pattern(d, nsd));
    double *val = nullptr;
    if (wantK) {
        if (!*K) {
            YG_TRY(new_matrix_from_pattern(d, format, K));
        } else if ((*K)->owner != d || (*K)->owner_format != format) {
            return fail(YG_BAD_ARG, "matrix was not assembled from this dofmap in this format");
        }
        yg_matrix A = *K;
        YG_CUDA(cudaMemsetAsync(A->d_val, 0, sizeof(double) * A->nnzb * A->block * A->block, ctx->stream));
        val = A->d_val;
    }
    PhysParams prm{};
    for (int i = 0; i < 8; ++i) prm.p[i] = physics->params[i];
    if (kind == YG_SUPG) {
        // supg_advection.hpp:78-88,110-122
        const double k = prm.p[0], h = prm.p[1], U0 = prm.p[2];
        const double Pe = U0 * h / (2 * k);
        const double alpha = (Pe == 0) ? 0.0 : std::cosh(Pe) / std::sinh(Pe) - 1.0 / Pe;
        prm.U[0] = U0;
        double normU = std::fabs(U0);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                prm.Kd[3 * a + b] = (a == b) ? k : 0.0;
                if (normU > 0) prm.Kd[3 * a + b] += (alpha * h / (normU * 2)) * (prm.U[a] * prm.U[b]);
            }
        for (int a = 0; a < 3; ++a) prm.Uhat[a] = normU > 0 ? (alpha * h / 2) * prm.U[a] / normU : 0.0;
    }
    for (const ElementGroup &g : d->groups) {
        yg_status s;
        switch (nsd) {
        case 1: s = dispatch_physics<1>(ctx, g, d, kind, dpn, prm, val, format, wantR ? residual->d : nullptr, wantK, wantR); break;
        case 2: s = dispatch_physics<2>(ctx, g, d, kind, dpn, prm, val, format, wantR ? residual->d : nullptr, wantK, wantR); break;
        default: s = dispatch_physics<3>(ctx, g, d, kind, dpn, prm, val, format, wantR ? residual->d : nullptr, wantK, wantR); break;
        }
        if (s != YG_OK) return s;
    }
    if (wantK && (*K)->d_val32) YG_TRY(yg_matrix_make_fp32(*K));
    return YG_OK;
}

extern "C" yg_status yg_dirichlet_apply(yg_matrix K, yg_vector rhs, const int64_t *bc_dofs, const double *bc_values,
                                        int64_t n_bc) {
    if (!K || !rhs || n_bc < 0 || (n_bc && (!bc_dofs || !bc_values))) return fail(YG_BAD_ARG, "yg_dirichlet_apply: bad argument");
    if (K->rows() != K->cols() || rhs->n != K->rows()) return fail(YG_BAD_ARG, "yg_dirichlet_apply: size mismatch");
    for (int64_t i = 0; i < n_bc; ++i)
        if (bc_dofs[i] < 0 || bc_dofs[i] >= K->rows()) return fail(YG_BAD_ARG, "BC dof %lld out of range", (long long)bc_dofs[i]);
    yg_context ctx = K->ctx;
    const int64_t n = K->rows();
    // scratch kept on the matrix between calls
    if (!K->d_bcmask) {
        yg_status s;
        if ((s = dev_alloc_t(ctx, &K->d_bcmask, n)) != YG_OK || (s = dev_alloc_t(ctx, &K->d_bcg, n)) != YG_OK ||
            (s = dev_alloc_t(ctx, &K->d_bcq, n)) != YG_OK)
            return s;
    }
    if (n_bc > K->bc_cap) {
        YG_CUDA(cudaStreamSynchronize(ctx->stream));
        dev_free(ctx, K->d_bcdofs);
        dev_free(ctx, K->d_bcvals);
        K->d_bcdofs = nullptr;
        K->d_bcvals = nullptr;
        K->bc_cap = 0;
        const int64_t cap = n_bc + n_bc / 2 + 16;
        YG_TRY(dev_alloc_t(ctx, &K->d_bcdofs, cap));
        YG_TRY(dev_alloc_t(ctx, &K->d_bcvals, cap));
        K->bc_cap = cap;
    }
    bool homogeneous = true;
    for (int64_t i = 0; i < n_bc && homogeneous; ++i) homogeneous = bc_values[i] == 0.0;
    uint8_t *mask = K->d_bcmask;
    double *g = K->d_bcg, *q = K->d_bcq;
    cudaStream_t st = ctx->stream;
    cudaMemsetAsync(mask, 0, n, st);
    cudaMemsetAsync(g, 0, sizeof(double) * n, st);
    yg_status s = YG_OK;
    if (n_bc) {
        // the host arrays are pageable: the copies complete before the call returns
        YG_CUDA(cudaMemcpyAsync(K->d_bcdofs, bc_dofs, sizeof(int64_t) * n_bc, cudaMemcpyHostToDevice, st));
        YG_CUDA(cudaMemcpyAsync(K->d_bcvals, bc_values, sizeof(double) * n_bc, cudaMemcpyHostToDevice, st));
        k_bc_scatter<<<stream_grid(ctx, n_bc), kThreads, 0, st>>>(n_bc, K->d_bcdofs, K->d_bcvals, mask, g);
        YG_LAUNCHED(ctx);
    }
    // F -= K g (skipped when every prescribed value is 0: K g = 0)
    if (!homogeneous) {
        s = spmv_launch(K, g, q, YG_PREC_FP64, nullptr, nullptr, spmv_default_grid(K));
        if (s == YG_OK) {
            k_sub_inplace<<<stream_grid(ctx, n), kThreads, 0, st>>>(n, rhs->d, q);
            YG_LAUNCHED(ctx);
        }
    }
    if (s == YG_OK && n_bc) {
        const int64_t warps_needed = K->nbrows;
        int64_t blocks = (warps_needed * 32 + kThreads - 1) / kThreads;
        const int64_t cap = (int64_t)ctx->num_sms * 16;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) blocks = 1;
        k_bc_zero<<<(int)blocks, kThreads, 0, st>>>(K->nbrows, K->block, K->d_rowptr, K->d_col, K->d_val, mask, g,
                                                    rhs->d);
        YG_LAUNCHED(ctx);
    }
    if (s == YG_OK && K->d_val32) s = yg_matrix_make_fp32(K);
    cudaError_t e = cudaStreamSynchronize(st);
    if (s != YG_OK) return s;
    if (e != cudaSuccess) return fail(YG_CUDA_ERROR, "Dirichlet apply: %s", cudaGetErrorString(e));
    return YG_OK;
}

// ------------------------------------------------------------------ gradient recovery

namespace yg {

// Element::update for one cell, cooperatively by the CTA (include/element/Element.hpp:109-149):
// the Jacobian sum_A x_A (x) dN_A/dxi, jxw = det J * w_q and the physical
// gradients G[(q*nen + A)*NSD + i] = sum_j Jinv(j, i) dN_A/dxi_j, from the
// cell's node coordinates xe (nen x 3, already in shared memory).  Ends with
// the CTA synchronised.
template <int NSD>
__device__ void cell_gradients(const double *__restrict__ xe, const double *__restrict__ tdN, const double *__restrict__ tw,
                               int nen, int nq, int tdim, double *__restrict__ G, double *__restrict__ jxw,
                               double *__restrict__ Ji) {
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int A = 0; A < nen; ++A) {
            const double *d = tdN + ((size_t)q * nen + A) * tdim;
#pragma unroll
            for (int i = 0; i < NSD; ++i)
#pragma unroll
                for (int j = 0; j < NSD; ++j) J[i][j] += xe[3 * A + i] * d[j];
        }
        double det, inv[3][3];
        if (NSD == 1) {
            det = J[0][0];
            inv[0][0] = 1.0 / J[0][0];
        } else if (NSD == 2) {
            det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
            const double di = 1.0 / det;
            inv[0][0] = J[1][1] * di; inv[1][1] = J[0][0] * di;
            inv[0][1] = -J[0][1] * di; inv[1][0] = -J[1][0] * di;
        } else {
            det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[2][0] * J[1][2]) +
                  J[0][2] * (J[1][0] * J[2][1] - J[2][0] * J[1][1]);
            const double di = 1.0 / det;
            inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * di;
            inv[0][1] = -(J[0][1] * J[2][2] - J[2][1] * J[0][2]) * di;
            inv[0][2] = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * di;
            inv[1][0] = -(J[1][0] * J[2][2] - J[2][0] * J[1][2]) * di;
            inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * di;
            inv[1][2] = -(J[0][0] * J[1][2] - J[1][0] * J[0][2]) * di;
            inv[2][0] = (J[1][0] * J[2][1] - J[2][0] * J[1][1]) * di;
            inv[2][1] = -(J[0][0] * J[2][1] - J[2][0] * J[0][1]) * di;
            inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * di;
        }
        jxw[q] = det * tw[q];
#pragma unroll
        for (int i = 0; i < NSD; ++i)
#pragma unroll
            for (int j = 0; j < NSD; ++j) Ji[9 * q + 3 * i + j] = inv[i][j];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nq * nen; idx += blockDim.x) {
        const int q = idx / nen;
        const double *d = tdN + (size_t)idx * tdim;
#pragma unroll
        for (int dd = 0; dd < NSD; ++dd) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < NSD; ++j) s += Ji[9 * q + 3 * j + dd] * d[j];
            G[(size_t)idx * NSD + dd] = s;
        }
    }
    __syncthreads();
}

// LocalSmoothingGradient<Physics> (include/assembly/LocalSmoothingGradient.hpp:20-94):
// per cell of dimension NSD (one CTA), per quadrature point, the gradient of each
// of the DPN solution components, qg(comp, i) = sum_A u_A dN_A/dx_i, is spread to
// the cell's dofs: vtg(dof, i) += N_A qg(comp_A, i) jxw and vol(dof) += N_A jxw.
// A CTA first sums its quadrature points, then adds into the global arrays; the
// cells of one launch share no node (one colour), so the adds need no atomics and
// the sums are deterministic.  The geometry is that of k_assemble's Element::update.
template <int NSD, int DPN>
__global__ void __launch_bounds__(128)
k_smooth_gradient(const int32_t *__restrict__ order, int ncell, const int32_t *__restrict__ off,
                  const int32_t *__restrict__ el, const double *__restrict__ nodes, const double *__restrict__ tab,
                  int nen, int nq, int tdim, const double *__restrict__ sol, double *__restrict__ vol,
                  double *__restrict__ vtg) {
    extern __shared__ double sm[];
    double *xe = sm;                           // nen*3
    double *G = xe + 3 * nen;                  // nq*nen*NSD
    double *jxw = G + (size_t)nq * nen * NSD;  // nq
    double *Ji = jxw + nq;                     // nq*9
    double *ul = Ji + 9 * nq;                  // nen*DPN
    double *qg = ul + nen * DPN;               // nq*DPN*NSD
    int32_t *gn = reinterpret_cast<int32_t *>(qg + (size_t)nq * DPN * NSD);  // nen
    const double *tN = tab;
    const double *tdN = tab + (size_t)nq * nen;
    const double *tw = tdN + (size_t)nq * nen * tdim;
    for (int t = blockIdx.x; t < ncell; t += gridDim.x) {
        const int c = order[t];
        const int base = off[c];
        for (int a = threadIdx.x; a < nen; a += blockDim.x) {
            const int n = el[base + a];
            gn[a] = n;
            xe[3 * a + 0] = nodes[3 * (int64_t)n + 0];
            xe[3 * a + 1] = nodes[3 * (int64_t)n + 1];
            xe[3 * a + 2] = nodes[3 * (int64_t)n + 2];
        }
        __syncthreads();
        for (int a = threadIdx.x; a < nen * DPN; a += blockDim.x) ul[a] = sol[(int64_t)gn[a / DPN] * DPN + a % DPN];
        cell_gradients<NSD>(xe, tdN, tw, nen, nq, tdim, G, jxw, Ji);
        // qg[(q*DPN + comp)*NSD + i] = sum over the cell's nodes A of u(A, comp) dN_A/dx_i at q
        for (int idx = threadIdx.x; idx < nq * DPN * NSD; idx += blockDim.x) {
            const int q = idx / (DPN * NSD), comp = (idx / NSD) % DPN, i = idx % NSD;
            double s = 0;
            for (int A = 0; A < nen; ++A) s += ul[A * DPN + comp] * G[((size_t)q * nen + A) * NSD + i];
            qg[idx] = s;
        }
        __syncthreads();
        for (int a = threadIdx.x; a < nen * DPN; a += blockDim.x) {
            const int A = a / DPN, comp = a % DPN;
            double v = 0, w[NSD];
#pragma unroll
            for (int i = 0; i < NSD; ++i) w[i] = 0;
            for (int q = 0; q < nq; ++q) {
                const double NA = tN[(size_t)q * nen + A];
                v += NA * jxw[q];
#pragma unroll
                for (int i = 0; i < NSD; ++i) w[i] += NA * qg[(q * DPN + comp) * NSD + i] * jxw[q];
            }
            const int64_t g = (int64_t)gn[A] * DPN + comp;
            vol[g] += v;
#pragma unroll
            for (int i = 0; i < NSD; ++i) vtg[g * NSD + i] += w[i];
        }
        __syncthreads();
    }
}

// ZZGradientRecovery<Physics> (include/assembly/ZZGradientRecovery.hpp:33-140), p = 1:
// every node fits a linear polynomial a_0 + a.(x - x_n) by least squares to the
// FE gradient sampled at the quadrature points of the cells around it; the
// recovered gradient is a_0.  Centred coordinates give the same fit as the
// reference's [1 x y z] basis with a better conditioned system.  This kernel
// accumulates, per node, the normal equations of its patch: the symmetric
// (NSD+1)^2 matrix sum P^T P (packed upper triangle) and P^T g (NSD+1 rows of
// NSD), P = [1, x_q - x_n].  One CTA per cell of one colour, as in
// k_smooth_gradient, so the sums need no atomics and are deterministic.
template <int NSD>
__global__ void __launch_bounds__(128)
k_zz_accumulate(const int32_t *__restrict__ order, int ncell, const int32_t *__restrict__ off,
                const int32_t *__restrict__ el, const double *__restrict__ nodes, const double *__restrict__ tab,
                int nen, int nq, int tdim, const double *__restrict__ sol, double *__restrict__ acc) {
    constexpr int NB = NSD + 1, NM = NB * (NB + 1) / 2, NA = NM + NB * NSD;
    extern __shared__ double sm[];
    double *xe = sm;                           // nen*3
    double *G = xe + 3 * nen;                  // nq*nen*NSD
    double *jxw = G + (size_t)nq * nen * NSD;  // nq
    double *Ji = jxw + nq;                     // nq*9
    double *ul = Ji + 9 * nq;                  // nen
    double *qg = ul + nen;                     // nq*NSD: field gradient at q
    double *xq = qg + (size_t)nq * NSD;        // nq*3: point location
    int32_t *gn = reinterpret_cast<int32_t *>(xq + (size_t)nq * 3);  // nen
    const double *tN = tab;
    const double *tdN = tab + (size_t)nq * nen;
    const double *tw = tdN + (size_t)nq * nen * tdim;
    for (int t = blockIdx.x; t < ncell; t += gridDim.x) {
        const int c = order[t];
        const int base = off[c];
        for (int a = threadIdx.x; a < nen; a += blockDim.x) {
            const int n = el[base + a];
            gn[a] = n;
            xe[3 * a + 0] = nodes[3 * (int64_t)n + 0];
            xe[3 * a + 1] = nodes[3 * (int64_t)n + 1];
            xe[3 * a + 2] = nodes[3 * (int64_t)n + 2];
        }
        __syncthreads();
        for (int a = threadIdx.x; a < nen; a += blockDim.x) ul[a] = sol[gn[a]];
        cell_gradients<NSD>(xe, tdN, tw, nen, nq, tdim, G, jxw, Ji);
        // sample point x_q = sum_A N_A x_A and field gradient sum_A u_A dN_A/dx
        for (int idx = threadIdx.x; idx < nq * 3; idx += blockDim.x) {
            const int q = idx / 3, k = idx % 3;
            double s = 0;
            for (int A = 0; A < nen; ++A) s += tN[(size_t)q * nen + A] * xe[3 * A + k];
            xq[idx] = s;
        }
        for (int idx = threadIdx.x; idx < nq * NSD; idx += blockDim.x) {
            const int q = idx / NSD, i = idx % NSD;
            double s = 0;
            for (int A = 0; A < nen; ++A) s += ul[A] * G[((size_t)q * nen + A) * NSD + i];
            qg[idx] = s;
        }
        __syncthreads();
        // node A of the cell: its patch rows, one per quadrature point
        for (int A = threadIdx.x; A < nen; A += blockDim.x) {
            double a[NA];
#pragma unroll
            for (int k = 0; k < NA; ++k) a[k] = 0;
            for (int q = 0; q < nq; ++q) {
                double P[NB];
                P[0] = 1;
#pragma unroll
                for (int i = 0; i < NSD; ++i) P[i + 1] = xq[3 * q + i] - xe[3 * A + i];
                int k = 0;
#pragma unroll
                for (int r = 0; r < NB; ++r)
#pragma unroll
                    for (int cc = r; cc < NB; ++cc) a[k++] += P[r] * P[cc];
#pragma unroll
                for (int r = 0; r < NB; ++r)
#pragma unroll
                    for (int i = 0; i < NSD; ++i) a[NM + r * NSD + i] += P[r] * qg[q * NSD + i];
            }
            double *dst = acc + (int64_t)gn[A] * NA;
#pragma unroll
            for (int k = 0; k < NA; ++k) dst[k] += a[k];
        }
        __syncthreads();
    }
}

// Per node: solve the (NSD+1)^2 normal equations by Cholesky and keep the
// constant term of each of the NSD fits.  A node with too few samples (a
// singular system) gets NaN; a node no cell of the dimension touches gets 0/0.
template <int NSD>
__global__ void k_zz_solve(int64_t n, const double *__restrict__ acc, double *__restrict__ grad) {
    constexpr int NB = NSD + 1, NM = NB * (NB + 1) / 2, NA = NM + NB * NSD;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const double *a = acc + v * NA;
        double L[NB][NB], y[NB][NSD];
        int k = 0;
#pragma unroll
        for (int r = 0; r < NB; ++r)
#pragma unroll
            for (int cc = r; cc < NB; ++cc) { L[cc][r] = a[k]; ++k; }  // lower triangle of the symmetric matrix
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            double d = L[j][j];
#pragma unroll
            for (int m = 0; m < j; ++m) d -= L[j][m] * L[j][m];
            d = sqrt(d);
            L[j][j] = d;
#pragma unroll
            for (int i = j + 1; i < NB; ++i) {
                double s = L[i][j];
#pragma unroll
                for (int m = 0; m < j; ++m) s -= L[i][m] * L[j][m];
                L[i][j] = s / d;
            }
        }
#pragma unroll
        for (int i = 0; i < NSD; ++i) {
            double z[NB];
#pragma unroll
            for (int r = 0; r < NB; ++r) {  // L z = P^T g
                double s = a[NM + r * NSD + i];
#pragma unroll
                for (int m = 0; m < r; ++m) s -= L[r][m] * z[m];
                z[r] = s / L[r][r];
            }
#pragma unroll
            for (int r = NB - 1; r >= 0; --r) {  // L^T y = z
                double s = z[r];
#pragma unroll
                for (int m = r + 1; m < NB; ++m) s -= L[m][r] * y[m][i];
                y[r][i] = s / L[r][r];
            }
            grad[v * NSD + i] = y[0][i];
        }
    }
}

__global__ void k_divide_rows(int64_t n, int nsd, const double *__restrict__ vol, double *__restrict__ g) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * nsd; i += (int64_t)gridDim.x * blockDim.x)
        g[i] = g[i] / vol[i / nsd];
}

template <int NSD, int DPN>
static yg_status launch_smooth_gradient(yg_context ctx, const ElementGroup &g, yg_dofmap d, const double *sol,
                                        double *vol, double *vtg) {
    const int nen = g.tab.nen, nq = g.tab.nq;
    const size_t smem = sizeof(double) * (3 * nen + (size_t)nq * nen * NSD + nq + 9 * nq + nen * DPN +
                                          (size_t)nq * DPN * NSD) + sizeof(int32_t) * nen + 16;
    auto kern = k_smooth_gradient<NSD, DPN>;
    // the element's shape gradients at every quadrature point sit in shared
    // memory: hexahedra of order 4 and above need more than a block can hold
    if (smem > ctx->smem_optin)
        return fail(YG_UNSUPPORTED, "LocalSmoothingGradient: element (nen %d, nq %d) needs %zu B of shared memory, "
                    "the device allows %zu", nen, nq, smem, ctx->smem_optin);
    if (smem > 48 * 1024) YG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (size_t c = 0; c + 1 < g.color_ptr.size(); ++c) {
        const int n = g.color_ptr[c + 1] - g.color_ptr[c];
        if (n == 0) continue;
        const int grid = std::min(n, ctx->num_sms * 16);
        kern<<<grid, 128, smem, ctx->stream>>>(g.d_order + g.color_ptr[c], n, d->d_offsets, d->d_elements, d->d_nodes,
                                               g.d_tab, nen, nq, g.tab.dim, sol, vol, vtg);
        YG_LAUNCHED(ctx);
    }
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

template <int NSD>
static yg_status smooth_gradient_dpn(yg_context ctx, const ElementGroup &g, yg_dofmap d, int dpn, const double *sol,
                                     double *vol, double *vtg) {
    if (dpn == 1) return launch_smooth_gradient<NSD, 1>(ctx, g, d, sol, vol, vtg);
    if (dpn == 2) return launch_smooth_gradient<NSD, 2>(ctx, g, d, sol, vol, vtg);
    return launch_smooth_gradient<NSD, 3>(ctx, g, d, sol, vol, vtg);
}

template <int NSD>
static yg_status launch_zz(yg_context ctx, const ElementGroup &g, yg_dofmap d, const double *sol, double *acc) {
    const int nen = g.tab.nen, nq = g.tab.nq;
    const size_t smem = sizeof(double) * (3 * nen + (size_t)nq * nen * NSD + nq + 9 * nq + nen + (size_t)nq * NSD +
                                          (size_t)nq * 3) + sizeof(int32_t) * nen + 16;
    auto kern = k_zz_accumulate<NSD>;
    if (smem > ctx->smem_optin)
        return fail(YG_UNSUPPORTED, "ZZGradientRecovery: element (nen %d, nq %d) needs %zu B of shared memory", nen, nq,
                    smem);
    if (smem > 48 * 1024) YG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (size_t c = 0; c + 1 < g.color_ptr.size(); ++c) {
        const int n = g.color_ptr[c + 1] - g.color_ptr[c];
        if (n == 0) continue;
        const int grid = std::min(n, ctx->num_sms * 16);
        kern<<<grid, 128, smem, ctx->stream>>>(g.d_order + g.color_ptr[c], n, d->d_offsets, d->d_elements, d->d_nodes,
                                               g.d_tab, nen, nq, g.tab.dim, sol, acc);
        YG_LAUNCHED(ctx);
    }
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

}  // namespace yg

extern "C" yg_status yg_zz_gradient_recovery(yg_dofmap d, int32_t nsd, yg_vector solution, yg_vector gradient) {
    if (!d || !solution || !gradient) return fail(YG_BAD_ARG, "yg_zz_gradient_recovery: NULL argument");
    if (nsd < 2 || nsd > 3) return fail(YG_BAD_ARG, "yg_zz_gradient_recovery: nsd must be 2 or 3");
    yg_context ctx = d->ctx;
    if (!ctx) return fail(YG_BAD_ARG, "yg_zz_gradient_recovery: dofmap was created without a context");
    // the reference asserts p = 1 (ZZGradientRecovery.hpp:44) and reads one dof per node
    if (d->host.poly_order != 1 || d->host.dof_per_node != 1)
        return fail(YG_UNSUPPORTED, "ZZGradientRecovery: p = 1 and one dof per node only (got p %d, dpn %d)",
                    d->host.poly_order, d->host.dof_per_node);
    const int64_t nn = d->host.n_nodes();
    if (solution->n != nn || gradient->n != nn * nsd)
        return fail(YG_BAD_ARG, "yg_zz_gradient_recovery: solution needs %lld entries, gradient %lld", (long long)nn,
                    (long long)(nn * nsd));
    YG_TRY(build_pattern(d, nsd));
    const int na = (nsd + 1) * (nsd + 2) / 2 + (nsd + 1) * nsd;
    double *acc = nullptr;
    YG_TRY(dev_alloc_t(ctx, &acc, nn * na));
    yg_status s = YG_OK;
    cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(double) * nn * na, ctx->stream);
    if (e != cudaSuccess) s = fail(YG_CUDA_ERROR, "ZZGradientRecovery: %s", cudaGetErrorString(e));
    for (const ElementGroup &g : d->groups) {
        if (s != YG_OK) break;
        s = nsd == 2 ? launch_zz<2>(ctx, g, d, solution->d, acc) : launch_zz<3>(ctx, g, d, solution->d, acc);
    }
    if (s == YG_OK && nn > 0) {
        if (nsd == 2) k_zz_solve<2><<<stream_grid(ctx, nn), kThreads, 0, ctx->stream>>>(nn, acc, gradient->d);
        else k_zz_solve<3><<<stream_grid(ctx, nn), kThreads, 0, ctx->stream>>>(nn, acc, gradient->d);
        YG_LAUNCHED(ctx);
    }
    dev_free(ctx, acc);
    if (s != YG_OK) return s;
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}

extern "C" yg_status yg_local_smoothing_gradient(yg_dofmap d, int32_t nsd, yg_vector solution, yg_vector gradient) {
    if (!d || !solution || !gradient) return fail(YG_BAD_ARG, "yg_local_smoothing_gradient: NULL argument");
    if (nsd < 1 || nsd > 3) return fail(YG_BAD_ARG, "yg_local_smoothing_gradient: nsd must be 1..3");
    yg_context ctx = d->ctx;
    if (!ctx) return fail(YG_BAD_ARG, "yg_local_smoothing_gradient: dofmap was created without a context");
    const int dpn = d->host.dof_per_node;
    if (dpn < 1 || dpn > 3) return fail(YG_UNSUPPORTED, "yg_local_smoothing_gradient: dof_per_node %d (1..3)", dpn);
    const int64_t ndofs = (int64_t)d->host.n_nodes() * dpn;
    if (solution->n != ndofs || gradient->n != ndofs * nsd)
        return fail(YG_BAD_ARG, "yg_local_smoothing_gradient: solution needs %lld entries, gradient %lld",
                    (long long)ndofs, (long long)(ndofs * nsd));
    YG_TRY(build_pattern(d, nsd));  // element groups and colourings of the cells of dimension nsd
    double *vol = nullptr;
    YG_TRY(dev_alloc_t(ctx, &vol, ndofs));
    yg_status s = YG_OK;
    cudaError_t e = cudaMemsetAsync(vol, 0, sizeof(double) * ndofs, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(gradient->d, 0, sizeof(double) * ndofs * nsd, ctx->stream);
    if (e != cudaSuccess) s = fail(YG_CUDA_ERROR, "LocalSmoothingGradient: %s", cudaGetErrorString(e));
    for (const ElementGroup &g : d->groups) {
        if (s != YG_OK) break;
        switch (nsd) {
        case 1: s = smooth_gradient_dpn<1>(ctx, g, d, dpn, solution->d, vol, gradient->d); break;
        case 2: s = smooth_gradient_dpn<2>(ctx, g, d, dpn, solution->d, vol, gradient->d); break;
        default: s = smooth_gradient_dpn<3>(ctx, g, d, dpn, solution->d, vol, gradient->d); break;
        }
        if (s != YG_OK) break;
    }
    if (s == YG_OK && ndofs > 0) {
        k_divide_rows<<<stream_grid(ctx, ndofs * nsd), kThreads, 0, ctx->stream>>>(ndofs, nsd, vol, gradient->d);
        YG_LAUNCHED(ctx);
    }
    dev_free(ctx, vol);
    if (s != YG_OK) return s;
    YG_CUDA(cudaGetLastError());
    return YG_OK;
}
