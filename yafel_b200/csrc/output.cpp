// output.cpp -- VTU output of a solution held on the device.
//
// Replaces SimulationOutput(fname_base, BackendType::VTU) + captureFrame(FESystem&)
// with its default capture (include/output/SimulationOutput.hpp:47-116,
// src/output/SimulationOutput.cpp, src/output/VTUBackend.cpp:20-269,
// src/output/OutputMesh.cpp:10-50): one ASCII UnstructuredGrid file whose points
// are the dof nodes and whose cells are the linear sub-cells of every element's
// local mesh, with one scalar array per solution component.  The text is the
// reference's, character for character: the same tags and order, numbers in the
// stream's default format (six significant digits, as printf "%g").
//
// The solution is streamed off the device in chunks through two pinned host
// buffers: the copy of the next chunk overlaps the formatting of this one.
#include "internal.h"
#include "host_fe.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace yg {

const HostDofmap &dofmap_host(yg_dofmap d);  // assembly.cu

namespace {

// Linear sub-cells of an element's local mesh and their VTK cell types
// (make_tensorproduct_element.cpp:35-110, make_simplex_element.cpp:41-90;
// VTUBackend.cpp:247-262 maps Line2/Quad4/Hex8/Tri3 to 3/9/12/5 and the
// Point1 cells of a tetrahedron's local mesh to 2).
struct SubCells {
    std::vector<int> nodes, offsets, types;
};

SubCells local_sub_cells(int topology, int dim, int p) {
    SubCells s;
    const int n = p + 1;
    s.offsets.push_back(0);
    auto add = [&](std::initializer_list<int> c, int type) {
        s.nodes.insert(s.nodes.end(), c);
        s.offsets.push_back((int)s.nodes.size());
        s.types.push_back(type);
    };
    if (topology == TOPO_TENSOR || dim == 1) {
        if (dim == 1) {
            for (int i = 0; i + 1 < n; ++i) add({i, i + 1}, 3);
        } else if (dim == 2) {
            for (int i = 0; i + 1 < n; ++i)
                for (int j = 0; j + 1 < n; ++j) add({i * n + j, i * n + j + 1, (i + 1) * n + j + 1, (i + 1) * n + j}, 9);
        } else {
            const int js = n, is = n * n;
            for (int i = 0; i + 1 < n; ++i)
                for (int j = 0; j + 1 < n; ++j)
                    for (int k = 0; k + 1 < n; ++k) {
                        const int c = i * is + j * js + k;
                        add({c, c + 1, c + 1 + js, c + js, c + is, c + is + 1, c + is + 1 + js, c + is + js}, 12);
                    }
        }
    } else if (dim == 2) {  // triangles: rows of the Blyth-Pozrikidis node layout
        int idx = 0;
        for (int layer = 0; layer < p; ++layer) {
            for (int i = 0; i < p - layer; ++i) {
                add({idx + i, idx + i + 1, idx + i + 1 + p - layer}, 5);
                if (i < p - layer - 1) add({idx + i + 1, idx + i + 2 + p - layer, idx + i + 1 + p - layer}, 5);
            }
            idx += p + 1 - layer;
        }
    } else {  // tetrahedra: one vertex cell per local node
        const int nen = (n * (n + 1) * (n + 2)) / 6;
        for (int a = 0; a < nen; ++a) add({a}, 2);
    }
    return s;
}

// Buffered text output: formats into a large buffer, writes it in blocks.
struct Writer {
    FILE *f = nullptr;
    std::vector<char> buf;
    size_t len = 0;
    bool ok = true;
    explicit Writer(FILE *fp) : f(fp), buf(1 << 22) {}
    void flush() {
        if (len && fwrite(buf.data(), 1, len, f) != len) ok = false;
        len = 0;
    }
    void reserve(size_t n) {
        if (len + n > buf.size()) flush();
    }
    void str(const char *s) {
        const size_t n = strlen(s);
        reserve(n);
        memcpy(buf.data() + len, s, n);
        len += n;
    }
    void num(double v, char sep) {  // the stream default: %g
        reserve(40);
        len += (size_t)snprintf(buf.data() + len, 40, "%g%c", v, sep);
    }
    void inum(long long v, char sep) {
        reserve(24);
        len += (size_t)snprintf(buf.data() + len, 24, "%lld%c", v, sep);
    }
};

}  // namespace
}  // namespace yg

using namespace yg;

extern "C" yg_status yg_output_vtu(yg_dofmap d, const char *fname_base, yg_vector solution) {
    if (!d || !fname_base) return fail(YG_BAD_ARG, "yg_output_vtu: NULL argument");
    const HostDofmap &h = dofmap_host(d);
    const int dpn = h.dof_per_node;
    const int32_t nn = h.n_nodes(), nc = h.n_cells();
    const int64_t nvals = solution ? solution->n : 0;
    if (solution && !solution->ctx) return fail(YG_BAD_ARG, "yg_output_vtu: vector without a context");
    // default capture: point data unless the vector holds dpn values per cell
    const bool cell_data = solution && (int64_t)dpn * nc == nvals;
    if (solution && !cell_data && nvals != (int64_t)dpn * nn)
        return fail(YG_BAD_ARG, "yg_output_vtu: the solution needs %lld (points) or %lld (cells) entries",
                    (long long)dpn * nn, (long long)dpn * nc);
    const std::string fname = std::string(fname_base) + ".vtu";
    FILE *fp = fopen(fname.c_str(), "wb");
    if (!fp) return fail(YG_BAD_ARG, "yg_output_vtu: cannot open %s", fname.c_str());
    std::unique_ptr<FILE, int (*)(FILE *)> guard(fp, fclose);
    Writer w(fp);

    // expanded sub-cell topology (OutputMesh.cpp:18-47)
    SubCells tabs[2][4];
    bool have[2][4] = {{false}};
    std::vector<int> per_cell(nc, 0);
    int64_t n_sub = 0, n_conn = 0;
    for (int32_t c = 0; c < nc; ++c) {
        const int t = h.topology[c], td = h.topo_dim[c];
        if (t == TOPO_NONE) continue;
        if (!have[t][td]) {
            tabs[t][td] = local_sub_cells(t, td, h.poly_order);
            have[t][td] = true;
        }
        per_cell[c] = (int)tabs[t][td].types.size();
        n_sub += per_cell[c];
        n_conn += (int64_t)tabs[t][td].nodes.size();
    }

    w.str("<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\">\n");
    w.str(("<UnstructuredGrid>\n<Piece NumberOfPoints=\"" + std::to_string(nn) + "\" NumberOfCells=\"" +
           std::to_string(n_sub) + "\">\n").c_str());
    w.str("<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (int32_t i = 0; i < nn; ++i) {
        w.num(h.nodes[3 * (int64_t)i], ' ');
        w.num(h.nodes[3 * (int64_t)i + 1], ' ');
        w.num(h.nodes[3 * (int64_t)i + 2], '\n');
    }
    w.str("</DataArray>\n</Points>\n<Cells>\n<DataArray type=\"UInt32\" Name=\"connectivity\" format=\"ascii\">\n");
    for (int32_t c = 0; c < nc; ++c) {
        if (!per_cell[c]) continue;
        const SubCells &s = tabs[h.topology[c]][h.topo_dim[c]];
        const int32_t *g = h.elements.data() + h.offsets[c];
        for (size_t k = 0; k + 1 < s.offsets.size(); ++k)
            for (int a = s.offsets[k]; a < s.offsets[k + 1]; ++a) w.inum(g[s.nodes[a]], a + 1 < s.offsets[k + 1] ? ' ' : '\n');
    }
    w.str("</DataArray>\n<DataArray type=\"UInt32\" Name=\"offsets\" format=\"ascii\">\n");
    int64_t off = 0;
    for (int32_t c = 0; c < nc; ++c) {
        if (!per_cell[c]) continue;
        const SubCells &s = tabs[h.topology[c]][h.topo_dim[c]];
        for (size_t k = 0; k + 1 < s.offsets.size(); ++k) {
            off += s.offsets[k + 1] - s.offsets[k];
            w.inum(off, '\n');
        }
    }
    w.str("</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n");
    for (int32_t c = 0; c < nc; ++c) {
        if (!per_cell[c]) continue;
        for (int ty : tabs[h.topology[c]][h.topo_dim[c]].types) w.inum(ty, '\n');
    }
    w.str("</DataArray>\n</Cells>\n");

    yg_status st = YG_OK;
    if (solution && nvals > 0) {
        // the whole vector, streamed in chunks through two pinned buffers
        yg_context ctx = solution->ctx;
        const int64_t chunk = std::min<int64_t>(nvals, int64_t(1) << 21);
        double *pin[2] = {nullptr, nullptr};
        cudaEvent_t ev[2] = {nullptr, nullptr};
        std::vector<double> vals((size_t)nvals);
        for (int b = 0; b < 2 && st == YG_OK; ++b) {
            if (cudaMallocHost(&pin[b], sizeof(double) * chunk) != cudaSuccess ||
                cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming) != cudaSuccess)
                st = fail(YG_CUDA_ERROR, "yg_output_vtu: pinned staging buffers");
        }
        auto issue = [&](int64_t start, int b) {
            const int64_t m = std::min(chunk, nvals - start);
            cudaMemcpyAsync(pin[b], solution->d + start, sizeof(double) * m, cudaMemcpyDeviceToHost, ctx->stream);
            cudaEventRecord(ev[b], ctx->stream);
        };
        if (st == YG_OK) issue(0, 0);
        for (int64_t start = 0, b = 0; st == YG_OK && start < nvals; start += chunk, b ^= 1) {
            if (start + chunk < nvals) issue(start + chunk, (int)(b ^ 1));
            if (cudaEventSynchronize(ev[b]) != cudaSuccess) { st = fail(YG_CUDA_ERROR, "yg_output_vtu: copy"); break; }
            memcpy(vals.data() + start, pin[b], sizeof(double) * std::min(chunk, nvals - start));
        }
        for (int b = 0; b < 2; ++b) {
            if (ev[b]) cudaEventDestroy(ev[b]);
            if (pin[b]) cudaFreeHost(pin[b]);
        }
        if (st == YG_OK) {
            // one scalar array per component (default_capture, SimulationOutput.hpp:66-88)
            w.str(cell_data ? "<CellData>\n" : "<PointData>\n");
            for (int comp = 0; comp < dpn; ++comp) {
                w.str(("<DataArray type=\"Float32\" format=\"ascii\" Name=\"Solution_" + std::to_string(comp) +
                       "\" NumberOfComponents=\"1\">\n").c_str());
                if (cell_data) {  // a parent cell's value on each of its sub-cells
                    for (int32_t c = 0; c < nc; ++c)
                        for (int k = 0; k < per_cell[c]; ++k) w.num(vals[(int64_t)c * dpn + comp], '\n');
                } else {
                    for (int32_t i = 0; i < nn; ++i) w.num(vals[(int64_t)i * dpn + comp], '\n');
                }
                w.str("</DataArray>\n");
            }
            w.str(cell_data ? "</CellData>\n" : "</PointData>\n");
        }
    }
    w.str("</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
    w.flush();
    if (st != YG_OK) return st;
    if (!w.ok) return fail(YG_BAD_ARG, "yg_output_vtu: write to %s failed", fname.c_str());
    return YG_OK;
}
