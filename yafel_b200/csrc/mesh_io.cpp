// mesh_io.cpp -- mesh ingest: Gmsh 2.x ASCII files into the explicit mesh arrays.
//
// Replaces Mesh(const std::string &fname) / Mesh::parse_gmsh
// (include/mesh/Mesh.hpp:56-59, src/mesh/Mesh.cpp:32-36,
// src/mesh/parse_gmsh.cpp:80-193).  Same reading as the reference: the $Nodes
// block fills node id-1 with its three coordinates; the $Elements block gives
// element id-1 its cell type (Gmsh 1/2/3/4/5/15 -> Line2/Tri3/Quad4/Tet4/Hex8/
// Point1, anything else None), its tags and its node count, while the element
// node lists are appended in file order (0-based); other sections are skipped.
// The whole file is read at once and parsed in memory.
#include "internal.h"

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

struct yg_mesh_t {
    std::vector<double> nodes;  // 3 per node
    std::vector<int32_t> cell_nodes, offsets, types, tag_offsets, tags;
};

namespace yg {
namespace {

int gmsh_cell_type(long t) {
    switch (t) {
    case 1: return 0;   // Line2
    case 2: return 1;   // Tri3
    case 3: return 3;   // Quad4
    case 4: return 2;   // Tet4
    case 5: return 4;   // Hex8
    case 15: return 5;  // Point1
    default: return 6;  // None
    }
}

// Tokens of one line (separated by blanks; a trailing carriage return is a blank).
void split(const char *b, const char *e, std::vector<std::pair<const char *, const char *>> &w) {
    w.clear();
    while (b < e) {
        while (b < e && (*b == ' ' || *b == '\t' || *b == '\r')) ++b;
        const char *s = b;
        while (b < e && *b != ' ' && *b != '\t' && *b != '\r') ++b;
        if (b > s) w.emplace_back(s, b);
    }
}

bool to_long(std::pair<const char *, const char *> t, long *v) {
    std::string s(t.first, t.second);
    char *end = nullptr;
    errno = 0;
    *v = strtol(s.c_str(), &end, 10);
    return errno == 0 && end && *end == 0;
}

bool to_double(std::pair<const char *, const char *> t, double *v) {
    std::string s(t.first, t.second);
    char *end = nullptr;
    errno = 0;
    *v = strtod(s.c_str(), &end);
    return end && *end == 0;
}

}  // namespace
}  // namespace yg

using namespace yg;

extern "C" yg_status yg_mesh_read_gmsh(const char *path, yg_mesh *out) {
    if (!path || !out) return fail(YG_BAD_ARG, "yg_mesh_read_gmsh: NULL argument");
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(YG_BAD_ARG, "Mesh::parse_gmsh: cannot open %s", path);
    std::vector<char> text;
    char chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) text.insert(text.end(), chunk, chunk + got);
    fclose(f);
    auto *m = new yg_mesh_t();
    enum { NONE, NODES, ELEMENTS } action = NONE;
    std::vector<std::pair<const char *, const char *>> w;
    std::vector<std::vector<int32_t>> tags;
    int64_t offset = 0, nlines = 0;
    const char *p = text.data(), *end = text.data() + text.size();
    auto fail_line = [&](const char *what) {
        delete m;
        return fail(YG_BAD_ARG, "Mesh::parse_gmsh: %s at line %lld of %s", what, (long long)nlines, path);
    };
    auto next_line = [&](const char *&b, const char *&e) {
        b = p;
        while (p < end && *p != '\n') ++p;
        e = p;
        if (p < end) ++p;
        ++nlines;
    };
    while (p < end) {
        const char *b, *e;
        next_line(b, e);
        split(b, e, w);
        if (w.empty()) continue;
        const std::string head(w[0].first, w[0].second);
        if (head == "$Nodes" || head == "$Elements") {
            const char *cb, *ce;
            next_line(cb, ce);
            split(cb, ce, w);
            long count = 0;
            if (w.empty() || !to_long(w[0], &count) || count < 0) return fail_line("bad count");
            if (head == "$Nodes") {
                action = NODES;
                m->nodes.assign(3 * (size_t)count, 0.0);
            } else {
                action = ELEMENTS;
                m->offsets.assign((size_t)count + 1, 0);
                m->types.assign((size_t)count, 0);  // value-initialised CellType, as cellTypes_.resize
                tags.assign((size_t)count, {});
                m->cell_nodes.reserve(4 * (size_t)count);
            }
            continue;
        }
        if (head == "$EndNodes" || head == "$EndElements") {
            action = NONE;
            continue;
        }
        if (action == NODES) {
            long id;
            if (w.size() < 4 || !to_long(w[0], &id)) return fail_line("bad node line");
            if (id < 1 || 3 * (size_t)id > m->nodes.size()) return fail_line("node id out of range");
            for (int k = 0; k < 3; ++k)
                if (!to_double(w[1 + k], &m->nodes[3 * (size_t)(id - 1) + k])) return fail_line("bad coordinate");
        } else if (action == ELEMENTS) {
            long id, type, ntags;
            if (w.size() < 3 || !to_long(w[0], &id) || !to_long(w[1], &type) || !to_long(w[2], &ntags))
                return fail_line("bad element line");
            if (id < 1 || (size_t)id > m->types.size()) return fail_line("element id out of range");
            if (ntags < 0 || (size_t)(3 + ntags) > w.size()) return fail_line("bad tag count");
            m->types[id - 1] = gmsh_cell_type(type);
            std::vector<int32_t> &t = tags[id - 1];
            t.clear();
            for (long i = 0; i < ntags; ++i) {
                long v;
                if (!to_long(w[3 + i], &v)) return fail_line("bad tag");
                t.push_back((int32_t)v);
            }
            const int64_t nodes_in_el = (int64_t)w.size() - ntags - 3;
            for (size_t i = 3 + ntags; i < w.size(); ++i) {
                long v;
                if (!to_long(w[i], &v)) return fail_line("bad node index");
                m->cell_nodes.push_back((int32_t)(v - 1));
            }
            m->offsets[id - 1] = (int32_t)offset;
            offset += nodes_in_el;
        }
    }
    if (!m->offsets.empty()) m->offsets.back() = (int32_t)offset;
    m->tag_offsets.assign(1, 0);
    for (auto &t : tags) {
        m->tags.insert(m->tags.end(), t.begin(), t.end());
        m->tag_offsets.push_back((int32_t)m->tags.size());
    }
    const int64_t nn = (int64_t)m->nodes.size() / 3;
    for (int32_t v : m->cell_nodes)
        if (v < 0 || v >= nn) {
            delete m;
            return fail(YG_BAD_ARG, "Mesh::parse_gmsh: an element references node %d of %lld in %s", v + 1,
                        (long long)nn, path);
        }
    *out = m;
    return YG_OK;
}

extern "C" yg_status yg_mesh_sizes(yg_mesh m, int32_t *n_nodes, int32_t *n_cells, int64_t *n_cell_nodes,
                                   int64_t *n_tags) {
    if (!m) return fail(YG_BAD_ARG, "yg_mesh_sizes: NULL mesh");
    if (n_nodes) *n_nodes = (int32_t)(m->nodes.size() / 3);
    if (n_cells) *n_cells = (int32_t)m->types.size();
    if (n_cell_nodes) *n_cell_nodes = (int64_t)m->cell_nodes.size();
    if (n_tags) *n_tags = (int64_t)m->tags.size();
    return YG_OK;
}

extern "C" yg_status yg_mesh_get(yg_mesh m, double *nodes_xyz, int32_t *cell_nodes, int32_t *cell_offsets,
                                 int32_t *cell_types, int32_t *tag_offsets, int32_t *tags) {
    if (!m) return fail(YG_BAD_ARG, "yg_mesh_get: NULL mesh");
    if (nodes_xyz) std::copy(m->nodes.begin(), m->nodes.end(), nodes_xyz);
    if (cell_nodes) std::copy(m->cell_nodes.begin(), m->cell_nodes.end(), cell_nodes);
    if (cell_offsets) std::copy(m->offsets.begin(), m->offsets.end(), cell_offsets);
    if (cell_types) std::copy(m->types.begin(), m->types.end(), cell_types);
    if (tag_offsets) std::copy(m->tag_offsets.begin(), m->tag_offsets.end(), tag_offsets);
    if (tags) std::copy(m->tags.begin(), m->tags.end(), tags);
    return YG_OK;
}

extern "C" yg_status yg_mesh_destroy(yg_mesh m) {
    delete m;
    return YG_OK;
}
