// host_fe.h -- host-side finite-element setup: quadrature, reference elements,
// the CG DoF numbering and element colouring.  Setup work that the reference
// also does on the host; its output is uploaded once per mesh.
#pragma once
#include <cstdint>
#include <vector>

namespace yg {

enum { TOPO_TENSOR = 0, TOPO_SIMPLEX = 1, TOPO_NONE = 2 };
enum { CELL_LINE2 = 0, CELL_TRI3 = 1, CELL_TET4 = 2, CELL_QUAD4 = 3, CELL_HEX8 = 4, CELL_POINT1 = 5 };

void gauss_legendre_1d(int n, double *x, double *w);
void gauss_lobatto_1d(int n, double *x, double *w);
int tensor_rule(bool lobatto, int dim, int order, std::vector<double> &pts, std::vector<double> &w);
int triangle_rule(int order, std::vector<double> &pts, std::vector<double> &w);
int tetrahedron_rule(int order, std::vector<double> &pts, std::vector<double> &w);

// Reference-element tables of one ElementType.
struct ElementTable {
    int topology = TOPO_NONE, dim = 0, p = 0;
    int nen = 0, nq = 0;
    std::vector<double> local_nodes;  // nen*3
    std::vector<double> qpts, qw;     // nq*3, nq
    std::vector<double> N;            // nq*nen
    std::vector<double> dN;           // nq*nen*dim
};
bool make_element_table(int topology, int dim, int p, ElementTable &T);

// Element topology and topological dimension of a mesh CellType code
// (DoFManager::CellType_to_ElementType, src/utils/DoFManager.cpp:107-141).
void cell_element_type(int cell_type, int &topology, int &topo_dim);

struct HostDofmap {
    int32_t dof_per_node = 1, poly_order = 1;
    std::vector<double> nodes;          // 3 per dof node
    std::vector<int32_t> offsets;       // n_cells+1
    std::vector<int32_t> elements;
    std::vector<int8_t> topology, topo_dim, porder;
    int32_t n_nodes() const { return (int32_t)(nodes.size() / 3); }
    int32_t n_cells() const { return (int32_t)topology.size(); }
};
// Meshes with at most this many raw element nodes are numbered with the
// reference's own comparison sort (see build_dofmap).
constexpr int64_t kReferenceOrderMaxRawNodes = int64_t(1) << 20;

// The raw-node layout of make_raw_dofs for p > 1: the local node table of each
// element type present, and d.offsets (the raw nodes of cell c start at
// d.offsets[c]); d.topology and d.topo_dim must be set.  Returns the number of
// raw nodes.
struct RawLayout {
    std::vector<double> loc[3][4];  // [topology][dim]: nloc x 3 local coordinates
    int nloc[3][4] = {{0}};
};
int64_t raw_node_layout(int32_t n_cells, int32_t p, HostDofmap &d, RawLayout &lay);
// True when the merge order must be the reference's own comparison sort
// (meshes of at most kReferenceOrderMaxRawNodes raw nodes, or simplices mixed
// with tensor cells at p >= 3); otherwise a stable sort gives the same numbering.
bool raw_mix_needs_reference_order(const HostDofmap &d, int64_t n_raw);

// DoFManager(M, CG, p, dpn): returns false for p < 1.
bool build_dofmap(const double *xyz, int32_t n_nodes, const int32_t *cell_nodes, const int32_t *cell_offsets,
                  const int32_t *cell_types, int32_t n_cells, int32_t p, int32_t dpn, HostDofmap &out);

// Greedy colouring of the cells with topo_dim == nsd so that cells of one
// colour share no node.  Returns the number of colours; cells of colour c are
// listed in ascending order in order[ptr[c] .. ptr[c+1]).
int color_cells(const HostDofmap &d, int nsd, int topology, std::vector<int32_t> &order, std::vector<int32_t> &ptr);

}  // namespace yg
