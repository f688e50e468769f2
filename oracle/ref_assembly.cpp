// ref_assembly.cpp -- C-ABI over the reference's own assembly half, compiled in
// place from the YAFEL source tree by oracle/Makefile against the from-scratch
// Eigen-API subset in oracle/ref_compat/ (Eigen is not installed).  TEST
// INFRASTRUCTURE ONLY: it generates golden fixtures, pins the C restatement, and
// is the reference's CPU path timed as the baseline; the product never loads it.
//
// Reference code that runs unmodified through these entry points:
//   src/utils/DoFManager.cpp:11-36,143-229,296-414   DoFManager (CG numbering)
//   src/element/*.cpp, include/element/Element.hpp   Element, ElementFactory, shape functions
//   src/quadrature/*.cpp                             quadrature rules
//   include/fe_system/FESystem.hpp:18-56             FESystem
//   include/assembly/CGAssembly.hpp:27-186           CGAssembly<Physics>
//   src/boundary_conditions/DirichletBC.cpp:58-89    DirichletBC::apply (ColMajor)
//   include/boundary_conditions/DirichletBC.hpp:80-89 selectByFunction
//   include/assembly/LocalSmoothingGradient.hpp:20-94 LocalSmoothingGradient<Physics>
//   include/assembly/ZZGradientRecovery.hpp:33-140   ZZGradientRecovery<Physics>
//   src/output/{SimulationOutput,OutputMesh,VTUBackend}.cpp  VTU output (default capture)
//   apps/supg_learning/supg_advection.hpp:19-132     AdvectionDiffusionSUPG<NSD> (the physics itself)
//
// The Poisson and elasticity Physics structs of the reference live in the apps'
// main.cpp files next to ViennaCL calls, so they cannot be compiled here; the
// two structs below are the plug-ins a user writes for CGAssembly, with the
// tangent and residual formulas of apps/BasicPoisson/main.cpp:31-60 and
// apps/BasicLinearElasticity/main.cpp:63-112 (same loops over A <= B with the
// mirrored entry), generalised to a sign and load parameters.
#include "assembly/CGAssembly.hpp"
#include "assembly/LocalSmoothingGradient.hpp"
#include "assembly/ZZGradientRecovery.hpp"
#include "boundary_conditions/DirichletBC.hpp"
#include "fe_system/FESystem.hpp"
#include "mesh/Mesh.hpp"
#include "output/SimulationOutput.hpp"
#include "utils/DoFManager.hpp"
#include "supg_learning/supg_advection.hpp"

#include <cmath>
#include <cstdint>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace yafel;

namespace {

// Physics parameters are process globals because the reference's Physics
// concept is a set of static functions (CGAssembly.hpp:134-139).
double g_sign = 1.0, g_f = 1.0, g_lambda = 1.0, g_mu = 1.0, g_body[3] = {0, 0, 0};

template <int NSD>
struct PoissonPhysics {
    static constexpr int nsd() { return NSD; }
    static void LocalResidual(const Element &E, int qpi, coordinate<> &, double,
                              Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &,
                              Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &R_el) {
        R_el += (g_f * E.jxw) * E.shapeValues[qpi];
    }
    static void LocalTangent(const Element &E, int, coordinate<> &, double,
                             Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &,
                             Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor>> &K_el) {
        const int n = static_cast<int>(K_el.rows());
        for (int A = 0; A < n; ++A) {
            for (int B = A; B < n; ++B) {
                double d = 0;
                for (int i = 0; i < NSD; ++i) d += E.shapeGrad(A, i) * E.shapeGrad(B, i);
                K_el(A, B) += g_sign * d * E.jxw;
                K_el(B, A) = K_el(A, B);
            }
        }
    }
};

template <int NSD>
struct ElasticityPhysics {
    static constexpr int nsd() { return NSD; }
    static void LocalResidual(const Element &E, int qpi, coordinate<> &, double,
                              Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &,
                              Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &R_el) {
        for (int A = 0; A < static_cast<int>(R_el.rows()); ++A)
            R_el(A) += g_body[A % NSD] * E.shapeValues[qpi](A / NSD) * E.jxw;
    }
    // K_{Ai,Bk} += sign * (lambda dA_i dB_k + mu (delta_ik dA.dB + dA_k dB_i)) jxw,
    // node blocks B >= A, the block below the diagonal mirrored.
    static void LocalTangent(const Element &E, int, coordinate<> &, double,
                             Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &,
                             Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor>> &K_el) {
        const int nn = static_cast<int>(K_el.rows()) / NSD;
        for (int An = 0; An < nn; ++An) {
            for (int Bn = An; Bn < nn; ++Bn) {
                double ab = 0;
                for (int d = 0; d < NSD; ++d) ab += E.shapeGrad(An, d) * E.shapeGrad(Bn, d);
                for (int i = 0; i < NSD; ++i) {
                    for (int k = 0; k < NSD; ++k) {
                        const double c = g_lambda * E.shapeGrad(An, i) * E.shapeGrad(Bn, k) +
                                         g_mu * ((i == k ? ab : 0.0) + E.shapeGrad(An, k) * E.shapeGrad(Bn, i));
                        K_el(An * NSD + i, Bn * NSD + k) += g_sign * c * E.jxw;
                        if (Bn != An) K_el(Bn * NSD + k, An * NSD + i) = K_el(An * NSD + i, Bn * NSD + k);
                    }
                }
            }
        }
    }
};

// Steady SUPG advection-diffusion with run-time constants: the tangent and
// residual of apps/supg_learning/supg_advection.hpp:24-131 (advection summed
// inside the Acomp loop, as there), with k, h, U0 and Q as parameters instead
// of that header's compile-time constants, for problems of any Peclet number.
double g_k = 0.1, g_h = 0.1, g_U0 = 1.0, g_Q = 0.0;

template <int NSD>
struct SupgPhysics {
    static constexpr int nsd() { return NSD; }
    static double alpha() {
        const double Pe = g_U0 * g_h / (2 * g_k);
        return Pe == 0 ? 0.0 : std::cosh(Pe) / std::sinh(Pe) - 1.0 / Pe;
    }
    static void LocalResidual(const Element &E, int qpi, coordinate<> &, double,
                              Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &,
                              Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &R_el) {
        const double a = alpha(), normU = std::abs(g_U0);
        double Uhat[NSD] = {0};
        if (normU > 0) Uhat[0] = (a * g_h / 2) * g_U0 * (1.0 / normU);
        for (int A = 0; A < E.localMesh.nNodes(); ++A)
            for (int i = 0; i < NSD; ++i)
                R_el(A) -= (E.shapeValues[qpi](A) * g_Q + Uhat[i] * E.shapeGrad(A, i)) * E.jxw;
    }
    static void LocalTangent(const Element &E, int qpi, coordinate<> &, double,
                             Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, 1>> &,
                             Eigen::Map<Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor>> &K_el) {
        const double a = alpha(), normU = std::abs(g_U0);
        double U[NSD] = {0}, K[NSD][NSD];
        U[0] = g_U0;
        for (int i = 0; i < NSD; ++i)
            for (int j = 0; j < NSD; ++j) K[i][j] = (i == j ? 1.0 : 0.0) * g_k;
        if (normU > 0) {
            const double c = a * g_h / (normU * 2);
            for (int i = 0; i < NSD; ++i)
                for (int j = 0; j < NSD; ++j) K[i][j] += c * (U[i] * U[j]);
        }
        const int n = E.localMesh.nNodes();
        for (int A = 0; A < n; ++A)
            for (int ac = 0; ac < NSD; ++ac)
                for (int B = 0; B < n; ++B)
                    for (int bc = 0; bc < NSD; ++bc)
                        K_el(A, B) += (E.shapeValues[qpi](A) * U[bc] * E.shapeGrad(B, bc) +
                                       E.shapeGrad(A, ac) * E.shapeGrad(B, bc) * K[ac][bc]) * E.jxw;
    }
};

struct RefMesh {
    Mesh mesh;
    DoFManager dofm;
    RefMesh(const Mesh &m, int p, int dpn) : mesh(m), dofm(mesh, DoFManager::ManagerType::CG, p, dpn) {}
};

struct RefSystem {
    RefMesh *m;
    FESystem sys;
    explicit RefSystem(RefMesh *mm, int nsd) : m(mm), sys(mm->dofm, nsd) {}
};

template <template <int> class P>
void assemble_nsd(FESystem &s, int nsd, const std::vector<AssemblyRequirement> &req) {
    if (nsd == 1) CGAssembly<P<1>>(s, req);
    if (nsd == 2) CGAssembly<P<2>>(s, req);
    if (nsd == 3) CGAssembly<P<3>>(s, req);
}

template <int NSD>
struct SupgSteady : AdvectionDiffusionSUPG<NSD, Steady> {};

}  // namespace

extern "C" {

// Worker threads of the OpenMP loops (CGAssembly's element loop). One thread
// makes the triplet list element-ordered, hence the duplicate sums deterministic.
void refa_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// Mesh(const std::string &fname) (parse_gmsh.cpp:80-171): sizes, then arrays
// (call with NULL arrays first).  tag_offsets/tags hold each cell's tags.
int refa_read_gmsh(const char *path, int *n_nodes, int *n_cells, int *n_cell_nodes, int *n_tags, double *xyz,
                   int *cell_nodes, int *offsets, int *types, int *tag_offsets, int *tags) {
    try {
        Mesh m{std::string(path)};
        *n_nodes = m.nNodes();
        *n_cells = m.nCells();
        *n_cell_nodes = static_cast<int>(m.getCellVector().size());
        int nt = 0;
        for (int c = 0; c < m.nCells(); ++c) nt += static_cast<int>(m.getCellTags(c).size());
        *n_tags = nt;
        if (!xyz) return 0;
        for (int i = 0; i < m.nNodes(); ++i)
            for (int k = 0; k < 3; ++k) xyz[3 * i + k] = m.getGeometryNodes()[i](k);
        for (std::size_t i = 0; i < m.getCellVector().size(); ++i) cell_nodes[i] = m.getCellVector()[i];
        for (std::size_t i = 0; i < m.getOffsetVector().size(); ++i) offsets[i] = m.getOffsetVector()[i];
        int k = 0;
        tag_offsets[0] = 0;
        for (int c = 0; c < m.nCells(); ++c) {
            types[c] = static_cast<int>(m.getCellType(c));
            for (int t : m.getCellTags(c)) tags[k++] = t;
            tag_offsets[c + 1] = k;
        }
        return 0;
    } catch (...) {
        return 1;
    }
}

// Mesh(DefinitionScheme::Explicit, nodes, cells, offsets, types, tags) + DoFManager(M, CG, p, dpn).
void *refa_dofmanager(const double *xyz, int n_nodes, const int *cells, const int *offsets, const int *types,
                      int n_cells, int p, int dpn) {
    std::vector<coordinate<>> nodes(n_nodes);
    for (int i = 0; i < n_nodes; ++i)
        for (int k = 0; k < 3; ++k) nodes[i](k) = xyz[3 * i + k];
    std::vector<int> cn(cells, cells + offsets[n_cells]);
    std::vector<int> off(offsets, offsets + n_cells + 1);
    std::vector<CellType> ct(n_cells);
    for (int c = 0; c < n_cells; ++c) ct[c] = static_cast<CellType>(types[c]);
    std::vector<std::vector<int>> tags(n_cells, std::vector<int>{0});
    Mesh m(Mesh::DefinitionScheme::Explicit, nodes, cn, off, ct, tags);
    try {
        return new RefMesh(m, p, dpn);
    } catch (...) {
        return nullptr;
    }
}
void refa_dofmanager_free(void *h) { delete static_cast<RefMesh *>(h); }
void refa_dofmanager_sizes(void *h, int *n_dof_nodes, int *n_cells, int *n_entries) {
    auto &d = static_cast<RefMesh *>(h)->dofm;
    *n_dof_nodes = d.nNodes();
    *n_cells = d.nCells();
    *n_entries = static_cast<int>(d.elements.size());
}
void refa_dofmanager_get(void *h, double *xyz, int *element_offsets, int *elements, int8_t *topo, int8_t *topo_dim,
                         int8_t *order) {
    auto &d = static_cast<RefMesh *>(h)->dofm;
    for (int i = 0; i < d.nNodes(); ++i)
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = d.dof_nodes[i](k);
    for (std::size_t i = 0; i < d.element_offsets.size(); ++i) element_offsets[i] = d.element_offsets[i];
    for (std::size_t i = 0; i < d.elements.size(); ++i) elements[i] = d.elements[i];
    for (int c = 0; c < d.nCells(); ++c) {
        topo[c] = static_cast<int8_t>(d.element_types[c].elementTopology);
        topo_dim[c] = d.element_types[c].topoDim;
        order[c] = d.element_types[c].polyOrder;
    }
}

// Element(ElementType{topology, dim, p}, 1, qrm) (src/element/Element.cpp:11-31):
// sizes of its tables; any output pointer may be NULL.  local_xyz: nen x 3 local
// nodes; qp_xyz: nq x 3 points; w: nq weights; N: nq x nen values;
// dN: nq x nen x dim reference gradients (shapeGradXi, row-major).
void refa_element(int topology, int dim, int p, int qrm, int *nen, int *nq, double *local_xyz, double *qp_xyz,
                  double *w, double *N, double *dN) {
    Element E(ElementType(static_cast<ElementTopology>(topology), dim, p), 1, qrm);
    const int ne = E.localMesh.nNodes(), q = E.nQP();
    *nen = ne;
    *nq = q;
    auto const &ln = E.localMesh.getGeometryNodes();
    for (int a = 0; a < ne && local_xyz; ++a)
        for (int k = 0; k < 3; ++k) local_xyz[3 * a + k] = ln[a](k);
    for (int i = 0; i < q; ++i) {
        for (int k = 0; k < 3 && qp_xyz; ++k) qp_xyz[3 * i + k] = E.quadratureRule.nodes[i](k);
        if (w) w[i] = E.quadratureRule.weights[i];
        for (int a = 0; a < ne; ++a) {
            if (N) N[(size_t)i * ne + a] = E.shapeValues[i](a);
            for (int d = 0; d < dim && dN; ++d) dN[((size_t)i * ne + a) * dim + d] = E.shapeGradXi[i](a, d);
        }
    }
}

// FESystem(dofm, nsd) + CGAssembly<Physics>(sys, {Residual?, Tangent?}).
// kind 0: Poisson {sign, f}; 1: elasticity {sign, lambda, mu, b0, b1, b2};
// 2: the reference's steady AdvectionDiffusionSUPG (its own constants);
// 3: the same SUPG formulas with params {k, h, U0, Q}.
void *refa_assemble(void *mesh, int kind, int nsd, const double *params, int want_tangent, int want_residual) {
    auto *m = static_cast<RefMesh *>(mesh);
    auto *s = new RefSystem(m, nsd);
    std::vector<AssemblyRequirement> req;
    if (want_residual) req.push_back(AssemblyRequirement::Residual);
    if (want_tangent) req.push_back(AssemblyRequirement::Tangent);
    if (kind == 0) {
        g_sign = params[0];
        g_f = params[1];
        assemble_nsd<PoissonPhysics>(s->sys, nsd, req);
    } else if (kind == 1) {
        g_sign = params[0];
        g_lambda = params[1];
        g_mu = params[2];
        for (int k = 0; k < 3; ++k) g_body[k] = params[3 + k];
        assemble_nsd<ElasticityPhysics>(s->sys, nsd, req);
    } else if (kind == 3) {
        g_k = params[0];
        g_h = params[1];
        g_U0 = params[2];
        g_Q = params[3];
        assemble_nsd<SupgPhysics>(s->sys, nsd, req);
    } else {
        assemble_nsd<SupgSteady>(s->sys, nsd, req);
    }
    return s;
}
void refa_system_free(void *h) { delete static_cast<RefSystem *>(h); }
void refa_system_sizes(void *h, int64_t *n_dofs, int64_t *nnz) {
    auto &s = static_cast<RefSystem *>(h)->sys;
    *n_dofs = s.getGlobalTangent().rows();
    *nnz = s.getGlobalTangent().nonZeros();
}
// The tangent in Eigen's ColMajor compressed form (column pointers, row indices,
// values) and the residual vector.
void refa_system_get(void *h, int *col_ptr, int *row_idx, double *val, double *residual) {
    auto &s = static_cast<RefSystem *>(h)->sys;
    auto &K = s.getGlobalTangent();
    for (Eigen::Index c = 0; c <= K.cols(); ++c) col_ptr[c] = K.outerIndexPtr()[c];
    for (Eigen::Index k = 0; k < K.nonZeros(); ++k) {
        row_idx[k] = K.innerIndexPtr()[k];
        val[k] = K.valuePtr()[k];
    }
    auto &R = s.getGlobalResidual();
    for (Eigen::Index i = 0; i < R.rows(); ++i) residual[i] = R(i);
}
void refa_system_set_residual(void *h, const double *r) {
    auto &R = static_cast<RefSystem *>(h)->sys.getGlobalResidual();
    for (Eigen::Index i = 0; i < R.rows(); ++i) R(i) = r[i];
}

// DirichletBC(dofm, value, comp) with selectByFunction(|x(axis) - coord| < tol),
// then apply(K, F): one BC object per call, applied to the system in place.
void refa_dirichlet_plane(void *h, int comp, int axis, double coord, double tol, double value, int *n_selected) {
    auto *s = static_cast<RefSystem *>(h);
    DirichletBC bc(s->m->dofm, value, comp);
    bc.selectByFunction([&](const coordinate<> &x) { return std::abs(x(axis) - coord) < tol; });
    if (n_selected) *n_selected = static_cast<int>(bc.getNodes().size());
    bc.apply(s->sys.getGlobalTangent(), s->sys.getGlobalResidual());
}
// The same with an explicit node list (DirichletBC::getNodes() filled directly).
void refa_dirichlet_nodes(void *h, int comp, const int *nodes, int n, double value) {
    auto *s = static_cast<RefSystem *>(h);
    DirichletBC bc(s->m->dofm, value, comp);
    bc.getNodes().assign(nodes, nodes + n);
    bc.apply(s->sys.getGlobalTangent(), s->sys.getGlobalResidual());
}

// LocalSmoothingGradient<Physics>(sys) on a given solution; gradient row-major (n_dofs x nsd).
void refa_local_smoothing_gradient(void *h, int nsd, const double *solution, double *gradient) {
    auto &s = static_cast<RefSystem *>(h)->sys;
    auto &U = s.getSolution();
    for (Eigen::Index i = 0; i < U.rows(); ++i) U(i) = solution[i];
    if (nsd == 1) LocalSmoothingGradient<PoissonPhysics<1>>(s);
    if (nsd == 2) LocalSmoothingGradient<PoissonPhysics<2>>(s);
    if (nsd == 3) LocalSmoothingGradient<PoissonPhysics<3>>(s);
    auto &G = s.getSolutionGradient();
    for (Eigen::Index i = 0; i < G.rows(); ++i)
        for (int d = 0; d < nsd; ++d) gradient[i * nsd + d] = G(i, d);
}

// ZZGradientRecovery<Physics>(sys) on a given solution (p = 1, one dof per
// node); gradient row-major (n_nodes x nsd).
void refa_zz_gradient(void *h, int nsd, const double *solution, double *gradient) {
    auto &s = static_cast<RefSystem *>(h)->sys;
    auto &U = s.getSolution();
    for (Eigen::Index i = 0; i < U.rows(); ++i) U(i) = solution[i];
    if (nsd == 2) ZZGradientRecovery<PoissonPhysics<2>>(s);
    if (nsd == 3) ZZGradientRecovery<PoissonPhysics<3>>(s);
    auto &G = s.getSolutionGradient();
    for (Eigen::Index i = 0; i < G.rows(); ++i)
        for (int d = 0; d < nsd; ++d) gradient[i * nsd + d] = G(i, d);
}

// SimulationOutput(fname_base, VTU).captureFrame(sys) with the default capture
// of the system's solution (with_solution) or a capture that adds no data.
void refa_write_vtu(void *h, const char *fname_base, const double *solution, int with_solution) {
    auto &s = static_cast<RefSystem *>(h)->sys;
    if (with_solution) {
        auto &U = s.getSolution();
        for (Eigen::Index i = 0; i < U.rows(); ++i) U(i) = solution[i];
    }
    SimulationOutput out(fname_base, BackendType::VTU);
    if (with_solution) {
        out.captureFrame(s);
    } else {
        std::function<void(FESystem &, OutputFrame &)> none = [](FESystem &, OutputFrame &) {};
        out.captureFrame(s, none);
    }
}

}  // extern "C"
