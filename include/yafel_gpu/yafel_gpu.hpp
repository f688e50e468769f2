// yafel_gpu.hpp -- header-only C++ adapters with the reference's spellings over
// the C ABI of yafel_gpu.h.  Code written against the reference's
//   DoFManager / FESystem / CGAssembly<Physics> / LocalSmoothingGradient<Physics> /
//   ZZGradientRecovery<Physics> / SimulationOutput (VTU) / Mesh(gmsh file) / DirichletBC
//   sparse_csr / sparse_bcsr / cg_solve / pcg_solve / bicgstab_solve /
//   JacobiPreconditioner / ILUPreconditioner / IdentityPreconditioner
// switches to the GPU by including this header and using namespace yafel::gpu.
// Failures throw std::runtime_error, as the reference throws where it reports
// errors (src/utils/DoFManager.cpp:162, EigenCholesky.hpp:45-53).
#pragma once

#include "../yafel_gpu.h"

#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace yafel {
namespace gpu {

inline void check(yg_status s, const char *what) {
    if (s != YG_OK) throw std::runtime_error(std::string(what) + ": " + yg_last_error());
}

// One device, one stream; process-wide default on device 0.
class Context {
public:
    explicit Context(int device = 0, uint64_t hbm_budget = 0) { check(yg_context_create(device, hbm_budget, &h_), "yg_context_create"); }
    ~Context() { yg_context_destroy(h_); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    yg_context get() const { return h_; }
    static Context &instance() {
        static Context c(0);
        return c;
    }

private:
    yg_context h_ = nullptr;
};

using coordinate = std::array<double, 3>;

// Vector<double> (include/old_handmade_linalg/Vector.hpp): host storage; solvers
// return results by value, like the reference.
template <typename T = double>
class Vector {
public:
    explicit Vector(std::size_t n = 0, T v = T(0)) : d_(n, v) {}
    T &operator()(std::size_t i) { return d_[i]; }
    T operator()(std::size_t i) const { return d_[i]; }
    std::size_t size() const { return d_.size(); }
    T *data() { return d_.data(); }
    const T *data() const { return d_.data(); }
    T dot(const Vector &o) const {
        T s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        std::size_t NN = (size() / 4) * 4;
        for (std::size_t i = 0; i < NN; i += 4) {
            s0 += d_[i] * o.d_[i]; s1 += d_[i + 1] * o.d_[i + 1]; s2 += d_[i + 2] * o.d_[i + 2]; s3 += d_[i + 3] * o.d_[i + 3];
        }
        for (std::size_t i = NN; i < size(); ++i) s0 += d_[i] * o.d_[i];
        return s0 + s1 + s2 + s3;
    }
    bool operator==(const Vector &o) const { return d_ == o.d_; }

private:
    std::vector<T> d_;
};

// RAII device vector
class DeviceVector {
public:
    DeviceVector(Context &ctx, int64_t n) { check(yg_vector_create(ctx.get(), n, &h_), "yg_vector_create"); }
    DeviceVector(Context &ctx, const Vector<double> &v) : DeviceVector(ctx, (int64_t)v.size()) { upload(v); }
    ~DeviceVector() { yg_vector_destroy(h_); }
    DeviceVector(const DeviceVector &) = delete;
    DeviceVector &operator=(const DeviceVector &) = delete;
    void upload(const Vector<double> &v) { check(yg_vector_upload(h_, v.data(), (int64_t)v.size()), "upload"); }
    Vector<double> download() const {
        Vector<double> v((std::size_t)yg_vector_size(h_));
        check(yg_vector_download(h_, v.data(), (int64_t)v.size()), "download");
        return v;
    }
    yg_vector get() const { return h_; }
    int64_t size() const { return yg_vector_size(h_); }

private:
    yg_vector h_ = nullptr;
};

// ------------------------------------------------------------------ sparse matrices

template <typename T>
using triplet = std::tuple<std::size_t, std::size_t, T>;

class matrix_base {
public:
    yg_matrix get() const { return h_.get(); }
    std::size_t rows() const { return (std::size_t)sizes()[0]; }
    std::size_t cols() const { return (std::size_t)sizes()[1]; }
    std::size_t nnz() const { return (std::size_t)sizes()[2]; }
    Context &context() const { return *ctx_; }

protected:
    matrix_base(Context &ctx, yg_matrix h) : ctx_(&ctx), h_(h, [](yg_matrix m) { yg_matrix_destroy(m); }) {}
    std::array<int64_t, 3> sizes() const {
        int64_t r, c, n;
        int32_t b;
        check(yg_matrix_sizes(h_.get(), &r, &c, &n, &b), "yg_matrix_sizes");
        return {r, c, n};
    }
    Context *ctx_;
    std::shared_ptr<yg_matrix_t> h_;
};

template <typename T>
static yg_matrix from_triplets(Context &ctx, int block, const std::vector<triplet<T>> &ts) {
    std::vector<uint64_t> r(ts.size()), c(ts.size());
    std::vector<double> v(ts.size());
    for (std::size_t i = 0; i < ts.size(); ++i) {
        r[i] = std::get<0>(ts[i]);
        c[i] = std::get<1>(ts[i]);
        v[i] = (double)std::get<2>(ts[i]);
    }
    yg_matrix h = nullptr;
    check(yg_matrix_from_triplets(ctx.get(), block, r.data(), c.data(), v.data(), ts.size(), &h), "sparse matrix from triplets");
    return h;
}

// sparse_csr<T>(triplets) (include/old_handmade_linalg/sparse_csr.hpp:90-149), on the GPU.
template <typename dataType = double>
class sparse_csr : public matrix_base {
public:
    using triplet = gpu::triplet<dataType>;
    explicit sparse_csr(const std::vector<triplet> &ts, Context &ctx = Context::instance())
        : matrix_base(ctx, from_triplets(ctx, 1, ts)) {}
    sparse_csr(Context &ctx, yg_matrix adopted) : matrix_base(ctx, adopted) {}
};

// sparse_bcsr<BLOCK,T>(triplets) (include/old_handmade_linalg/sparse_bcsr.hpp:93-176), on the GPU.
template <unsigned BLOCK, typename dataType = double>
class sparse_bcsr : public matrix_base {
public:
    using triplet = gpu::triplet<dataType>;
    explicit sparse_bcsr(const std::vector<triplet> &ts, Context &ctx = Context::instance())
        : matrix_base(ctx, from_triplets(ctx, BLOCK, ts)) {}
    sparse_bcsr(Context &ctx, yg_matrix adopted) : matrix_base(ctx, adopted) {}
};

// operator*(A, x) -> new Vector (operators.hpp:117-131)
inline Vector<double> operator*(const matrix_base &A, const Vector<double> &x) {
    DeviceVector dx(A.context(), x), dy(A.context(), (int64_t)A.rows());
    check(yg_spmv(A.get(), dx.get(), dy.get()), "spmv");
    return dy.download();
}

// ------------------------------------------------------------------ preconditioners

class Preconditioner {
public:
    yg_precond get() const { return h_.get(); }
    // M.solve(z) in place (Preconditioner.hpp:9-21)
    void solve(Vector<double> &z) const {
        DeviceVector d(*ctx_, z);
        check(yg_precond_apply(h_.get(), d.get()), "M.solve");
        z = d.download();
    }

protected:
    Preconditioner(const matrix_base &A, int kind) : ctx_(&A.context()) {
        yg_precond p = nullptr;
        check(yg_precond_create(A.get(), kind, &p), "preconditioner");
        h_.reset(p, [](yg_precond q) { yg_precond_destroy(q); });
    }
    Context *ctx_;
    std::shared_ptr<yg_precond_t> h_;
};

template <typename dataType = double>
class JacobiPreconditioner : public Preconditioner {
public:
    explicit JacobiPreconditioner(const matrix_base &A) : Preconditioner(A, YG_PRECOND_JACOBI) {}
};
template <typename dataType = double>
class ILUPreconditioner : public Preconditioner {
public:
    explicit ILUPreconditioner(const matrix_base &A) : Preconditioner(A, YG_PRECOND_ILU0) {}
};
template <typename MT = void, typename dataType = double>
class IdentityPreconditioner : public Preconditioner {
public:
    explicit IdentityPreconditioner(const matrix_base &A) : Preconditioner(A, YG_PRECOND_IDENTITY) {}
};

// ------------------------------------------------------------------ solvers

constexpr double CG_SOLVER_TOL = 1.0e-14;  // cg_solve.hpp:21

inline Vector<double> solve_impl(const matrix_base &A, const Preconditioner *M, const Vector<double> &rhs,
                                 const Vector<double> &x0, double TOL, bool bicg, yg_solve_stats *stats = nullptr) {
    DeviceVector b(A.context(), rhs), x(A.context(), x0);
    yg_solve_opts o{YG_CRIT_REFERENCE, YG_PREC_FP64, TOL, 0, 0, 0};
    yg_solve_stats st{};
    yg_status s = bicg ? yg_bicgstab(A.get(), M ? M->get() : nullptr, b.get(), x.get(), &o, &st)
                       : yg_cg(A.get(), M ? M->get() : nullptr, b.get(), x.get(), &o, &st);
    // the reference returns silently after maxiter (cg_solve.hpp:56); so do we
    if (s != YG_OK && s != YG_NOT_CONVERGED) check(s, bicg ? "bicgstab_solve" : "cg_solve");
    if (stats) *stats = st;
    return x.download();
}

// cg_solve(A, rhs[, x0][, TOL]) (solver/iterative/cg_solve.hpp:23-81)
inline Vector<double> cg_solve(const matrix_base &A, const Vector<double> &rhs, const Vector<double> &x0,
                               double TOL = CG_SOLVER_TOL) {
    return solve_impl(A, nullptr, rhs, x0, TOL, false);
}
inline Vector<double> cg_solve(const matrix_base &A, const Vector<double> &rhs, double TOL = CG_SOLVER_TOL) {
    return cg_solve(A, rhs, Vector<double>(rhs.size(), 0.0), TOL);
}
// pcg_solve(A, rhs, M[, x0][, TOL]) (pcg_solve.hpp:115-178); the reference's
// 4-argument overload drops M (pcg_solve.hpp:31) and does not compile when
// instantiated; here it passes M on.
inline Vector<double> pcg_solve(const matrix_base &A, const Vector<double> &rhs, const Preconditioner &M,
                                const Vector<double> &x0, double TOL = CG_SOLVER_TOL) {
    return solve_impl(A, &M, rhs, x0, TOL, false);
}
inline Vector<double> pcg_solve(const matrix_base &A, const Vector<double> &rhs, const Preconditioner &M,
                                double TOL = CG_SOLVER_TOL) {
    return pcg_solve(A, rhs, M, Vector<double>(rhs.size(), 0.0), TOL);
}
// bicgstab_solve(A, rhs[, x0]) (bicgstab_solve.hpp:207-283)
inline Vector<double> bicgstab_solve(const matrix_base &A, const Vector<double> &rhs, const Vector<double> &x0) {
    return solve_impl(A, nullptr, rhs, x0, 1.0e-14, true);
}
inline Vector<double> bicgstab_solve(const matrix_base &A, const Vector<double> &rhs) {
    return bicgstab_solve(A, rhs, Vector<double>(rhs.size(), 0.0));
}

// ------------------------------------------------------------------ mesh, DoFs, system

enum class CellType : int { Line2 = 0, Tri3 = 1, Tet4 = 2, Quad4 = 3, Hex8 = 4, Point1 = 5, None = 6 };

// Mesh(DefinitionScheme::Explicit, nodes, cellNodes, offsets, cellTypes, cellTags)
// (include/mesh/Mesh.hpp:48-53)
struct Mesh {
    std::vector<coordinate> nodes;
    std::vector<int> cellNodes, offsets;
    std::vector<CellType> cellTypes;
    std::vector<std::vector<int>> cellTags;
    int nCells() const { return (int)cellTypes.size(); }
    int nNodes() const { return (int)nodes.size(); }
};

class DoFManager {
public:
    enum class ManagerType { CG, DG };
    DoFManager(const Mesh &M, ManagerType type, int polyOrder, int dof_per_node = 1, Context &ctx = Context::instance())
        : dof_per_node(dof_per_node), polyOrder(polyOrder), ctx_(&ctx) {
        if (type != ManagerType::CG) throw std::runtime_error("DoFManager: only ManagerType::CG is on the GPU path");
        std::vector<double> xyz(3 * M.nodes.size());
        for (std::size_t i = 0; i < M.nodes.size(); ++i)
            for (int k = 0; k < 3; ++k) xyz[3 * i + k] = M.nodes[i][k];
        std::vector<int32_t> ct(M.cellTypes.size());
        for (std::size_t i = 0; i < ct.size(); ++i) ct[i] = (int32_t)M.cellTypes[i];
        yg_dofmap d = nullptr;
        check(yg_dofmap_create(ctx.get(), xyz.data(), M.nNodes(), M.cellNodes.data(), M.offsets.data(), ct.data(),
                               M.nCells(), polyOrder, dof_per_node, &d),
              "DoFManager");
        h_.reset(d, [](yg_dofmap p) { yg_dofmap_destroy(p); });
        int32_t nn, nc;
        int64_t ne, nd;
        check(yg_dofmap_sizes(d, &nn, &nc, &ne, &nd), "yg_dofmap_sizes");
        std::vector<double> X(3 * (std::size_t)nn);
        element_offsets.resize(nc + 1);
        elements.resize(ne);
        check(yg_dofmap_get(d, X.data(), element_offsets.data(), elements.data(), nullptr, nullptr, nullptr), "yg_dofmap_get");
        dof_nodes.resize(nn);
        for (int32_t i = 0; i < nn; ++i) dof_nodes[i] = {X[3 * i], X[3 * i + 1], X[3 * i + 2]};
        cell_region_idx.resize(M.nCells());
        for (int c = 0; c < M.nCells(); ++c)
            cell_region_idx[c] = (c < (int)M.cellTags.size() && !M.cellTags[c].empty()) ? M.cellTags[c][0] : 0;
    }
    void getGlobalDofs(int elnum, std::vector<int> &out) const {
        out.clear();
        for (int i = element_offsets[elnum]; i < element_offsets[elnum + 1]; ++i)
            for (int d = 0; d < dof_per_node; ++d) out.push_back(elements[i] * dof_per_node + d);
    }
    void getGlobalNodes(int elnum, std::vector<int> &out) const {
        out.assign(elements.begin() + element_offsets[elnum], elements.begin() + element_offsets[elnum + 1]);
    }
    int nCells() const { return (int)element_offsets.size() - 1; }
    int nNodes() const { return (int)dof_nodes.size(); }
    yg_dofmap get() const { return h_.get(); }
    Context &context() const { return *ctx_; }

    int dof_per_node, polyOrder;
    std::vector<coordinate> dof_nodes;
    std::vector<int> element_offsets, elements, cell_region_idx;

private:
    Context *ctx_;
    std::shared_ptr<yg_dofmap_t> h_;
};

// FESystem(DoFManager&, dim) (include/fe_system/FESystem.hpp:18-56): tangent,
// residual and solution live on the device.
class FESystem {
public:
    explicit FESystem(DoFManager &dofm, int dim = 0, int format = YG_FORMAT_BCSR)
        : dofm(dofm), dim_(dim), format_(format),
          residual_(dofm.context(), (int64_t)dofm.nNodes() * dofm.dof_per_node),
          solution_(dofm.context(), (int64_t)dofm.nNodes() * dofm.dof_per_node) {}
    matrix_base &getGlobalTangent() {
        if (!tangent_) throw std::runtime_error("FESystem: tangent not assembled");
        return *tangent_;
    }
    DeviceVector &getGlobalResidual() { return residual_; }
    DeviceVector &getSolution() { return solution_; }
    // the nodal gradient of the last LocalSmoothingGradient call: n_dofs * nsd
    // entries, row-major (one row of nsd derivatives per dof)
    DeviceVector &getSolutionGradient() {
        if (!gradient_) throw std::runtime_error("FESystem: no solution gradient computed");
        return *gradient_;
    }
    void reset_gradient(int nsd) {
        const int64_t n = (int64_t)dofm.nNodes() * dofm.dof_per_node * nsd;
        if (!gradient_ || gradient_->size() != n) gradient_.reset(new DeviceVector(dofm.context(), n));
    }
    DoFManager &getDoFManager() { return dofm; }
    double &currentTime() { return time_; }
    int format() const { return format_; }
    void adopt_tangent(yg_matrix K) {
        if (!tangent_) tangent_.reset(new sparse_csr<double>(dofm.context(), K));
    }
    yg_matrix tangent_handle() const { return tangent_ ? tangent_->get() : nullptr; }

    DoFManager &dofm;

private:
    int dim_, format_;
    double time_ = 0;
    DeviceVector residual_, solution_;
    std::unique_ptr<matrix_base> tangent_;
    std::unique_ptr<DeviceVector> gradient_;
};

enum class AssemblyRequirement : int { Residual, Tangent, DtMass, LumpedDtMassInverse, DtDtMass };

// Device physics with the reference apps' Physics names; static members give
// the parameters (the reference's Physics is a struct of static functions).
template <int NSD>
struct PoissonEquation {
    static constexpr int nsd() { return NSD; }
    double sign = 1.0, f = 1.0;
    yg_physics physics() const { yg_physics p{YG_POISSON, NSD, {sign, f}}; return p; }
};
template <int NSD>
struct LinearElasticity {
    static constexpr int nsd() { return NSD; }
    double Youngs = 1.0, nu = 0.3, sign = 1.0;
    std::array<double, 3> body{{0, 0, 0}};
    yg_physics physics() const {
        double lambda = (Youngs * nu) / ((1 + nu) * (1 - 2 * nu)), mu = Youngs / (2 * (1 + nu));
        yg_physics p{YG_ELASTICITY, NSD, {sign, lambda, mu, body[0], body[1], body[2]}};
        return p;
    }
};
template <int NSD>
struct AdvectionDiffusionSUPG {
    static constexpr int nsd() { return NSD; }
    double k = 0.1, h = 0.1, U0 = 1.0, Q = 0.0;  // supg_advection.hpp:110-113
    yg_physics physics() const { yg_physics p{YG_SUPG, NSD, {k, h, U0, Q}}; return p; }
};

// CGAssembly<Physics>(FESystem&, requirements) (include/assembly/CGAssembly.hpp:27-186)
template <typename Physics>
void CGAssembly(FESystem &fe, std::vector<AssemblyRequirement> requirements = {AssemblyRequirement::Residual,
                                                                              AssemblyRequirement::Tangent},
                const Physics &physics = Physics()) {
    uint32_t mask = 0;
    for (auto r : requirements) {
        if (r == AssemblyRequirement::Residual) mask |= YG_REQ_RESIDUAL;
        if (r == AssemblyRequirement::Tangent) mask |= YG_REQ_TANGENT;
    }
    yg_physics p = physics.physics();
    yg_matrix K = fe.tangent_handle();
    check(yg_assemble(fe.dofm.get(), &p, mask, fe.format(), &K, fe.getGlobalResidual().get()), "CGAssembly");
    if (mask & YG_REQ_TANGENT) fe.adopt_tangent(K);
}

// LocalSmoothingGradient<Physics>(FESystem&)
// (include/assembly/LocalSmoothingGradient.hpp:20-94): the gradient of the
// solution averaged to the dofs with weights N_A jxw over the cells of dimension
// Physics::nsd(); read it with fe.getSolutionGradient().
template <typename Physics>
void LocalSmoothingGradient(FESystem &fe) {
    fe.reset_gradient(Physics::nsd());
    check(yg_local_smoothing_gradient(fe.dofm.get(), Physics::nsd(), fe.getSolution().get(),
                                      fe.getSolutionGradient().get()),
          "LocalSmoothingGradient");
}

// ZZGradientRecovery<Physics>(FESystem&) (include/assembly/ZZGradientRecovery.hpp:33-140):
// Zienkiewicz-Zhu patch recovery of the gradient of a p = 1 scalar solution;
// read it with fe.getSolutionGradient() (n_nodes * nsd entries, row-major).
template <typename Physics>
void ZZGradientRecovery(FESystem &fe) {
    fe.reset_gradient(Physics::nsd());
    check(yg_zz_gradient_recovery(fe.dofm.get(), Physics::nsd(), fe.getSolution().get(),
                                  fe.getSolutionGradient().get()),
          "ZZGradientRecovery");
}

// SimulationOutput (include/output/SimulationOutput.hpp:22-116) with the VTU
// backend: captureFrame(fe) writes fname_base.vtu, the reference's text.
enum class BackendType { VTU };
class SimulationOutput {
public:
    explicit SimulationOutput(std::string fname_base = "output", BackendType = BackendType::VTU)
        : base_(std::move(fname_base)) {}
    void captureFrame(FESystem &fe) {
        check(yg_output_vtu(fe.getDoFManager().get(), base_.c_str(), fe.getSolution().get()),
              "SimulationOutput::captureFrame");
    }

private:
    std::string base_;
};

// Mesh(const std::string &fname) (src/mesh/parse_gmsh.cpp:80-193): a Gmsh 2.x file.
inline Mesh read_gmsh(const std::string &fname) {
    yg_mesh h = nullptr;
    check(yg_mesh_read_gmsh(fname.c_str(), &h), "Mesh(fname)");
    int32_t nn = 0, nc = 0;
    int64_t ncn = 0, nt = 0;
    yg_mesh_sizes(h, &nn, &nc, &ncn, &nt);
    std::vector<double> xyz(3 * (size_t)nn);
    std::vector<int32_t> cn(ncn), off(nc + 1), ct(nc), to(nc + 1), tg(nt);
    yg_mesh_get(h, xyz.data(), cn.data(), off.data(), ct.data(), to.data(), tg.data());
    yg_mesh_destroy(h);
    Mesh m;
    m.nodes.resize(nn);
    for (int32_t i = 0; i < nn; ++i) m.nodes[i] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    m.cellNodes.assign(cn.begin(), cn.end());
    m.offsets.assign(off.begin(), off.end());
    for (int32_t c = 0; c < nc; ++c) {
        m.cellTypes.push_back(static_cast<CellType>(ct[c]));
        m.cellTags.emplace_back(tg.begin() + to[c], tg.begin() + to[c + 1]);
    }
    return m;
}

// DirichletBC (include/boundary_conditions/DirichletBC.hpp:23-89)
class DirichletBC {
public:
    DirichletBC(const DoFManager &dofm, double bcval, int comp = 0)
        : dofm_(dofm), component_(comp), value_func_([bcval](const coordinate &, double) { return bcval; }) {}
    DirichletBC(const DoFManager &dofm, std::function<double(const coordinate &, double)> f, int comp = 0)
        : dofm_(dofm), component_(comp), value_func_(std::move(f)) {}
    template <typename Lambda>
    void selectByFunction(Lambda &&func) {
        for (int i = 0; i < dofm_.nNodes(); ++i)
            if (func(dofm_.dof_nodes[i])) bc_nodes_.push_back(i);
    }
    void selectByRegionID(int region_id) {
        std::vector<int> nodes;
        for (int c = 0; c < dofm_.nCells(); ++c)
            if (dofm_.cell_region_idx[c] == region_id) {
                dofm_.getGlobalNodes(c, nodes);
                for (int n : nodes) bc_nodes_.push_back(n);
            }
        // std::unique over the list, as DirichletBC.cpp:116-117 does
        std::vector<int> u;
        for (int n : bc_nodes_) if (u.empty() || u.back() != n) u.push_back(n);
        bc_nodes_.swap(u);
    }
    void apply(matrix_base &A, DeviceVector &rhs, double time = 0.0) {
        std::vector<int64_t> dofs;
        std::vector<double> vals;
        for (int n : bc_nodes_) {
            dofs.push_back((int64_t)n * dofm_.dof_per_node + component_);
            vals.push_back(value_func_(dofm_.dof_nodes[n], time));
        }
        check(yg_dirichlet_apply(A.get(), rhs.get(), dofs.data(), vals.data(), (int64_t)dofs.size()), "DirichletBC::apply");
    }
    std::vector<int> &getNodes() { return bc_nodes_; }

private:
    const DoFManager &dofm_;
    int component_;
    std::function<double(const coordinate &, double)> value_func_;
    std::vector<int> bc_nodes_;
};

// Solve the assembled system on the device to a relative residual (no host
// round trip of the matrix); returns the statistics.
inline yg_solve_stats solve_system(FESystem &fe, const Preconditioner *M, double relres = 1e-10,
                                   int precision = YG_PREC_FP64) {
    yg_solve_opts o{YG_CRIT_RELRES, precision, relres, 0, 0, 0};
    yg_solve_stats st{};
    yg_status s = yg_cg(fe.getGlobalTangent().get(), M ? M->get() : nullptr, fe.getGlobalResidual().get(),
                        fe.getSolution().get(), &o, &st);
    if (s != YG_OK && s != YG_NOT_CONVERGED) check(s, "solve_system");
    return st;
}

}  // namespace gpu
}  // namespace yafel
