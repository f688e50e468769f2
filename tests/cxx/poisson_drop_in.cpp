// A reference-style application written against the C++ adapters: the
// BasicPoisson flow (apps/BasicPoisson/main.cpp:94-120) and the handmade
// linear-algebra tests (test/test_cg_solve.cpp), on the GPU.  Prints
// "name value" lines that tests/test_gpu_cxx.py checks against the oracle.
#include "yafel_gpu/yafel_gpu.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>

using namespace yafel::gpu;

int main(int argc, char **argv) {
    int n = argc > 1 ? std::atoi(argv[1]) : 16;
    // unit square, n x n Q1 cells, corners in the element's x-fastest order
    Mesh M;
    for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) M.nodes.push_back({double(i) / n, double(j) / n, 0.0});
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            int a = j * (n + 1) + i;
            M.offsets.push_back((int)M.cellNodes.size());
            for (int c : {a, a + 1, a + n + 1, a + n + 2}) M.cellNodes.push_back(c);
            M.cellTypes.push_back(CellType::Quad4);
        }
    M.offsets.push_back((int)M.cellNodes.size());

    DoFManager dofm(M, DoFManager::ManagerType::CG, 1, 1);
    FESystem feSystem(dofm, 2, YG_FORMAT_CSR);
    CGAssembly<PoissonEquation<2>>(feSystem);
    DirichletBC bc0(dofm, 0.0);
    bc0.selectByFunction([](const coordinate &x) {
        return std::abs(x[0]) < 1e-6 || std::abs(x[0] - 1) < 1e-6 || std::abs(x[1]) < 1e-6 || std::abs(x[1] - 1) < 1e-6;
    });
    bc0.apply(feSystem.getGlobalTangent(), feSystem.getGlobalResidual());
    JacobiPreconditioner<double> Mj(feSystem.getGlobalTangent());
    yg_solve_stats st = solve_system(feSystem, &Mj, 1e-10);
    Vector<double> u = feSystem.getSolution().download();
    double umax = 0;
    for (std::size_t i = 0; i < u.size(); ++i) umax = std::fmax(umax, u(i));
    std::printf("dofs %zu\nnnz %zu\niterations %lld\nrelres %.3e\numax %.17g\n", u.size(),
                feSystem.getGlobalTangent().nnz(), (long long)st.iterations, st.rel_residual, umax);

    // test/test_cg_solve.cpp test_2 with the reference's own call spellings
    std::vector<triplet<double>> ts;
    for (std::size_t i = 0; i < 10; ++i) ts.emplace_back(i, i, -2.0);
    for (std::size_t i = 1; i < 10; ++i) { ts.emplace_back(i, i - 1, 1.0); ts.emplace_back(i - 1, i, 1.0); }
    sparse_csr<double> A(ts);
    Vector<double> xref(10);
    for (int i = 0; i < 10; ++i) xref(i) = i;
    Vector<double> rhs = A * xref;
    Vector<double> x = cg_solve(A, rhs);
    double err = 0;
    for (int i = 0; i < 10; ++i) err += (x(i) - xref(i)) * (x(i) - xref(i));
    std::printf("laplace_err2 %.3e\n", err);
    JacobiPreconditioner<double> MJ(A);
    Vector<double> xp = pcg_solve(A, rhs, MJ, Vector<double>(10, 0.0), 1e-20);
    double errp = 0;
    for (int i = 0; i < 10; ++i) errp += (xp(i) - xref(i)) * (xp(i) - xref(i));
    std::printf("laplace_pcg_err2 %.3e\n", errp);
    return 0;
}
