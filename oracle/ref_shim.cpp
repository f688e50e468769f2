// ref_shim.cpp -- C-ABI over the reference's own handmade linear algebra and
// quadrature, compiled in place from the YAFEL source tree by oracle/Makefile
// into oracle/_ref/libyafel_ref.so.  TEST INFRASTRUCTURE ONLY: used to pin the
// oracle and as the timed CPU baseline; the product never loads it.
//
// Wrapped reference code:
//   include/old_handmade_linalg/sparse_csr.hpp:90-149      sparse_csr(triplets)
//   include/old_handmade_linalg/sparse_bcsr.hpp:93-176     sparse_bcsr<B>(triplets)
//   include/old_handmade_linalg/csr_spmv.hpp:25-56         csr_spmv (OpenMP)
//   include/old_handmade_linalg/bcsr_spmv.hpp:23-62        bcsr_spmv
//   include/old_handmade_linalg/solver/iterative/*.hpp     cg/pcg/bicgstab, Jacobi, ILU(0)
//   src/quadrature/QuadratureRule.cpp, TriangleQuadratureRules.cpp
#include "old_handmade_linalg/sparse_csr.hpp"
#include "old_handmade_linalg/sparse_bcsr.hpp"
#include "old_handmade_linalg/Vector.hpp"
#include "old_handmade_linalg/operators.hpp"
#include "old_handmade_linalg/solver/iterative/cg_solve.hpp"
#include "old_handmade_linalg/solver/iterative/pcg_solve.hpp"
#include "old_handmade_linalg/solver/iterative/bicgstab_solve.hpp"
#include "old_handmade_linalg/solver/iterative/JacobiPreconditioner.hpp"
#include "old_handmade_linalg/solver/iterative/ILUPreconditioner.hpp"
#include "quadrature/QuadratureRule.hpp"

#include <cstdint>
#include <vector>
#include <tuple>

using namespace yafel;
using Trip = std::tuple<std::size_t, std::size_t, double>;

static std::vector<Trip> make_trips(const int64_t *r, const int64_t *c, const double *v, int64_t n) {
    std::vector<Trip> t;
    t.reserve(n);
    for (int64_t i = 0; i < n; ++i) t.emplace_back((std::size_t)r[i], (std::size_t)c[i], v[i]);
    return t;
}
static Vector<double> to_vec(const double *x, int64_t n) {
    Vector<double> v((std::size_t)n, 0.0);
    for (int64_t i = 0; i < n; ++i) v(i) = x[i];
    return v;
}


// ---- quadrature ----
extern "C" int ref_gauss_1d(int lobatto, int n, double *x, double *w) {
    QuadratureRule q(n, lobatto ? QuadratureRule::QuadratureType::GAUSS_LOBATTO
                                : QuadratureRule::QuadratureType::GAUSS_LEGENDRE);
    for (std::size_t i = 0; i < q.weights.size(); ++i) { x[i] = q.nodes[i](0); w[i] = q.weights[i]; }
    return (int)q.weights.size();
}
extern "C" int ref_tensor_rule(int lobatto, int dim, int order, double *pts, double *w) {
    auto q = QuadratureRule::make_tensor_product(
        lobatto ? QuadratureRule::QuadratureType::GAUSS_LOBATTO : QuadratureRule::QuadratureType::GAUSS_LEGENDRE,
        dim, order);
    for (std::size_t i = 0; i < q.weights.size(); ++i) {
        for (int k = 0; k < 3; ++k) pts[3 * i + k] = q.nodes[i](k);
        w[i] = q.weights[i];
    }
    return (int)q.weights.size();
}
extern "C" int ref_triangle_rule(int order, double *pts, double *w) {
    QuadratureRule q;
    q.get_triangle_quadrature(order);
    for (std::size_t i = 0; i < q.weights.size(); ++i) {
        for (int k = 0; k < 3; ++k) pts[3 * i + k] = q.nodes[i](k);
        w[i] = q.weights[i];
    }
    return (int)q.weights.size();
}

// ---- sparse_csr ----
extern "C" void *ref_csr_from_triplets(const int64_t *r, const int64_t *c, const double *v, int64_t n) {
    return new sparse_csr<double>(make_trips(r, c, v, n));
}
extern "C" void ref_csr_info(void *h, int64_t *rows, int64_t *cols, int64_t *nnz) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    *rows = (int64_t)A->rows(); *cols = (int64_t)A->cols(); *nnz = (int64_t)A->nnz();
}
extern "C" void ref_csr_get(void *h, int64_t *row_ptr, int64_t *col, double *val) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    for (std::size_t i = 0; i < A->row_ptr.size(); ++i) row_ptr[i] = (int64_t)A->row_ptr[i];
    for (std::size_t i = 0; i < A->col_index.size(); ++i) { col[i] = (int64_t)A->col_index[i]; val[i] = A->_data[i]; }
}
// The bridge from the current stack to the handmade one (the reference has
// none): Eigen's ColMajor compressed tangent (column pointers, row indices,
// values) as a triplet list, then the reference's own sparse_csr(triplets).
extern "C" void *ref_csr_from_csc(int64_t n, const int *col_ptr, const int *row_idx, const double *val) {
    std::vector<Trip> t;
    t.reserve((std::size_t)col_ptr[n]);
    for (int64_t c = 0; c < n; ++c)
        for (int k = col_ptr[c]; k < col_ptr[c + 1]; ++k) t.emplace_back((std::size_t)row_idx[k], (std::size_t)c, val[k]);
    return new sparse_csr<double>(t);
}
extern "C" void ref_csr_free(void *h) { delete static_cast<sparse_csr<double> *>(h); }
extern "C" void ref_csr_spmv(void *h, const double *x, double *y) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    Vector<double> xv = to_vec(x, (int64_t)A->cols());
    Vector<double> yv = (*A) * xv;
    for (std::size_t i = 0; i < yv.size(); ++i) y[i] = yv(i);
}

// ---- sparse_bcsr<B> ----
template <unsigned B>
static void *bcsr_make(const int64_t *r, const int64_t *c, const double *v, int64_t n) {
    return new sparse_bcsr<B, double>(make_trips(r, c, v, n));
}
extern "C" void *ref_bcsr_from_triplets(int block, const int64_t *r, const int64_t *c, const double *v, int64_t n) {
    if (block == 1) return bcsr_make<1>(r, c, v, n);
    if (block == 2) return bcsr_make<2>(r, c, v, n);
    if (block == 3) return bcsr_make<3>(r, c, v, n);
    return nullptr;
}
template <unsigned B>
static void bcsr_info_t(void *h, int64_t *nbrows, int64_t *nnzb) {
    auto *A = static_cast<sparse_bcsr<B, double> *>(h);
    *nbrows = (int64_t)A->brow_ptr.size() - 1;
    *nnzb = (int64_t)A->bcol_index.size();
}
extern "C" void ref_bcsr_info(int block, void *h, int64_t *nbrows, int64_t *nnzb) {
    if (block == 1) bcsr_info_t<1>(h, nbrows, nnzb);
    if (block == 2) bcsr_info_t<2>(h, nbrows, nnzb);
    if (block == 3) bcsr_info_t<3>(h, nbrows, nnzb);
}
template <unsigned B>
static void bcsr_get_t(void *h, int64_t *brow_ptr, int64_t *bcol, double *val) {
    auto *A = static_cast<sparse_bcsr<B, double> *>(h);
    for (std::size_t i = 0; i < A->brow_ptr.size(); ++i) brow_ptr[i] = (int64_t)A->brow_ptr[i];
    for (std::size_t i = 0; i < A->bcol_index.size(); ++i) bcol[i] = (int64_t)A->bcol_index[i];
    for (std::size_t i = 0; i < A->data.size(); ++i) val[i] = A->data[i];
}
extern "C" void ref_bcsr_get(int block, void *h, int64_t *brow_ptr, int64_t *bcol, double *val) {
    if (block == 1) bcsr_get_t<1>(h, brow_ptr, bcol, val);
    if (block == 2) bcsr_get_t<2>(h, brow_ptr, bcol, val);
    if (block == 3) bcsr_get_t<3>(h, brow_ptr, bcol, val);
}
template <unsigned B>
static void bcsr_spmv_t(void *h, const double *x, double *y) {
    auto *A = static_cast<sparse_bcsr<B, double> *>(h);
    Vector<double> xv = to_vec(x, (int64_t)A->cols());
    Vector<double> yv = (*A) * xv;
    for (std::size_t i = 0; i < yv.size(); ++i) y[i] = yv(i);
}
extern "C" void ref_bcsr_spmv(int block, void *h, const double *x, double *y) {
    if (block == 1) bcsr_spmv_t<1>(h, x, y);
    if (block == 2) bcsr_spmv_t<2>(h, x, y);
    if (block == 3) bcsr_spmv_t<3>(h, x, y);
}
extern "C" void ref_bcsr_free(int block, void *h) {
    if (block == 1) delete static_cast<sparse_bcsr<1, double> *>(h);
    if (block == 2) delete static_cast<sparse_bcsr<2, double> *>(h);
    if (block == 3) delete static_cast<sparse_bcsr<3, double> *>(h);
}

// ---- solvers (x0 in x, solution out in x) ----
extern "C" void ref_cg(void *h, const double *b, double *x, double tol) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    int64_t n = (int64_t)A->rows();
    auto r = cg_solve(*A, to_vec(b, n), to_vec(x, n), tol);
    for (int64_t i = 0; i < n; ++i) x[i] = r(i);
}
template <unsigned B>
static void bcsr_cg_t(void *h, const double *b, double *x, double tol) {
    auto *A = static_cast<sparse_bcsr<B, double> *>(h);
    int64_t n = (int64_t)A->rows();
    auto r = cg_solve(*A, to_vec(b, n), to_vec(x, n), tol);
    for (int64_t i = 0; i < n; ++i) x[i] = r(i);
}
extern "C" void ref_bcsr_cg(int block, void *h, const double *b, double *x, double tol) {
    if (block == 1) bcsr_cg_t<1>(h, b, x, tol);
    if (block == 2) bcsr_cg_t<2>(h, b, x, tol);
    if (block == 3) bcsr_cg_t<3>(h, b, x, tol);
}
extern "C" void ref_pcg_jacobi(void *h, const double *b, double *x, double tol) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    int64_t n = (int64_t)A->rows();
    JacobiPreconditioner<double> M(*A);
    auto r = pcg_solve(*A, to_vec(b, n), M, to_vec(x, n), tol);
    for (int64_t i = 0; i < n; ++i) x[i] = r(i);
}
extern "C" void ref_pcg_ilu(void *h, const double *b, double *x, double tol) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    int64_t n = (int64_t)A->rows();
    ILUPreconditioner<double> M(*A);
    auto r = pcg_solve(*A, to_vec(b, n), M, to_vec(x, n), tol);
    for (int64_t i = 0; i < n; ++i) x[i] = r(i);
}
extern "C" void ref_bicgstab(void *h, const double *b, double *x) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    int64_t n = (int64_t)A->rows();
    auto r = bicgstab_solve(*A, to_vec(b, n), to_vec(x, n));
    for (int64_t i = 0; i < n; ++i) x[i] = r(i);
}
// ILU(0) factors as a CSR handle (same pattern as A)
extern "C" void *ref_ilu_factor(void *h) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    ILUPreconditioner<double> M(*A);
    return new sparse_csr<double>(M.getILU());
}
extern "C" void ref_ilu_apply(void *h, double *z) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    ILUPreconditioner<double> M(*A);
    int64_t n = (int64_t)A->rows();
    Vector<double> v = to_vec(z, n);
    M.solve(v);
    for (int64_t i = 0; i < n; ++i) z[i] = v(i);
}
extern "C" void ref_jacobi_apply(void *h, double *z) {
    auto *A = static_cast<sparse_csr<double> *>(h);
    JacobiPreconditioner<double> M(*A);
    int64_t n = (int64_t)A->rows();
    Vector<double> v = to_vec(z, n);
    M.solve(v);
    for (int64_t i = 0; i < n; ++i) z[i] = v(i);
}

