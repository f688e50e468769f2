/*
 * yafel_oracle.h -- CPU restatement of the reference's continuous-Galerkin
 * assemble + solve path.  TEST INFRASTRUCTURE ONLY: the product never links,
 * loads or calls this code.  Tests, the smoke check and the bench's CPU
 * baseline use it as the checker.
 *
 * Every function names the reference file:line it restates (paths are relative
 * to the YAFEL source tree).  Parity pinning: the linear-algebra half and the
 * quadrature are checked against the reference's own code compiled under
 * oracle/_ref (see oracle/Makefile); the assembly half (which needs Eigen3,
 * absent here) is checked against the known answers the reference's tests
 * state (GL/GLL weight sums, Q1 corner gradients, integral of x over the unit
 * square) and against properties (row sums of the Laplacian, patch tests).
 */
#ifndef YAFEL_ORACLE_H
#define YAFEL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Cell types: same codes as the reference's CellType enum
 * (include/mesh/mesh_typedefs.hpp:42-50). */
enum { OR_LINE2 = 0, OR_TRI3 = 1, OR_TET4 = 2, OR_QUAD4 = 3, OR_HEX8 = 4, OR_POINT1 = 5 };
/* Element topologies (include/element/ElementType.hpp:22-27). */
enum { OR_TENSOR = 0, OR_SIMPLEX = 1, OR_NONE = 2 };
/* Physics kinds restated from the reference apps. */
enum { OR_POISSON = 0, OR_ELASTICITY = 1, OR_SUPG = 2 };
/* Preconditioners / stopping criteria. */
enum { OR_PRECOND_NONE = 0, OR_PRECOND_JACOBI = 1, OR_PRECOND_ILU0 = 2 };
enum { OR_CRIT_REFERENCE = 0, OR_CRIT_RELRES = 1 };

typedef struct {
    int64_t nrows, ncols, nnz;
    int64_t *row_ptr; /* nrows+1 */
    int64_t *col;     /* nnz */
    double *val;      /* nnz */
} or_csr;

typedef struct {
    int32_t block;
    int64_t nbrows, nbcols, nnzb;
    int64_t *brow_ptr; /* nbrows+1 */
    int64_t *bcol;     /* nnzb */
    double *val;       /* nnzb*block*block, row-major inside a block */
} or_bcsr;

typedef struct {
    int32_t n_nodes;
    double *nodes;       /* 3*n_nodes */
    int32_t n_cells;
    int32_t *offsets;    /* n_cells+1 */
    int32_t *elements;   /* offsets[n_cells] */
    int8_t *topology;    /* per cell: OR_TENSOR/OR_SIMPLEX/OR_NONE */
    int8_t *topo_dim;    /* per cell */
    int8_t *poly_order;  /* per cell */
} or_dofmap;

/* ---- quadrature (src/quadrature/QuadratureRule.cpp) ---- */
void or_gauss_legendre_1d(int n, double *x, double *w);
void or_gauss_lobatto_1d(int n, double *x, double *w);
int or_tensor_rule(int lobatto, int dim, int order, double *pts, double *w);
int or_triangle_rule(int order, double *pts, double *w);
int or_triangle_rule_collapsed(int order, double *pts, double *w);
void or_set_triangle_rule(int order, const double *pts, const double *w, int n);

/* ---- reference elements ---- */
int or_local_nodes(int topology, int dim, int p, double *pts);
int or_shape_functions(int topology, int dim, int p, const double *qpts, int nq,
                       double *N, double *dN);
int or_element_rule(int topology, int dim, int p, double *pts, double *w);

/* ---- DoFManager ---- */
or_dofmap *or_dofmanager(const double *xyz, int32_t n_nodes, const int32_t *cell_nodes,
                         const int32_t *cell_offsets, const int32_t *cell_types, int32_t n_cells,
                         int32_t p);
void or_free_dofmap(or_dofmap *d);

/* ---- assembly ---- */
or_csr *or_assemble(const or_dofmap *d, int32_t dpn, int32_t nsd, int32_t physics,
                    const double *params, double *residual /* nullable, n_nodes*dpn */);
void or_dirichlet_apply(or_csr *A, double *rhs, const uint8_t *mask, const double *vals);
/* LocalSmoothingGradient: grad is n_nodes*dpn rows of nsd (row-major). */
void or_local_smoothing_gradient(const or_dofmap *d, int32_t dpn, int32_t nsd, const double *sol, double *grad);

/* ---- sparse containers ---- */
or_csr *or_csr_from_triplets(const int64_t *r, const int64_t *c, const double *v, int64_t n);
or_bcsr *or_bcsr_from_triplets(int32_t block, const int64_t *r, const int64_t *c,
                               const double *v, int64_t n);
or_bcsr *or_bcsr_from_csr(const or_csr *A, int32_t block);
void or_free_csr(or_csr *A);
void or_free_bcsr(or_bcsr *A);

/* ---- kernels / solvers ---- */
void or_csr_spmv(const or_csr *A, const double *x, double *y);
void or_bcsr_spmv(const or_bcsr *A, const double *x, double *y);
or_csr *or_ilu0(const or_csr *A);
void or_ilu_solve(const or_csr *F, double *z);
int64_t or_cg(const or_csr *A, const double *b, double *x, int32_t precond, int32_t criterion,
              double tol, int64_t maxiter, double *relres);
int64_t or_bicgstab(const or_csr *A, const double *b, double *x, int32_t criterion, double tol,
                    int64_t maxiter, double *relres);
double or_true_relres(const or_csr *A, const double *b, const double *x);
int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
