/*
 * yafel_gpu.h -- C ABI of the B200 continuous-Galerkin assemble + solve path.
 *
 * The library (yafel_b200/libyafel_b200.so) replaces, for one GPU, the
 * reference's path from the DoF numbering through element assembly, Dirichlet
 * conditions, sparse storage, SpMV, preconditioners and Krylov solvers.  Each
 * entry point names the reference interface it replaces (paths relative to the
 * YAFEL source tree).  Plain pointers and sizes only; all handles are opaque;
 * every call returns a yg_status and never throws.  Host arrays are copied; the
 * library owns all device memory behind a handle.  Calls on one context are
 * not thread-safe (the reference's objects are not either); use one context per
 * thread.
 */
#ifndef YAFEL_GPU_H
#define YAFEL_GPU_H

#include <stddef.h>
#include <stdint.h>

/* Symbols of the shared library; hidden-by-default builds export only these. */
#if defined(YG_BUILD) && defined(__GNUC__)
#define YG_API __attribute__((visibility("default")))
#else
#define YG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum yg_status {
    YG_OK = 0,
    YG_NOT_CONVERGED = 1, /* iteration cap reached (the reference returns silently: cg_solve.hpp:56) */
    YG_BREAKDOWN = 2,     /* p.Ap <= 0, rho = 0 or omega = 0 in a Krylov recurrence */
    YG_NAN = 3,           /* a non-finite scalar appeared */
    YG_TIMEOUT = 4,       /* a bounded device wait expired */
    YG_OUT_OF_MEMORY = 5,
    YG_OVER_BUDGET = 6,   /* the request exceeds the context's HBM budget */
    YG_BAD_ARG = 7,
    YG_CUDA_ERROR = 8,
    YG_UNSUPPORTED = 9,
    YG_ZERO_PIVOT = 10,   /* reported, not fatal: the reference warns and continues */
    YG_RUNNING = 11       /* a batched or served solve still in progress */
} yg_status;

typedef struct yg_context_t *yg_context;
typedef struct yg_dofmap_t *yg_dofmap;
typedef struct yg_matrix_t *yg_matrix;
typedef struct yg_vector_t *yg_vector;
typedef struct yg_precond_t *yg_precond;
typedef struct yg_mesh_t *yg_mesh;

/* ------------------------------------------------------------------ context */

/* One CUDA device, one stream, an HBM budget (0 = no limit).  No reference
 * counterpart: the reference runs in one host process. */
YG_API yg_status yg_context_create(int32_t device, uint64_t hbm_budget_bytes, yg_context *out);
YG_API yg_status yg_context_destroy(yg_context ctx);
YG_API yg_status yg_context_synchronize(yg_context ctx);
YG_API yg_status yg_context_memory(yg_context ctx, uint64_t *in_use, uint64_t *budget);
/* Kernels this context has launched so far (instrumentation for benchmarks). */
YG_API int64_t yg_context_launches(yg_context ctx);
/* Message of the last failed call on this thread; never NULL. */
YG_API const char *yg_last_error(void);
YG_API const char *yg_status_string(yg_status s);

/* ------------------------------------------------------------------ vectors */

/* Device FP64 vector.  Replaces Vector<double> (include/old_handmade_linalg/Vector.hpp:9-158). */
YG_API yg_status yg_vector_create(yg_context ctx, int64_t n, yg_vector *out);
YG_API yg_status yg_vector_destroy(yg_vector v);
YG_API int64_t yg_vector_size(yg_vector v);
YG_API yg_status yg_vector_upload(yg_vector v, const double *host, int64_t n);
YG_API yg_status yg_vector_download(yg_vector v, double *host, int64_t n);
YG_API yg_status yg_vector_fill(yg_vector v, double value);
YG_API yg_status yg_vector_copy(yg_vector dst, yg_vector src);
/* Deterministic dot product; replaces VectorExpression::dot (VectorExpression.hpp:33-54). */
YG_API yg_status yg_vector_dot(yg_vector a, yg_vector b, double *out);
/* y += alpha*x; replaces Vector::operator+= of a scaled expression (Vector.hpp:48-150). */
YG_API yg_status yg_vector_axpy(double alpha, yg_vector x, yg_vector y);

/* ------------------------------------------------------------------ DoFManager */

/* Mesh cell types use the reference's CellType codes (include/mesh/mesh_typedefs.hpp:42-50). */
enum { YG_CELL_LINE2 = 0, YG_CELL_TRI3 = 1, YG_CELL_TET4 = 2, YG_CELL_QUAD4 = 3, YG_CELL_HEX8 = 4, YG_CELL_POINT1 = 5,
       YG_CELL_NONE = 6 };

/* Mesh(const std::string &fname) (include/mesh/Mesh.hpp:56-59, src/mesh/parse_gmsh.cpp:80-193):
 * reads a Gmsh 2.x ASCII file ($Nodes, $Elements; other sections skipped) into
 * host arrays in the layout of Mesh(DefinitionScheme::Explicit, ...): node id-1
 * gets its coordinates, element id-1 its CellType (Gmsh 1/2/3/4/5/15 ->
 * Line2/Tri3/Quad4/Tet4/Hex8/Point1, else None), tags and node count, the node
 * lists follow in file order, 0-based.  YG_BAD_ARG names the offending line. */
YG_API yg_status yg_mesh_read_gmsh(const char *path, yg_mesh *out);
/* Sizes: nodes, cells, entries of the cell-node list, entries of the tag list. */
YG_API yg_status yg_mesh_sizes(yg_mesh m, int32_t *n_nodes, int32_t *n_cells, int64_t *n_cell_nodes,
                        int64_t *n_tags);
/* Copies of the arrays (any pointer may be NULL): nodes (3 per node), cell nodes,
 * cell offsets (n_cells+1), CellType codes, and each cell's tags as
 * tags[tag_offsets[c] .. tag_offsets[c+1]) (Mesh::getCellTags; the first tag is
 * the region id DoFManager keeps, DoFManager.cpp:22-25). */
YG_API yg_status yg_mesh_get(yg_mesh m, double *nodes_xyz, int32_t *cell_nodes, int32_t *cell_offsets,
                      int32_t *cell_types, int32_t *tag_offsets, int32_t *tags);
YG_API yg_status yg_mesh_destroy(yg_mesh m);
/* Element topologies (include/element/ElementType.hpp:22-27). */
enum { YG_TOPO_TENSOR = 0, YG_TOPO_SIMPLEX = 1, YG_TOPO_NONE = 2 };

/* DoFManager(const Mesh&, ManagerType::CG, polyOrder, dof_per_node)
 * (include/utils/DoFManager.hpp:25, src/utils/DoFManager.cpp:11-36,143-229,340-414).
 * nodes_xyz: 3 per node; cells as in Mesh(DefinitionScheme::Explicit, ...)
 * (include/mesh/Mesh.hpp:48-53).  Numbering is identical to the reference's:
 * p=1 keeps the mesh numbering; p>1 merges coincident element nodes sorted on
 * snapped (z,y,x).  Fails with YG_BAD_ARG for polyOrder < 1, as the reference
 * throws (DoFManager.cpp:162).  ctx may be NULL: the numbering is then built on
 * the host only (no device memory) and the dofmap cannot be assembled. */
YG_API yg_status yg_dofmap_create(yg_context ctx, const double *nodes_xyz, int32_t n_nodes,
                           const int32_t *cell_nodes, const int32_t *cell_offsets,
                           const int32_t *cell_types, int32_t n_cells, int32_t poly_order,
                           int32_t dof_per_node, yg_dofmap *out);
/* The same numbering computed on the GPU whatever the mesh size (p > 1; p = 1
 * keeps the mesh numbering): raw nodes, snapped keys, a stable radix sort and
 * the merge run on the device, the result is also copied to the host.
 * yg_dofmap_create does this by itself for meshes of more than 2^20 raw nodes
 * (no simplex/tensor mix at p >= 3), where its host path uses the same stable
 * order, so both give identical bits.  On smaller meshes the host keeps the
 * coincident node that the reference's std::sort leaves first; this entry keeps
 * the first in raw order, so merged coordinates can differ in the last bits
 * (numbering identical).  YG_UNSUPPORTED if the snapped keys need more than 64
 * bits. */
YG_API yg_status yg_dofmap_create_on_device(yg_context ctx, const double *nodes_xyz, int32_t n_nodes,
                                     const int32_t *cell_nodes, const int32_t *cell_offsets,
                                     const int32_t *cell_types, int32_t n_cells, int32_t poly_order,
                                     int32_t dof_per_node, yg_dofmap *out);
/* The DoFManager of a structured box generated on the device, with no mesh from
 * the host: dim 2 gives nx*ny Quad4 cells on [0,lx]x[0,ly], dim 3 nx*ny*nz Hex8
 * cells on [0,lx]x[0,ly]x[0,lz]; nodes x fastest at i*(lx/nx) (the last at lx);
 * cell corners in the element's x-fastest order for p = 1 (the DoFManager keeps
 * the mesh, DoFManager.cpp:153-160) and counter-clockwise, bottom face first,
 * for p > 1 (the corner maps of DoFManager.cpp:296-338).  p > 1 is numbered on
 * the device as by yg_dofmap_create_on_device. */
YG_API yg_status yg_dofmap_create_box(yg_context ctx, int32_t dim, int32_t nx, int32_t ny, int32_t nz, double lx,
                               double ly, double lz, int32_t poly_order, int32_t dof_per_node, yg_dofmap *out);
YG_API yg_status yg_dofmap_destroy(yg_dofmap d);
/* Sizes of dof_nodes, cells, the elements array, and dofs = dof_nodes*dof_per_node. */
YG_API yg_status yg_dofmap_sizes(yg_dofmap d, int32_t *n_dof_nodes, int32_t *n_cells,
                          int64_t *n_element_nodes, int64_t *n_dofs);
/* Copies of dof_nodes, element_offsets, elements and element_types
 * (DoFManager.hpp:67-73); any pointer may be NULL. */
YG_API yg_status yg_dofmap_get(yg_dofmap d, double *dof_nodes_xyz, int32_t *element_offsets,
                        int32_t *elements, int8_t *topology, int8_t *topo_dim, int8_t *poly_order);
/* A dofmap from a numbering the caller already has: the public members of a
 * host DoFManager (dof_nodes, element_offsets, elements, element_types;
 * include/utils/DoFManager.hpp:62-70) after DoFManager(M, CG, p, dpn).  For a
 * caller that keeps the reference's own DoFManager and hands only assembly and
 * the solve to the GPU.  cell_types are the mesh CellType codes of each cell
 * (they give the element topology and dimension); every cell has poly_order.
 * Fails with YG_BAD_ARG when an element lists a node outside dof_nodes or its
 * node count is not that of its element type. */
YG_API yg_status yg_dofmap_create_from_numbering(yg_context ctx, const double *dof_nodes_xyz, int32_t n_dof_nodes,
                                          const int32_t *element_offsets, const int32_t *elements,
                                          const int32_t *cell_types, int32_t n_cells, int32_t poly_order,
                                          int32_t dof_per_node, yg_dofmap *out);
/* Element(ElementType{topology, dim, p}) tables as the GPU uses them
 * (src/element/Element.cpp:11-31, make_tensorproduct_element.cpp:17-145,
 * make_simplex_element.cpp:17-142, ShapeFunctionUtils.cpp:16-304): local node
 * coordinates (nen x 3), volume quadrature points (nq x 3) and weights (nq),
 * shape values N (nq x nen) and reference gradients dN/dxi (nq x nen x dim).
 * Host only.  Call with NULL arrays to get nen and nq; YG_UNSUPPORTED for an
 * element the reference cannot build either (tetrahedra above p = 2). */
YG_API yg_status yg_element_table(int32_t topology, int32_t dim, int32_t poly_order, int32_t *nen, int32_t *nq,
                           double *local_nodes_xyz, double *qp_xyz, double *qw, double *N, double *dN);

/* ------------------------------------------------------------------ assembly */

/* Device physics registered for CGAssembly<Physics>; a host-side Physics struct
 * cannot run on the GPU, so each is a kernel with parameters.
 *  YG_POISSON     params = {sign, f}: K_AB += sign*gradN_A.gradN_B*jxw, R_A += f*N_A*jxw
 *                 (apps/BasicPoisson/main.cpp:31-60 uses sign=-1; sign=+1 is the SPD form)
 *  YG_ELASTICITY  params = {sign, lambda, mu, b0, b1, b2}: K_{Ai,Bk} += sign*C_ikjl
 *                 dN_A/dx_j dN_B/dx_l jxw, R_{Ai} += b_i*N_A*jxw
 *                 (apps/BasicLinearElasticity/main.cpp:41-113)
 *  YG_SUPG        params = {k, h, U0, Q}: steady SUPG advection-diffusion with U=(U0,0,0)
 *                 (apps/supg_learning/supg_advection.hpp:19-132) */
enum { YG_POISSON = 0, YG_ELASTICITY = 1, YG_SUPG = 2 };
typedef struct yg_physics {
    int32_t kind;
    int32_t nsd; /* Physics::nsd(); cells of another topological dimension are skipped */
    double params[8];
} yg_physics;

/* AssemblyRequirement (include/assembly/AssemblyRequirement.hpp:12-19) as bits. */
enum { YG_REQ_RESIDUAL = 1, YG_REQ_TANGENT = 2 };
/* Storage of the assembled tangent: scalar CSR, or BCSR with dof_per_node-sized
 * blocks (dof = node*dof_per_node + comp, so node blocks are natural). */
enum { YG_FORMAT_CSR = 0, YG_FORMAT_BCSR = 1 };

/* CGAssembly<Physics>(FESystem&, requirements) (include/assembly/CGAssembly.hpp:27-186).
 * Tangent: if *K is NULL a new matrix (pattern built on the GPU) is returned; if
 * *K came from an earlier call on the same dofmap and format, its values are
 * replaced, like setFromTriplets (CGAssembly.hpp:185).  Residual: added into
 * `residual` (length n_dofs), like GlobalResidual += private_residual
 * (CGAssembly.hpp:181).  Duplicate summation is deterministic (element-coloured
 * scatter, colours in ascending order).  An element's shape gradients at all its
 * quadrature points are staged in shared memory, which limits hexahedra to
 * p <= 3 (p = 4 needs 375 KB); larger elements return YG_UNSUPPORTED. */
YG_API yg_status yg_assemble(yg_dofmap d, const yg_physics *physics, uint32_t requirements,
                      int32_t format, yg_matrix *K, yg_vector residual);

/* LocalSmoothingGradient<Physics>(FESystem&) (include/assembly/LocalSmoothingGradient.hpp:20-94):
 * the nodal gradient of `solution` (n_dofs entries) over the cells of dimension
 * nsd, written to `gradient` (n_dofs * nsd entries, row-major: dof-major, then
 * the nsd derivatives): the element gradient at each quadrature point, weighted
 * by N_A jxw, summed per dof and divided by the sum of N_A jxw (a dof no such
 * cell touches gets 0/0).  Deterministic (element-coloured sums).  Same element
 * limit as yg_assemble (hexahedra p <= 3, else YG_UNSUPPORTED). */
YG_API yg_status yg_local_smoothing_gradient(yg_dofmap d, int32_t nsd, yg_vector solution, yg_vector gradient);

/* ZZGradientRecovery<Physics>(FESystem&) (include/assembly/ZZGradientRecovery.hpp:33-140):
 * Zienkiewicz-Zhu patch recovery of the nodal gradient of a p = 1 scalar field
 * (one dof per node, as the reference asserts): each node fits a linear
 * polynomial by least squares to the FE gradient at the quadrature points of
 * the cells of dimension nsd (2 or 3) around it and takes its value at the
 * node.  `gradient` has n_nodes * nsd entries, row-major.  Solved through the
 * patch's normal equations in coordinates centred at the node (the reference
 * uses a column-pivoted QR in absolute coordinates; same fit to rounding).
 * A node whose patch has fewer samples than nsd + 1 gets NaN.  Deterministic. */
YG_API yg_status yg_zz_gradient_recovery(yg_dofmap d, int32_t nsd, yg_vector solution, yg_vector gradient);

/* DirichletBC::apply(A, rhs) for one BC object (src/boundary_conditions/DirichletBC.cpp:27-89):
 * rhs -= A*g, zero the BC rows and columns, unit diagonal, rhs_bc = g.  bc_dofs
 * are global dofs (node*dof_per_node + component), bc_values their g. */
YG_API yg_status yg_dirichlet_apply(yg_matrix K, yg_vector rhs, const int64_t *bc_dofs,
                             const double *bc_values, int64_t n_bc);

/* ------------------------------------------------------------------ output */

/* SimulationOutput(fname_base, BackendType::VTU).captureFrame(FESystem&) with the
 * default capture (include/output/SimulationOutput.hpp:47-116,
 * src/output/VTUBackend.cpp:20-269, src/output/OutputMesh.cpp:10-50): writes
 * fname_base.vtu, an ASCII UnstructuredGrid of the dof nodes and the linear
 * sub-cells of every element, with the components of `solution` (device, NULL
 * for the mesh alone) as scalar arrays Solution_0.. -- point data when it holds
 * dof_per_node values per dof node, cell data when it holds dof_per_node values
 * per cell.  The text is the reference's character for character (six
 * significant digits).  The vector is copied off the device in chunks through
 * pinned buffers.  The HDF5 backend is not provided (no HDF5 library here). */
YG_API yg_status yg_output_vtu(yg_dofmap d, const char *fname_base, yg_vector solution);

/* ------------------------------------------------------------------ matrices */

/* sparse_csr<T>(triplets) for block=1 (include/old_handmade_linalg/sparse_csr.hpp:90-149)
 * and sparse_bcsr<B,T>(triplets) for block=B (sparse_bcsr.hpp:93-176): duplicates
 * summed, rows/cols = max index + 1 (BCSR: rounded up to whole blocks).  Triplet
 * indices are size_t in the reference (sparse_matrix.hpp:19). */
YG_API yg_status yg_matrix_from_triplets(yg_context ctx, int32_t block, const uint64_t *rows,
                                  const uint64_t *cols, const double *vals, uint64_t n,
                                  yg_matrix *out);
/* Import an already compressed matrix (row_ptr/col_index/_data of sparse_csr,
 * sparse_csr.hpp:63-65, or brow_ptr/bcol_index/data of sparse_bcsr,
 * sparse_bcsr.hpp:31-33). Column indices must be sorted within each row. */
YG_API yg_status yg_matrix_from_csr(yg_context ctx, int32_t block, int64_t nbrows, int64_t nbcols,
                             const int64_t *brow_ptr, const int64_t *bcol, const double *vals,
                             yg_matrix *out);
YG_API yg_status yg_matrix_destroy(yg_matrix A);
/* rows(), cols(), nnz() (scalar entries) and the block size. */
YG_API yg_status yg_matrix_sizes(yg_matrix A, int64_t *rows, int64_t *cols, int64_t *nnz, int32_t *block);
/* Export in the reference layout (block row pointer, block columns, values with
 * row-major blocks); any pointer may be NULL. */
YG_API yg_status yg_matrix_get(yg_matrix A, int64_t *brow_ptr, int64_t *bcol, double *vals);
/* Keep an FP32 copy of the values for mixed-precision SpMV (no reference counterpart). */
YG_API yg_status yg_matrix_make_fp32(yg_matrix A);

/* y = A*x: csr_spmv / bcsr_spmv via operator* (include/old_handmade_linalg/csr_spmv.hpp:25-56,
 * bcsr_spmv.hpp:23-62, operators.hpp:117-131).  precision: YG_PREC_FP64,
 * YG_PREC_MIXED (FP32 values, FP64 vectors and accumulation) or
 * YG_SPMV_MIXED_CORRECTED (no reference counterpart): FP32 values plus, per
 * block row r, y_r += C_r x_r with C_r the FP64 sum over the row's blocks of
 * A_rj - fl32(A_rj) -- the operator the mixed-precision solvers iterate with;
 * it keeps A's block row sums, so it is exact on per-component constant x
 * (square matrices only). */
enum { YG_PREC_FP64 = 0, YG_PREC_MIXED = 1, YG_PREC_MIXED_IR = 2, YG_SPMV_MIXED_CORRECTED = 3 };
YG_API yg_status yg_spmv(yg_matrix A, yg_vector x, yg_vector y);
YG_API yg_status yg_spmv_ex(yg_matrix A, yg_vector x, yg_vector y, int32_t precision);

/* SpMV kernel choice (no reference counterpart; the reference has one loop).
 * variant 0: flat, `lanes` lanes per block row read the value stream coalesced;
 * variant 1: each warp stages its rows' values in shared memory with cp.async
 * (2x2 and 3x3 blocks); variant 2: bulk asynchronous copies (cp.async.bulk) of
 * row chunks into per-warp rings (2x2 and 3x3 blocks, `lanes` 1..32 selects the
 * ring shape); variant 3: bulk copies of tiles of whole rows with at most 256,
 * 512 or 1024 entries (CSR only, `lanes` 1, 2, 4, 8 selects the shape; every
 * row must hold 1..capacity entries); variant 4: one bulk copy pair per whole
 * block row into per-warp rings, every lane's x gathers issued before its
 * products, a transposed butterfly for the B row sums (2x2 and 3x3 blocks,
 * `lanes` 1, 2: rows of up to 128 blocks, 4, 8: up to 64 blocks).  variant -1 re-runs the device autotuner, which times
 * the candidates on this matrix and keeps the fastest (it also runs on the
 * first SpMV or solve of a matrix). */
YG_API yg_status yg_matrix_set_spmv(yg_matrix A, int32_t variant, int32_t lanes);
/* As yg_matrix_set_spmv for one value precision only: YG_PREC_FP64 sets the
 * kernel of FP64 values, any other precision that of the FP32 copy (no
 * reference counterpart; pins the autotuner's choice, e.g. under a profiler). */
YG_API yg_status yg_matrix_set_spmv_for(yg_matrix A, int32_t precision, int32_t variant, int32_t lanes);
YG_API yg_status yg_matrix_get_spmv(yg_matrix A, int32_t *variant, int32_t *lanes);
/* The SpMV kernel used for FP64 values (precision YG_PREC_FP64) or for the FP32
 * value copy (any other precision). */
YG_API yg_status yg_matrix_get_spmv_for(yg_matrix A, int32_t precision, int32_t *variant, int32_t *lanes);
/* Average device time of `reps` back-to-back SpMVs (CUDA events on the
 * context's stream), for roofline measurements. */
YG_API yg_status yg_spmv_bench(yg_matrix A, yg_vector x, yg_vector y, int32_t precision, int32_t reps,
                               double *ms_per_launch);

/* ------------------------------------------------------------------ preconditioners */

/* IdentityPreconditioner (IdentityPreconditioner.hpp:20-29), JacobiPreconditioner
 * (JacobiPreconditioner.hpp:11-54: z_i = r_i / a_ii, a zero diagonal gives inf as
 * in the reference), ILUPreconditioner (ILUPreconditioner.hpp:96-329: ILU(0) on
 * the pattern of A, no pivoting, zero pivots skipped; solve = forward
 * substitution with unit L then backward substitution with U). */
enum { YG_PRECOND_IDENTITY = 0, YG_PRECOND_JACOBI = 1, YG_PRECOND_ILU0 = 2 };
YG_API yg_status yg_precond_create(yg_matrix A, int32_t kind, yg_precond *out);
/* M.solve(z) in place (Preconditioner.hpp:9-21). */
YG_API yg_status yg_precond_apply(yg_precond M, yg_vector z);
/* Frees M; valid after A has been destroyed (M keeps A's context, not A), but
 * not after that context has been destroyed. */
YG_API yg_status yg_precond_destroy(yg_precond M);
/* Number of zero pivots skipped while factoring (ILU(0)) or zero diagonals (Jacobi). */
YG_API int64_t yg_precond_zero_pivots(yg_precond M);
/* ILU(0) only (no reference counterpart): the dependency levels of its forward
 * and backward triangular sweeps -- the grid-wide barriers each apply waits
 * on; 0 and 0 for the other kinds. */
YG_API yg_status yg_precond_levels(yg_precond M, int64_t *lower, int64_t *upper);

/* ------------------------------------------------------------------ solvers */

/* Stopping criteria.  REFERENCE reproduces the reference's own test:
 *   cg_solve:   r.r / r0.r0 < tol, at most N iterations (cg_solve.hpp:45-69)
 *   pcg_solve:  r.z / r0.z0 < tol, at most N iterations (pcg_solve.hpp:141-167)
 *   bicgstab:   ||Ax-b||^2/||b||^2 < tol checked every max(N/100,1) iterations
 *               (bicgstab_solve.hpp:227-272)
 * RELRES stops when ||b - A x|| <= tol ||b||, recomputed in FP64 on the GPU
 * before returning (the recursive residual is only a trigger). */
enum { YG_CRIT_REFERENCE = 0, YG_CRIT_RELRES = 1 };
typedef struct yg_solve_opts {
    int32_t criterion;  /* YG_CRIT_* */
    int32_t precision;  /* YG_PREC_FP64; YG_PREC_MIXED: the iteration's SpMV reads FP32 values (FP64
                           vectors, accumulation and dots; the FP32 operator carries the row-sum
                           correction of YG_SPMV_MIXED_CORRECTED) and the residual is replaced by the FP64
                           true residual b - A x whenever it fell 10x -- each replacement is an FP64
                           refinement step; YG_PREC_MIXED_IR: restarted FP64 iterative refinement
                           around FP32-SpMV PCG inner solves */
    double tol;         /* see criterion */
    int64_t maxiter;    /* 0 = the reference's default (N for CG) */
    int32_t check_every;/* iterations between host convergence checks (0 = automatic) */
    int32_t profile;    /* 1: time every SpMV of the iteration with CUDA events (stats.spmv_*) */
} yg_solve_opts;
typedef struct yg_solve_stats {
    int64_t iterations;       /* Krylov iterations (inner iterations summed for MIXED) */
    double rel_residual;      /* ||b - A x|| / ||b|| recomputed in FP64 */
    int32_t status;           /* yg_status of the solve */
    int32_t refinements;      /* FP64 residual replacements / refinement steps */
    double device_ms;         /* device time of the solve (CUDA events) */
    double spmv_ms;           /* with opts.profile: summed device time of the iteration SpMVs */
    int64_t spmv_launches;    /* with opts.profile: number of SpMVs timed */
} yg_solve_stats;

/* cg_solve(A, rhs, x0, TOL) / pcg_solve(A, rhs, M, x0, TOL)
 * (solver/iterative/cg_solve.hpp:23-81, pcg_solve.hpp:115-178).  M may be NULL
 * (plain CG).  x holds x0 on entry and the solution on return. */
YG_API yg_status yg_cg(yg_matrix A, yg_precond M, yg_vector b, yg_vector x, const yg_solve_opts *opts,
                yg_solve_stats *stats);
/* bicgstab_solve(A, rhs, x0) (solver/iterative/bicgstab_solve.hpp:207-283), with an
 * optional right preconditioner and an iteration cap (the reference has none). */
YG_API yg_status yg_bicgstab(yg_matrix A, yg_precond M, yg_vector b, yg_vector x,
                      const yg_solve_opts *opts, yg_solve_stats *stats);

/* ------------------------------------------------------------------ batched and served solves */

/* Many independent systems advanced together by shared persistent-grid kernels
 * (relative-residual criterion): symmetric positive definite systems by
 * Jacobi-PCG, non-symmetric ones by BiCGSTAB with right Jacobi
 * preconditioning, in the same launches.  No reference counterpart: the
 * reference solves one system per pcg_solve / bicgstab_solve call.  Each system
 * keeps its own matrix (CSR or 2x2/3x3 BCSR), right-hand side and iterate,
 * which must stay alive while it is in the batch; x holds x0 when added and the
 * solution when finished.  They may belong to another context of the same
 * device (a second stream, so that systems are assembled while a block runs):
 * yg_batch_add waits for that context's pending work, and the caller frees them
 * only after the slot is removed between a wait and the next launch.  Systems may be added and removed between calls of
 * yg_batch_run (continuous batching); work advances in blocks of iterations
 * captured in one CUDA graph followed by an FP64 verification pass (true
 * residual b - A x for converged systems, BiCGSTAB restarts after a breakdown,
 * and the residual replacement of YG_PREC_MIXED).  A system's result does not
 * depend on the other systems in the batch. */
typedef struct yg_batch_t *yg_batch;
enum { YG_METHOD_CG = 0, YG_METHOD_BICGSTAB = 1 };
YG_API yg_status yg_batch_create(yg_context ctx, int32_t capacity, yg_batch *out);
YG_API yg_status yg_batch_destroy(yg_batch B);
/* method: YG_METHOD_CG (Jacobi-PCG) or YG_METHOD_BICGSTAB; opts: criterion must
 * be YG_CRIT_RELRES, precision YG_PREC_FP64 or YG_PREC_MIXED. */
YG_API yg_status yg_batch_add(yg_batch B, yg_matrix A, yg_vector b, yg_vector x, int32_t method,
                              const yg_solve_opts *opts, int32_t *slot);
/* Device bytes yg_batch_add allocates for a system of `rows` rows (work vectors
 * and tile table), for admission against a memory budget. */
YG_API int64_t yg_batch_work_bytes(int64_t rows, int32_t method);
YG_API yg_status yg_batch_remove(yg_batch B, int32_t slot);
/* Solve a slot's system again from its current x (the caller may have changed
 * x or b in place); slot -1 resets every system in the batch. */
YG_API yg_status yg_batch_reset(yg_batch B, int32_t slot);
/* Run at most max_blocks blocks of iterations (0 = until no system is active);
 * *n_active receives the number of systems still iterating. */
YG_API yg_status yg_batch_run(yg_batch B, int32_t max_blocks, int32_t *n_active);
/* One block of iterations without waiting (the host may prepare new systems
 * meanwhile), then yg_batch_wait for it; systems are added or removed only
 * between a wait and the next launch. */
YG_API yg_status yg_batch_launch(yg_batch B);
YG_API yg_status yg_batch_wait(yg_batch B, int32_t *n_active);
/* Systems added from now on whose FP64 matrix holds at least `bytes` bytes run
 * their iteration SpMV as one launch of the single-system kernel (autotuned for
 * that matrix, dot products fused) inside the batch's graph instead of sharing
 * the batched SpMV kernels; 0 turns this off.  Default 128 MiB. */
YG_API yg_status yg_batch_set_solo_bytes(yg_batch B, int64_t bytes);
/* *ready = 1 when no block is in flight or the launched block has completed
 * (yg_batch_wait then returns without blocking), 0 while it runs.  Never blocks. */
YG_API yg_status yg_batch_ready(yg_batch B, int32_t *ready);
/* Status (YG_OK when converged and verified in FP64, YG_RUNNING while it
 * iterates), iterations and FP64 relative residual of a slot. */
YG_API yg_status yg_batch_stats(yg_batch B, int32_t slot, yg_solve_stats *stats);
/* Autotune, per block size, the SpMV variant (0: tiles staged in shared memory
 * by bulk asynchronous copies, 1: direct loads), tiles per work item and lanes
 * per block row, for the systems present. */
YG_API yg_status yg_batch_tune(yg_batch B);
/* The tuning in use: out[3*(b-1) + {0,1,2}] = variant, lanes, tiles per item
 * for block size b = 1, 2, 3. */
YG_API yg_status yg_batch_get_tuning(yg_batch B, int32_t *out);
/* Set the tuning of one block size (variant 0 or 1; lanes 1, 2, 4, ..., 32 --
 * lanes 1 means a lane per block with a segmented row sum in variant 0 and a
 * thread per row in variant 1; tiles per work item >= 1), between runs. */
YG_API yg_status yg_batch_set_tuning(yg_batch B, int32_t block, int32_t variant, int32_t lanes, int32_t tiles);

/* A continuous-batching solve server on one context.  No reference
 * counterpart.  A request is submitted with an estimate of the device bytes it
 * needs; yg_server_admit hands out queued requests in arrival order while the
 * admitted ones fit in the budget (the head of the queue waits for room); the
 * caller builds an admitted request's system on the device and attaches it;
 * attached systems advance together in one batch (PCG and BiCGSTAB).  Between
 * yg_server_launch and yg_server_wait one block of iterations runs without
 * blocking the host (build the next admitted systems meanwhile; attach only
 * after the wait).  The wait retires finished requests: list them with
 * yg_server_finished, read their stats with yg_server_poll and their solution
 * from the x that was attached, then yg_server_release them, which returns
 * their bytes to the budget. */
typedef struct yg_server_t *yg_server;
YG_API yg_status yg_server_create(yg_context ctx, uint64_t budget_bytes, int32_t max_active, yg_server *out);
YG_API yg_status yg_server_destroy(yg_server S);
YG_API yg_status yg_server_submit(yg_server S, uint64_t bytes, int64_t *id);
/* *id = the next admitted request, or -1 when none fits now. */
YG_API yg_status yg_server_admit(yg_server S, int64_t *id);
YG_API yg_status yg_server_attach(yg_server S, int64_t id, yg_matrix A, yg_vector b, yg_vector x, int32_t method,
                                  const yg_solve_opts *opts);
YG_API yg_status yg_server_launch(yg_server S);
YG_API yg_status yg_server_wait(yg_server S, int32_t *n_finished);
/* yg_batch_set_solo_bytes for the server's batch: requests attached from now on
 * whose FP64 matrix holds at least `bytes` run their iteration SpMV as their own
 * single-system launch inside the batch's graph. */
YG_API yg_status yg_server_set_solo_spmv_bytes(yg_server S, int64_t bytes);
/* *ready = 1 when no block is in flight or it has completed, 0 while it runs
 * (build admitted requests until then).  Never blocks. */
YG_API yg_status yg_server_ready(yg_server S, int32_t *ready);
YG_API yg_status yg_server_finished(yg_server S, int64_t *ids, int32_t cap, int32_t *n);
/* stats->status is YG_RUNNING until the request finished. */
YG_API yg_status yg_server_poll(yg_server S, int64_t id, yg_solve_stats *stats);
YG_API yg_status yg_server_release(yg_server S, int64_t id);
YG_API yg_status yg_server_info(yg_server S, int64_t *queued, int64_t *active, uint64_t *bytes_held);
/* Autotune the shared batch's SpMV on the systems attached now (between a wait
 * and the next launch). */
YG_API yg_status yg_server_tune(yg_server S);
/* Systems of at least `rows` rows (0: none) skip the batch: each wait solves
 * one of them alone, to completion, with yg_cg or yg_bicgstab (Jacobi), before
 * it waits for the block in flight; on the matrix's own context, so with the
 * systems built on another context the solve and the block overlap. */
YG_API yg_status yg_server_set_solo_rows(yg_server S, int64_t rows);

/* ------------------------------------------------------------------ allocation-free dot product */

/* *out = sum_i x[i]*y[i], with x, y and out device pointers and stream a
 * cudaStream_t (NULL: the default stream of the current device).  No
 * counterpart in the reference, which has no device code.
 *
 * For callers that must not allocate device memory when they need a
 * reduction: a host framework that has reserved the device's memory for its
 * own pool (cudaMalloc would fail or grow past the budget it accounts for), or
 * a latency-bound loop between solver steps (cudaMalloc and cudaFree
 * synchronise the device).  It needs no yg_context, whose creation allocates.
 * The call allocates nothing: its partial sums live in a fixed 64 KiB array of
 * this library's device code, one per device; nothing in it has to start at
 * zero.  Limits: n <= 67,108,864 (8192 partial sums of 8192 values each);
 * larger n fails with YG_BAD_ARG and a message (use yg_vector_dot).  The first
 * call on each device looks up the array's address (cudaGetSymbolAddress),
 * which may load this library's device code: make that first call before any
 * stream capture.  Calls that overlap on the same device (other streams or
 * host threads) share the array and race; order them on one stream.  The
 * launch is asynchronous: *out is ready when the stream reaches it. */
YG_API yg_status yg_dot_static_scratch(const double *x, const double *y, int64_t n, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
