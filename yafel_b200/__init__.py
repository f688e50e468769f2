"""yafel_b200 -- YAFEL's continuous-Galerkin assemble + solve path on one B200.

The names follow the reference's API so that code written against it reads the
same: ``DoFManager``, ``FESystem``, ``CGAssembly``, ``DirichletBC``,
``sparse_csr``/``sparse_bcsr``, ``cg_solve``/``pcg_solve``/``bicgstab_solve``,
``JacobiPreconditioner``/``ILUPreconditioner``/``IdentityPreconditioner``.
Everything below calls the C ABI of include/yafel_gpu.h (libyafel_b200.so,
hand-written sm_100a kernels); there is no CPU fallback.
"""
import ctypes as C
import sys

import numpy as np

from ._lib import (lib, check, YafelError, Physics, SolveOpts, SolveStats, YG_OK,
                   YG_NOT_CONVERGED, YG_BREAKDOWN, YG_NAN, YG_OVER_BUDGET, YG_BAD_ARG,
                   YG_UNSUPPORTED)
from . import meshgen

__all__ = ["Context", "default_context", "Mesh", "DoFManager", "FESystem", "CGAssembly", "LocalSmoothingGradient",
           "AssemblyRequirement", "PoissonEquation", "LinearElasticity", "AdvectionDiffusionSUPG",
           "DirichletBC", "DeviceVector", "sparse_csr", "sparse_bcsr", "JacobiPreconditioner",
           "ILUPreconditioner", "IdentityPreconditioner", "cg_solve", "pcg_solve",
           "bicgstab_solve", "solve", "Batch", "YafelError", "meshgen", "CG_SOLVER_TOL"]

# cg_solve.hpp:21, pcg_solve.hpp:21, bicgstab_solve.hpp:13
CG_SOLVER_TOL = 1.0e-14

CSR, BCSR = 0, 1
PREC_FP64, PREC_MIXED, PREC_MIXED_IR = 0, 1, 2
SPMV_MIXED_CORRECTED = 3  # FP32 values + FP64 row-sum correction (the mixed solvers' operator)
METHOD_CG, METHOD_BICGSTAB = 0, 1
CRIT_REFERENCE, CRIT_RELRES = 0, 1
POISSON, ELASTICITY, SUPG = 0, 1, 2


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _alive(ctx):
    """Handles are released only while the interpreter runs and the owning
    context is open; at shutdown the context's teardown frees everything."""
    return not sys.is_finalizing() and (ctx is None or getattr(ctx, "h", None))


class Context:
    """A CUDA device, one stream and an HBM budget (bytes, 0 = unlimited)."""

    def __init__(self, device=0, hbm_budget=0):
        h = C.c_void_p()
        check(lib().yg_context_create(device, int(hbm_budget), C.byref(h)), "context")
        self.h = h

    def synchronize(self):
        check(lib().yg_context_synchronize(self.h))

    def memory(self):
        a, b = C.c_uint64(), C.c_uint64()
        check(lib().yg_context_memory(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    @property
    def launches(self):
        return lib().yg_context_launches(self.h)

    def close(self):
        if getattr(self, "h", None) and not sys.is_finalizing():
            lib().yg_context_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DEFAULT = None


def default_context():
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Context(0)
    return _DEFAULT


# ------------------------------------------------------------------ vectors

class DeviceVector:
    """Device-resident FP64 vector (the GPU counterpart of Vector<double>)."""

    def __init__(self, n_or_array, ctx=None):
        self.ctx = ctx or default_context()
        arr = None
        if np.isscalar(n_or_array):
            n = int(n_or_array)
        else:
            arr = np.ascontiguousarray(n_or_array, dtype=np.float64)
            n = arr.size
        h = C.c_void_p()
        check(lib().yg_vector_create(self.ctx.h, n, C.byref(h)), "vector")
        self.h, self.n = h, n
        if arr is not None:
            self.upload(arr)

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        check(lib().yg_vector_upload(self.h, _ptr(a), a.size), "upload")

    def numpy(self):
        out = np.empty(self.n)
        check(lib().yg_vector_download(self.h, _ptr(out), self.n), "download")
        return out

    def fill(self, v):
        check(lib().yg_vector_fill(self.h, float(v)))

    def dot(self, other):
        r = C.c_double()
        check(lib().yg_vector_dot(self.h, other.h, C.byref(r)))
        return r.value

    def axpy(self, alpha, x):
        check(lib().yg_vector_axpy(float(alpha), x.h, self.h))

    def size(self):
        return self.n

    def __len__(self):
        return self.n

    def __del__(self):
        if getattr(self, "h", None) and _alive(getattr(self, "ctx", None)):
            lib().yg_vector_destroy(self.h)
        self.h = None


def _as_device(v, ctx):
    if isinstance(v, DeviceVector):
        return v, False
    return DeviceVector(np.asarray(v, dtype=np.float64), ctx), True


# ------------------------------------------------------------------ mesh & DoFs

class Mesh:
    """Explicit mesh: Mesh(DefinitionScheme::Explicit, nodes, cellNodes, offsets,
    cellTypes, cellTags) (include/mesh/Mesh.hpp:48-53)."""

    def __init__(self, nodes, cell_nodes, offsets, cell_types, cell_tags=None):
        self.nodes = np.ascontiguousarray(np.asarray(nodes, dtype=np.float64).reshape(-1, 3))
        self.cell_nodes = np.ascontiguousarray(cell_nodes, dtype=np.int32)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        self.cell_types = np.ascontiguousarray(cell_types, dtype=np.int32)
        self.cell_tags = (np.zeros(self.cell_types.size, np.int32) if cell_tags is None
                          else np.ascontiguousarray(cell_tags, dtype=np.int32))

    @classmethod
    def from_dict(cls, m):
        return cls(m["nodes"], m["cell_nodes"], m["offsets"], m["cell_types"], m.get("cell_tags"))

    @classmethod
    def from_gmsh(cls, path):
        """Mesh(const std::string &fname) (src/mesh/parse_gmsh.cpp:80-193): a Gmsh
        2.x ASCII file; cell_tags holds each cell's first tag (its region id) and
        tags_all the full per-cell tag lists."""
        h = C.c_void_p()
        check(lib().yg_mesh_read_gmsh(str(path).encode(), C.byref(h)), "Mesh(gmsh)")
        try:
            a, b, c, d = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
            check(lib().yg_mesh_sizes(h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
            nodes = np.zeros((a.value, 3))
            cn = np.zeros(max(1, c.value), np.int32)
            off = np.zeros(b.value + 1, np.int32)
            ct = np.zeros(max(1, b.value), np.int32)
            to = np.zeros(b.value + 1, np.int32)
            tg = np.zeros(max(1, d.value), np.int32)
            check(lib().yg_mesh_get(h, _ptr(nodes), _ptr(cn), _ptr(off), _ptr(ct), _ptr(to), _ptr(tg)))
        finally:
            lib().yg_mesh_destroy(h)
        tags = [tg[to[i]:to[i + 1]].copy() for i in range(b.value)]
        first = np.array([t[0] if t.size else 0 for t in tags], np.int32)
        m = cls(nodes, cn[:c.value], off, ct[:b.value], first)
        m.tags_all = tags
        return m

    def to_dict(self):
        return {"nodes": self.nodes, "cell_nodes": self.cell_nodes, "offsets": self.offsets,
                "cell_types": self.cell_types, "cell_tags": self.cell_tags}

    def nCells(self):
        return int(self.cell_types.size)

    def nNodes(self):
        return int(self.nodes.shape[0])


class DoFManager:
    """DoFManager(M, ManagerType::CG, polyOrder, dof_per_node)
    (src/utils/DoFManager.cpp:11-36); numbering identical to the reference's."""

    def __init__(self, mesh, polyOrder=1, dof_per_node=1, ctx=None, host_only=False, numbering=None,
                 on_device=False):
        """numbering: optional (dof_nodes n x 3, element_offsets, elements) of a
        DoFManager the caller already built (the reference's own, say); the
        mesh then only supplies the cell types.  on_device: number on the GPU
        whatever the size (yg_dofmap_create_on_device)."""
        if isinstance(mesh, dict):
            mesh = Mesh.from_dict(mesh)
        self.ctx = None if host_only else (ctx or default_context())
        self.mesh = mesh
        h = C.c_void_p()
        cx = self.ctx.h if self.ctx else None
        if numbering is None:
            fn = lib().yg_dofmap_create_on_device if on_device else lib().yg_dofmap_create
            check(fn(cx, _ptr(mesh.nodes), mesh.nNodes(), _ptr(mesh.cell_nodes),
                                         _ptr(mesh.offsets), _ptr(mesh.cell_types), mesh.nCells(), int(polyOrder),
                                         int(dof_per_node), C.byref(h)), "DoFManager")
        else:
            dn = np.ascontiguousarray(np.asarray(numbering[0], dtype=np.float64).reshape(-1, 3))
            eo = np.ascontiguousarray(numbering[1], dtype=np.int32)
            el = np.ascontiguousarray(numbering[2], dtype=np.int32)
            check(lib().yg_dofmap_create_from_numbering(cx, _ptr(dn), dn.shape[0], _ptr(eo), _ptr(el),
                                                        _ptr(mesh.cell_types), mesh.nCells(), int(polyOrder),
                                                        int(dof_per_node), C.byref(h)), "DoFManager")
        self.h = h
        self.polyOrder, self.dof_per_node = int(polyOrder), int(dof_per_node)
        a, b, c, d = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
        check(lib().yg_dofmap_sizes(h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        self._n_nodes, self._n_cells, self._n_el, self.ndofs = a.value, b.value, c.value, d.value
        self._cache = None
        self.cell_region_idx = mesh.cell_tags

    @classmethod
    def box(cls, dim, n, lengths=(1.0, 1.0, 1.0), polyOrder=1, dof_per_node=1, ctx=None):
        """The DoFManager of a structured box generated on the GPU
        (yg_dofmap_create_box): n = (nx, ny[, nz]) cells, the mesh of
        meshgen.structured_quad/hex in the corner order the element expects."""
        self = cls.__new__(cls)
        self.ctx = ctx or default_context()
        self.mesh = None
        nx, ny = int(n[0]), int(n[1])
        nz = int(n[2]) if dim == 3 else 0
        h = C.c_void_p()
        check(lib().yg_dofmap_create_box(self.ctx.h, dim, nx, ny, nz, float(lengths[0]), float(lengths[1]),
                                         float(lengths[2]) if dim == 3 else 0.0, int(polyOrder), int(dof_per_node),
                                         C.byref(h)), "DoFManager.box")
        self.h = h
        self.polyOrder, self.dof_per_node = int(polyOrder), int(dof_per_node)
        a, b, c, d = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
        check(lib().yg_dofmap_sizes(h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        self._n_nodes, self._n_cells, self._n_el, self.ndofs = a.value, b.value, c.value, d.value
        self._cache = None
        self.cell_region_idx = np.zeros(self._n_cells, np.int32)
        return self

    def _fetch(self):
        if self._cache is None:
            nodes = np.empty((self._n_nodes, 3))
            off = np.empty(self._n_cells + 1, np.int32)
            el = np.empty(max(self._n_el, 1), np.int32)
            topo = np.empty(max(self._n_cells, 1), np.int8)
            tdim = np.empty(max(self._n_cells, 1), np.int8)
            por = np.empty(max(self._n_cells, 1), np.int8)
            check(lib().yg_dofmap_get(self.h, _ptr(nodes), _ptr(off), _ptr(el), _ptr(topo), _ptr(tdim), _ptr(por)))
            self._cache = (nodes, off, el[:self._n_el], topo[:self._n_cells], tdim[:self._n_cells], por[:self._n_cells])
        return self._cache

    @property
    def dof_nodes(self):
        return self._fetch()[0]

    @property
    def element_offsets(self):
        return self._fetch()[1]

    @property
    def elements(self):
        return self._fetch()[2]

    @property
    def element_topology(self):
        return self._fetch()[3]

    @property
    def element_topo_dim(self):
        return self._fetch()[4]

    def nNodes(self):
        return self._n_nodes

    def nCells(self):
        return self._n_cells

    def getGlobalNodes(self, elnum):
        off = self.element_offsets
        return self.elements[off[elnum]:off[elnum + 1]].copy()

    def getGlobalDofs(self, elnum):
        nodes = self.getGlobalNodes(elnum)
        d = self.dof_per_node
        return (nodes[:, None] * d + np.arange(d)[None, :]).ravel()

    def __del__(self):
        if getattr(self, "h", None) and _alive(getattr(self, "ctx", None)):
            lib().yg_dofmap_destroy(self.h)
        self.h = None


def element_table(topology, dim, polyOrder):
    """The reference element tables the GPU kernels use for ElementType
    {topology, dim, polyOrder}: (local nodes nen x 3, quadrature points nq x 3,
    weights nq, N nq x nen, dN/dxi nq x nen x dim)."""
    nen, nq = C.c_int32(), C.c_int32()
    check(lib().yg_element_table(topology, dim, polyOrder, C.byref(nen), C.byref(nq), None, None, None, None, None),
          "element_table")
    a, q = nen.value, nq.value
    L, X, W = np.zeros((a, 3)), np.zeros((q, 3)), np.zeros(q)
    N, dN = np.zeros((q, a)), np.zeros((q, a, dim))
    check(lib().yg_element_table(topology, dim, polyOrder, C.byref(nen), C.byref(nq), _ptr(L), _ptr(X), _ptr(W),
                                 _ptr(N), _ptr(dN)), "element_table")
    return L, X, W, N, dN


# ------------------------------------------------------------------ physics

class PoissonEquation:
    """K_AB += sign grad N_A . grad N_B jxw, R_A += f N_A jxw
    (apps/BasicPoisson/main.cpp:25-61 is sign=-1, f=100; sign=+1 is SPD)."""

    def __init__(self, nsd, f=1.0, sign=1.0):
        self._nsd, self.f, self.sign = nsd, f, sign

    def nsd(self):
        return self._nsd

    def struct(self):
        p = Physics(POISSON, self._nsd)
        p.params[0], p.params[1] = self.sign, self.f
        return p


class LinearElasticity:
    """Isotropic linear elasticity (apps/BasicLinearElasticity/main.cpp:41-113):
    lambda = E nu/((1+nu)(1-2nu)), mu = E/(2(1+nu)); body force b per component."""

    def __init__(self, nsd, E=1.0, nu=0.3, body=(0.0, 0.0, 0.0), sign=1.0):
        self._nsd, self.E, self.nu, self.body, self.sign = nsd, E, nu, tuple(body), sign
        self.lam = (E * nu) / ((1 + nu) * (1 - 2 * nu))
        self.mu = E / (2 * (1 + nu))

    def nsd(self):
        return self._nsd

    def struct(self):
        p = Physics(ELASTICITY, self._nsd)
        vals = [self.sign, self.lam, self.mu] + list(self.body) + [0.0] * (3 - len(self.body))
        for i, v in enumerate(vals[:8]):
            p.params[i] = v
        return p


class AdvectionDiffusionSUPG:
    """Steady SUPG advection-diffusion (apps/supg_learning/supg_advection.hpp:19-132)
    with parameters k, h, U0, Q (the reference fixes k=0.1, h=0.1, U0=1, Q=0);
    Peclet number U0 h / (2k)."""

    def __init__(self, nsd, k=0.1, h=0.1, U0=1.0, Q=0.0):
        self._nsd, self.k, self.h, self.U0, self.Q = nsd, k, h, U0, Q

    def nsd(self):
        return self._nsd

    def struct(self):
        p = Physics(SUPG, self._nsd)
        p.params[0], p.params[1], p.params[2], p.params[3] = self.k, self.h, self.U0, self.Q
        return p


class AssemblyRequirement:
    """AssemblyRequirement (include/assembly/AssemblyRequirement.hpp:12-19)."""
    Residual = 1
    Tangent = 2


# ------------------------------------------------------------------ matrices

class _Matrix:
    block = 1

    def __init__(self, handle, ctx):
        self.h, self.ctx = handle, ctx
        r, c, n, b = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        check(lib().yg_matrix_sizes(handle, C.byref(r), C.byref(c), C.byref(n), C.byref(b)))
        self._rows, self._cols, self._nnz, self.block = r.value, c.value, n.value, b.value

    def rows(self):
        return self._rows

    def cols(self):
        return self._cols

    def nnz(self):
        return self._nnz

    def arrays(self):
        """(block row_ptr, block col_index, values) in the reference layout."""
        nb = self._rows // self.block
        nnzb = self._nnz // (self.block * self.block)
        rp = np.empty(nb + 1, np.int64)
        col = np.empty(max(nnzb, 1), np.int64)
        val = np.empty(max(self._nnz, 1))
        check(lib().yg_matrix_get(self.h, _ptr(rp), _ptr(col), _ptr(val)))
        return rp, col[:nnzb], val[:self._nnz]

    def copy_triplets(self):
        rp, col, val = self.arrays()
        B = self.block
        nb = rp.size - 1
        brow = np.repeat(np.arange(nb, dtype=np.int64), np.diff(rp))
        i = np.arange(B)
        rows = (brow[:, None, None] * B + i[None, :, None]).repeat(B, axis=2).ravel()
        cols = (col[:, None, None] * B + i[None, None, :]).repeat(B, axis=1).ravel()
        return rows, cols, val.copy()

    def make_fp32(self):
        check(lib().yg_matrix_make_fp32(self.h))

    def set_spmv(self, variant, lanes=32):
        """variant 0 flat (lanes per row), 1 shared-memory staged, 2 bulk-copy
        row chunks (2x2/3x3 blocks), 3 bulk-copy row tiles (CSR), 4 bulk-copy
        whole rows (2x2/3x3 blocks, rows of up to 128 or 64 blocks), -1 autotune."""
        check(lib().yg_matrix_set_spmv(self.h, int(variant), int(lanes)))

    def set_spmv_for(self, precision, variant, lanes):
        """Pin the SpMV kernel of one value precision (PREC_FP64, or the FP32 copy)."""
        check(lib().yg_matrix_set_spmv_for(self.h, int(precision), int(variant), int(lanes)))

    def get_spmv(self, precision=PREC_FP64):
        """(variant, lanes) of the SpMV kernel for FP64 values or, with another
        precision, for the FP32 value copy."""
        v, l = C.c_int32(), C.c_int32()
        check(lib().yg_matrix_get_spmv_for(self.h, int(precision), C.byref(v), C.byref(l)))
        return v.value, l.value

    def spmv_bench(self, reps=10, precision=PREC_FP64, x=None):
        """Average device milliseconds of one SpMV (CUDA events)."""
        xd = x if x is not None else DeviceVector(np.ones(self._cols), self.ctx)
        yd = DeviceVector(self._rows, self.ctx)
        ms = C.c_double()
        check(lib().yg_spmv_bench(self.h, xd.h, yd.h, precision, int(reps), C.byref(ms)))
        return ms.value

    def spmv(self, x, y=None, precision=PREC_FP64):
        xd, _ = _as_device(x, self.ctx)
        yd = y if y is not None else DeviceVector(self._rows, self.ctx)
        check(lib().yg_spmv_ex(self.h, xd.h, yd.h, precision), "spmv")
        return yd

    def __mul__(self, x):
        """A*x with a host vector returns a host vector (operators.hpp:117-131)."""
        if isinstance(x, DeviceVector):
            return self.spmv(x)
        return self.spmv(np.asarray(x, dtype=np.float64)).numpy()

    def __del__(self):
        if getattr(self, "h", None) and _alive(getattr(self, "ctx", None)):
            lib().yg_matrix_destroy(self.h)
        self.h = None


def _triplet_arrays(ts):
    if isinstance(ts, tuple) and len(ts) == 3 and hasattr(ts[0], "__len__"):
        r, c, v = ts
    else:
        ts = list(ts)
        r = [t[0] for t in ts]
        c = [t[1] for t in ts]
        v = [t[2] for t in ts]
    return (np.ascontiguousarray(r, dtype=np.uint64), np.ascontiguousarray(c, dtype=np.uint64),
            np.ascontiguousarray(v, dtype=np.float64))


class sparse_csr(_Matrix):
    """sparse_csr<double>(triplets) (include/old_handmade_linalg/sparse_csr.hpp:90-149),
    stored on the GPU.  ``triplets`` is a list of (i, j, value) or a tuple of arrays."""

    def __init__(self, triplets=None, ctx=None, _handle=None):
        ctx = ctx or default_context()
        if _handle is None:
            r, c, v = _triplet_arrays(triplets)
            h = C.c_void_p()
            check(lib().yg_matrix_from_triplets(ctx.h, 1, _ptr(r), _ptr(c), _ptr(v), r.size, C.byref(h)), "sparse_csr")
            _handle = h
        _Matrix.__init__(self, _handle, ctx)

    @classmethod
    def from_csr(cls, row_ptr, col_index, data, ncols=None, ctx=None):
        ctx = ctx or default_context()
        rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
        col = np.ascontiguousarray(col_index, dtype=np.int64)
        val = np.ascontiguousarray(data, dtype=np.float64)
        n = rp.size - 1
        h = C.c_void_p()
        check(lib().yg_matrix_from_csr(ctx.h, 1, n, n if ncols is None else ncols, _ptr(rp), _ptr(col), _ptr(val),
                                       C.byref(h)), "sparse_csr")
        return cls(ctx=ctx, _handle=h)


class sparse_bcsr(_Matrix):
    """sparse_bcsr<BLOCK,double>(triplets) (include/old_handmade_linalg/sparse_bcsr.hpp:93-176)."""

    def __init__(self, BLOCK, triplets=None, ctx=None, _handle=None):
        ctx = ctx or default_context()
        if _handle is None:
            r, c, v = _triplet_arrays(triplets)
            h = C.c_void_p()
            check(lib().yg_matrix_from_triplets(ctx.h, int(BLOCK), _ptr(r), _ptr(c), _ptr(v), r.size, C.byref(h)),
                  "sparse_bcsr")
            _handle = h
        _Matrix.__init__(self, _handle, ctx)

    @classmethod
    def from_bcsr(cls, BLOCK, brow_ptr, bcol_index, data, nbcols=None, ctx=None):
        ctx = ctx or default_context()
        rp = np.ascontiguousarray(brow_ptr, dtype=np.int64)
        col = np.ascontiguousarray(bcol_index, dtype=np.int64)
        val = np.ascontiguousarray(data, dtype=np.float64)
        n = rp.size - 1
        h = C.c_void_p()
        check(lib().yg_matrix_from_csr(ctx.h, int(BLOCK), n, n if nbcols is None else nbcols, _ptr(rp), _ptr(col),
                                       _ptr(val), C.byref(h)), "sparse_bcsr")
        return cls(BLOCK, ctx=ctx, _handle=h)


def _wrap_matrix(handle, ctx):
    m = _Matrix.__new__(sparse_bcsr)
    _Matrix.__init__(m, handle, ctx)
    if m.block == 1:
        m.__class__ = sparse_csr
    return m


# ------------------------------------------------------------------ FE system

class FESystem:
    """FESystem(DoFManager&, dim) (include/fe_system/FESystem.hpp:18-56): holds the
    global tangent, residual and solution on the device."""

    def __init__(self, dofm, dim=0, format=BCSR):
        self.dofm, self.dim, self.format = dofm, dim, format
        self.ctx = dofm.ctx
        n = dofm.ndofs
        self.global_residual = DeviceVector(n, self.ctx)
        self.solution = DeviceVector(n, self.ctx)
        self.solution_gradient = None
        self.global_tangent = None
        self.time = 0.0

    def getGlobalTangent(self):
        return self.global_tangent

    def getGlobalResidual(self):
        return self.global_residual

    def getSolution(self):
        return self.solution

    def getSolutionGradient(self):
        """The nodal gradient of the last LocalSmoothingGradient call: a
        DeviceVector of n_dofs * nsd entries (row-major, one row per dof)."""
        return self.solution_gradient

    def getDoFManager(self):
        return self.dofm

    def currentTime(self):
        return self.time


def CGAssembly(physics, feSystem, requirements=(AssemblyRequirement.Residual, AssemblyRequirement.Tangent),
               format=None):
    """CGAssembly<Physics>(FESystem&, requirements) (include/assembly/CGAssembly.hpp:27-186)."""
    mask = 0
    for r in requirements:
        mask |= int(r)
    fmt = feSystem.format if format is None else format
    st = physics.struct()
    K = feSystem.global_tangent
    h = C.c_void_p(K.h.value if K is not None else None)
    check(lib().yg_assemble(feSystem.dofm.h, C.byref(st), mask, fmt, C.byref(h),
                            feSystem.global_residual.h), "CGAssembly")
    if K is None and (mask & AssemblyRequirement.Tangent):
        feSystem.global_tangent = _wrap_matrix(h, feSystem.ctx)
    return feSystem


def LocalSmoothingGradient(physics, feSystem):
    """LocalSmoothingGradient<Physics>(FESystem&)
    (include/assembly/LocalSmoothingGradient.hpp:20-94): the gradient of the
    FESystem's solution averaged to the dofs with weights N_A jxw over the cells
    of dimension physics.nsd(); stored as the FESystem's solution gradient."""
    nsd = physics.nsd()
    g = DeviceVector(feSystem.dofm.ndofs * nsd, feSystem.ctx)
    check(lib().yg_local_smoothing_gradient(feSystem.dofm.h, nsd, feSystem.solution.h, g.h), "LocalSmoothingGradient")
    feSystem.solution_gradient = g
    return feSystem


def ZZGradientRecovery(physics, feSystem):
    """ZZGradientRecovery<Physics>(FESystem&)
    (include/assembly/ZZGradientRecovery.hpp:33-140): Zienkiewicz-Zhu patch
    recovery of the gradient of the FESystem's p = 1 scalar solution, stored as
    the FESystem's solution gradient (n_nodes x nsd)."""
    nsd = physics.nsd()
    g = DeviceVector(feSystem.dofm.nNodes() * nsd, feSystem.ctx)
    check(lib().yg_zz_gradient_recovery(feSystem.dofm.h, nsd, feSystem.solution.h, g.h), "ZZGradientRecovery")
    feSystem.solution_gradient = g
    return feSystem


class SimulationOutput:
    """SimulationOutput(fname_base, BackendType::VTU) (include/output/SimulationOutput.hpp:22-116):
    captureFrame(feSystem) writes fname_base.vtu -- the dof nodes, the linear
    sub-cells of every element and the solution's components as Solution_0..
    (the reference's default capture), in the reference's ASCII format."""

    def __init__(self, fname_base="output", backend="VTU"):
        if backend != "VTU":
            raise ValueError("only the VTU backend is provided (no HDF5 library)")
        self.fname_base = fname_base

    def captureFrame(self, feSystem, solution=None):
        sol = feSystem.solution if solution is None else solution
        check(lib().yg_output_vtu(feSystem.dofm.h, self.fname_base.encode(), sol.h if sol is not None else None),
              "SimulationOutput.captureFrame")


class DirichletBC:
    """DirichletBC(dofm, value, comp) (include/boundary_conditions/DirichletBC.hpp:23-89);
    value is a number or a function f(x, t)."""

    def __init__(self, dofm, bcval=0.0, comp=0):
        self.dofm, self.component = dofm, int(comp)
        self.value_func = bcval if callable(bcval) else (lambda x, t, v=float(bcval): v)
        self.constant = None if callable(bcval) else float(bcval)
        self.bc_nodes = np.zeros(0, np.int64)

    def selectByFunction(self, func):
        """Nodes whose coordinate satisfies func (DirichletBC.hpp:80-89); func may be
        vectorised over an (n,3) array or scalar over one point."""
        X = self.dofm.dof_nodes
        try:
            m = np.asarray(func(X))
            if m.shape != (X.shape[0],):
                raise TypeError
        except Exception:
            m = np.array([bool(func(x)) for x in X])
        self.bc_nodes = np.concatenate([self.bc_nodes, np.nonzero(m)[0].astype(np.int64)])

    def selectByRegionID(self, region_id):
        """Nodes of cells tagged region_id, with consecutive duplicates removed
        (src/boundary_conditions/DirichletBC.cpp:10-24)."""
        tags = self.dofm.cell_region_idx
        off, el = self.dofm.element_offsets, self.dofm.elements
        nodes = [el[off[c]:off[c + 1]] for c in np.nonzero(tags == region_id)[0]]
        nodes = np.concatenate(nodes).astype(np.int64) if nodes else np.zeros(0, np.int64)
        if nodes.size:
            keep = np.ones(nodes.size, bool)
            keep[1:] = nodes[1:] != nodes[:-1]
            nodes = nodes[keep]
        self.bc_nodes = np.concatenate([self.bc_nodes, nodes])

    def getNodes(self):
        return self.bc_nodes

    def dofs_and_values(self, time=0.0):
        d = self.dofm.dof_per_node
        dofs = self.bc_nodes * d + self.component
        if self.constant is not None:  # a constant value needs no node coordinates
            vals = np.full(self.bc_nodes.size, self.constant)
        else:
            X = self.dofm.dof_nodes[self.bc_nodes] if self.bc_nodes.size else np.zeros((0, 3))
            vals = np.array([self.value_func(x, time) for x in X], dtype=np.float64)
        return np.ascontiguousarray(dofs, dtype=np.int64), np.ascontiguousarray(vals)

    def apply(self, A, rhs, time=0.0):
        dofs, vals = self.dofs_and_values(time)
        check(lib().yg_dirichlet_apply(A.h, rhs.h, _ptr(dofs), _ptr(vals), dofs.size), "DirichletBC::apply")


# ------------------------------------------------------------------ preconditioners & solvers

class _Precond:
    kind = 0

    def __init__(self, A):
        self.A = A
        h = C.c_void_p()
        check(lib().yg_precond_create(A.h, self.kind, C.byref(h)), type(self).__name__)
        self.h = h
        self.zero_pivots = lib().yg_precond_zero_pivots(h)

    @property
    def levels(self):
        """(forward, backward) dependency levels of an ILU(0) apply; (0, 0) otherwise."""
        lo, up = C.c_int64(), C.c_int64()
        check(lib().yg_precond_levels(self.h, C.byref(lo), C.byref(up)))
        return lo.value, up.value

    def solve(self, z):
        """M.solve(z) in place (Preconditioner.hpp:9-21); z is a DeviceVector or a
        numpy array (modified in place)."""
        if isinstance(z, DeviceVector):
            check(lib().yg_precond_apply(self.h, z.h))
            return z
        d = DeviceVector(z, self.A.ctx)
        check(lib().yg_precond_apply(self.h, d.h))
        z[:] = d.numpy()
        return z

    def __del__(self):
        if getattr(self, "h", None) and _alive(getattr(self.A, "ctx", None)):
            lib().yg_precond_destroy(self.h)
        self.h = None


class IdentityPreconditioner(_Precond):
    kind = 0


class JacobiPreconditioner(_Precond):
    kind = 1


class ILUPreconditioner(_Precond):
    kind = 2


def solve(A, b, x0=None, M=None, method="cg", criterion=CRIT_RELRES, tol=1e-10, maxiter=0,
          precision=PREC_FP64, check_every=0, raise_on_failure=False, profile=False):
    """Solve on the GPU and return (x, stats).  b and x0 may be host arrays or
    DeviceVectors; x is a DeviceVector."""
    ctx = A.ctx
    bd, _ = _as_device(b, ctx)
    if x0 is None:
        xd = DeviceVector(A.rows(), ctx)
    elif isinstance(x0, DeviceVector):
        xd = x0
    else:
        xd = DeviceVector(np.asarray(x0, dtype=np.float64), ctx)
    opts = SolveOpts(criterion, precision, tol, maxiter, check_every, int(bool(profile)))
    st = SolveStats()
    fn = lib().yg_cg if method == "cg" else lib().yg_bicgstab
    s = fn(A.h, M.h if M is not None else None, bd.h, xd.h, C.byref(opts), C.byref(st))
    if s not in (YG_OK, YG_NOT_CONVERGED, YG_BREAKDOWN, YG_NAN) or (raise_on_failure and s != YG_OK):
        check(s, method)
    return xd, st


def cg_solve(A, rhs, x0=None, TOL=CG_SOLVER_TOL):
    """cg_solve(A, rhs[, x0][, TOL]) (solver/iterative/cg_solve.hpp:23-81): stops when
    r.r/r0.r0 < TOL or after N iterations; returns the solution as a host vector."""
    x, _ = solve(A, rhs, x0, None, "cg", CRIT_REFERENCE, TOL)
    return x.numpy()


def pcg_solve(A, rhs, M, x0=None, TOL=CG_SOLVER_TOL):
    """pcg_solve(A, rhs, M, x0, TOL) (pcg_solve.hpp:126-178): stops when
    r.z/r0.z0 < TOL or after N iterations."""
    x, _ = solve(A, rhs, x0, M, "cg", CRIT_REFERENCE, TOL)
    return x.numpy()


def bicgstab_solve(A, rhs, x0=None, TOL=CG_SOLVER_TOL):
    """bicgstab_solve(A, rhs[, x0]) (bicgstab_solve.hpp:207-283): true residual
    ||Ax-b||^2/||b||^2 < TOL every max(N/100,1) iterations."""
    x, _ = solve(A, rhs, x0, None, "bicgstab", CRIT_REFERENCE, TOL)
    return x.numpy()


# ------------------------------------------------------------------ batched / served solves

class Batch:
    """Many systems advanced together (yg_batch_*): add (A, b, x0) triples, run
    until all converge or step block by block while adding/removing systems."""

    def __init__(self, capacity, ctx=None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().yg_batch_create(self.ctx.h, int(capacity), C.byref(h)), "Batch")
        self.h = h
        self._keep = {}

    def add(self, A, b, x0=None, tol=1e-10, precision=PREC_FP64, maxiter=0, method="cg"):
        """Add A x = b (x0 default 0); method "cg" (Jacobi-PCG, SPD systems) or
        "bicgstab" (right Jacobi-preconditioned BiCGSTAB).  Returns the slot."""
        bd, _ = _as_device(b, self.ctx)
        xd = x0 if isinstance(x0, DeviceVector) else DeviceVector(
            np.zeros(A.rows()) if x0 is None else np.asarray(x0, dtype=np.float64), self.ctx)
        opts = SolveOpts(CRIT_RELRES, precision, tol, maxiter, 0, 0)
        slot = C.c_int32()
        m = {"cg": METHOD_CG, "bicgstab": METHOD_BICGSTAB}[method]
        check(lib().yg_batch_add(self.h, A.h, bd.h, xd.h, m, C.byref(opts), C.byref(slot)), "Batch.add")
        self._keep[slot.value] = (A, bd, xd)
        return slot.value

    def remove(self, slot):
        check(lib().yg_batch_remove(self.h, int(slot)), "Batch.remove")
        self._keep.pop(slot, None)

    def reset(self, slot=-1):
        """Solve again from the current x of `slot` (every slot when -1)."""
        check(lib().yg_batch_reset(self.h, int(slot)), "Batch.reset")

    def run(self, max_blocks=0):
        n = C.c_int32()
        check(lib().yg_batch_run(self.h, int(max_blocks), C.byref(n)), "Batch.run")
        return n.value

    def tune(self):
        check(lib().yg_batch_tune(self.h), "Batch.tune")

    def tuning(self):
        """{block size: (variant, lanes, tiles per item)} in use."""
        a = (C.c_int32 * 9)()
        check(lib().yg_batch_get_tuning(self.h, a), "Batch.tuning")
        return {b: (a[3 * (b - 1)], a[3 * (b - 1) + 1], a[3 * (b - 1) + 2]) for b in (1, 2, 3)}

    def set_tuning(self, block, variant, lanes, tiles):
        check(lib().yg_batch_set_tuning(self.h, int(block), int(variant), int(lanes), int(tiles)), "Batch.set_tuning")

    def launch(self):
        """One block of iterations without waiting; pair with wait()."""
        check(lib().yg_batch_launch(self.h), "Batch.launch")

    def wait(self):
        n = C.c_int32()
        check(lib().yg_batch_wait(self.h, C.byref(n)), "Batch.wait")
        return n.value

    def set_solo_bytes(self, nbytes):
        """Systems added from now on whose FP64 matrix holds at least `nbytes`
        run their iteration SpMV as their own single-system launch (0: never)."""
        check(lib().yg_batch_set_solo_bytes(self.h, int(nbytes)), "Batch.set_solo_bytes")

    def ready(self):
        """True when no block is in flight or the launched one has completed."""
        r = C.c_int32()
        check(lib().yg_batch_ready(self.h, C.byref(r)), "Batch.ready")
        return bool(r.value)

    def stats(self, slot):
        st = SolveStats()
        check(lib().yg_batch_stats(self.h, int(slot), C.byref(st)), "Batch.stats")
        return st

    def solution(self, slot):
        return self._keep[slot][2]

    def __del__(self):
        if getattr(self, "h", None) and _alive(getattr(self, "ctx", None)):
            lib().yg_batch_destroy(self.h)
        self.h = None


class Server:
    """Continuous-batching solve server (yg_server_*): requests are submitted
    with a device-byte estimate, admitted in arrival order under an HBM budget,
    built by the caller, attached, and advanced together in one batch."""

    def __init__(self, budget_bytes, max_active=1024, ctx=None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().yg_server_create(self.ctx.h, int(budget_bytes), int(max_active), C.byref(h)), "Server")
        self.h = h
        self._keep = {}

    def submit(self, est_bytes):
        r = C.c_int64()
        check(lib().yg_server_submit(self.h, int(est_bytes), C.byref(r)), "Server.submit")
        return r.value

    def admit(self):
        """Id of the next admitted request, or None."""
        r = C.c_int64()
        check(lib().yg_server_admit(self.h, C.byref(r)), "Server.admit")
        return None if r.value < 0 else r.value

    def attach(self, rid, A, b, x, method="cg", tol=1e-10, precision=PREC_FP64, maxiter=0):
        opts = SolveOpts(CRIT_RELRES, precision, tol, maxiter, 0, 0)
        m = {"cg": METHOD_CG, "bicgstab": METHOD_BICGSTAB}[method]
        check(lib().yg_server_attach(self.h, int(rid), A.h, b.h, x.h, m, C.byref(opts)), "Server.attach")
        self._keep[rid] = (A, b, x)

    def launch(self):
        check(lib().yg_server_launch(self.h), "Server.launch")

    def wait(self):
        n = C.c_int32()
        check(lib().yg_server_wait(self.h, C.byref(n)), "Server.wait")
        return n.value

    def set_solo_spmv_bytes(self, nbytes):
        """Requests attached from now on whose FP64 matrix holds at least
        `nbytes` run their iteration SpMV as their own launch (0: never)."""
        check(lib().yg_server_set_solo_spmv_bytes(self.h, int(nbytes)), "Server.set_solo_spmv_bytes")

    def ready(self):
        """True when no block is in flight or the launched one has completed
        (build admitted requests until then)."""
        r = C.c_int32()
        check(lib().yg_server_ready(self.h, C.byref(r)), "Server.ready")
        return bool(r.value)

    def finished(self):
        ids = (C.c_int64 * 4096)()
        n = C.c_int32()
        out = []
        while True:
            check(lib().yg_server_finished(self.h, ids, 4096, C.byref(n)), "Server.finished")
            out.extend(ids[i] for i in range(n.value))
            if n.value < 4096:
                return out

    def poll(self, rid):
        st = SolveStats()
        check(lib().yg_server_poll(self.h, int(rid), C.byref(st)), "Server.poll")
        return st

    def solution(self, rid):
        return self._keep[rid][2]

    def release(self, rid):
        check(lib().yg_server_release(self.h, int(rid)), "Server.release")
        self._keep.pop(rid, None)

    def tune(self):
        check(lib().yg_server_tune(self.h), "Server.tune")

    def set_solo_rows(self, rows):
        """Systems of at least `rows` rows are solved alone (0: batch everything)."""
        check(lib().yg_server_set_solo_rows(self.h, int(rows)), "Server.set_solo_rows")

    def info(self):
        q, a, b = C.c_int64(), C.c_int64(), C.c_uint64()
        check(lib().yg_server_info(self.h, C.byref(q), C.byref(a), C.byref(b)), "Server.info")
        return {"queued": q.value, "active": a.value, "bytes_held": b.value}

    def __del__(self):
        if getattr(self, "h", None) and _alive(getattr(self, "ctx", None)):
            lib().yg_server_destroy(self.h)
        self.h = None
