"""ctypes front end of the checker libraries (test infrastructure only).

``liboracle.so`` is the C restatement of the reference path (oracle/yafel_oracle.c);
``_ref/libyafel_ref.so`` is the reference's own handmade linear algebra and
quadrature compiled in place (oracle/Makefile).  Only tests, the smoke check
and the bench's CPU-baseline leg import this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

TENSOR, SIMPLEX, NONE = 0, 1, 2
POISSON, ELASTICITY, SUPG = 0, 1, 2
SUPG_PARAM = 3  # reference assembly only: SUPG formulas with run-time k, h, U0, Q
PRECOND_NONE, PRECOND_JACOBI, PRECOND_ILU0 = 0, 1, 2
CRIT_REFERENCE, CRIT_RELRES = 0, 1


class _Csr(C.Structure):
    _fields_ = [("nrows", C.c_int64), ("ncols", C.c_int64), ("nnz", C.c_int64),
                ("row_ptr", C.POINTER(C.c_int64)), ("col", C.POINTER(C.c_int64)),
                ("val", C.POINTER(C.c_double))]


class _Bcsr(C.Structure):
    _fields_ = [("block", C.c_int32), ("nbrows", C.c_int64), ("nbcols", C.c_int64),
                ("nnzb", C.c_int64), ("brow_ptr", C.POINTER(C.c_int64)),
                ("bcol", C.POINTER(C.c_int64)), ("val", C.POINTER(C.c_double))]


class _Dofmap(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("nodes", C.POINTER(C.c_double)),
                ("n_cells", C.c_int32), ("offsets", C.POINTER(C.c_int32)),
                ("elements", C.POINTER(C.c_int32)), ("topology", C.POINTER(C.c_int8)),
                ("topo_dim", C.POINTER(C.c_int8)), ("poly_order", C.POINTER(C.c_int8))]


def build():
    """Compile liboracle.so (and _ref when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.or_gauss_legendre_1d.argtypes = [C.c_int, f64p, f64p]
        L.or_gauss_lobatto_1d.argtypes = [C.c_int, f64p, f64p]
        L.or_tensor_rule.argtypes = [C.c_int, C.c_int, C.c_int, f64p, f64p]
        L.or_triangle_rule.argtypes = [C.c_int, f64p, f64p]
        L.or_triangle_rule_collapsed.argtypes = [C.c_int, f64p, f64p]
        L.or_set_triangle_rule.argtypes = [C.c_int, f64p, f64p, C.c_int]
        L.or_local_nodes.argtypes = [C.c_int, C.c_int, C.c_int, f64p]
        L.or_element_rule.argtypes = [C.c_int, C.c_int, C.c_int, f64p, f64p]
        L.or_shape_functions.argtypes = [C.c_int, C.c_int, C.c_int, f64p, C.c_int, f64p, f64p]
        L.or_dofmanager.argtypes = [f64p, C.c_int32, i32p, i32p, i32p, C.c_int32, C.c_int32]
        L.or_dofmanager.restype = C.POINTER(_Dofmap)
        L.or_free_dofmap.argtypes = [C.POINTER(_Dofmap)]
        L.or_assemble.argtypes = [C.POINTER(_Dofmap), C.c_int32, C.c_int32, C.c_int32, f64p, C.c_void_p]
        L.or_assemble.restype = C.POINTER(_Csr)
        L.or_local_smoothing_gradient.argtypes = [C.POINTER(_Dofmap), C.c_int32, C.c_int32, f64p, f64p]
        L.or_local_smoothing_gradient.restype = None
        L.or_dirichlet_apply.argtypes = [C.POINTER(_Csr), f64p, u8p, f64p]
        L.or_csr_from_triplets.argtypes = [i64p, i64p, f64p, C.c_int64]
        L.or_csr_from_triplets.restype = C.POINTER(_Csr)
        L.or_bcsr_from_triplets.argtypes = [C.c_int32, i64p, i64p, f64p, C.c_int64]
        L.or_bcsr_from_triplets.restype = C.POINTER(_Bcsr)
        L.or_free_csr.argtypes = [C.POINTER(_Csr)]
        L.or_free_bcsr.argtypes = [C.POINTER(_Bcsr)]
        L.or_csr_spmv.argtypes = [C.POINTER(_Csr), f64p, f64p]
        L.or_bcsr_spmv.argtypes = [C.POINTER(_Bcsr), f64p, f64p]
        L.or_ilu0.argtypes = [C.POINTER(_Csr)]
        L.or_ilu0.restype = C.POINTER(_Csr)
        L.or_ilu_solve.argtypes = [C.POINTER(_Csr), f64p]
        L.or_cg.argtypes = [C.POINTER(_Csr), f64p, f64p, C.c_int32, C.c_int32, C.c_double,
                            C.c_int64, C.POINTER(C.c_double)]
        L.or_cg.restype = C.c_int64
        L.or_bicgstab.argtypes = [C.POINTER(_Csr), f64p, f64p, C.c_int32, C.c_double, C.c_int64,
                                  C.POINTER(C.c_double)]
        L.or_bicgstab.restype = C.c_int64
        L.or_true_relres.argtypes = [C.POINTER(_Csr), f64p, f64p]
        L.or_true_relres.restype = C.c_double
        L.or_num_threads.restype = C.c_int
        _install_reference_triangle_rules(L)
        _LIB = L
    return _LIB


def _install_reference_triangle_rules(L):
    """The reference integrates triangles with its tabulated (Dunavant) rules,
    whose 15-digit constants are part of its arithmetic; the oracle uses the same
    rules, read from the fixture that tests/golden/make_golden.py generated by
    running the reference's own TriangleQuadratureRules.cpp.  Without the fixture
    the oracle falls back to an exact collapsed Gauss-Legendre rule."""
    path = os.path.join(os.path.dirname(HERE), "tests", "golden", "quadrature.npz")
    if not os.path.exists(path):
        return
    g = np.load(path)
    for order in range(1, 7):
        key = "tri_%d_p" % order
        if key in g:
            p = np.ascontiguousarray(g[key], dtype=np.float64).ravel()
            w = np.ascontiguousarray(g["tri_%d_w" % order], dtype=np.float64)
            L.or_set_triangle_rule(order, p, w, w.size)


def triangle_rule_collapsed(order):
    pts, w = np.zeros(3 * 4096), np.zeros(4096)
    nq = lib().or_triangle_rule_collapsed(order, pts, w)
    return pts[:3 * nq].reshape(nq, 3), w[:nq]


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libyafel_ref.so"))


def ref():
    """The reference's own linear algebra / quadrature (compiled in place)."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libyafel_ref.so")
        if not os.path.exists(path):
            build()
        R = C.CDLL(path)
        R.ref_gauss_1d.argtypes = [C.c_int, C.c_int, f64p, f64p]
        R.ref_tensor_rule.argtypes = [C.c_int, C.c_int, C.c_int, f64p, f64p]
        R.ref_triangle_rule.argtypes = [C.c_int, f64p, f64p]
        R.ref_csr_from_triplets.argtypes = [i64p, i64p, f64p, C.c_int64]
        R.ref_csr_from_triplets.restype = C.c_void_p
        R.ref_csr_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 3
        R.ref_csr_get.argtypes = [C.c_void_p, i64p, i64p, f64p]
        R.ref_csr_free.argtypes = [C.c_void_p]
        R.ref_csr_from_csc.argtypes = [C.c_int64, i32p, i32p, f64p]
        R.ref_csr_from_csc.restype = C.c_void_p
        R.ref_csr_spmv.argtypes = [C.c_void_p, f64p, f64p]
        R.ref_bcsr_from_triplets.argtypes = [C.c_int, i64p, i64p, f64p, C.c_int64]
        R.ref_bcsr_from_triplets.restype = C.c_void_p
        R.ref_bcsr_info.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        R.ref_bcsr_get.argtypes = [C.c_int, C.c_void_p, i64p, i64p, f64p]
        R.ref_bcsr_spmv.argtypes = [C.c_int, C.c_void_p, f64p, f64p]
        R.ref_bcsr_free.argtypes = [C.c_int, C.c_void_p]
        R.ref_cg.argtypes = [C.c_void_p, f64p, f64p, C.c_double]
        R.ref_bcsr_cg.argtypes = [C.c_int, C.c_void_p, f64p, f64p, C.c_double]
        R.ref_pcg_jacobi.argtypes = [C.c_void_p, f64p, f64p, C.c_double]
        R.ref_pcg_ilu.argtypes = [C.c_void_p, f64p, f64p, C.c_double]
        R.ref_bicgstab.argtypes = [C.c_void_p, f64p, f64p]
        R.ref_ilu_factor.argtypes = [C.c_void_p]
        R.ref_ilu_factor.restype = C.c_void_p
        R.ref_ilu_apply.argtypes = [C.c_void_p, f64p]
        R.ref_jacobi_apply.argtypes = [C.c_void_p, f64p]
        # the assembly half (ref_assembly.cpp)
        R.refa_set_threads.argtypes = [C.c_int]
        R.refa_dofmanager.argtypes = [f64p, C.c_int, i32p, i32p, i32p, C.c_int, C.c_int, C.c_int]
        R.refa_dofmanager.restype = C.c_void_p
        R.refa_dofmanager_free.argtypes = [C.c_void_p]
        R.refa_dofmanager_sizes.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3
        R.refa_dofmanager_get.argtypes = [C.c_void_p, f64p, i32p, i32p, i8p, i8p, i8p]
        R.refa_assemble.argtypes = [C.c_void_p, C.c_int, C.c_int, f64p, C.c_int, C.c_int]
        R.refa_assemble.restype = C.c_void_p
        R.refa_system_free.argtypes = [C.c_void_p]
        R.refa_system_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        R.refa_system_get.argtypes = [C.c_void_p, i32p, i32p, f64p, f64p]
        R.refa_system_set_residual.argtypes = [C.c_void_p, f64p]
        R.refa_dirichlet_plane.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                           C.c_double, C.POINTER(C.c_int)]
        R.refa_dirichlet_nodes.argtypes = [C.c_void_p, C.c_int, i32p, C.c_int, C.c_double]
        R.refa_local_smoothing_gradient.argtypes = [C.c_void_p, C.c_int, f64p, f64p]
        R.refa_element.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_int)] * 2 + [C.c_void_p] * 5
        R.refa_zz_gradient.argtypes = [C.c_void_p, C.c_int, f64p, f64p]
        R.refa_write_vtu.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int]
        R.refa_read_gmsh.argtypes = [C.c_char_p] + [C.POINTER(C.c_int)] * 4 + [C.c_void_p] * 6
        _REF = R
    return _REF


def ref_element(topology, dim, p, qrm=2):
    """The reference's Element(ElementType{topology, dim, p}, 1, qrm) tables:
    (local nodes nen x 3, quadrature points nq x 3, weights, N nq x nen,
    dN/dxi nq x nen x dim)."""
    R = ref()
    nen, nq = C.c_int(), C.c_int()
    R.refa_element(topology, dim, p, qrm, C.byref(nen), C.byref(nq), None, None, None, None, None)
    a, q = nen.value, nq.value
    L, X, W = np.zeros((a, 3)), np.zeros((q, 3)), np.zeros(q)
    N, dN = np.zeros((q, a)), np.zeros((q, a, dim))
    ptr = lambda x: x.ctypes.data_as(C.c_void_p)
    R.refa_element(topology, dim, p, qrm, C.byref(nen), C.byref(nq), ptr(L), ptr(X), ptr(W), ptr(N), ptr(dN))
    return L, X, W, N, dN


def ref_read_gmsh(path):
    """The reference's Mesh(fname) (src/mesh/parse_gmsh.cpp): dict of nodes,
    cell_nodes, offsets, cell_types, tag_offsets, tags."""
    R = ref()
    a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    if R.refa_read_gmsh(path.encode(), C.byref(a), C.byref(b), C.byref(c), C.byref(d), None, None, None, None,
                        None, None):
        raise RuntimeError("Mesh::parse_gmsh failed")
    out = {"nodes": np.zeros((a.value, 3)), "cell_nodes": np.zeros(max(1, c.value), np.int32),
           "offsets": np.zeros(b.value + 1, np.int32), "cell_types": np.zeros(max(1, b.value), np.int32),
           "tag_offsets": np.zeros(b.value + 1, np.int32), "tags": np.zeros(max(1, d.value), np.int32)}
    ptr = lambda x: x.ctypes.data_as(C.c_void_p)
    R.refa_read_gmsh(path.encode(), C.byref(a), C.byref(b), C.byref(c), C.byref(d), ptr(out["nodes"]),
                     ptr(out["cell_nodes"]), ptr(out["offsets"]), ptr(out["cell_types"]), ptr(out["tag_offsets"]),
                     ptr(out["tags"]))
    out["cell_nodes"], out["cell_types"] = out["cell_nodes"][:c.value], out["cell_types"][:b.value]
    out["tags"] = out["tags"][:d.value]
    return out


class RefDofManager:
    """The reference's own Mesh + DoFManager(M, CG, p, dpn) (src/utils/DoFManager.cpp),
    compiled in place; arrays copied out after construction."""

    def __init__(self, mesh, p, dpn=1):
        R = ref()
        nodes = np.ascontiguousarray(mesh["nodes"], dtype=np.float64).ravel()
        cn = np.ascontiguousarray(mesh["cell_nodes"], dtype=np.int32)
        off = np.ascontiguousarray(mesh["offsets"], dtype=np.int32)
        ct = np.ascontiguousarray(mesh["cell_types"], dtype=np.int32)
        self.h = R.refa_dofmanager(nodes, nodes.size // 3, cn, off, ct, ct.size, p, dpn)
        if not self.h:
            raise RuntimeError("DoFManager: Invalid polynomial order")
        self.dpn = dpn
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        R.refa_dofmanager_sizes(self.h, C.byref(a), C.byref(b), C.byref(c))
        self.n_nodes, self.n_cells = a.value, b.value
        self.nodes = np.zeros(3 * max(1, a.value))
        self.offsets = np.zeros(b.value + 1, np.int32)
        self.elements = np.zeros(max(1, c.value), np.int32)
        self.topology = np.zeros(max(1, b.value), np.int8)
        self.topo_dim = np.zeros(max(1, b.value), np.int8)
        self.poly_order = np.zeros(max(1, b.value), np.int8)
        R.refa_dofmanager_get(self.h, self.nodes, self.offsets, self.elements, self.topology,
                              self.topo_dim, self.poly_order)
        self.nodes = self.nodes[:3 * a.value].reshape(-1, 3)
        self.elements = self.elements[:c.value]
        self.topology, self.topo_dim = self.topology[:b.value], self.topo_dim[:b.value]
        self.poly_order = self.poly_order[:b.value]

    def __del__(self):
        if getattr(self, "h", None) and _REF is not None:
            _REF.refa_dofmanager_free(self.h)
            self.h = None


class RefSystem:
    """FESystem + CGAssembly<Physics> of the reference (include/assembly/CGAssembly.hpp),
    run single-threaded so that duplicates are summed in element order.
    physics: POISSON {sign, f}, ELASTICITY {sign, lambda, mu, b0, b1, b2},
    SUPG (the reference's AdvectionDiffusionSUPG with its own constants), or
    SUPG_PARAM {k, h, U0, Q} (the same formulas with run-time constants)."""

    def __init__(self, dm, nsd, physics, params=None, tangent=True, residual=True, threads=1):
        R = ref()
        self.dm = dm
        prm = np.zeros(8)
        if params is not None:
            prm[:len(params)] = params
        R.refa_set_threads(threads)
        self.h = R.refa_assemble(dm.h, physics, nsd, prm, int(tangent), int(residual))
        n, nnz = C.c_int64(), C.c_int64()
        R.refa_system_sizes(self.h, C.byref(n), C.byref(nnz))
        self.n, self.nnz = n.value, nnz.value

    def matrix(self):
        """(Csr of K, residual): Eigen's ColMajor storage transposed to row-major."""
        cp = np.zeros(self.n + 1, np.int32)
        ri = np.zeros(max(1, self.nnz), np.int32)
        v = np.zeros(max(1, self.nnz))
        res = np.zeros(max(1, self.n))
        ref().refa_system_get(self.h, cp, ri, v, res)
        ri, v = ri[:self.nnz], v[:self.nnz]
        cols = np.repeat(np.arange(self.n, dtype=np.int64), np.diff(cp))
        order = np.lexsort((cols, ri))
        row_ptr = np.zeros(self.n + 1, np.int64)
        np.add.at(row_ptr, ri.astype(np.int64) + 1, 1)
        return Csr(self.n, self.n, np.cumsum(row_ptr), cols[order], v[order]), res[:self.n]

    def csc(self):
        """Eigen's ColMajor arrays of the tangent (column pointers, row indices,
        values) and the residual, copied out."""
        cp = np.zeros(self.n + 1, np.int32)
        ri = np.zeros(max(1, self.nnz), np.int32)
        v = np.zeros(max(1, self.nnz))
        res = np.zeros(max(1, self.n))
        ref().refa_system_get(self.h, cp, ri, v, res)
        return cp, ri, v, res[:self.n]

    def to_ref_csr(self):
        """The tangent as the reference's handmade sparse_csr (its triplet
        constructor over Eigen's entries) and the residual."""
        cp, ri, v, res = self.csc()
        return RefCsr.from_handle(ref().ref_csr_from_csc(self.n, cp, ri, v)), res

    def set_residual(self, r):
        ref().refa_system_set_residual(self.h, np.ascontiguousarray(r, dtype=np.float64))

    def dirichlet_plane(self, comp, axis, coord, value=0.0, tol=1e-9):
        """DirichletBC(dofm, value, comp).selectByFunction(|x[axis]-coord| < tol).apply(K, F)."""
        n = C.c_int()
        ref().refa_dirichlet_plane(self.h, comp, axis, coord, tol, value, C.byref(n))
        return n.value

    def dirichlet_nodes(self, comp, nodes, value=0.0):
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        ref().refa_dirichlet_nodes(self.h, comp, nodes, nodes.size, value)

    def local_smoothing_gradient(self, nsd, sol):
        out = np.zeros((self.n, nsd))
        ref().refa_local_smoothing_gradient(self.h, nsd, np.ascontiguousarray(sol, dtype=np.float64), out)
        return out

    def write_vtu(self, fname_base, sol=None):
        """SimulationOutput(fname_base, VTU).captureFrame(system) (default capture
        of `sol`, or no data); returns the file's text."""
        a = None if sol is None else np.ascontiguousarray(sol, dtype=np.float64)
        ref().refa_write_vtu(self.h, fname_base.encode(), None if a is None else a.ctypes.data_as(C.c_void_p),
                             0 if a is None else 1)
        with open(fname_base + ".vtu") as f:
            return f.read()

    def zz_gradient(self, nsd, sol):
        """ZZGradientRecovery (include/assembly/ZZGradientRecovery.hpp:33-140): the
        patch-recovered nodal gradient of a p = 1 scalar field, (n_nodes, nsd)."""
        out = np.zeros((self.n, nsd))
        ref().refa_zz_gradient(self.h, nsd, np.ascontiguousarray(sol, dtype=np.float64), out)
        return out

    def __del__(self):
        if getattr(self, "h", None) and _REF is not None:
            _REF.refa_system_free(self.h)
            self.h = None


# ---------------------------------------------------------------- helpers

class Csr:
    """Host CSR (int64 indices, float64 values) owned by numpy."""

    def __init__(self, nrows, ncols, row_ptr, col, val):
        self.nrows, self.ncols = int(nrows), int(ncols)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int64)
        self.val = np.ascontiguousarray(val, dtype=np.float64)

    @property
    def nnz(self):
        return int(self.col.size)

    def _struct(self):
        s = _Csr(self.nrows, self.ncols, self.nnz,
                 self.row_ptr.ctypes.data_as(C.POINTER(C.c_int64)),
                 self.col.ctypes.data_as(C.POINTER(C.c_int64)),
                 self.val.ctypes.data_as(C.POINTER(C.c_double)))
        return s

    def spmv(self, x):
        y = np.empty(self.nrows)
        s = self._struct()
        lib().or_csr_spmv(C.byref(s), np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def copy(self):
        return Csr(self.nrows, self.ncols, self.row_ptr.copy(), self.col.copy(), self.val.copy())

    def diagonal(self):
        d = np.zeros(self.nrows)
        rows = np.repeat(np.arange(self.nrows), np.diff(self.row_ptr))
        m = rows == self.col
        d[rows[m]] = self.val[m]
        return d


def _csr_from_ptr(p):
    s = p.contents
    n, nnz = s.nrows, s.nnz
    rp = np.ctypeslib.as_array(s.row_ptr, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(s.col, shape=(max(nnz, 1),))[:nnz].copy()
    val = np.ctypeslib.as_array(s.val, shape=(max(nnz, 1),))[:nnz].copy()
    out = Csr(n, s.ncols, rp, col, val)
    lib().or_free_csr(p)
    return out


def gauss_1d(n, lobatto=False):
    x, w = np.zeros(n), np.zeros(n)
    (lib().or_gauss_lobatto_1d if lobatto else lib().or_gauss_legendre_1d)(n, x, w)
    return x, w


def tensor_rule(dim, order, lobatto=False):
    pts, w = np.zeros(3 * 4096), np.zeros(4096)
    nq = lib().or_tensor_rule(int(lobatto), dim, order, pts, w)
    return pts[:3 * nq].reshape(nq, 3), w[:nq]


def triangle_rule(order):
    pts, w = np.zeros(3 * 4096), np.zeros(4096)
    nq = lib().or_triangle_rule(order, pts, w)
    return pts[:3 * nq].reshape(nq, 3), w[:nq]


def element_rule(topology, dim, p):
    pts, w = np.zeros(3 * 4096), np.zeros(4096)
    nq = lib().or_element_rule(topology, dim, p, pts, w)
    return pts[:3 * nq].reshape(nq, 3), w[:nq]


def local_nodes(topology, dim, p):
    pts = np.zeros(3 * 512)
    n = lib().or_local_nodes(topology, dim, p, pts)
    return pts[:3 * n].reshape(n, 3)


def shape_functions(topology, dim, p, qpts):
    qpts = np.ascontiguousarray(qpts, dtype=np.float64).reshape(-1, 3)
    nq = qpts.shape[0]
    nen = local_nodes(topology, dim, p).shape[0]
    N, dN = np.zeros(nq * nen), np.zeros(nq * nen * dim)
    r = lib().or_shape_functions(topology, dim, p, qpts.ravel(), nq, N, dN)
    assert r == nen
    return N.reshape(nq, nen), dN.reshape(nq, nen, dim)


class DofMap:
    def __init__(self, ptr):
        self._p = ptr
        s = ptr.contents
        self.n_nodes, self.n_cells = s.n_nodes, s.n_cells
        self.nodes = np.ctypeslib.as_array(s.nodes, shape=(max(1, 3 * s.n_nodes),))[:3 * s.n_nodes].reshape(-1, 3).copy()
        self.offsets = np.ctypeslib.as_array(s.offsets, shape=(s.n_cells + 1,)).copy()
        ne = int(self.offsets[-1])
        self.elements = np.ctypeslib.as_array(s.elements, shape=(max(ne, 1),))[:ne].copy()
        self.topology = np.ctypeslib.as_array(s.topology, shape=(max(1, s.n_cells),))[:s.n_cells].copy()
        self.topo_dim = np.ctypeslib.as_array(s.topo_dim, shape=(max(1, s.n_cells),))[:s.n_cells].copy()

    def __del__(self):
        if getattr(self, "_p", None) is not None and _LIB is not None:
            _LIB.or_free_dofmap(self._p)
            self._p = None


class ArrayDofMap:
    """An oracle dofmap over caller-held numbering arrays (the reference's own
    DoFManager output, say), for assembling on exactly that numbering."""

    _TOPO = {0: (TENSOR, 1), 1: (SIMPLEX, 2), 2: (SIMPLEX, 3), 3: (TENSOR, 2), 4: (TENSOR, 3)}

    def __init__(self, dof_nodes, element_offsets, elements, cell_types, p):
        self.nodes = np.ascontiguousarray(np.asarray(dof_nodes, dtype=np.float64).reshape(-1, 3))
        self.offsets = np.ascontiguousarray(element_offsets, dtype=np.int32)
        self.elements = np.ascontiguousarray(elements, dtype=np.int32)
        ct = np.asarray(cell_types)
        self.topology = np.array([self._TOPO.get(int(c), (NONE, 0))[0] for c in ct], np.int8)
        self.topo_dim = np.array([self._TOPO.get(int(c), (NONE, 0))[1] for c in ct], np.int8)
        self.poly_order = np.full(ct.size, p, np.int8)
        self.n_nodes, self.n_cells = self.nodes.shape[0], ct.size
        self._s = _Dofmap(self.n_nodes, self.nodes.ctypes.data_as(C.POINTER(C.c_double)), self.n_cells,
                          self.offsets.ctypes.data_as(C.POINTER(C.c_int32)),
                          self.elements.ctypes.data_as(C.POINTER(C.c_int32)),
                          self.topology.ctypes.data_as(C.POINTER(C.c_int8)),
                          self.topo_dim.ctypes.data_as(C.POINTER(C.c_int8)),
                          self.poly_order.ctypes.data_as(C.POINTER(C.c_int8)))
        self._p = C.pointer(self._s)


def dofmanager(mesh, p):
    nodes = np.ascontiguousarray(mesh["nodes"], dtype=np.float64).ravel()
    cn = np.ascontiguousarray(mesh["cell_nodes"], dtype=np.int32)
    off = np.ascontiguousarray(mesh["offsets"], dtype=np.int32)
    ct = np.ascontiguousarray(mesh["cell_types"], dtype=np.int32)
    ptr = lib().or_dofmanager(nodes, nodes.size // 3, cn, off, ct, ct.size, p)
    if not ptr:
        raise RuntimeError("DoFManager: Invalid polynomial order")
    return DofMap(ptr)


def assemble(dm, dpn, nsd, physics, params, residual=True):
    params = np.zeros(8) if params is None else np.ascontiguousarray(
        np.pad(np.asarray(params, dtype=np.float64), (0, max(0, 8 - len(params)))), dtype=np.float64)
    R = np.zeros(dm.n_nodes * dpn) if residual else None
    p = lib().or_assemble(dm._p, dpn, nsd, physics, params,
                          R.ctypes.data_as(C.c_void_p) if R is not None else None)
    return _csr_from_ptr(p), R


def local_smoothing_gradient(dm, dpn, nsd, sol):
    """LocalSmoothingGradient (include/assembly/LocalSmoothingGradient.hpp:20-94):
    the nodal gradient, shape (n_nodes*dpn, nsd)."""
    sol = np.ascontiguousarray(sol, dtype=np.float64)
    out = np.zeros((dm.n_nodes * dpn, nsd))
    lib().or_local_smoothing_gradient(dm._p, dpn, nsd, sol, out)
    return out


def dirichlet_apply(A, rhs, mask, vals):
    s = A._struct()
    lib().or_dirichlet_apply(C.byref(s), rhs, np.ascontiguousarray(mask, dtype=np.uint8),
                             np.ascontiguousarray(vals, dtype=np.float64))


def csr_from_triplets(r, c, v):
    r = np.ascontiguousarray(r, dtype=np.int64)
    c = np.ascontiguousarray(c, dtype=np.int64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    return _csr_from_ptr(lib().or_csr_from_triplets(r, c, v, r.size))


def bcsr_from_triplets(block, r, c, v):
    r = np.ascontiguousarray(r, dtype=np.int64)
    c = np.ascontiguousarray(c, dtype=np.int64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    p = lib().or_bcsr_from_triplets(block, r, c, v, r.size)
    s = p.contents
    nb = s.nnzb
    out = dict(block=block, nbrows=s.nbrows, nbcols=s.nbcols, nnzb=nb,
               brow_ptr=np.ctypeslib.as_array(s.brow_ptr, shape=(s.nbrows + 1,)).copy(),
               bcol=np.ctypeslib.as_array(s.bcol, shape=(max(nb, 1),))[:nb].copy(),
               val=np.ctypeslib.as_array(s.val, shape=(max(nb * block * block, 1),))[:nb * block * block].copy())
    lib().or_free_bcsr(p)
    return out


def bcsr_spmv(B, x):
    s = _Bcsr(B["block"], B["nbrows"], B["nbcols"], B["nnzb"],
              B["brow_ptr"].ctypes.data_as(C.POINTER(C.c_int64)),
              B["bcol"].ctypes.data_as(C.POINTER(C.c_int64)),
              B["val"].ctypes.data_as(C.POINTER(C.c_double)))
    y = np.zeros(B["nbrows"] * B["block"])
    lib().or_bcsr_spmv(C.byref(s), np.ascontiguousarray(x, dtype=np.float64), y)
    return y


def ilu0(A):
    s = A._struct()
    return _csr_from_ptr(lib().or_ilu0(C.byref(s)))


def ilu_solve(F, z):
    z = np.ascontiguousarray(z, dtype=np.float64).copy()
    s = F._struct()
    lib().or_ilu_solve(C.byref(s), z)
    return z


def cg(A, b, x0=None, precond=PRECOND_NONE, criterion=CRIT_RELRES, tol=1e-10, maxiter=0):
    x = np.zeros(A.nrows) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
    rr = C.c_double(0)
    s = A._struct()
    it = lib().or_cg(C.byref(s), np.ascontiguousarray(b, dtype=np.float64), x, precond, criterion,
                     tol, maxiter, C.byref(rr))
    return x, int(it), rr.value


def bicgstab(A, b, x0=None, criterion=CRIT_RELRES, tol=1e-10, maxiter=0):
    x = np.zeros(A.nrows) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
    rr = C.c_double(0)
    s = A._struct()
    it = lib().or_bicgstab(C.byref(s), np.ascontiguousarray(b, dtype=np.float64), x, criterion,
                           tol, maxiter, C.byref(rr))
    return x, int(it), rr.value


def true_relres(A, b, x):
    s = A._struct()
    return lib().or_true_relres(C.byref(s), np.ascontiguousarray(b, dtype=np.float64),
                                np.ascontiguousarray(x, dtype=np.float64))


# ------------------------------------------------- the reference itself (_ref)

class RefCsr:
    """The reference's sparse_csr<double>, built from triplets by its own ctor."""

    def __init__(self, r, c, v):
        R = ref()
        self._r, self._c, self._v = (np.ascontiguousarray(r, dtype=np.int64),
                                     np.ascontiguousarray(c, dtype=np.int64),
                                     np.ascontiguousarray(v, dtype=np.float64))
        self.h = R.ref_csr_from_triplets(self._r, self._c, self._v, self._r.size)
        a, b, n = C.c_int64(), C.c_int64(), C.c_int64()
        R.ref_csr_info(self.h, C.byref(a), C.byref(b), C.byref(n))
        self.nrows, self.ncols, self.nnz = a.value, b.value, n.value

    @classmethod
    def from_handle(cls, h):
        self = cls.__new__(cls)
        self.h = h
        a, b, n = C.c_int64(), C.c_int64(), C.c_int64()
        ref().ref_csr_info(self.h, C.byref(a), C.byref(b), C.byref(n))
        self.nrows, self.ncols, self.nnz = a.value, b.value, n.value
        return self

    def arrays(self):
        rp = np.zeros(self.nrows + 1, np.int64)
        col = np.zeros(max(self.nnz, 1), np.int64)
        val = np.zeros(max(self.nnz, 1))
        ref().ref_csr_get(self.h, rp, col, val)
        return rp, col[:self.nnz], val[:self.nnz]

    def spmv(self, x):
        y = np.zeros(self.nrows)
        ref().ref_csr_spmv(self.h, np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def cg(self, b, x0, tol):
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        ref().ref_cg(self.h, np.ascontiguousarray(b, dtype=np.float64), x, tol)
        return x

    def true_relres(self, b, x):
        """||b - A x|| / ||b|| with A x from the reference's csr_spmv."""
        r = np.asarray(b, dtype=np.float64) - self.spmv(x)
        return float(np.linalg.norm(r) / np.linalg.norm(b))

    def pcg_jacobi(self, b, x0, tol):
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        ref().ref_pcg_jacobi(self.h, np.ascontiguousarray(b, dtype=np.float64), x, tol)
        return x

    def pcg_ilu(self, b, x0, tol):
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        ref().ref_pcg_ilu(self.h, np.ascontiguousarray(b, dtype=np.float64), x, tol)
        return x

    def bicgstab(self, b, x0):
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        ref().ref_bicgstab(self.h, np.ascontiguousarray(b, dtype=np.float64), x)
        return x

    def ilu_factor_values(self):
        h = ref().ref_ilu_factor(self.h)
        rp = np.zeros(self.nrows + 1, np.int64)
        col = np.zeros(max(self.nnz, 1), np.int64)
        val = np.zeros(max(self.nnz, 1))
        ref().ref_csr_get(h, rp, col, val)
        ref().ref_csr_free(h)
        return val[:self.nnz]

    def __del__(self):
        if getattr(self, "h", None) and _REF is not None:
            _REF.ref_csr_free(self.h)
            self.h = None


def csr_to_triplets(A):
    rows = np.repeat(np.arange(A.nrows, dtype=np.int64), np.diff(A.row_ptr))
    return rows, A.col.copy(), A.val.copy()
