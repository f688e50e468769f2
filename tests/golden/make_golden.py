"""Generate the golden fixtures in this directory from the reference's own code.

Run here (where the reference tree exists and oracle/_ref is built):
    python tests/golden/make_golden.py
The fixtures hold outputs of the reference's own code compiled in place by
oracle/Makefile: its handmade linear algebra and quadrature on the inputs its
own tests use (test/test_sparse_csr.cpp, test_sparse_bcsr.cpp,
test_cg_solve.cpp, test_bicgstab_solve.cpp, test_ILU.cpp) and on a small
assembled Poisson system (linalg.npz, quadrature.npz, poisson8.npz); and its
assembly half -- Element tables, DoFManager numbering, CGAssembly values and
residuals, DirichletBC::apply, LocalSmoothingGradient, ZZGradientRecovery and
the VTU writer's text, and its Gmsh reader on files written here -- on small
seeded quadrilateral, triangle, mixed, hexahedron and tetrahedron meshes at
orders 1-3 (elements.npz, assembly_ref.npz, zz_ref.npz, vtu_ref.npz,
gmsh_ref.npz), built
against the from-scratch Eigen-API subset in oracle/ref_compat (Eigen itself is
not installed).
They pin the oracle without the reference tree being present.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from yafel_b200 import meshgen  # noqa: E402


def quadrature():
    R = O.ref()
    out = {}
    for lob in (0, 1):
        for n in range(2, 10 if lob == 0 else 11):  # the reference's GL loop never ends at n=10
            x, w = np.zeros(n), np.zeros(n)
            R.ref_gauss_1d(lob, n, x, w)
            out["g1d_%d_%d_x" % (lob, n)] = x
            out["g1d_%d_%d_w" % (lob, n)] = w
    for dim in (1, 2, 3):
        for order in range(1, 10):
            p, w = np.zeros(3 * 4096), np.zeros(4096)
            nq = R.ref_tensor_rule(0, dim, order, p, w)
            out["tp_%d_%d_p" % (dim, order)] = p[:3 * nq].reshape(nq, 3)
            out["tp_%d_%d_w" % (dim, order)] = w[:nq]
    for order in range(1, 7):
        p, w = np.zeros(3 * 256), np.zeros(256)
        nq = R.ref_triangle_rule(order, p, w)
        out["tri_%d_p" % order] = p[:3 * nq].reshape(nq, 3)
        out["tri_%d_w" % order] = w[:nq]
    np.savez_compressed(os.path.join(HERE, "quadrature.npz"), **out)


def laplace_5pt(N):
    """2D five-point Laplacian of test/test_ILU.cpp:13-33 (diag -4, neighbours 1)."""
    NN = N * N
    r, c, v = [], [], []
    for i in range(NN):
        r.append(i); c.append(i); v.append(-4.0)
        if i >= 1: r.append(i); c.append(i - 1); v.append(1.0)
        if i >= N: r.append(i); c.append(i - N); v.append(1.0)
        if i < NN - 1: r.append(i); c.append(i + 1); v.append(1.0)
        if i < NN - N: r.append(i); c.append(i + N); v.append(1.0)
    return np.array(r), np.array(c), np.array(v)


def linalg():
    out = {}
    rng = np.random.Generator(np.random.PCG64(20261203))
    # test_sparse_csr.cpp test_3: accumulation into two nonzeros
    N = 10
    r = np.array([N - 1, 0] * N); c = r.copy(); v = np.ones(2 * N)
    A = O.RefCsr(r, c, v)
    out["dup_in"] = np.stack([r, c, v])
    out["dup_rp"], out["dup_col"], out["dup_val"] = A.arrays()
    # test_sparse_csr.cpp test_4: random integer matrix, seeded here
    r = rng.integers(0, 20, 500); c = rng.integers(0, 20, 500); v = rng.integers(-10, 11, 500).astype(float)
    A = O.RefCsr(r, c, v)
    out["rand_in"] = np.stack([r, c, v])
    out["rand_rp"], out["rand_col"], out["rand_val"] = A.arrays()
    # test_sparse_bcsr.cpp test_1: 60x60 dense fill read back through BCSR<3>
    ii, jj = np.meshgrid(np.arange(60), np.arange(60), indexing="ij")
    r, c, v = ii.ravel(), jj.ravel(), (ii * 60 + jj).ravel().astype(float)
    R = O.ref()
    h = R.ref_bcsr_from_triplets(3, np.ascontiguousarray(r, np.int64), np.ascontiguousarray(c, np.int64),
                                 np.ascontiguousarray(v), r.size)
    import ctypes as C
    nb, nnzb = C.c_int64(), C.c_int64()
    R.ref_bcsr_info(3, h, C.byref(nb), C.byref(nnzb))
    brp = np.zeros(nb.value + 1, np.int64); bcol = np.zeros(nnzb.value, np.int64); bval = np.zeros(9 * nnzb.value)
    R.ref_bcsr_get(3, h, brp, bcol, bval)
    x = rng.standard_normal(60)
    y = np.zeros(60)
    R.ref_bcsr_spmv(3, h, x, y)
    R.ref_bcsr_free(3, h)
    out["bcsr60_rp"], out["bcsr60_col"], out["bcsr60_val"] = brp, bcol, bval
    out["bcsr60_x"], out["bcsr60_y"] = x, y
    # test_cg_solve.cpp / test_bicgstab_solve.cpp test_2: tridiag(1,-2,1), x_ref = i
    N = 10
    r = list(range(N)) + list(range(1, N)) + list(range(0, N - 1))
    c = list(range(N)) + list(range(0, N - 1)) + list(range(1, N))
    v = [-2.0] * N + [1.0] * (2 * (N - 1))
    A = O.RefCsr(r, c, v)
    b = A.spmv(np.arange(N, dtype=float))
    out["lap_in"] = np.stack([np.array(r), np.array(c), np.array(v)])
    out["lap_b"] = b
    out["lap_cg"] = A.cg(b, np.zeros(N), 1e-14)
    out["lap_bicgstab"] = A.bicgstab(b, np.zeros(N))
    # test_cg_solve.cpp test_1: identity with integer rhs -> exact
    rhs = rng.integers(0, 100, 10).astype(float)
    A = O.RefCsr(np.arange(10), np.arange(10), np.ones(10))
    out["ident_b"] = rhs
    out["ident_cg"] = A.cg(rhs, np.zeros(10), 1e-14)
    # test_ILU.cpp: ILU(0) factors of the 5x5-grid Laplacian
    r, c, v = laplace_5pt(5)
    A = O.RefCsr(r, c, v)
    out["ilu5_in"] = np.stack([r, c, v])
    out["ilu5_lu"] = A.ilu_factor_values()
    z = rng.standard_normal(25)
    out["ilu5_z"] = z
    zz = z.copy(); O.ref().ref_ilu_apply(A.h, zz)
    out["ilu5_apply"] = zz
    np.savez_compressed(os.path.join(HERE, "linalg.npz"), **out)


def poisson_system():
    """8x8 Q1 Poisson (SPD sign, f=1), Dirichlet u=0 on the boundary, assembled by
    the oracle; solved by the reference's pcg_solve (Jacobi and ILU) and cg_solve."""
    m = meshgen.structured_quad(8, 8, order="tensor")
    dm = O.dofmanager(m, 1)
    K, R = O.assemble(dm, 1, 2, O.POISSON, [1.0, 1.0])
    X = dm.nodes
    mask = ((np.abs(X[:, 0]) < 1e-9) | (np.abs(X[:, 0] - 1) < 1e-9) |
            (np.abs(X[:, 1]) < 1e-9) | (np.abs(X[:, 1] - 1) < 1e-9)).astype(np.uint8)
    O.dirichlet_apply(K, R, mask, np.zeros(K.nrows))
    r, c, v = O.csr_to_triplets(K)
    A = O.RefCsr(r, c, v)
    out = {"rp": K.row_ptr, "col": K.col, "val": K.val, "b": R, "mask": mask}
    out["pcg_jacobi"] = A.pcg_jacobi(R, np.zeros(K.nrows), 1e-20)
    out["pcg_ilu"] = A.pcg_ilu(R, np.zeros(K.nrows), 1e-20)
    out["cg"] = A.cg(R, np.zeros(K.nrows), 1e-20)
    out["ilu_lu"] = A.ilu_factor_values()
    np.savez_compressed(os.path.join(HERE, "poisson8.npz"), **out)


# ------------------------------------------------ the reference's assembly half

ELEMENT_TYPES = ([(0, 1, p) for p in (1, 2, 3, 4)] + [(0, 2, p) for p in (1, 2, 3, 4)] +
                 [(0, 3, p) for p in (1, 2, 3)] + [(1, 2, p) for p in (1, 2, 3)] + [(1, 3, p) for p in (1, 2)])


def elements():
    """Element tables (local nodes, quadrature, N, dN/dxi) of the reference's own
    Element(ElementType{topology, dim, p}) (src/element/*.cpp, compiled against
    oracle/ref_compat)."""
    out = {}
    for topo, dim, p in ELEMENT_TYPES:
        L, X, W, N, dN = O.ref_element(topo, dim, p)
        k = "e%d_%d_%d_" % (topo, dim, p)
        out[k + "L"], out[k + "X"], out[k + "W"], out[k + "N"], out[k + "dN"] = L, X, W, N, dN
    np.savez_compressed(os.path.join(HERE, "elements.npz"), **out)


def _jitter(mesh, h, amount, seed):
    """Move the interior nodes of a structured mesh by U(-amount, amount)*h."""
    m = dict(mesh)
    X = m["nodes"].copy()
    lo, hi = X.min(0), X.max(0)
    inner = np.all((X > lo + 1e-9) | (hi - lo < 1e-12), axis=1) & np.all((X < hi - 1e-9) | (hi - lo < 1e-12), axis=1)
    rng = np.random.Generator(np.random.PCG64(seed))
    d = rng.uniform(-amount, amount, size=X.shape) * np.asarray(h)
    d[:, (hi - lo) < 1e-12] = 0
    X[inner] += d[inner]
    m["nodes"] = X
    return m


def assembly_meshes(kind, p):
    o = meshgen.corner_order(p)
    if kind == "quad":
        return _jitter(meshgen.structured_quad(4, 3, order=o), (0.25, 1 / 3, 0), 0.2, 11), 2
    if kind == "mixed":
        return meshgen.jittered_mixed(4, 4, seed=5, order=o), 2
    if kind == "tri":
        return meshgen.jittered_mixed(3, 3, seed=8, tri_fraction=1.0, order=o), 2
    if kind == "hex":
        return _jitter(meshgen.structured_hex(2, 2, 2, order=o), (0.5, 0.5, 0.5), 0.15, 12), 3
    if kind == "tet":
        return meshgen.structured_tet(2, 2, 2, seed=13, jitter=0.15), 3
    raise ValueError(kind)


LAM, MU = 0.5769230769230769, 0.38461538461538464  # E=1, nu=0.3
# (name, mesh kind, p, physics, params); dpn = nsd for elasticity, else 1
ASSEMBLY_CASES = (
    [("quad_poisson_p%d" % p, "quad", p, O.POISSON, [1.0, 1.3]) for p in (1, 2, 3)] +
    [("quad_poisson_refsign_p2", "quad", 2, O.POISSON, [-1.0, 100.0])] +
    [("quad_elast_p%d" % p, "quad", p, O.ELASTICITY, [1.0, LAM, MU, 0.5, -1.0]) for p in (1, 2, 3)] +
    [("mixed_poisson_p%d" % p, "mixed", p, O.POISSON, [1.0, 1.0]) for p in (1, 2, 3)] +
    [("mixed_elast_p%d" % p, "mixed", p, O.ELASTICITY, [1.0, LAM, MU, 0.0, -1.0]) for p in (2, 3)] +
    [("mixed_supg_p%d" % p, "mixed", p, O.SUPG, None) for p in (1, 2, 3)] +
    [("tri_poisson_p%d" % p, "tri", p, O.POISSON, [1.0, 2.0]) for p in (1, 2, 3)] +
    [("hex_poisson_p%d" % p, "hex", p, O.POISSON, [1.0, 1.0]) for p in (1, 2, 3)] +
    [("hex_elast_p%d" % p, "hex", p, O.ELASTICITY, [1.0, LAM, MU, 1.0, 0.0, -0.5]) for p in (1, 2)] +
    [("hex_supg_p2", "hex", 2, O.SUPG, None)] +
    [("tet_poisson_p%d" % p, "tet", p, O.POISSON, [1.0, 1.0]) for p in (1, 2)] +
    [("tet_elast_p%d" % p, "tet", p, O.ELASTICITY, [1.0, LAM, MU, 0.0, 0.0, 1.0]) for p in (1, 2)]
)
# the reference's AdvectionDiffusionSUPG constants (apps/supg_learning/supg_advection.hpp:110-113)
SUPG_PARAMS = [0.1, 0.1, 1.0, 0.0]


def smooth_field(X, comp):
    """A non-linear field sampled at the dof nodes, for the gradient fixtures."""
    return np.sin(2 * X[:, 0]) + X[:, 0] * X[:, 1] ** 2 + 0.5 * X[:, 2] + comp * (X[:, 0] - X[:, 1] ** 2)


def assembly():
    """The reference's DoFManager, CGAssembly<Physics>, DirichletBC::apply and
    LocalSmoothingGradient run on small seeded meshes (one thread, so that
    duplicate sums follow element order)."""
    out = {}
    for name, kind, p, phys, params in ASSEMBLY_CASES:
        mesh, nsd = assembly_meshes(kind, p)
        dpn = nsd if phys == O.ELASTICITY else 1
        dm = O.RefDofManager(mesh, p, dpn)
        sysm = O.RefSystem(dm, nsd, phys, params)
        K, R = sysm.matrix()
        k = name + "/"
        for key in ("nodes", "cell_nodes", "offsets", "cell_types"):
            out[k + "mesh_" + key] = mesh[key]
        out[k + "dof_nodes"], out[k + "element_offsets"], out[k + "elements"] = dm.nodes, dm.offsets, dm.elements
        out[k + "row_ptr"], out[k + "col"] = K.row_ptr.astype(np.int32), K.col.astype(np.int32)
        out[k + "val"], out[k + "residual"] = K.val, R
        # two Dirichlet objects: comp 0 = 0.25 on x = min, comp dpn-1 = -0.5 on y = min
        X = dm.nodes
        nsel0 = sysm.dirichlet_plane(0, 0, X[:, 0].min(), 0.25)
        nsel1 = sysm.dirichlet_plane(dpn - 1, 1, X[:, 1].min(), -0.5)
        Kb, Rb = sysm.matrix()
        out[k + "bc_val"], out[k + "bc_rhs"], out[k + "bc_count"] = Kb.val, Rb, np.array([nsel0, nsel1])
        u = np.stack([smooth_field(X, c) for c in range(dpn)], axis=1).ravel()
        out[k + "grad_u"] = u
        out[k + "grad"] = sysm.local_smoothing_gradient(nsd, u)
        out[k + "meta"] = np.array([p, dpn, nsd, phys] + list(params if params is not None else SUPG_PARAMS))
    np.savez_compressed(os.path.join(HERE, "assembly_ref.npz"), **out)


def zz():
    """The reference's ZZGradientRecovery (p = 1, one dof per node) of a
    non-linear field on the p = 1 meshes of assembly_meshes."""
    out = {}
    for kind in ("quad", "mixed", "tri", "hex", "tet"):
        mesh, nsd = assembly_meshes(kind, 1)
        dm = O.RefDofManager(mesh, 1, 1)
        sysm = O.RefSystem(dm, nsd, O.POISSON, [1.0, 1.0])
        u = smooth_field(dm.nodes, 0)
        k = kind + "/"
        for key in ("nodes", "cell_nodes", "offsets", "cell_types"):
            out[k + "mesh_" + key] = mesh[key]
        out[k + "u"], out[k + "grad"], out[k + "nsd"] = u, sysm.zz_gradient(nsd, u), np.array(nsd)
    np.savez_compressed(os.path.join(HERE, "zz_ref.npz"), **out)


VTU_CASES = [("quad", 2, 1), ("mixed", 3, 1), ("tri", 1, 1), ("hex", 2, 3), ("tet", 2, 1)]


def vtu():
    """The reference's SimulationOutput(VTU).captureFrame text, mesh only and with
    the default capture of a solution (dof_per_node components)."""
    import tempfile
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for kind, p, dpn in VTU_CASES:
            mesh, nsd = assembly_meshes(kind, p)
            dm = O.RefDofManager(mesh, p, dpn)
            phys = O.ELASTICITY if dpn > 1 else O.POISSON
            sysm = O.RefSystem(dm, nsd, phys, [1.0, 1.0, 1.0])
            u = np.stack([smooth_field(dm.nodes, c) for c in range(dpn)], axis=1).ravel()
            k = "%s_p%d/" % (kind, p)
            for key in ("nodes", "cell_nodes", "offsets", "cell_types"):
                out[k + "mesh_" + key] = mesh[key]
            out[k + "meta"] = np.array([p, dpn])
            out[k + "u"] = u
            out[k + "text_mesh"] = np.array(sysm.write_vtu(os.path.join(tmp, "m")))
            out[k + "text_solution"] = np.array(sysm.write_vtu(os.path.join(tmp, "s"), u))
    np.savez_compressed(os.path.join(HERE, "vtu_ref.npz"), **out)


GMSH_TYPE = {0: 1, 1: 2, 3: 3, 2: 4, 4: 5, 5: 15}  # CellType code -> Gmsh element type


def gmsh_text(mesh, extra_cells=(), seed=0):
    """A Gmsh 2.2 ASCII file of `mesh` (written here, not taken from the
    reference): a $MeshFormat header, $Nodes with 17 significant digits, and
    $Elements with two tags each (physical, elementary) -- the mesh's cells, then
    `extra_cells` (cell type code or raw Gmsh type as ("gmsh", t), node list)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    X = mesh["nodes"]
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$Nodes", str(X.shape[0])]
    lines += ["%d %.17g %.17g %.17g" % (i + 1, x, y, z) for i, (x, y, z) in enumerate(X)]
    lines += ["$EndNodes"]
    cells = []
    off, cn, ct = mesh["offsets"], mesh["cell_nodes"], mesh["cell_types"]
    for c in range(ct.size):
        cells.append((GMSH_TYPE[int(ct[c])], list(cn[off[c]:off[c + 1]])))
    for t, nodes in extra_cells:
        cells.append((t[1] if isinstance(t, tuple) else GMSH_TYPE[t], list(nodes)))
    lines += ["$Elements", str(len(cells))]
    for i, (t, nodes) in enumerate(cells):
        tags = rng.integers(1, 9, 2)
        lines.append("%d %d 2 %d %d " % (i + 1, t, tags[0], tags[1]) + " ".join(str(n + 1) for n in nodes))
    lines += ["$EndElements", "$PhysicalNames", "1", "2 1 \"domain\"", "$EndPhysicalNames"]
    return "\n".join(lines) + "\n"


def gmsh():
    """The reference's Mesh(fname) on Gmsh files written by gmsh_text: a mixed
    tri+quad mesh with boundary Line2 and corner Point1 cells, a hexahedron mesh,
    a tetrahedron mesh and a file holding a second-order line (unknown to the
    reference: CellType None); plus the reference's DoFManager numbering of the
    mixed mesh at p = 2 (lower-dimensional cells included)."""
    import tempfile
    out = {}
    m2 = meshgen.jittered_mixed(4, 3, seed=9, order="ccw")
    X = m2["nodes"]
    bottom = np.nonzero(np.abs(X[:, 1]) < 1e-12)[0]
    bottom = bottom[np.argsort(X[bottom, 0])]
    extra2 = [(0, [bottom[i], bottom[i + 1]]) for i in range(bottom.size - 1)] + [(5, [0]), (5, [4])]
    files = {"mixed2d": gmsh_text(m2, extra2, seed=1),
             "hex": gmsh_text(meshgen.structured_hex(2, 2, 1, order="ccw"), seed=2),
             "tet": gmsh_text(meshgen.structured_tet(1, 2, 1, seed=3, jitter=0.1), seed=3),
             "unknown_type": gmsh_text(meshgen.structured_quad(2, 1, order="ccw"), [(("gmsh", 8), [0, 1, 2])], seed=4)}
    with tempfile.TemporaryDirectory() as tmp:
        for name, text in files.items():
            path = os.path.join(tmp, name + ".msh")
            with open(path, "w") as f:
                f.write(text)
            r = O.ref_read_gmsh(path)
            out[name + "/text"] = np.array(text)
            for key, v in r.items():
                out[name + "/" + key] = v
        mesh = {k: out["mixed2d/" + k] for k in ("nodes", "cell_nodes", "offsets", "cell_types")}
        dm = O.RefDofManager(mesh, 2, 1)
        out["mixed2d/p2_dof_nodes"], out["mixed2d/p2_offsets"], out["mixed2d/p2_elements"] = dm.nodes, dm.offsets, dm.elements
    np.savez_compressed(os.path.join(HERE, "gmsh_ref.npz"), **out)


if __name__ == "__main__":
    O.build()
    if not O.ref_available():
        sys.exit("oracle/_ref/libyafel_ref.so is missing: build it where the reference tree exists")
    quadrature()
    linalg()
    poisson_system()
    elements()
    assembly()
    zz()
    vtu()
    gmsh()
    print("golden fixtures written to", HERE)
