"""GPU assembly against the reference itself.

tests/golden/assembly_ref.npz holds the reference's own DoFManager numbering,
CGAssembly<Physics> tangent and residual, DirichletBC::apply result and
LocalSmoothingGradient on small seeded quadrilateral, triangle, mixed,
hexahedron and tetrahedron meshes at orders 1-3 (Poisson in both signs,
elasticity, SUPG), produced by tests/golden/make_golden.py from the
reference's sources compiled in place.  The CUDA path must reproduce:

* the numbering and the sparsity pattern bit for bit;
* tangent values within 1e-13 of the row's largest entry, the residual within
  1e-13 of its largest entry (the reference's duplicate sums follow its
  triplet order, the GPU's its element colours);
* the same after the two Dirichlet objects, and the smoothed gradient of a
  non-linear field within 1e-12.

Every case runs in scalar CSR and in dof_per_node-block BCSR, once on the
GPU's own numbering and once on the reference's numbering handed over through
yg_dofmap_create_from_numbering.
"""
import os

import numpy as np
import pytest

import yafel_b200 as yb
from yafel_b200 import _lib

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
AS = np.load(os.path.join(HERE, "golden", "assembly_ref.npz"))
CASES = sorted({k.split("/")[0] for k in AS.files})
VAL_TOL = 1e-13


def case(name):
    k = name + "/"
    c = {key[len(k):]: AS[key] for key in AS.files if key.startswith(k)}
    c["mesh"] = {"nodes": c["mesh_nodes"], "cell_nodes": c["mesh_cell_nodes"], "offsets": c["mesh_offsets"],
                 "cell_types": c["mesh_cell_types"]}
    m = c["meta"]
    c["p"], c["dpn"], c["nsd"], c["phys"] = int(m[0]), int(m[1]), int(m[2]), int(m[3])
    c["params"] = [float(v) for v in m[4:]]
    return c


class RawPhysics:
    """A registered device physics with its parameter vector as stored in the fixture."""

    def __init__(self, kind, nsd, params):
        self.kind, self._nsd, self.params = kind, nsd, params

    def nsd(self):
        return self._nsd

    def struct(self):
        p = _lib.Physics(self.kind, self._nsd)
        for i, v in enumerate(self.params[:8]):
            p.params[i] = v
        return p


def scalar_csr(K):
    rp, col, val = K.arrays()
    if K.block == 1:
        return rp, col, val
    r, c, v = K.copy_triplets()
    o = np.lexsort((c, r))
    r, c, v = r[o], c[o], v[o]
    srp = np.zeros(K.rows() + 1, np.int64)
    np.add.at(srp, r + 1, 1)
    return np.cumsum(srp), c, v


def check_values(K, c, key):
    rp, col, val = scalar_csr(K)
    assert np.array_equal(rp, c["row_ptr"]) and np.array_equal(col, c["col"]), "pattern"
    ref = c[key]
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    rm = np.zeros(rp.size - 1)
    np.maximum.at(rm, rows, np.abs(ref))
    err = np.abs(val - ref)
    assert np.all(err <= VAL_TOL * np.maximum(rm[rows], 1e-300)), "max error %.3e" % err.max()


def check_vector(v, ref, tol=VAL_TOL):
    assert np.abs(v - ref).max() <= tol * max(np.abs(ref).max(), 1e-300)


def check_gradient(G, ref, tol=1e-12):
    """The smoothed gradient at the nodes whose lumped volume is not zero.

    A quadratic triangle's vertex shape functions integrate to zero, so a node
    that is a vertex of quadratic triangles only divides a rounding-noise sum by
    a rounding-noise volume (LocalSmoothingGradient.hpp:75-91): the reference
    gives values of 1e9 and more there, whose digits carry nothing.  Those nodes
    are told by the size of the reference value against the median."""
    n = np.linalg.norm(ref, axis=1)
    ok = n <= 1e4 * np.median(n)
    assert ok.mean() > 0.5
    check_vector(G[ok], ref[ok], tol)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("numbering", ["gpu", "reference"])
@pytest.mark.parametrize("fmt", ["bcsr", "csr"])
def test_assembly_matches_reference(ctx, name, numbering, fmt):
    c = case(name)
    if numbering == "gpu":
        dm = yb.DoFManager(c["mesh"], c["p"], c["dpn"])
        assert np.array_equal(dm.element_offsets, c["element_offsets"])
        assert np.array_equal(dm.elements, c["elements"])
        assert np.array_equal(dm.dof_nodes, c["dof_nodes"])
    else:
        dm = yb.DoFManager(c["mesh"], c["p"], c["dpn"],
                           numbering=(c["dof_nodes"], c["element_offsets"], c["elements"]))
    fe = yb.FESystem(dm, c["nsd"], format=yb.BCSR if fmt == "bcsr" else yb.CSR)
    phys = RawPhysics(c["phys"], c["nsd"], c["params"])
    yb.CGAssembly(phys, fe)
    K, F = fe.getGlobalTangent(), fe.getGlobalResidual()
    check_values(K, c, "val")
    check_vector(F.numpy(), c["residual"])
    # DirichletBC: comp 0 = 0.25 on x = min, then comp dpn-1 = -0.5 on y = min
    X = dm.dof_nodes
    counts = []
    for comp, axis, value in ((0, 0, 0.25), (c["dpn"] - 1, 1, -0.5)):
        bc = yb.DirichletBC(dm, value, comp)
        bc.selectByFunction(lambda P, a=axis, m=X[:, axis].min(): np.abs(P[:, a] - m) < 1e-9)
        bc.apply(K, F)
        counts.append(bc.getNodes().size)
    assert counts == list(c["bc_count"])
    check_values(K, c, "bc_val")
    check_vector(F.numpy(), c["bc_rhs"])
    # LocalSmoothingGradient of a non-linear field
    fe.getSolution().upload(c["grad_u"])
    yb.LocalSmoothingGradient(phys, fe)
    G = fe.solution_gradient.numpy().reshape(-1, c["nsd"])
    check_gradient(G, c["grad"])


def test_numbering_handed_over_is_checked(ctx):
    c = case("quad_poisson_p2")
    bad = c["elements"].copy()
    bad[3] = c["dof_nodes"].shape[0]  # a node past the end
    with pytest.raises(RuntimeError):
        yb.DoFManager(c["mesh"], 2, 1, numbering=(c["dof_nodes"], c["element_offsets"], bad))
    short = c["element_offsets"].copy()
    short[1] -= 1  # element 0 one node short of a Q2 quadrilateral
    with pytest.raises(RuntimeError):
        yb.DoFManager(c["mesh"], 2, 1, numbering=(c["dof_nodes"], short, c["elements"]))
