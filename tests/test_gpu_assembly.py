"""GPU parity of the assembly path (DoF map, pattern, element kernels, Dirichlet)
against the oracle: patterns and numbering bit-exact, FP64 values within
1e-13 of the row's largest entry (the reference's duplicate-summation order is
thread dependent, CGAssembly.hpp:175-182, so per-entry bit equality is not a
property the reference itself has)."""
import numpy as np
import pytest

import yafel_b200 as yb
from oracle import oracle as O
from yafel_b200 import meshgen

pytestmark = pytest.mark.gpu

VAL_TOL = 1e-13


def scalar_csr(K):
    """GPU matrix -> scalar (row_ptr, col, val) in row/column order."""
    rp, col, val = K.arrays()
    B = K.block
    if B == 1:
        return rp, col, val
    r, c, v = K.copy_triplets()
    o = np.lexsort((c, r))
    r, c, v = r[o], c[o], v[o]
    srp = np.zeros(K.rows() + 1, np.int64)
    np.add.at(srp, r + 1, 1)
    return np.cumsum(srp), c, v


def compare(K_gpu, K_or):
    rp, col, val = scalar_csr(K_gpu)
    assert np.array_equal(rp, K_or.row_ptr), "row pointers differ"
    assert np.array_equal(col, K_or.col), "column indices differ"
    rows = np.repeat(np.arange(K_or.nrows), np.diff(K_or.row_ptr))
    rowmax = np.zeros(K_or.nrows)
    np.maximum.at(rowmax, rows, np.abs(K_or.val))
    err = np.abs(val - K_or.val)
    assert np.all(err <= VAL_TOL * np.maximum(rowmax[rows], 1e-300)), err.max()


def oracle_dofmap(mesh, p, dm):
    """The oracle's numbering must equal the GPU's element lists; the oracle
    then assembles on the GPU's merged coordinates, which are the reference's
    (test_gpu_assembly_ref.py) -- the oracle's own choice among coincident raw
    nodes differs from the reference's where triangles meet quadrilaterals at
    p >= 3."""
    odm = O.dofmanager(mesh, p)
    assert np.array_equal(dm.element_offsets, odm.offsets) and np.array_equal(dm.elements, odm.elements)
    assert np.abs(dm.dof_nodes - odm.nodes).max() <= (1e-6 if p >= 3 else 1e-15)
    return O.ArrayDofMap(dm.dof_nodes, dm.element_offsets, dm.elements, mesh["cell_types"], p)


PHYS = {
    "poisson": (O.POISSON, lambda nsd: yb.PoissonEquation(nsd, f=1.3, sign=1.0), [1.0, 1.3]),
    "poisson_ref_sign": (O.POISSON, lambda nsd: yb.PoissonEquation(nsd, f=100.0, sign=-1.0), [-1.0, 100.0]),
    "elasticity": (O.ELASTICITY, lambda nsd: yb.LinearElasticity(nsd, E=1.0, nu=0.3, body=(0.5, -1.0, 2.0)),
                   None),
    "supg": (O.SUPG, lambda nsd: yb.AdvectionDiffusionSUPG(nsd, k=0.02, h=0.1, U0=1.0), [0.02, 0.1, 1.0, 0.0]),
}

CASES = [
    ("quad", 1, "poisson"), ("quad", 2, "poisson"), ("quad", 3, "poisson"), ("quad", 1, "poisson_ref_sign"),
    ("hex", 1, "poisson"), ("hex", 2, "poisson"), ("hex", 3, "poisson"),
    ("quad", 1, "elasticity"), ("quad", 2, "elasticity"), ("quad", 3, "elasticity"),
    ("hex", 1, "elasticity"), ("hex", 2, "elasticity"), ("hex", 3, "elasticity"),
    ("mixed", 1, "poisson"), ("mixed", 2, "poisson"), ("mixed", 3, "poisson"),
    ("mixed", 2, "elasticity"), ("mixed", 3, "elasticity"),
    ("quad", 1, "supg"), ("quad", 2, "supg"), ("mixed", 2, "supg"), ("hex", 2, "supg"),
]


def make_mesh(kind, p):
    o = meshgen.corner_order(p)
    if kind == "quad":
        return meshgen.structured_quad(9, 7, order=o), 2
    if kind == "hex":
        return meshgen.structured_hex(4, 3, 3, order=o), 3
    return meshgen.jittered_mixed(8, 9, seed=21, order=o), 2


@pytest.mark.parametrize("kind,p,phys", CASES)
@pytest.mark.parametrize("fmt", ["bcsr", "csr"])
def test_assembly_matches_oracle(ctx, kind, p, phys, fmt):
    mesh, nsd = make_mesh(kind, p)
    okind, mk, oparams = PHYS[phys]
    physics = mk(nsd)
    dpn = nsd if okind == O.ELASTICITY else 1
    if oparams is None:
        oparams = [1.0, physics.lam, physics.mu] + list(physics.body)
    dm = yb.DoFManager(mesh, p, dpn)
    fe = yb.FESystem(dm, nsd, format=yb.BCSR if fmt == "bcsr" else yb.CSR)
    yb.CGAssembly(physics, fe)
    odm = oracle_dofmap(mesh, p, dm)
    Ko, Ro = O.assemble(odm, dpn, nsd, okind, oparams)
    compare(fe.getGlobalTangent(), Ko)
    R = fe.getGlobalResidual().numpy()
    assert np.abs(R - Ro).max() <= 1e-13 * max(np.abs(Ro).max(), 1e-300)


def test_assembly_is_deterministic_and_reassembles_in_place(ctx):
    mesh = meshgen.structured_hex(5, 4, 4)
    dm = yb.DoFManager(mesh, 2, 3)
    fe = yb.FESystem(dm, 3)
    phys = yb.LinearElasticity(3)
    yb.CGAssembly(phys, fe, [yb.AssemblyRequirement.Tangent])
    v1 = fe.getGlobalTangent().arrays()[2]
    yb.CGAssembly(phys, fe, [yb.AssemblyRequirement.Tangent])  # replaces values (setFromTriplets)
    v2 = fe.getGlobalTangent().arrays()[2]
    assert np.array_equal(v1, v2)
    # residual accumulates like GlobalResidual += private_residual
    yb.CGAssembly(yb.LinearElasticity(3, body=(1, 0, 0)), fe, [yb.AssemblyRequirement.Residual])
    r1 = fe.getGlobalResidual().numpy()
    yb.CGAssembly(yb.LinearElasticity(3, body=(1, 0, 0)), fe, [yb.AssemblyRequirement.Residual])
    assert np.allclose(fe.getGlobalResidual().numpy(), 2 * r1, rtol=1e-15, atol=0)


@pytest.mark.parametrize("fmt", ["bcsr", "csr"])
def test_dirichlet_apply_matches_oracle(ctx, fmt):
    mesh = meshgen.structured_quad(10, 8, order="ccw")
    dm = yb.DoFManager(mesh, 2, 2)
    fe = yb.FESystem(dm, 2, format=yb.BCSR if fmt == "bcsr" else yb.CSR)
    phys = yb.LinearElasticity(2, body=(0.0, -1.0))
    yb.CGAssembly(phys, fe)
    bc0 = yb.DirichletBC(dm, lambda x, t: 0.1 * x[1], 0)
    bc0.selectByFunction(lambda X: np.abs(X[:, 0]) < 1e-6)
    bc1 = yb.DirichletBC(dm, 0.25, 1)
    bc1.selectByFunction(lambda X: np.abs(X[:, 0]) < 1e-6)
    K, F = fe.getGlobalTangent(), fe.getGlobalResidual()
    bc0.apply(K, F)
    bc1.apply(K, F)
    odm = oracle_dofmap(mesh, 2, dm)
    Ko, Fo = O.assemble(odm, 2, 2, O.ELASTICITY, [1.0, phys.lam, phys.mu, 0.0, -1.0])
    for bc in (bc0, bc1):
        d, v = bc.dofs_and_values()
        mask = np.zeros(Ko.nrows, np.uint8)
        vals = np.zeros(Ko.nrows)
        mask[d] = 1
        vals[d] = v
        O.dirichlet_apply(Ko, Fo, mask, vals)
    compare(K, Ko)
    assert np.abs(F.numpy() - Fo).max() <= 1e-13 * np.abs(Fo).max()


def test_poisson_64x64_q1_end_to_end(ctx):
    """The 64x64 Q1 Poisson case: numbering, pattern (nnz 37,249), values,
    Dirichlet, Jacobi-PCG to 1e-10 -- against the oracle end to end."""
    mesh = meshgen.structured_quad(64, 64, order="tensor")
    dm = yb.DoFManager(mesh, 1, 1)
    fe = yb.FESystem(dm, 2, format=yb.CSR)
    yb.CGAssembly(yb.PoissonEquation(2, f=1.0), fe)
    bc = yb.DirichletBC(dm, 0.0)
    bc.selectByFunction(lambda X: (np.abs(X[:, 0]) < 1e-6) | (np.abs(X[:, 0] - 1) < 1e-6) |
                        (np.abs(X[:, 1]) < 1e-6) | (np.abs(X[:, 1] - 1) < 1e-6))
    K, F = fe.getGlobalTangent(), fe.getGlobalResidual()
    bc.apply(K, F)
    assert K.nnz() == 37249 and K.rows() == 4225 and bc.getNodes().size == 256
    x, st = yb.solve(K, F, M=yb.JacobiPreconditioner(K), tol=1e-10)
    assert st.status == 0 and st.rel_residual <= 1e-10
    odm = O.dofmanager(mesh, 1)
    Ko, Fo = O.assemble(odm, 1, 2, O.POISSON, [1.0, 1.0])
    mask = np.zeros(Ko.nrows, np.uint8)
    mask[bc.getNodes()] = 1
    O.dirichlet_apply(Ko, Fo, mask, np.zeros(Ko.nrows))
    compare(K, Ko)
    xs = x.numpy()
    assert O.true_relres(Ko, Fo, xs) <= 1e-10
    xo, _, _ = O.cg(Ko, Fo, precond=O.PRECOND_JACOBI, tol=1e-12)
    assert np.linalg.norm(xs - xo) <= 1e-8 * np.linalg.norm(xo)
