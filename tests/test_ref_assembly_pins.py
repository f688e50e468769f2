"""The assembly half pinned to the reference itself (CPU).

tests/golden/elements.npz and assembly_ref.npz hold outputs of the reference's
own Element, DoFManager, CGAssembly<Physics>, DirichletBC::apply and
LocalSmoothingGradient, compiled in place against a from-scratch Eigen-API
subset (oracle/Makefile, tests/golden/make_golden.py).  Here they pin:

* the product's host code -- element tables (yg_element_table) and the DoF
  numbering (yg_dofmap_create without a context) -- bit for bit;
* the oracle's C restatement (oracle/yafel_oracle.c): numbering, pattern,
  values within 1e-13 of the row's largest entry, residual, Dirichlet and the
  smoothed gradient, all assembled on the reference's numbering.

The oracle restatement has no tetrahedra; those cases are pinned on the GPU
directly against the fixtures (tests/test_gpu_assembly_ref.py).
"""
import os

import numpy as np
import pytest

import yafel_b200 as yb
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
EL = np.load(os.path.join(HERE, "golden", "elements.npz"))
AS = np.load(os.path.join(HERE, "golden", "assembly_ref.npz"))
CASES = sorted({k.split("/")[0] for k in AS.files})
ETYPES = sorted({tuple(int(v) for v in k[1:].split("_")[:3]) for k in EL.files})
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


def row_max(row_ptr, val):
    rows = np.repeat(np.arange(row_ptr.size - 1), np.diff(row_ptr))
    rm = np.zeros(row_ptr.size - 1)
    np.maximum.at(rm, rows, np.abs(val))
    return rm[rows]


def assert_values(val, ref_val, row_ptr, tol=VAL_TOL):
    err = np.abs(val - ref_val)
    bound = tol * np.maximum(row_max(row_ptr, ref_val), 1e-300)
    assert np.all(err <= bound), "max relative error %.3e" % (err / np.maximum(bound / tol, 1e-300)).max()


def test_fixture_inventory():
    kinds = {c.split("_")[0] for c in CASES}
    assert kinds == {"quad", "mixed", "tri", "hex", "tet"}
    assert len(CASES) >= 28 and len(ETYPES) >= 16


@pytest.mark.parametrize("etype", ETYPES, ids=lambda t: "topo%d_dim%d_p%d" % t)
def test_product_element_tables_match_reference(etype):
    topo, dim, p = etype
    k = "e%d_%d_%d_" % etype
    L, X, W, N, dN = yb.element_table(topo, dim, p)
    assert np.array_equal(L, EL[k + "L"]), "local nodes"
    assert np.array_equal(X, EL[k + "X"]) and np.array_equal(W, EL[k + "W"]), "quadrature"
    if topo == O.SIMPLEX:  # the same Vandermonde construction: identical bits
        assert np.array_equal(N, EL[k + "N"]) and np.array_equal(dN, EL[k + "dN"])
    else:  # 1-D Lagrange products instead of a Vandermonde solve: equal to rounding
        assert np.abs(N - EL[k + "N"]).max() <= 1e-14
        assert np.abs(dN - EL[k + "dN"]).max() <= 1e-14 * max(1.0, np.abs(EL[k + "dN"]).max())


@pytest.mark.parametrize("etype", [t for t in ETYPES if not (t[0] == 1 and t[1] == 3)],
                         ids=lambda t: "topo%d_dim%d_p%d" % t)
def test_oracle_element_tables_match_reference(etype):
    topo, dim, p = etype
    k = "e%d_%d_%d_" % etype
    assert np.array_equal(O.local_nodes(topo, dim, p), EL[k + "L"])
    X, W = O.element_rule(topo, dim, p)
    assert np.array_equal(X, EL[k + "X"]) and np.array_equal(W, EL[k + "W"])
    N, dN = O.shape_functions(topo, dim, p, X)
    assert np.abs(N - EL[k + "N"]).max() <= 1e-14
    assert np.abs(dN - EL[k + "dN"]).max() <= 1e-14 * max(1.0, np.abs(EL[k + "dN"]).max())


@pytest.mark.parametrize("name", CASES)
def test_product_numbering_matches_reference(name):
    c = case(name)
    dm = yb.DoFManager(c["mesh"], c["p"], c["dpn"], host_only=True)
    assert np.array_equal(dm.element_offsets, c["element_offsets"])
    assert np.array_equal(dm.elements, c["elements"])
    assert np.array_equal(dm.dof_nodes, c["dof_nodes"]), "merged node coordinates"


@pytest.mark.parametrize("name", [n for n in CASES if not n.startswith("tet")])
def test_oracle_matches_reference(name):
    c = case(name)
    # numbering: element lists exact; merged coordinates to rounding, except
    # where triangles meet quadrilaterals at p >= 3 (the reference's unstable
    # std::sort picks which coincident raw node is kept; see DESIGN)
    od = O.dofmanager(c["mesh"], c["p"])
    assert np.array_equal(od.offsets, c["element_offsets"]) and np.array_equal(od.elements, c["elements"])
    tol = 1e-6 if (name.startswith("mixed") and c["p"] >= 3) else 1e-15
    assert np.abs(od.nodes - c["dof_nodes"]).max() <= tol
    # assembly on the reference's own numbering
    dm = O.ArrayDofMap(c["dof_nodes"], c["element_offsets"], c["elements"], c["mesh"]["cell_types"], c["p"])
    K, R = O.assemble(dm, c["dpn"], c["nsd"], c["phys"], c["params"])
    assert np.array_equal(K.row_ptr, c["row_ptr"]) and np.array_equal(K.col, c["col"]), "pattern"
    assert_values(K.val, c["val"], c["row_ptr"])
    assert np.abs(R - c["residual"]).max() <= VAL_TOL * max(np.abs(c["residual"]).max(), 1e-300)
    # Dirichlet: comp 0 = 0.25 on x = min, comp dpn-1 = -0.5 on y = min
    X = c["dof_nodes"]
    for comp, axis, value in ((0, 0, 0.25), (c["dpn"] - 1, 1, -0.5)):
        sel = np.nonzero(np.abs(X[:, axis] - X[:, axis].min()) < 1e-9)[0]
        mask = np.zeros(K.nrows, np.uint8)
        vals = np.zeros(K.nrows)
        mask[sel * c["dpn"] + comp] = 1
        vals[sel * c["dpn"] + comp] = value
        O.dirichlet_apply(K, R, mask, vals)
    assert_values(K.val, c["bc_val"], c["row_ptr"])
    assert np.abs(R - c["bc_rhs"]).max() <= VAL_TOL * max(np.abs(c["bc_rhs"]).max(), 1e-300)
    # LocalSmoothingGradient of a non-linear field
    # (nodes that are vertices of quadratic triangles only have a zero lumped
    # volume, LocalSmoothingGradient.hpp:75-91: noise over noise, not compared)
    G = O.local_smoothing_gradient(dm, c["dpn"], c["nsd"], c["grad_u"])
    n = np.linalg.norm(c["grad"], axis=1)
    ok = n <= 1e4 * np.median(n)
    assert ok.mean() > 0.5
    assert np.abs(G[ok] - c["grad"][ok]).max() <= 1e-12 * np.abs(c["grad"][ok]).max()


def test_reference_quirks_visible_in_fixtures():
    """Properties of the reference's own output that the product keeps."""
    # the SUPG tangent is not symmetric (advection), the SPD Poisson one is
    c = case("mixed_supg_p2")
    n = c["row_ptr"].size - 1
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(c["row_ptr"]))
    A[rows, c["col"]] = c["val"]
    assert np.abs(A - A.T).max() > 1e-3
    c = case("quad_poisson_p2")
    n = c["row_ptr"].size - 1
    A = np.zeros((n, n))
    A[np.repeat(np.arange(n), np.diff(c["row_ptr"])), c["col"]] = c["val"]
    assert np.abs(A - A.T).max() <= 1e-15 * np.abs(A).max()
    # Laplacian rows sum to zero before boundary conditions
    assert np.abs(A.sum(1)).max() <= 1e-13 * np.abs(A).max()
    # the reference-sign Poisson system is the negative of the SPD one at f scaled
    c2 = case("quad_poisson_refsign_p2")
    assert np.array_equal(c2["col"], c["col"]) and np.allclose(c2["val"], -c["val"], rtol=1e-15, atol=0)
    # simplices: the Vandermonde is built on nodes moved by 1e-9..1e-8
    # (ShapeFunctionUtils.cpp:169-172, 240-246), so the reference gradients
    # reproduce the linear map x(xi) = xi only to ~1e-8 (the Jacobian of the
    # reference cell itself is not exactly the identity)
    for k in ("e1_2_2_", "e1_3_1_", "e1_3_2_"):
        L, dN = EL[k + "L"], EL[k + "dN"]
        dim = dN.shape[2]
        J = np.einsum("ai,qaj->qij", L[:, :dim], dN)
        assert 1e-10 < np.abs(J - np.eye(dim)).max() < 1e-7
