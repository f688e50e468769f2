"""Pin the oracle (the CPU restatement under oracle/) before trusting it:
against the reference's own code (golden fixtures made from oracle/_ref, and
oracle/_ref itself when present) and against the known answers the reference's
tests state.  CPU only."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from yafel_b200 import meshgen

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name))


# ---------------------------------------------------------------- quadrature

def test_gauss_1d_bit_exact_vs_reference_fixture():
    g = gold("quadrature.npz")
    for lob in (0, 1):
        for n in range(2, 10):
            x, w = O.gauss_1d(n, bool(lob))
            assert np.array_equal(x, g["g1d_%d_%d_x" % (lob, n)]), (lob, n)
            assert np.array_equal(w, g["g1d_%d_%d_w" % (lob, n)]), (lob, n)


def test_tensor_rules_bit_exact_vs_reference_fixture():
    g = gold("quadrature.npz")
    for dim in (1, 2, 3):
        for order in range(1, 10):
            p, w = O.tensor_rule(dim, order)
            assert np.array_equal(p, g["tp_%d_%d_p" % (dim, order)])
            assert np.array_equal(w, g["tp_%d_%d_w" % (dim, order)])


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_weights_sum_known_answer(dim):
    # test/test_GaussLegQuadrature.cpp:9-17, test_GaussLobQuadrature.cpp:9-16
    for order in range(1, 9):
        _, w = O.tensor_rule(dim, order)
        assert abs(w.sum() - 2.0 ** dim) < 1e-13
        _, w = O.tensor_rule(dim, order, lobatto=True)
        assert abs(w.sum() - 2.0 ** dim) < 1e-13


def test_triangle_rule_matches_reference_table_on_polynomials():
    """The oracle's collapsed-GL triangle rule and the reference's tabulated rule
    integrate every monomial of degree <= order to the same value."""
    g = gold("quadrature.npz")
    for order in range(1, 7):
        pr, wr = g["tri_%d_p" % order], g["tri_%d_w" % order]
        po, wo = O.triangle_rule_collapsed(order)
        pt, wt = O.triangle_rule(order)
        assert np.array_equal(pt, pr) and np.array_equal(wt, wr)
        for a in range(order + 1):
            for b in range(order + 1 - a):
                ir = np.sum(wr * pr[:, 0] ** a * pr[:, 1] ** b)
                io = np.sum(wo * po[:, 0] ** a * po[:, 1] ** b)
                assert abs(ir - io) < 1e-13, (order, a, b, ir, io)


# ---------------------------------------------------------------- elements

def test_q1_corner_gradients_known_answer():
    # test/test_LinQuadElement.cpp:96-118: Q1 reference gradients at corners are +-1/2
    nodes = O.local_nodes(O.TENSOR, 2, 1)
    N, dN = O.shape_functions(O.TENSOR, 2, 1, nodes)
    assert np.allclose(N, np.eye(4), atol=1e-15)
    assert np.allclose(np.abs(dN[0][dN[0] != 0]), 0.5)
    assert np.allclose(dN[0], [[-0.5, -0.5], [0.5, 0.0], [0.0, 0.5], [0.0, 0.0]], atol=1e-15)


@pytest.mark.parametrize("topo,dim,p", [(0, 1, 3), (0, 2, 1), (0, 2, 2), (0, 2, 3), (0, 3, 1), (0, 3, 2),
                                        (0, 3, 3), (1, 2, 1), (1, 2, 2), (1, 2, 3)])
def test_shape_functions_nodal_and_partition_of_unity(topo, dim, p):
    nodes = O.local_nodes(topo, dim, p)
    q, _ = O.element_rule(topo, dim, p)
    N, dN = O.shape_functions(topo, dim, p, q)
    assert np.abs(N.sum(1) - 1).max() < 1e-12
    assert np.abs(dN.sum(1)).max() < 1e-11
    if topo == 1:
        # triangles: the reference's basis is singular at the top vertex, which its
        # Vandermonde moves to y=0.999999999 (ShapeFunctionUtils.cpp:169-172); the
        # nodal basis is the Lagrange basis of that moved point set
        nodes = nodes.copy()
        nodes[:, 1] = np.minimum(nodes[:, 1], 0.999999999)
    Nn, _ = O.shape_functions(topo, dim, p, nodes)
    assert np.abs(Nn - np.eye(len(nodes))).max() < 1e-9


def test_integral_of_x_over_unit_square_known_answer():
    # test/test_LinQuadElement.cpp:34-92: int_Omega x = 1/2 on 1 and 10x10 Q1 meshes
    for n in (1, 10):
        dm = O.dofmanager(meshgen.structured_quad(n, n, order="tensor"), 1)
        _, R = O.assemble(dm, 1, 2, O.POISSON, [1.0, 1.0])
        assert abs((R * dm.nodes[:, 0]).sum() - 0.5) < 1e-14


def test_rectilinear_counts_known_answer():
    # test/test_RectilinearMesh.cpp: node and cell counts of structured meshes
    m = meshgen.structured_quad(4, 3)
    assert m["nodes"].shape[0] == 20 and m["cell_types"].size == 12
    m = meshgen.structured_hex(2, 3, 4)
    assert m["nodes"].shape[0] == 60 and m["cell_types"].size == 24


@pytest.mark.parametrize("p", [1, 2, 3])
def test_laplacian_row_sums_and_rigid_modes(p):
    dm = O.dofmanager(meshgen.structured_quad(5, 4, order=meshgen.corner_order(p)), p)
    K, R = O.assemble(dm, 1, 2, O.POISSON, [1.0, 1.0])
    assert np.abs(K.spmv(np.ones(K.nrows))).max() < 1e-12
    assert abs(R.sum() - 1.0) < 1e-12
    dm = O.dofmanager(meshgen.structured_hex(2, 2, 2, order=meshgen.corner_order(p)), p)
    K, _ = O.assemble(dm, 3, 3, O.ELASTICITY, [1.0, 0.5769, 0.3846, 0, 0, 0])
    for c in range(3):
        u = np.zeros(K.nrows)
        u[c::3] = 1.0
        assert np.abs(K.spmv(u)).max() < 1e-12
    X = dm.nodes
    u = np.zeros(K.nrows)  # infinitesimal rotation about z
    u[0::3], u[1::3] = -X[:, 1], X[:, 0]
    assert np.abs(K.spmv(u)).max() < 1e-12


def test_dofmanager_structured_q2_numbering_is_x_fastest():
    dm = O.dofmanager(meshgen.structured_hex(3, 2, 2), 2)
    X = dm.nodes
    assert dm.n_nodes == 7 * 5 * 5
    order = np.lexsort((X[:, 0], X[:, 1], X[:, 2]))
    assert np.array_equal(order, np.arange(dm.n_nodes))


def test_patch_test_linear_field_mixed_mesh():
    """A linear field is reproduced exactly: K u_lin = boundary terms only, so
    interior rows of K u vanish (a property the reference's assembly has)."""
    for p in (1, 2, 3):
        dm = O.dofmanager(meshgen.jittered_mixed(6, 6, seed=5, order=meshgen.corner_order(p)), p)
        K, _ = O.assemble(dm, 1, 2, O.POISSON, [1.0, 0.0])
        X = dm.nodes
        u = 0.3 + 1.7 * X[:, 0] - 0.9 * X[:, 1]
        r = K.spmv(u)
        interior = (X[:, 0] > 1e-9) & (X[:, 0] < 1 - 1e-9) & (X[:, 1] > 1e-9) & (X[:, 1] < 1 - 1e-9)
        # the triangle basis is the Lagrange basis of nodes moved by 1e-9
        # (ShapeFunctionUtils.cpp:169-172), so linear fields are reproduced to ~1e-9
        assert np.abs(r[interior]).max() < 1e-8


# ---------------------------------------------------------------- linear algebra

def test_csr_from_triplets_vs_reference_fixture():
    g = gold("linalg.npz")
    for key in ("dup", "rand"):
        r, c, v = g[key + "_in"]
        A = O.csr_from_triplets(r.astype(np.int64), c.astype(np.int64), v)
        assert np.array_equal(A.row_ptr, g[key + "_rp"])
        assert np.array_equal(A.col, g[key + "_col"])
        assert np.array_equal(A.val, g[key + "_val"])
    # test_sparse_csr.cpp test_3: two nonzeros of value N
    A = O.csr_from_triplets(*[x.astype(np.int64) if i < 2 else x for i, x in enumerate(g["dup_in"])])
    assert A.nnz == 2 and A.nrows == 10 and np.all(A.val == 10)


def test_bcsr_from_triplets_vs_reference_fixture():
    g = gold("linalg.npz")
    ii, jj = np.meshgrid(np.arange(60), np.arange(60), indexing="ij")
    B = O.bcsr_from_triplets(3, ii.ravel(), jj.ravel(), (ii * 60 + jj).ravel().astype(float))
    assert np.array_equal(B["brow_ptr"], g["bcsr60_rp"])
    assert np.array_equal(B["bcol"], g["bcsr60_col"])
    assert np.array_equal(B["val"], g["bcsr60_val"])
    y = O.bcsr_spmv(B, g["bcsr60_x"])
    assert np.allclose(y, g["bcsr60_y"], rtol=1e-15, atol=1e-12)


def test_cg_and_bicgstab_reference_tests():
    g = gold("linalg.npz")
    r, c, v = g["lap_in"]
    A = O.csr_from_triplets(r.astype(np.int64), c.astype(np.int64), v)
    b = g["lap_b"]
    x, _, _ = O.cg(A, b, criterion=O.CRIT_REFERENCE, tol=1e-14)
    # test_cg_solve.cpp test_2: ||x - x_ref||^2 < 1e-10
    assert np.sum((x - np.arange(10)) ** 2) < 1e-10
    assert np.allclose(x, g["lap_cg"], rtol=1e-12, atol=1e-12)
    x, _, _ = O.bicgstab(A, b, criterion=O.CRIT_REFERENCE, tol=1e-14)
    assert np.sum((x - np.arange(10)) ** 2) < 1e-10
    assert np.allclose(x, g["lap_bicgstab"], rtol=1e-10, atol=1e-10)
    # test_cg_solve.cpp test_1: identity, exact equality
    I = O.csr_from_triplets(np.arange(10), np.arange(10), np.ones(10))
    x, _, _ = O.cg(I, g["ident_b"], criterion=O.CRIT_REFERENCE, tol=1e-14)
    assert np.array_equal(x, g["ident_b"]) and np.array_equal(x, g["ident_cg"])


def test_ilu0_factors_vs_reference_fixture():
    g = gold("linalg.npz")
    r, c, v = g["ilu5_in"]
    A = O.csr_from_triplets(r.astype(np.int64), c.astype(np.int64), v)
    F = O.ilu0(A)
    assert np.allclose(F.val, g["ilu5_lu"], rtol=1e-15, atol=1e-15)
    z = O.ilu_solve(F, g["ilu5_z"])
    assert np.allclose(z, g["ilu5_apply"], rtol=1e-13, atol=1e-14)


def test_poisson8_pcg_vs_reference_fixture():
    g = gold("poisson8.npz")
    A = O.Csr(g["rp"].size - 1, g["rp"].size - 1, g["rp"], g["col"], g["val"])
    F = O.ilu0(A)
    assert np.allclose(F.val, g["ilu_lu"], rtol=1e-14, atol=1e-15)
    for pc, key in ((O.PRECOND_JACOBI, "pcg_jacobi"), (O.PRECOND_ILU0, "pcg_ilu"), (O.PRECOND_NONE, "cg")):
        x, _, rel = O.cg(A, g["b"], precond=pc, criterion=O.CRIT_REFERENCE, tol=1e-20)
        assert np.abs(x - g[key]).max() <= 1e-12 * np.abs(g[key]).max()


def test_oracle_assembly_matches_reference_csr_construction():
    """The oracle's duplicate summation and the reference's sparse_csr(triplets)
    give the same pattern and values for an assembled system."""
    dm = O.dofmanager(meshgen.structured_quad(6, 5, order="tensor"), 1)
    K, _ = O.assemble(dm, 1, 2, O.POISSON, [1.0, 1.0])
    if not O.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree once)")
    r, c, v = O.csr_to_triplets(K)
    R = O.RefCsr(r, c, v)
    rp, col, val = R.arrays()
    assert np.array_equal(rp, K.row_ptr) and np.array_equal(col, K.col)
    assert np.allclose(val, K.val, rtol=1e-15, atol=1e-15)
