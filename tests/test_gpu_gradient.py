"""LocalSmoothingGradient on the GPU (yg_local_smoothing_gradient) against the
oracle's restatement of include/assembly/LocalSmoothingGradient.hpp:20-94, on the
same numbering: random solution fields on jittered mixed triangle/quad meshes
(orders 1 and 3; quads at order 2, where a quadratic triangle's vertex functions
integrate to zero) and hex meshes, scalar and vector fields; and the exact
constant gradient of a linear field.  ZZGradientRecovery (yg_zz_gradient_recovery)
against the reference's own, run on the fixtures of tests/golden/zz_ref.npz."""
import os

import numpy as np
import pytest

import yafel_b200 as yb
from oracle import oracle as O
from yafel_b200 import meshgen

pytestmark = pytest.mark.gpu

CASES = [  # (dimension, order, dofs per node, cells per side)
    (2, 1, 1, 9), (2, 1, 2, 7), (2, 2, 2, 6), (2, 3, 1, 5), (3, 1, 1, 4), (3, 2, 3, 3), (3, 3, 1, 2),
]


def mesh_for(dim, p, n):
    if dim == 2:
        return meshgen.jittered_mixed(n, n + 1, seed=11 * p + n, tri_fraction=0.0 if p == 2 else 0.5,
                                      order=meshgen.corner_order(p))
    return meshgen.structured_hex(n, n + 1, n, order=meshgen.corner_order(p))


@pytest.mark.parametrize("dim,p,dpn,n", CASES)
def test_gradient_matches_oracle(ctx, dim, p, dpn, n):
    mesh = mesh_for(dim, p, n)
    dm = yb.DoFManager(mesh, p, dpn, ctx=ctx)
    fe = yb.FESystem(dm, dim)
    u = np.random.Generator(np.random.PCG64(5 * p + dpn)).standard_normal(dm.ndofs)
    fe.getSolution().upload(u)
    yb.LocalSmoothingGradient(yb.PoissonEquation(dim), fe)
    g = fe.getSolutionGradient().numpy().reshape(-1, dim)
    # the oracle on the GPU's numbering (the reference's merged coordinates)
    odm = O.ArrayDofMap(dm.dof_nodes, dm.element_offsets, dm.elements, mesh["cell_types"], p)
    go = O.local_smoothing_gradient(odm, dpn, dim, u)
    assert g.shape == go.shape
    assert np.abs(g - go).max() <= 1e-11 * np.abs(go).max(), (dim, p, dpn)
    # same bits on a second call
    yb.LocalSmoothingGradient(yb.PoissonEquation(dim), fe)
    assert np.array_equal(fe.getSolutionGradient().numpy().reshape(-1, dim), g)


@pytest.mark.parametrize("dim,p,dpn,n", [(2, 3, 2, 4), (3, 2, 1, 3)])
def test_linear_field_has_its_constant_gradient(ctx, dim, p, dpn, n):
    mesh = mesh_for(dim, p, n)
    dm = yb.DoFManager(mesh, p, dpn, ctx=ctx)
    fe = yb.FESystem(dm, dim)
    X = dm.dof_nodes[:, :dim]
    a = np.arange(1, dpn * dim + 1, dtype=float).reshape(dpn, dim) * 0.25 - 0.5
    u = np.stack([X @ a[c] + c for c in range(dpn)], axis=1).ravel()
    fe.getSolution().upload(u)
    yb.LocalSmoothingGradient(yb.PoissonEquation(dim), fe)
    g = fe.getSolutionGradient().numpy().reshape(-1, dim)
    assert np.abs(g - np.tile(a, (dm.dof_nodes.shape[0], 1))).max() <= 1e-11


ZZ = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "zz_ref.npz"))


@pytest.mark.parametrize("kind", ["quad", "mixed", "tri", "hex", "tet"])
def test_zz_recovery_matches_reference(ctx, kind):
    """ZZGradientRecovery on the GPU against the reference's own (compiled in
    place, column-pivoted QR in absolute coordinates) on a non-linear field:
    the GPU solves the same least-squares fits through normal equations in
    coordinates centred at the node, so the two agree to rounding."""
    k = kind + "/"
    mesh = {"nodes": ZZ[k + "mesh_nodes"], "cell_nodes": ZZ[k + "mesh_cell_nodes"],
            "offsets": ZZ[k + "mesh_offsets"], "cell_types": ZZ[k + "mesh_cell_types"]}
    nsd = int(ZZ[k + "nsd"])
    dm = yb.DoFManager(mesh, 1, 1, ctx=ctx)
    fe = yb.FESystem(dm, nsd)
    fe.getSolution().upload(ZZ[k + "u"])
    yb.ZZGradientRecovery(yb.PoissonEquation(nsd), fe)
    g = fe.getSolutionGradient().numpy().reshape(-1, nsd)
    ref = ZZ[k + "grad"]
    assert np.abs(g - ref).max() <= 1e-10 * np.abs(ref).max(), np.abs(g - ref).max()
    # deterministic
    yb.ZZGradientRecovery(yb.PoissonEquation(nsd), fe)
    assert np.array_equal(fe.getSolutionGradient().numpy().reshape(-1, nsd), g)


def test_zz_recovers_linear_fields_exactly_and_rejects_p2(ctx):
    mesh = meshgen.jittered_mixed(12, 10, seed=4, order="tensor")
    dm = yb.DoFManager(mesh, 1, 1, ctx=ctx)
    fe = yb.FESystem(dm, 2)
    X = dm.dof_nodes
    fe.getSolution().upload(0.5 + 3.0 * X[:, 0] - 2.0 * X[:, 1])
    yb.ZZGradientRecovery(yb.PoissonEquation(2), fe)
    g = fe.getSolutionGradient().numpy().reshape(-1, 2)
    assert np.abs(g - np.array([3.0, -2.0])).max() <= 1e-11
    dm2 = yb.DoFManager(meshgen.structured_quad(4, 4), 2, 1, ctx=ctx)
    with pytest.raises(yb.YafelError):
        yb.ZZGradientRecovery(yb.PoissonEquation(2), yb.FESystem(dm2, 2))
