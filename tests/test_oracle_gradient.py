"""The oracle's LocalSmoothingGradient restatement (no GPU needed): for a field
that is linear in x, every element's gradient is exact, so the weighted nodal
average returns the field's constant gradient at every dof (up to rounding), on
jittered mixed triangle/quad meshes of orders 1 and 3 (quads at order 2) and hex
meshes, scalar and vector fields."""
import numpy as np
import pytest

from oracle import oracle as O
from yafel_b200 import meshgen


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("dpn", [1, 2])
def test_linear_field_2d_mixed_mesh(p, dpn):
    # order 2: quads only -- a quadratic triangle's vertex functions integrate to
    # zero, so at a vertex that only such triangles touch the reference divides
    # a rounding-level sum by a rounding-level volume
    mesh = meshgen.jittered_mixed(5, 4, seed=3 + p, tri_fraction=0.0 if p == 2 else 0.5,
                                  order=meshgen.corner_order(p))
    dm = O.dofmanager(mesh, p)
    X = dm.nodes
    a = np.array([[1.5, -0.25], [0.5, 2.0]])[:dpn]
    u = np.stack([X[:, 0] * a[c, 0] + X[:, 1] * a[c, 1] + 0.3 * c for c in range(dpn)], axis=1).ravel()
    g = O.local_smoothing_gradient(dm, dpn, 2, u)
    expect = np.tile(a, (dm.n_nodes, 1))
    assert np.abs(g - expect).max() <= 1e-12


@pytest.mark.parametrize("p", [1, 2])
def test_linear_field_3d_hex(p):
    mesh = meshgen.structured_hex(3, 2, 2, order=meshgen.corner_order(p))
    dm = O.dofmanager(mesh, p)
    X = dm.nodes
    a = np.array([[0.5, -1.0, 2.0], [1.0, 0.0, -0.5], [0.25, 0.75, 1.25]])
    u = np.stack([X @ a[c] for c in range(3)], axis=1).ravel()
    g = O.local_smoothing_gradient(dm, 3, 3, u)
    assert np.abs(g - np.tile(a, (dm.n_nodes, 1))).max() <= 1e-12
    gs = O.local_smoothing_gradient(dm, 1, 3, X @ a[0])
    assert np.abs(gs - a[0]).max() <= 1e-12


def test_quadratic_field_is_averaged():
    # u = x^2 on a P1 mesh: element gradients are constant per element, the nodal
    # average lies between the neighbouring element values
    mesh = meshgen.structured_quad(4, 4, order=meshgen.corner_order(1))
    dm = O.dofmanager(mesh, 1)
    X = dm.nodes
    g = O.local_smoothing_gradient(dm, 1, 2, X[:, 0] ** 2)
    assert np.all(g[:, 0] >= -1e-12) and np.all(g[:, 0] <= 2.0 + 1e-12)
    assert np.abs(g[:, 1]).max() <= 1e-12
