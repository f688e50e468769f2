"""The DoF numbering on the GPU (dofmap_gpu.cu) against the host numbering
(itself pinned to the reference in test_ref_assembly_pins.py): above 2^20 raw
nodes yg_dofmap_create numbers on the device and must give the host's bits;
yg_dofmap_create_on_device forces it on small meshes too, where the element
lists are identical and merged coordinates agree to rounding (the host keeps
the coincident node the reference's std::sort leaves first, the device the
first in raw order)."""
import numpy as np
import pytest

import yafel_b200 as yb
from yafel_b200 import meshgen

pytestmark = pytest.mark.gpu


def test_large_mesh_is_numbered_on_device_with_the_host_bits(ctx):
    mesh = meshgen.structured_hex(40, 40, 40, order="ccw")  # 64,000 Q2 cells, 1,728,000 raw nodes
    launches = ctx.launches
    dev = yb.DoFManager(mesh, 2, 3, ctx=ctx)
    assert ctx.launches > launches  # the numbering ran kernels
    host = yb.DoFManager(mesh, 2, 3, host_only=True)
    assert np.array_equal(dev.element_offsets, host.element_offsets)
    assert np.array_equal(dev.elements, host.elements)
    assert np.array_equal(dev.dof_nodes, host.dof_nodes)
    assert dev.nNodes() == 81 ** 3


@pytest.mark.parametrize("kind,p", [("quad", 2), ("quad", 3), ("mixed", 2), ("mixed", 3), ("hex", 2), ("hex", 3),
                                    ("tet", 2), ("tri", 3)])
def test_forced_device_numbering_on_small_meshes(ctx, kind, p):
    if kind == "quad":
        mesh = meshgen.jittered_mixed(9, 7, seed=3, tri_fraction=0.0)
    elif kind == "mixed":
        mesh = meshgen.jittered_mixed(9, 7, seed=3)
    elif kind == "tri":
        mesh = meshgen.jittered_mixed(6, 6, seed=4, tri_fraction=1.0)
    elif kind == "hex":
        mesh = meshgen.structured_hex(4, 3, 3)
    else:
        mesh = meshgen.structured_tet(3, 2, 2, seed=5, jitter=0.2)
    dev = yb.DoFManager(mesh, p, 1, ctx=ctx, on_device=True)
    host = yb.DoFManager(mesh, p, 1, host_only=True)
    assert np.array_equal(dev.element_offsets, host.element_offsets)
    assert np.array_equal(dev.elements, host.elements)
    tol = 1e-6 if (kind == "mixed" and p == 3) else 1e-15
    assert np.abs(dev.dof_nodes - host.dof_nodes).max() <= tol


def test_device_numbered_mesh_assembles_and_solves(ctx):
    mesh = meshgen.structured_hex(6, 6, 6, order="ccw")
    dm = yb.DoFManager(mesh, 2, 3, ctx=ctx, on_device=True)
    fe = yb.FESystem(dm, 3)
    yb.CGAssembly(yb.LinearElasticity(3, body=(0.0, 0.0, -1.0)), fe)
    for c in range(3):
        bc = yb.DirichletBC(dm, 0.0, c)
        bc.selectByFunction(lambda X: np.abs(X[:, 0]) < 1e-9)
        bc.apply(fe.getGlobalTangent(), fe.getGlobalResidual())
    K = fe.getGlobalTangent()
    x, st = yb.solve(K, fe.getGlobalResidual(), M=yb.JacobiPreconditioner(K), tol=1e-10)
    assert st.status == 0 and st.rel_residual <= 1e-10


@pytest.mark.parametrize("dim,n,p", [(3, (40, 40, 40), 2), (3, (5, 4, 3), 2), (3, (4, 3, 2), 3), (3, (6, 5, 4), 1),
                                     (2, (13, 9), 2), (2, (7, 6), 3), (2, (8, 8), 1)])
def test_box_generated_on_device(ctx, dim, n, p):
    lengths = (1.0, 2.5, 0.75)
    dev = yb.DoFManager.box(dim, n, lengths, p, 1, ctx=ctx)
    order = meshgen.corner_order(p)
    mesh = (meshgen.structured_hex(*n, *lengths, order=order) if dim == 3
            else meshgen.structured_quad(*n, *lengths[:2], order=order))
    host = yb.DoFManager(mesh, p, 1, host_only=True)
    assert np.array_equal(dev.element_offsets, host.element_offsets)
    assert np.array_equal(dev.elements, host.elements)
    exact = p == 1 or np.prod(n) * (p + 1) ** dim > (1 << 20)  # the host's stable order
    if exact:
        assert np.array_equal(dev.dof_nodes, host.dof_nodes)
    else:
        assert np.abs(dev.dof_nodes - host.dof_nodes).max() <= 1e-15 * max(lengths)
