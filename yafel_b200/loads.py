"""Consistent nodal loads of a surface traction on tensor-product cells.

The reference assembles no boundary-face terms on the CG path (CGAssembly
touches volume quadrature only, include/assembly/CGAssembly.hpp:129-145),
although it has the pieces: Element::face_update (include/element/Element.hpp:151-199)
and the boundary quadrature of make_tensorproduct_element.cpp:130-143.  This
module supplies the uniform-traction load that the elasticity workload needs:
F_{A,i} += t_i * integral over the face of N_A dS, with the face's own
tensor-product Lagrange basis on its GLL nodes and a Gauss-Legendre rule of
exactness 2p, evaluated on the host at set-up.
"""
import numpy as np


def _gll(n):
    """Gauss-Lobatto points on [-1,1] (same values as the element's local nodes)."""
    if n == 2:
        return np.array([-1.0, 1.0])
    # roots of (1-x^2) P'_{n-1}(x): interior points from the Legendre derivative
    c = np.zeros(n)
    c[-1] = 1
    inner = np.polynomial.legendre.Legendre(c).deriv().roots()
    return np.concatenate([[-1.0], np.sort(inner.real), [1.0]])


def _lagrange(nodes, t):
    n = nodes.size
    V = np.ones((t.size, n))
    D = np.zeros((t.size, n))
    for j in range(n):
        others = np.delete(nodes, j)
        den = np.prod(nodes[j] - others)
        V[:, j] = np.prod(t[:, None] - others[None, :], axis=1) / den
        s = np.zeros(t.size)
        for m in range(others.size):
            s += np.prod(np.delete(t[:, None] - others[None, :], m, axis=1), axis=1)
        D[:, j] = s / den
    return V, D


def hex_face_traction(dofm, on_face, traction):
    """Nodal load vector (length dofm.ndofs) of a uniform traction on every hex
    face whose nodes all satisfy on_face(X) (vectorised predicate on (n,3) coords).

    Cells must be order-p tensor-product hexes numbered x fastest (the element's
    local node order).  dof = node*dof_per_node + component."""
    p = dofm.polyOrder
    n = p + 1
    X = dofm.dof_nodes
    off, el = dofm.element_offsets, dofm.elements
    nen = n ** 3
    cells = np.nonzero(np.diff(off) == nen)[0]
    conn = np.stack([el[off[c]:off[c] + nen] for c in cells]) if cells.size else np.zeros((0, nen), np.int64)
    flag = on_face(X)
    idx = np.arange(nen)
    ii, jj, kk = idx // (n * n), (idx // n) % n, idx % n  # z, y, x local indices
    faces = [kk == 0, kk == n - 1, jj == 0, jj == n - 1, ii == 0, ii == n - 1]
    gl_x, gl_w = np.polynomial.legendre.leggauss(max(1, (2 * p + 1) // 2 + (2 * p + 1) % 2))
    nodes1d = _gll(n)
    V, D = _lagrange(nodes1d, gl_x)
    F = np.zeros(dofm.ndofs)
    dpn = dofm.dof_per_node
    t = np.asarray(traction, dtype=np.float64)
    for fm in faces:
        local = np.nonzero(fm)[0]            # (n*n) face nodes, ordered by the remaining two indices
        fn = conn[:, local]                  # cells x face nodes
        hit = flag[fn].all(axis=1)
        if not hit.any():
            continue
        fn = fn[hit]
        Xf = X[fn]                            # faces x n*n x 3, face-node grid (slow, fast)
        Xf = Xf.reshape(-1, n, n, 3)
        # 2-D basis on the face: value V[q,a], derivative D[q,a] per direction
        for qa in range(gl_x.size):
            for qb in range(gl_x.size):
                Na = np.outer(V[qa], V[qb])           # n x n (slow, fast)
                dxa = np.einsum("ab,fabk->fk", np.outer(D[qa], V[qb]), Xf)
                dxb = np.einsum("ab,fabk->fk", np.outer(V[qa], D[qb]), Xf)
                J = np.linalg.norm(np.cross(dxa, dxb), axis=1)
                w = gl_w[qa] * gl_w[qb]
                contrib = (J * w)[:, None] * Na.reshape(1, -1)   # faces x n*n
                for c in range(min(dpn, t.size)):
                    if t[c] != 0:
                        np.add.at(F, fn.ravel() * dpn + c, (t[c] * contrib).ravel())
    return F
