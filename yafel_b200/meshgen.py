"""Synthetic mesh generators producing the reference's explicit Mesh layout.

The layout is the one ``Mesh(DefinitionScheme::Explicit, nodes, cellNodes,
offsets, cellTypes)`` takes (include/mesh/Mesh.hpp:48-53): node coordinates
(always three components), a flat cell->node list with CSR offsets, and one
CellType code per cell (include/mesh/mesh_typedefs.hpp:42-50: Line2=0, Tri3=1,
Tet4=2, Quad4=3, Hex8=4, Point1=5).  Corner order follows the bilinear and
trilinear maps of DoFManager::interpolate_from_corners
(src/utils/DoFManager.cpp:296-338): counter-clockwise, bottom face first.

Corner order matters twice in the reference.  For polynomial order p>1 the
DoFManager places each cell's nodes with those counter-clockwise maps.  For p=1
it keeps the mesh's cell list as the element's node list
(src/utils/DoFManager.cpp:153-160), and a tensor-product element numbers its
nodes x fastest (src/element/make_tensorproduct_element.cpp:158-193), so a
counter-clockwise quad or hex is read as a twisted element.  Generators
therefore take ``order="ccw"`` (for p>1, and what Gmsh writes) or
``order="tensor"`` (x-fastest corners, what a p=1 tensor element expects);
``corner_order(p)`` picks the one that gives an untwisted element.
"""
import numpy as np

LINE2, TRI3, TET4, QUAD4, HEX8, POINT1 = 0, 1, 2, 3, 4, 5


def _mesh(nodes, cells, nper, ctypes):
    cells = np.ascontiguousarray(cells, dtype=np.int32).ravel()
    if np.isscalar(nper):
        offsets = np.arange(0, cells.size + 1, nper, dtype=np.int32)
    else:
        offsets = np.concatenate([[0], np.cumsum(nper)]).astype(np.int32)
    return {"nodes": np.ascontiguousarray(nodes, dtype=np.float64),
            "cell_nodes": cells, "offsets": offsets,
            "cell_types": np.ascontiguousarray(ctypes, dtype=np.int32)}


def corner_order(p):
    """Corner order that the reference reads as an untwisted element at order p."""
    return "tensor" if p == 1 else "ccw"


def structured_quad(nx, ny, lx=1.0, ly=1.0, order="ccw"):
    """nx*ny Quad4 cells on [0,lx]x[0,ly]; nodes x fastest."""
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    nodes = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (j * (nx + 1) + i).ravel()
    if order == "ccw":
        cells = np.stack([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1], axis=1)
    else:
        cells = np.stack([n0, n0 + 1, n0 + nx + 1, n0 + nx + 2], axis=1)
    return _mesh(nodes, cells, 4, np.full(nx * ny, QUAD4))


def structured_hex(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0, order="ccw"):
    """nx*ny*nz Hex8 cells on a box; nodes x fastest, then y, then z."""
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    sx, sy = 1, nx + 1
    sz = (nx + 1) * (ny + 1)
    n0 = (k * sz + j * sy + i).ravel()
    if order == "ccw":
        cells = np.stack([n0, n0 + sx, n0 + sx + sy, n0 + sy,
                          n0 + sz, n0 + sz + sx, n0 + sz + sx + sy, n0 + sz + sy], axis=1)
    else:
        cells = np.stack([n0, n0 + sx, n0 + sy, n0 + sx + sy,
                          n0 + sz, n0 + sz + sx, n0 + sz + sy, n0 + sz + sx + sy], axis=1)
    return _mesh(nodes, cells, 8, np.full(nx * ny * nz, HEX8))


def jittered_mixed(nx, ny, seed, tri_fraction=0.5, jitter=0.2, lx=1.0, ly=1.0, order="ccw"):
    """Structured nx*ny grid whose cells are quads, or split into two triangles
    by a seeded coin; interior nodes moved by U(-jitter, jitter)*h per
    coordinate.  Deterministic for a given seed (numpy PCG64)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = structured_quad(nx, ny, lx, ly)
    nodes = m["nodes"].copy()
    hx, hy = lx / nx, ly / ny
    ix = np.tile(np.arange(nx + 1), ny + 1)
    iy = np.repeat(np.arange(ny + 1), nx + 1)
    interior = (ix > 0) & (ix < nx) & (iy > 0) & (iy < ny)
    d = rng.uniform(-jitter, jitter, size=(nodes.shape[0], 2))
    nodes[interior, 0] += d[interior, 0] * hx
    nodes[interior, 1] += d[interior, 1] * hy
    quads = m["cell_nodes"].reshape(-1, 4)
    split = rng.uniform(size=quads.shape[0]) < tri_fraction
    cells, nper, types = [], [], []
    for q, s in zip(quads, split):
        if s:
            cells += [q[0], q[1], q[2], q[0], q[2], q[3]]
            nper += [3, 3]
            types += [TRI3, TRI3]
        else:
            cells += list(q) if order == "ccw" else [q[0], q[1], q[3], q[2]]
            nper.append(4)
            types.append(QUAD4)
    return _mesh(nodes, np.array(cells), np.array(nper), np.array(types))


def structured_tet(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0, seed=None, jitter=0.0):
    """nx*ny*nz boxes, each split into six Tet4 cells around its main diagonal
    (Freudenthal-Kuhn), corners ordered so that every tetrahedron has positive
    volume under the map (1-x-y-z) c0 + x c1 + y c2 + z c3 that
    DoFManager::interpolate_from_corners uses for Tet4
    (src/utils/DoFManager.cpp:307-311).  With a seed, interior nodes move by
    U(-jitter, jitter) times the box size per coordinate (numpy PCG64)."""
    m = structured_hex(nx, ny, nz, lx, ly, lz, order="tensor")
    nodes = m["nodes"].copy()
    if seed is not None and jitter > 0:
        rng = np.random.Generator(np.random.PCG64(seed))
        h = np.array([lx / nx, ly / ny, lz / nz])
        ix = np.round(nodes / h).astype(np.int64)
        interior = ((ix[:, 0] > 0) & (ix[:, 0] < nx) & (ix[:, 1] > 0) & (ix[:, 1] < ny) &
                    (ix[:, 2] > 0) & (ix[:, 2] < nz))
        d = rng.uniform(-jitter, jitter, size=nodes.shape) * h
        nodes[interior] += d[interior]
    hexes = m["cell_nodes"].reshape(-1, 8)  # tensor order: corner (i,j,k) at i + 2j + 4k
    # paths from corner 0 to corner 7 along the three axes in every order
    paths = [(1, 2, 4), (1, 4, 2), (2, 1, 4), (2, 4, 1), (4, 1, 2), (4, 2, 1)]
    tets = []
    for hx in hexes:
        for a, b, c in paths:
            t = [hx[0], hx[a], hx[a + b], hx[7]]
            x = nodes[t]
            if np.linalg.det(np.stack([x[1] - x[0], x[2] - x[0], x[3] - x[0]])) < 0:
                t[1], t[2] = t[2], t[1]
            tets.append(t)
    return _mesh(nodes, np.array(tets), 4, np.full(len(tets), TET4))
