"""Mesh ingest (yg_mesh_read_gmsh / Mesh.from_gmsh) against the reference's own
Mesh(fname) (src/mesh/parse_gmsh.cpp, compiled in place) on Gmsh 2.2 files
written by tests/golden/make_golden.py: nodes, cell lists, offsets, cell types
(an unknown Gmsh type gives None) and tags bit for bit; and the DoF numbering of
a mesh read this way, boundary lines and corner points included, against the
reference's DoFManager at p = 2.  Host code only (no GPU)."""
import os

import numpy as np
import pytest

import yafel_b200 as yb

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "gmsh_ref.npz"))
FILES = sorted({k.split("/")[0] for k in G.files})


@pytest.mark.parametrize("name", FILES)
def test_gmsh_reader_matches_reference(tmp_path, name):
    path = tmp_path / (name + ".msh")
    path.write_text(str(G[name + "/text"]))
    m = yb.Mesh.from_gmsh(path)
    assert np.array_equal(m.nodes, G[name + "/nodes"])
    assert np.array_equal(m.cell_nodes, G[name + "/cell_nodes"])
    assert np.array_equal(m.offsets, G[name + "/offsets"])
    assert np.array_equal(m.cell_types, G[name + "/cell_types"])
    to, tg = G[name + "/tag_offsets"], G[name + "/tags"]
    assert all(np.array_equal(m.tags_all[c], tg[to[c]:to[c + 1]]) for c in range(m.nCells()))
    assert np.array_equal(m.cell_tags, tg[to[:-1]])


def test_numbering_of_a_read_mesh_with_lower_dimensional_cells(tmp_path):
    path = tmp_path / "m.msh"
    path.write_text(str(G["mixed2d/text"]))
    m = yb.Mesh.from_gmsh(path)
    assert set(np.unique(m.cell_types)) == {0, 1, 3, 5}  # lines, triangles, quads, points
    dm = yb.DoFManager(m, 2, 1, host_only=True)
    assert np.array_equal(dm.elements, G["mixed2d/p2_elements"])
    assert np.array_equal(dm.dof_nodes, G["mixed2d/p2_dof_nodes"])
    # offsets: equal except at the Point1 cells (ElementTopology::None), which the
    # reference skips before recording their offset, leaving 0 there
    # (DoFManager.cpp:196-199) -- which also empties the range of the cell before
    # them; here a None cell gets an empty range at the running offset
    ref_off = G["mixed2d/p2_offsets"]
    none = np.nonzero(m.cell_types == 5)[0]
    keep = np.setdiff1d(np.arange(ref_off.size), none)
    assert np.array_equal(dm.element_offsets[keep], ref_off[keep]) and np.all(ref_off[none] == 0)
    assert np.all(np.diff(dm.element_offsets) >= 0) and np.all(np.diff(dm.element_offsets)[none] == 0)


def test_bad_files_are_reported(tmp_path):
    with pytest.raises(yb.YafelError):
        yb.Mesh.from_gmsh(tmp_path / "missing.msh")
    bad = tmp_path / "bad.msh"
    bad.write_text("$Nodes\n2\n1 0 0 0\n3 1 0 0\n$EndNodes\n")  # node id past the count
    with pytest.raises(yb.YafelError, match="line 4"):
        yb.Mesh.from_gmsh(bad)
