"""The VTU writer (yg_output_vtu, SimulationOutput.captureFrame) against the
reference's own SimulationOutput(VTU) + default capture, compiled in place: the
file text must be identical, character for character (tests/golden/vtu_ref.npz,
made by tests/golden/make_golden.py).  The mesh part is host code and is checked
on the CPU; the solution arrays come off the device and are checked on the GPU."""
import os

import numpy as np
import pytest

import yafel_b200 as yb
from yafel_b200 import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
V = np.load(os.path.join(HERE, "golden", "vtu_ref.npz"))
CASES = sorted({k.split("/")[0] for k in V.files})


def case(name):
    k = name + "/"
    mesh = {key[len(k) + 5:]: V[key] for key in V.files if key.startswith(k + "mesh_")}
    p, dpn = (int(v) for v in V[k + "meta"])
    return mesh, p, dpn, V[k + "u"], str(V[k + "text_mesh"]), str(V[k + "text_solution"])


@pytest.mark.parametrize("name", CASES)
def test_mesh_text_matches_reference(tmp_path, name):
    mesh, p, dpn, _, text, _ = case(name)
    dm = yb.DoFManager(mesh, p, dpn, host_only=True)
    base = str(tmp_path / "out")
    _lib.check(_lib.lib().yg_output_vtu(dm.h, base.encode(), None), "vtu")
    assert open(base + ".vtu").read() == text


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_solution_text_matches_reference(ctx, tmp_path, name):
    mesh, p, dpn, u, _, text = case(name)
    dm = yb.DoFManager(mesh, p, dpn)
    fe = yb.FESystem(dm, 2 if np.ptp(mesh["nodes"][:, 2]) == 0 else 3)
    fe.getSolution().upload(u)
    base = str(tmp_path / "sol")
    yb.SimulationOutput(base).captureFrame(fe)
    assert open(base + ".vtu").read() == text


@pytest.mark.gpu
def test_large_solution_streams_in_chunks(ctx, tmp_path):
    """A vector longer than one staging chunk (2^21 values) is written whole."""
    n = (1 << 21) + 1000  # a line of Line2 cells, just over one chunk of nodes
    x = np.linspace(0.0, 1.0, n)
    mesh = {"nodes": np.stack([x, np.zeros(n), np.zeros(n)], axis=1),
            "cell_nodes": np.stack([np.arange(n - 1), np.arange(1, n)], axis=1).ravel().astype(np.int32),
            "offsets": np.arange(0, 2 * n - 1, 2, dtype=np.int32), "cell_types": np.zeros(n - 1, np.int32)}
    dm = yb.DoFManager(mesh, 1, 1)
    fe = yb.FESystem(dm, 1)
    n = dm.ndofs
    vals = np.arange(n, dtype=np.float64) * 0.5
    fe.getSolution().upload(vals)
    base = str(tmp_path / "big")
    yb.SimulationOutput(base).captureFrame(fe)
    text = open(base + ".vtu").read()
    block = text.split('Name="Solution_0" NumberOfComponents="1">\n')[1].split("</DataArray>")[0]
    got = np.array(block.split(), dtype=np.float64)
    assert got.size == n and np.array_equal(got, np.array(["%g" % v for v in vals], dtype=np.float64))
