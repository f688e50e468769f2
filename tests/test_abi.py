"""The C-ABI library loads, exports every entry point include/yafel_gpu.h
declares, and its host-side DoF numbering equals the oracle's.  CPU only: no
call here touches a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from yafel_b200 import meshgen
from yafel_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"^YG_API\s+[\w\s\*]+?\b(yg_\w+)\s*\(", src, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 30
    for n in sorted(names):
        assert hasattr(L, n), n
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_status_strings_and_error_paths_without_gpu():
    L = _lib.lib()
    assert L.yg_status_string(0) == b"ok"
    assert L.yg_status_string(6) == b"over HBM budget"
    # a NULL output pointer is rejected before any device work
    assert L.yg_context_create(0, 0, None) == _lib.YG_BAD_ARG
    assert b"NULL" in L.yg_last_error()


def host_dofmap(mesh, p, dpn=1):
    L = _lib.lib()
    nodes = np.ascontiguousarray(mesh["nodes"], dtype=np.float64)
    cn, off, ct = mesh["cell_nodes"], mesh["offsets"], mesh["cell_types"]
    h = C.c_void_p()
    s = L.yg_dofmap_create(None, nodes.ctypes.data, nodes.shape[0], cn.ctypes.data, off.ctypes.data,
                           ct.ctypes.data, ct.size, p, dpn, C.byref(h))
    if s != 0:
        raise RuntimeError(L.yg_last_error())
    a, b, c, d = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
    L.yg_dofmap_sizes(h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
    X = np.empty((a.value, 3))
    o = np.empty(b.value + 1, np.int32)
    e = np.empty(max(c.value, 1), np.int32)
    L.yg_dofmap_get(h, X.ctypes.data, o.ctypes.data, e.ctypes.data, None, None, None)
    L.yg_dofmap_destroy(h)
    return X, o, e[:c.value]


@pytest.mark.parametrize("kind,p", [("quad", 1), ("quad", 2), ("quad", 3), ("hex", 1), ("hex", 2), ("hex", 3),
                                    ("mixed", 1), ("mixed", 2), ("mixed", 3)])
def test_dof_numbering_bit_exact_vs_oracle(kind, p):
    if kind == "quad":
        m = meshgen.structured_quad(7, 5, order=meshgen.corner_order(p))
    elif kind == "hex":
        m = meshgen.structured_hex(3, 4, 2, order=meshgen.corner_order(p))
    else:
        m = meshgen.jittered_mixed(9, 7, seed=11, order=meshgen.corner_order(p))
    X, off, el = host_dofmap(m, p)
    ref = O.dofmanager(m, p)
    assert X.shape[0] == ref.n_nodes
    assert np.array_equal(off, ref.offsets)
    assert np.array_equal(el, ref.elements)
    # merged coordinates: the library keeps the coincident raw node that the
    # reference's std::sort puts first (pinned bit for bit against the reference
    # in test_ref_assembly_pins.py); the oracle keeps the lowest raw index.  They
    # agree to rounding, except where triangles meet quadrilaterals at p >= 3.
    tol = 1e-6 if (kind == "mixed" and p >= 3) else 1e-15
    assert np.abs(X - ref.nodes).max() <= tol


def test_dofmanager_rejects_order_zero():
    m = meshgen.structured_quad(2, 2)
    with pytest.raises(RuntimeError):
        host_dofmap(m, 0)
