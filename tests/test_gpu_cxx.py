"""The C++ drop-in adapters (include/yafel_gpu/yafel_gpu.hpp) compile against the
C ABI and run a reference-style application on the GPU; results are checked
against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from yafel_b200 import meshgen, _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_example(tmp_path):
    _lib.lib()  # builds libyafel_b200.so if absent
    exe = str(tmp_path / "poisson_drop_in")
    libdir = os.path.join(ROOT, "yafel_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "poisson_drop_in.cpp"),
                    os.path.join(libdir, "libyafel_b200.so"), "-Wl,-rpath," + libdir, "-o", exe], check=True)
    return exe


def test_cxx_adapter_compiles(tmp_path):
    assert os.path.exists(build_example(tmp_path))


def test_cxx_gradient_adapter_compiles(tmp_path):
    obj = str(tmp_path / "gradient_compile.o")
    subprocess.run(["g++", "-std=c++17", "-O2", "-c", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "gradient_compile.cpp"), "-o", obj], check=True)
    assert os.path.exists(obj)


@pytest.mark.gpu
def test_cxx_drop_in_poisson_matches_oracle(tmp_path):
    exe = build_example(tmp_path)
    out = subprocess.run([exe, "16"], check=True, capture_output=True, text=True, timeout=120).stdout
    vals = dict(line.split() for line in out.strip().splitlines())
    dm = O.dofmanager(meshgen.structured_quad(16, 16, order="tensor"), 1)
    K, F = O.assemble(dm, 1, 2, O.POISSON, [1.0, 1.0])
    X = dm.nodes
    mask = ((np.abs(X[:, 0]) < 1e-6) | (np.abs(X[:, 0] - 1) < 1e-6) |
            (np.abs(X[:, 1]) < 1e-6) | (np.abs(X[:, 1] - 1) < 1e-6)).astype(np.uint8)
    O.dirichlet_apply(K, F, mask, np.zeros(K.nrows))
    x, _, _ = O.cg(K, F, precond=O.PRECOND_JACOBI, tol=1e-13)
    assert int(vals["dofs"]) == K.nrows and int(vals["nnz"]) == K.nnz
    assert float(vals["relres"]) <= 1e-10
    assert abs(float(vals["umax"]) - x.max()) <= 1e-9 * x.max()
    assert float(vals["laplace_err2"]) < 1e-10 and float(vals["laplace_pcg_err2"]) < 1e-10
