"""Failure paths of the solvers, injected on the host (no GPU fault, trap or
hang): a NaN in the right-hand side, an HBM budget below the matrix, the
iteration cap, a BiCGSTAB breakdown, and a NaN system among healthy ones in a
batch and in the server.  The reference reports none of these: its cg_solve
and pcg_solve stop silently at the iteration cap (cg_solve.hpp:46,56) and its
bicgstab_solve divides by a zero r0.v (bicgstab_solve.hpp:53); here each ends
with a status and the context stays usable."""
import numpy as np
import pytest

import yafel_b200 as yb
from oracle import oracle as O
from yafel_b200 import _lib, meshgen, workloads

pytestmark = pytest.mark.gpu


def poisson(n=32):
    """n x n Q1 Poisson with u = 0 on the boundary, assembled by the oracle."""
    dm = O.dofmanager(meshgen.structured_quad(n, n, order="tensor"), 1)
    K, R = O.assemble(dm, 1, 2, O.POISSON, [1.0, 1.0])
    X = dm.nodes
    mask = ((X[:, 0] < 1e-9) | (X[:, 0] > 1 - 1e-9) | (X[:, 1] < 1e-9) | (X[:, 1] > 1 - 1e-9)).astype(np.uint8)
    O.dirichlet_apply(K, R, mask, np.zeros(K.nrows))
    return K, R


@pytest.mark.parametrize("method,precision", [("cg", yb.PREC_FP64), ("cg", yb.PREC_MIXED),
                                              ("bicgstab", yb.PREC_FP64)])
def test_nan_rhs_reports_nan(ctx, method, precision):
    K, R = poisson()
    A = yb.sparse_csr.from_csr(K.row_ptr, K.col, K.val)
    b = R.copy()
    b[17] = np.nan
    x, st = yb.solve(A, b, M=yb.JacobiPreconditioner(A), method=method, tol=1e-10, precision=precision)
    assert st.status == _lib.YG_NAN, st.status
    # the context is still usable: the same system without the NaN converges
    x, st = yb.solve(A, R, M=yb.JacobiPreconditioner(A), method=method, tol=1e-10, precision=precision)
    assert st.status == _lib.YG_OK and st.rel_residual <= 1e-10


def test_bicgstab_in_mixed_precision_is_unsupported(ctx):
    """BiCGSTAB runs in FP64 only; another precision is refused before any launch."""
    K, R = poisson()
    A = yb.sparse_csr.from_csr(K.row_ptr, K.col, K.val)
    with pytest.raises(yb.YafelError) as e:
        yb.solve(A, R, M=yb.JacobiPreconditioner(A), method="bicgstab", precision=yb.PREC_MIXED)
    assert e.value.status == _lib.YG_UNSUPPORTED


def test_preconditioner_outlives_its_matrix(ctx):
    """A garbage-collected cycle finalises objects in any order: a preconditioner
    freed after its matrix touches only its own context."""
    K, R = poisson()
    A = yb.sparse_csr.from_csr(K.row_ptr, K.col, K.val)
    for P in (yb.JacobiPreconditioner, yb.ILUPreconditioner):
        M = P(A)
        B = yb.sparse_csr.from_csr(K.row_ptr, K.col, K.val)
        M2 = P(B)
        _lib.check(_lib.lib().yg_matrix_destroy(B.h))
        B.h = None
        _lib.check(_lib.lib().yg_precond_destroy(M2.h))
        M2.h = None
    x, st = yb.solve(A, R, M=M, tol=1e-10)
    assert st.status == _lib.YG_OK


def test_budget_below_the_matrix_is_over_budget():
    small = yb.Context(0, hbm_budget=2 << 20)  # 2 MiB
    mesh = meshgen.structured_hex(6, 6, 6, order="ccw")
    dm = yb.DoFManager(mesh, 2, 3, ctx=small)  # 2197 nodes: fits
    fe = yb.FESystem(dm, 3)
    with pytest.raises(yb.YafelError) as e:
        yb.CGAssembly(yb.LinearElasticity(3), fe)  # 3x3 blocks: ~11 MB of values
    assert e.value.status == _lib.YG_OVER_BUDGET
    # a system that fits still assembles and solves on the same context
    dm2 = yb.DoFManager(meshgen.structured_quad(8, 8, order="tensor"), 1, 1, ctx=small)
    fe2 = yb.FESystem(dm2, 2, format=yb.CSR)
    yb.CGAssembly(yb.PoissonEquation(2), fe2)
    bc = yb.DirichletBC(dm2, 0.0)
    bc.selectByFunction(lambda X: (X[:, 0] < 1e-9) | (X[:, 0] > 1 - 1e-9))
    bc.apply(fe2.getGlobalTangent(), fe2.getGlobalResidual())
    x, st = yb.solve(fe2.getGlobalTangent(), fe2.getGlobalResidual(), M=yb.JacobiPreconditioner(fe2.getGlobalTangent()))
    assert st.status == _lib.YG_OK and st.rel_residual <= 1e-10
    small.close()


@pytest.mark.parametrize("method", ["cg", "bicgstab"])
def test_iteration_cap_reports_not_converged_with_the_fp64_residual(ctx, method):
    K, R = poisson()
    A = yb.sparse_csr.from_csr(K.row_ptr, K.col, K.val)
    x, st = yb.solve(A, R, M=yb.JacobiPreconditioner(A), method=method, tol=1e-10, maxiter=5)
    assert st.status == _lib.YG_NOT_CONVERGED
    assert st.iterations == 5
    rel = O.true_relres(K, R, x.numpy())
    assert rel > 1e-10
    assert abs(st.rel_residual - rel) <= 1e-8 * rel  # the reported residual is the true FP64 one


def test_iteration_cap_race_repeated(ctx):
    """The PCG direction kernel must read the iteration count that the previous
    kernel recorded, not the one block 0 increments in the same launch: a CG
    solve on a multi-block grid stopped by its cap gives the same iteration
    count and the same bits every time."""
    K, R = poisson(48)  # 2401 rows: many blocks of the persistent grid
    A = yb.sparse_csr.from_csr(K.row_ptr, K.col, K.val)
    M = yb.JacobiPreconditioner(A)
    first = None
    for _ in range(100):
        x, st = yb.solve(A, R, M=M, tol=1e-14, maxiter=37)
        assert st.status == _lib.YG_NOT_CONVERGED and st.iterations == 37
        xs = x.numpy()
        if first is None:
            first = xs
        assert np.array_equal(xs, first)


def test_bicgstab_breakdown_is_reported(ctx):
    """A skew-symmetric matrix gives r0.(A r0) = 0 exactly for r0 = e_1, so
    every BiCGSTAB start breaks down; after its restarts from the true residual
    the solver reports a breakdown instead of dividing by zero."""
    n = 40
    r = np.concatenate([np.arange(n - 1), np.arange(1, n)])
    c = np.concatenate([np.arange(1, n), np.arange(n - 1)])
    v = np.concatenate([np.ones(n - 1), -np.ones(n - 1)])
    A = yb.sparse_csr((r.astype(np.uint64), c.astype(np.uint64), v))
    b = np.zeros(n)
    b[0] = 1.0
    x, st = yb.solve(A, b, method="bicgstab", tol=1e-10)
    assert st.status == _lib.YG_BREAKDOWN, st.status
    assert np.all(np.isfinite(x.numpy()))


def _specs():
    return [dict(workloads.problem_spec(i, lo=1e3, hi=8e3)) for i in range(4)]


def test_nan_system_in_a_batch_leaves_the_others_bit_identical(ctx):
    specs = _specs()
    built = [workloads.assemble(s, ctx) for s in specs]
    alone = []
    for s, (_, K, b, _) in zip(specs, built):
        B = yb.Batch(1, ctx)
        slot = B.add(K, b, method=workloads.method(s))
        assert B.run() == 0
        alone.append(B.solution(slot).numpy())
    # the same systems plus a copy of system 1 whose right-hand side holds a NaN
    _, K1, b1, _ = built[1]
    bad = b1.numpy()
    bad[3] = np.nan
    B = yb.Batch(8, ctx)
    slots = [B.add(K, b, method=workloads.method(s)) for s, (_, K, b, _) in zip(specs, built)]
    nan_slot = B.add(K1, bad, method=workloads.method(specs[1]))
    B.run()
    assert B.stats(nan_slot).status == _lib.YG_NAN
    for i, s in enumerate(slots):
        st = B.stats(s)
        assert st.status == _lib.YG_OK and st.rel_residual <= 1e-10
        assert np.array_equal(B.solution(s).numpy(), alone[i]), i


def test_nan_request_in_the_server_leaves_the_others_bit_identical(ctx):
    specs = _specs()
    S = yb.Server(int(1e10), max_active=16, ctx=ctx)
    rids = {}
    for i, s in enumerate(specs):
        rids[S.submit(workloads.est_bytes(s))] = i
    nan_rid = S.submit(workloads.est_bytes(specs[2]))
    keep, results = {}, {}
    while True:
        rid = S.admit()
        if rid is None:
            break
        i = rids.get(rid, 2)
        _, K, b, _ = workloads.assemble(specs[i], ctx)
        if rid == nan_rid:
            h = b.numpy()
            h[0] = np.nan
            b = yb.DeviceVector(h, ctx)
        x = yb.DeviceVector(K.rows(), ctx)
        x.fill(0.0)
        S.attach(rid, K, b, x, method=workloads.method(specs[i]))
        keep[rid] = (K, b, x)
    while len(results) < len(specs) + 1:
        S.launch()
        S.wait()
        for rid in S.finished():
            st = S.poll(rid)
            results[rid] = (st.status, S.solution(rid).numpy())
            S.release(rid)
    assert results[nan_rid][0] == _lib.YG_NAN
    for rid, i in rids.items():
        status, x = results[rid]
        assert status == _lib.YG_OK
        _, K, b, _ = workloads.assemble(specs[i], ctx)
        B = yb.Batch(1, ctx)
        slot = B.add(K, b, method=workloads.method(specs[i]))
        assert B.run() == 0
        assert np.array_equal(B.solution(slot).numpy(), x), i
