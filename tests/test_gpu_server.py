"""The continuous-batching solve server (yg_server_*): requests of every kind
(2D/3D Poisson, elasticity, SUPG by BiCGSTAB) are admitted in arrival order
under an HBM budget small enough to make the queue wait, every request reaches
a 1e-10 relative residual, the held bytes never exceed the budget, and each
batched result equals the one the system gets when solved alone in a batch;
with a solo threshold, the large systems are solved alone in between."""
import numpy as np
import pytest

import yafel_b200 as yb
from yafel_b200 import workloads

pytestmark = pytest.mark.gpu

SPECS = workloads.serving_specs(12, lo=1e3, hi=2e4)


@pytest.mark.parametrize("solo_rows", [0, 4000])
def test_server_admits_by_budget_and_solves_everything(ctx, solo_rows):
    assert {s["kind"] for s in SPECS} == {"poisson", "elasticity", "supg"}
    assert {s["dim"] for s in SPECS} == {2, 3}
    est = [workloads.est_bytes(s) for s in SPECS]
    budget = 2 * max(est)
    S = yb.Server(budget, max_active=8, ctx=ctx)
    S.set_solo_rows(solo_rows)
    ids = {S.submit(e): i for i, e in enumerate(est)}
    built, results, waited_for_room, rows = {}, {}, False, {}
    while len(results) < len(SPECS):
        while True:
            rid = S.admit()
            if rid is None:
                break
            spec = SPECS[ids[rid]]
            mesh, K, b, _ = workloads.assemble(spec, ctx)
            x = yb.DeviceVector(K.rows(), ctx)
            x.fill(0.0)
            S.attach(rid, K, b, x, method=workloads.method(spec))
            built[rid] = (K, b)
            rows[ids[rid]] = K.rows()
        info = S.info()
        assert info["bytes_held"] <= budget
        if info["queued"] > 0:
            waited_for_room = True
        S.launch()
        S.wait()
        for rid in S.finished():
            st = S.poll(rid)
            results[ids[rid]] = (st.status, st.rel_residual, S.solution(rid).numpy())
            S.release(rid)
            built.pop(rid)
    assert waited_for_room
    for i, (status, rel, x) in results.items():
        assert status == 0 and rel <= 1e-10, (SPECS[i], status, rel)
    if solo_rows:
        assert any(r >= solo_rows for r in rows.values()) and any(r < solo_rows for r in rows.values())
    # a batched system's result equals the one it gets alone in a batch
    for i in [k for k in (0, 5, 11) if not solo_rows or rows[k] < solo_rows]:
        mesh, K, b, _ = workloads.assemble(SPECS[i], ctx)
        B = yb.Batch(1, ctx)
        s = B.add(K, b, method=workloads.method(SPECS[i]))
        assert B.run() == 0
        assert np.array_equal(B.solution(s).numpy(), results[i][2]), i


def test_server_with_requests_built_on_a_second_context(ctx):
    """Requests assembled on another context of the device (its own stream) while
    a block runs: ready() reports the block's completion without blocking, the
    attached systems converge, and their results equal those of the same systems
    built on the server's own context."""
    bctx = yb.Context(0)
    S = yb.Server(int(1e11), max_active=16, ctx=ctx)
    ids = {S.submit(workloads.est_bytes(s)): i for i, s in enumerate(SPECS)}
    pending, results, keep = [], {}, {}

    def build_one():
        rid = S.admit()
        if rid is None:
            return False
        spec = SPECS[ids[rid]]
        _, K, b, _ = workloads.assemble(spec, bctx)
        x = yb.DeviceVector(K.rows(), bctx)
        x.fill(0.0)
        pending.append((rid, K, b, x))
        return True

    build_one()
    assert S.ready()  # nothing in flight
    while len(results) < len(SPECS):
        for rid, K, b, x in pending:
            S.attach(rid, K, b, x, method=workloads.method(SPECS[ids[rid]]))
            keep[rid] = (K, b, x)
        pending.clear()
        S.launch()
        while not S.ready():
            if not build_one():
                break
        S.wait()
        assert S.ready()
        for rid in S.finished():
            st = S.poll(rid)
            results[ids[rid]] = (st.status, st.rel_residual, S.solution(rid).numpy())
            S.release(rid)
            keep.pop(rid)
        if S.info()["active"] == 0 and not pending:
            build_one()
    for i, (status, rel, _) in results.items():
        assert status == 0 and rel <= 1e-10, (SPECS[i], status, rel)
    for i in (0, 4, 9):
        _, K, b, _ = workloads.assemble(SPECS[i], ctx)
        B = yb.Batch(1, ctx)
        s = B.add(K, b, method=workloads.method(SPECS[i]))
        assert B.run() == 0
        assert np.array_equal(B.solution(s).numpy(), results[i][2]), i
