"""Batched and continuous-batching solves (yg_batch_*): every system converges to
a 1e-10 relative residual (checked in FP64 against the oracle-assembled system),
and a system's result is the same alone and in the mix."""
import numpy as np
import pytest

import yafel_b200 as yb
from oracle import oracle as O
from yafel_b200 import workloads

pytestmark = pytest.mark.gpu


def assemble_problem(spec, ctx):
    return workloads.assemble(spec, ctx)


def oracle_relres(spec, mesh, dofs, b_host, x):
    # the oracle assembles on the library's numbering, which is the reference's
    # (its merged coordinates can differ from the oracle's own choice where
    # triangles meet quadrilaterals at order 3)
    hd = yb.DoFManager(mesh, spec["order"], spec["dpn"], host_only=True)
    odm = O.ArrayDofMap(hd.dof_nodes, hd.element_offsets, hd.elements, mesh["cell_types"], spec["order"])
    if spec["kind"] == "supg":
        kind = O.SUPG
        h = 1.0 / spec["n"]
        params = [h / (2.0 * spec["peclet"]), h, 1.0, 0.0]
    elif spec["kind"] == "poisson":
        kind, params = O.POISSON, [1.0, 0.0]
    else:
        kind, params = O.ELASTICITY, [1.0, 0.576923076923077, 0.3846153846153846, 0, 0, 0]
    K, _ = O.assemble(odm, spec["dpn"], spec["dim"], kind, params)
    mask = np.zeros(K.nrows, np.uint8)
    mask[dofs] = 1
    bb = workloads.rhs(spec, K.nrows)
    O.dirichlet_apply(K, bb, mask, np.zeros(K.nrows))
    assert np.allclose(bb, b_host, rtol=0, atol=1e-12 * np.abs(bb).max())
    return O.true_relres(K, bb, x)


SPECS = [dict(workloads.problem_spec(i, lo=1e3, hi=2e4)) for i in range(6)]


@pytest.mark.parametrize("precision", [yb.PREC_FP64, yb.PREC_MIXED])
def test_batch_converges_and_matches_single_solves(ctx, precision):
    probs = [assemble_problem(s, ctx) for s in SPECS]
    B = yb.Batch(len(probs), ctx)
    slots = [B.add(K, b, precision=precision) for (_, K, b, _) in probs]
    B.tune()
    assert B.run() == 0
    for spec, (mesh, K, b, dofs), s in zip(SPECS, probs, slots):
        st = B.stats(s)
        assert st.status == 0 and st.rel_residual <= 1e-10, (spec, st.status, st.rel_residual)
        x = B.solution(s).numpy()
        assert oracle_relres(spec, mesh, dofs, b.numpy(), x) <= 1e-10
        xs, sts = yb.solve(K, b, M=yb.JacobiPreconditioner(K), tol=1e-10)
        assert sts.status == 0
        assert np.linalg.norm(x - xs.numpy()) <= 1e-6 * np.linalg.norm(xs.numpy())


def test_continuous_batching_same_result_alone_and_in_mix(ctx):
    probs = [assemble_problem(s, ctx) for s in SPECS]
    # alone: each system in a batch of its own
    alone = []
    for (_, K, b, _) in probs:
        B1 = yb.Batch(1, ctx)
        s = B1.add(K, b)
        B1.run()
        alone.append(B1.solution(s).numpy())
    # mixed, with arrivals and a departure while others iterate
    B = yb.Batch(4, ctx)
    live = {}
    queue = list(range(len(probs)))
    done = {}
    for _ in range(200):
        while queue and len(live) < 4:
            i = queue.pop(0)
            live[B.add(probs[i][1], probs[i][2])] = i
        active = B.run(max_blocks=1)
        for s, i in list(live.items()):
            st = B.stats(s)
            if st.status == 0:
                done[i] = B.solution(s).numpy().copy()
                B.remove(s)
                del live[s]
        if not queue and not live:
            break
    assert len(done) == len(probs)
    for i in range(len(probs)):
        assert np.array_equal(done[i], alone[i]), i


def test_reset_solves_again_to_the_same_bits(ctx):
    probs = [assemble_problem(s, ctx) for s in SPECS[:3]]
    B = yb.Batch(3, ctx)
    slots = [B.add(K, b) for (_, K, b, _) in probs]
    assert B.run() == 0
    first = [B.solution(s).numpy().copy() for s in slots]
    for s in slots:
        B.solution(s).fill(0.0)
    B.reset()
    assert B.run() == 0
    for s, f in zip(slots, first):
        assert B.stats(s).status == 0
        assert np.array_equal(B.solution(s).numpy(), f)


MIXED_SPECS = [workloads.problem_spec(i, lo=1e3, hi=1e4, kinds=("supg", "poisson", "elasticity")) for i in range(8)]


@pytest.mark.parametrize("precision", [yb.PREC_FP64, yb.PREC_MIXED])
def test_batch_bicgstab_beside_pcg(ctx, precision):
    """SUPG advection-diffusion systems (BiCGSTAB) and SPD systems (PCG) in one
    batch: all reach 1e-10 (checked on the oracle-assembled system) and the
    BiCGSTAB results agree with the single-system yg_bicgstab."""
    assert any(s["kind"] == "supg" for s in MIXED_SPECS) and any(s["kind"] != "supg" for s in MIXED_SPECS)
    probs = [assemble_problem(s, ctx) for s in MIXED_SPECS]
    B = yb.Batch(len(probs), ctx)
    slots = [B.add(K, b, precision=precision, method=workloads.method(s)) for s, (_, K, b, _) in zip(MIXED_SPECS, probs)]
    B.tune()
    assert B.run() == 0
    for spec, (mesh, K, b, dofs), s in zip(MIXED_SPECS, probs, slots):
        st = B.stats(s)
        assert st.status == 0 and st.rel_residual <= 1e-10, (spec, st.status, st.rel_residual)
        x = B.solution(s).numpy()
        assert oracle_relres(spec, mesh, dofs, b.numpy(), x) <= 1e-10, spec
        if spec["kind"] == "supg":
            xs, sts = yb.solve(K, b, M=yb.JacobiPreconditioner(K), method="bicgstab", tol=1e-10)
            assert sts.status == 0
            assert np.linalg.norm(x - xs.numpy()) <= 1e-6 * np.linalg.norm(xs.numpy())


def test_bicgstab_same_result_alone_and_in_mix(ctx):
    probs = [assemble_problem(s, ctx) for s in MIXED_SPECS]
    methods = [workloads.method(s) for s in MIXED_SPECS]
    alone = []
    for (_, K, b, _), m in zip(probs, methods):
        B1 = yb.Batch(1, ctx)
        s = B1.add(K, b, method=m)
        assert B1.run() == 0
        alone.append(B1.solution(s).numpy())
    B = yb.Batch(len(probs), ctx)
    slots = [B.add(K, b, method=m) for (_, K, b, _), m in zip(probs, methods)]
    assert B.run() == 0
    for i, s in enumerate(slots):
        assert np.array_equal(B.solution(s).numpy(), alone[i]), i


@pytest.mark.parametrize("variant,lanes,tiles", [(0, 1, 4), (0, 2, 1), (0, 32, 16), (1, 1, 4), (1, 4, 1),
                                                 (1, 32, 16)])
def test_every_spmv_variant_solves_the_mix(ctx, variant, lanes, tiles):
    """Each SpMV variant (staged tiles with a lane per block and segmented row
    sums, or L lanes per row; direct loads with a thread or L lanes per row) on
    PCG and BiCGSTAB systems of 1x1 and 2x2 blocks: every system reaches 1e-10."""
    probs = [assemble_problem(s, ctx) for s in MIXED_SPECS]
    B = yb.Batch(len(probs), ctx)
    slots = [B.add(K, b, method=workloads.method(s)) for s, (_, K, b, _) in zip(MIXED_SPECS, probs)]
    for blk in (1, 2, 3):
        B.set_tuning(blk, variant, lanes, tiles)
    assert B.run() == 0
    for spec, (mesh, K, b, dofs), s in zip(MIXED_SPECS, probs, slots):
        st = B.stats(s)
        assert st.status == 0 and st.rel_residual <= 1e-10, (spec, st.status, st.rel_residual)
        assert oracle_relres(spec, mesh, dofs, b.numpy(), B.solution(s).numpy()) <= 1e-10


@pytest.mark.parametrize("precision", [yb.PREC_FP64, yb.PREC_MIXED])
def test_systems_with_their_own_spmv_launch(ctx, precision):
    """Systems above the matrix-size threshold run their iteration SpMV as a
    single-system launch inside the batch's graph (PCG and BiCGSTAB): they reach
    1e-10 on the oracle-assembled system, agree with the shared-kernel solution,
    give the same bits alone and in the mix, and a system of that kind added
    while the batch runs (a new graph) converges too."""
    probs = [assemble_problem(s, ctx) for s in MIXED_SPECS]
    sizes = sorted(K.nnz() * 8 for (_, K, _, _) in probs)
    threshold = sizes[len(sizes) // 2]
    solo = [K.nnz() * 8 >= threshold for (_, K, _, _) in probs]
    assert any(solo) and not all(solo)
    meth = [workloads.method(s) for s in MIXED_SPECS]
    assert any(m == "bicgstab" and o for m, o in zip(meth, solo)) or any(m == "cg" and o for m, o in zip(meth, solo))

    def run(idx, thr, late=None):
        B = yb.Batch(len(MIXED_SPECS), ctx)
        B.set_solo_bytes(thr)
        slots = {i: B.add(probs[i][1], probs[i][2], precision=precision, method=meth[i]) for i in idx}
        if late is not None:
            B.run(max_blocks=2)
            slots[late] = B.add(probs[late][1], probs[late][2], precision=precision, method=meth[late])
        assert B.run() == 0
        out = {}
        for i, s in slots.items():
            st = B.stats(s)
            assert st.status == 0 and st.rel_residual <= 1e-10, (MIXED_SPECS[i], st.status, st.rel_residual)
            out[i] = B.solution(s).numpy()
        return out

    everything = list(range(len(MIXED_SPECS)))
    own = run(everything, threshold)
    shared = run(everything, 0)
    for i in everything:
        spec, (mesh, K, b, dofs) = MIXED_SPECS[i], probs[i]
        assert oracle_relres(spec, mesh, dofs, b.numpy(), own[i]) <= 1e-10, spec
        assert np.linalg.norm(own[i] - shared[i]) <= 1e-6 * np.linalg.norm(shared[i]), spec
    first_solo = solo.index(True)
    alone = run([first_solo], threshold)
    assert np.array_equal(alone[first_solo], own[first_solo])
    late = max(i for i in everything if solo[i])
    rest = [i for i in everything if i != late]
    mixed_late = run(rest, threshold, late=late)
    assert np.array_equal(mixed_late[late], own[late])
