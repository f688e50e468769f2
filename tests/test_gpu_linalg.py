"""GPU parity of the sparse linear algebra (CUDA path through the C ABI) against
the oracle and the reference's own outputs."""
import os

import numpy as np
import pytest

import yafel_b200 as yb
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name))


def random_block_matrix(nb, B, per_row, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    rows, cols = [], []
    for i in range(nb):
        cs = np.unique(np.concatenate([[i], rng.integers(0, nb, per_row)]))
        rows.append(np.full(cs.size, i))
        cols.append(cs)
    brow = np.concatenate(rows)
    bcol = np.concatenate(cols)
    rp = np.concatenate([[0], np.cumsum([c.size for c in cols])]).astype(np.int64)
    val = rng.standard_normal(bcol.size * B * B)
    return rp, bcol.astype(np.int64), val


def bcsr_to_oracle_csr(rp, col, val, B):
    nb = rp.size - 1
    brow = np.repeat(np.arange(nb), np.diff(rp))
    i = np.arange(B)
    r = (brow[:, None, None] * B + i[None, :, None]).repeat(B, axis=2).ravel()
    c = (col[:, None, None] * B + i[None, None, :]).repeat(B, axis=1).ravel()
    return O.csr_from_triplets(r, c, val)


@pytest.mark.parametrize("B,per_row", [(1, 3), (1, 40), (2, 9), (3, 5), (3, 70)])
def test_spmv_matches_oracle(ctx, B, per_row):
    rp, col, val = random_block_matrix(3000, B, per_row, seed=B * 100 + per_row)
    A = yb.sparse_bcsr.from_bcsr(B, rp, col, val) if B > 1 else yb.sparse_csr.from_csr(rp, col, val)
    Ao = bcsr_to_oracle_csr(rp, col, val, B)
    x = np.random.Generator(np.random.PCG64(7)).standard_normal(A.cols())
    yo = Ao.spmv(x)
    scale = np.abs(val).max() * np.abs(x).max() * (per_row + 1) * B
    tma = [(2, L) for L in (32, 1, 2, 4, 8, 16)]
    tiles = [(3, L) for L in (1, 2, 4, 8)]
    rows = [(4, L) for L in (1, 2, 4, 8) if per_row < (128 if L <= 2 else 64)]
    variants = [(0, 4), (0, 32)] + ([(1, 32)] + tma + rows if B in (2, 3) else tiles) + [(-1, 32)]
    for v, L in variants:
        A.set_spmv(v, L)
        y = A * x
        assert np.abs(y - yo).max() <= 1e-14 * scale, (v, L)
        # determinism: same bits twice
        assert np.array_equal(y, A * x)
        if v == 3:
            # row tiles sum each row's rounded products left to right from 0, as the
            # oracle's csr_spmv loop does (built without contraction): same bits
            assert np.array_equal(y, yo), L
        if B in (2, 3) or v == 3:
            y32 = A.spmv(x, precision=yb.PREC_MIXED).numpy()
            yo32 = bcsr_to_oracle_csr(rp, col, val.astype(np.float32).astype(np.float64), B).spmv(x)
            assert np.abs(y32 - yo32).max() <= 1e-13 * np.abs(yo32).max(), (v, L)
            if v == 3:
                assert np.array_equal(y32, yo32), L


def test_csr_row_tiles_edge_cases(ctx):
    """Row tiles (SpMV variant 3): a row longer than a tile's capacity rules out
    that capacity only; an empty row rules the variant out; a one-row matrix and
    rows of one entry work; the autotuner skips what does not apply."""
    rng = np.random.Generator(np.random.PCG64(11))
    n = 700
    cols = [np.unique(np.concatenate([[i], rng.integers(0, n, 6)])) for i in range(n)]
    cols[5] = np.unique(np.concatenate([[5], rng.choice(n, 400, replace=False)]))  # 400+ entries
    rp = np.concatenate([[0], np.cumsum([c.size for c in cols])]).astype(np.int64)
    col = np.concatenate(cols).astype(np.int64)
    val = rng.standard_normal(col.size)
    A = yb.sparse_csr.from_csr(rp, col, val)
    x = rng.standard_normal(n)
    yo = O.Csr(n, n, rp, col, val).spmv(x)
    with pytest.raises(Exception):
        A.set_spmv(3, 4)  # capacity 256 < the long row
    for L in (1, 2, 8):  # capacities 512, 512, 1024
        A.set_spmv(3, L)
        assert np.array_equal(A * x, yo), L
    A.set_spmv(-1)
    assert np.abs(A * x - yo).max() <= 1e-13 * np.abs(yo).max()
    # an empty row
    rp2 = np.array([0, 2, 2, 3], dtype=np.int64)
    col2 = np.array([0, 2, 2], dtype=np.int64)
    val2 = np.array([1.0, 2.0, 3.0])
    A2 = yb.sparse_csr.from_csr(rp2, col2, val2)
    with pytest.raises(Exception):
        A2.set_spmv(3, 1)
    A2.set_spmv(-1)
    assert np.array_equal(A2 * np.array([1.0, 1.0, 1.0]), np.array([3.0, 0.0, 3.0]))
    # one row; rows of a single entry (diagonal)
    A3 = yb.sparse_csr.from_csr(np.array([0, 3]), np.array([0, 1, 2]), np.array([1.0, 2.0, 4.0]), ncols=3)
    A3.set_spmv(3, 2)
    assert np.array_equal(A3 * np.ones(3), np.array([7.0]))
    d = rng.standard_normal(5000)
    A4 = yb.sparse_csr.from_csr(np.arange(5001), np.arange(5000), d)
    for L in (1, 2, 4, 8):
        A4.set_spmv(3, L)
        assert np.array_equal(A4 * x[:1].repeat(5000), d * x[0]), L


def corrected_fp32_oracle(rp, col, val, B, x):
    """A32 x + C x_own: FP32-rounded values, plus per block row the FP64 sum of
    (A - fl32(A)) over its blocks times the row's own entries of x."""
    v32 = val.astype(np.float32).astype(np.float64)
    y = bcsr_to_oracle_csr(rp, col, v32, B).spmv(x)
    nb = rp.size - 1
    brow = np.repeat(np.arange(nb), np.diff(rp))
    C = np.zeros((nb, B, B))
    np.add.at(C, brow, (val - v32).reshape(-1, B, B))
    return y + np.einsum("rik,rk->ri", C, x.reshape(nb, B)).ravel()


@pytest.mark.parametrize("B,per_row", [(1, 30), (2, 9), (3, 40)])
def test_spmv_mixed_corrected(ctx, B, per_row):
    """The corrected FP32 operator of the mixed-precision solvers (FP32 values
    plus the FP64 row-sum correction) in every SpMV variant against the same
    operator in numpy; on a per-component constant x it reproduces the FP64
    product to FP64 rounding, where the plain FP32 values are off by about
    1e-8 of the scale."""
    rp, col, val = random_block_matrix(2500, B, per_row, seed=40 + B)
    A = yb.sparse_bcsr.from_bcsr(B, rp, col, val) if B > 1 else yb.sparse_csr.from_csr(rp, col, val)
    rng = np.random.Generator(np.random.PCG64(5))
    x = rng.standard_normal(A.cols())
    yo = corrected_fp32_oracle(rp, col, val, B, x)
    scale = np.abs(val).max() * np.abs(x).max() * (per_row + 1) * B
    xc = np.tile(np.arange(1.0, B + 1.0), A.cols() // B)
    y64c = bcsr_to_oracle_csr(rp, col, val, B).spmv(xc)
    variants = [(0, 8), (0, 32)] + ([(1, 32), (2, 4), (2, 8), (2, 32), (4, 1), (4, 2)] if B > 1 else [(3, 2)]) + [(-1, 32)]
    for v, L in variants:
        A.set_spmv(v, L)
        y = A.spmv(x, precision=yb.SPMV_MIXED_CORRECTED).numpy()
        assert np.abs(y - yo).max() <= 1e-14 * scale, (v, L)
        yc = A.spmv(xc, precision=yb.SPMV_MIXED_CORRECTED).numpy()
        assert np.abs(yc - y64c).max() <= 1e-14 * scale, (v, L)
    y32c = A.spmv(xc, precision=yb.PREC_MIXED).numpy()
    assert np.abs(y32c - y64c).max() > 1e-12 * scale  # the plain FP32 values are not exact there
    # a non-square matrix has no correction
    if B == 1:
        R = yb.sparse_csr.from_csr(np.array([0, 2, 3]), np.array([0, 2, 1]), np.array([1.0, 2.0, 3.0]), ncols=3)
        with pytest.raises(Exception):
            R.spmv(np.ones(3), precision=yb.SPMV_MIXED_CORRECTED)
    with pytest.raises(Exception):
        A.spmv(x, precision=7)


@pytest.mark.parametrize("B", [2, 3])
def test_whole_row_edge_cases(ctx, B):
    """Whole-row SpMV (variant 4): rows of 0 blocks (allowed), 1 block, exactly
    a stage's capacity (64 and 128 blocks), a row longer than a capacity (only
    the larger capacity remains), one row, fewer rows than warps; FP64 and FP32
    values, plain and corrected; the same bits from run to run."""
    rng = np.random.Generator(np.random.PCG64(70 + B))
    n = 1200
    lens = rng.integers(1, 60, n)
    lens[::89] = 0      # empty block rows
    lens[5::97] = 1
    lens[11] = 64
    lens[700] = 128     # longer than the 64-block stages
    cols = [np.sort(rng.choice(n, L, replace=False)) for L in lens]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    col = np.concatenate(cols).astype(np.int64)
    val = rng.standard_normal(col.size * B * B)
    A = yb.sparse_bcsr.from_bcsr(B, rp, col, val)
    x = rng.standard_normal(n * B)
    yo = bcsr_to_oracle_csr(rp, col, val, B).spmv(x)
    yo32 = bcsr_to_oracle_csr(rp, col, val.astype(np.float32).astype(np.float64), B).spmv(x)
    yoc = corrected_fp32_oracle(rp, col, val, B, x)
    scale = np.abs(val).max() * np.abs(x).max() * 129 * B
    for L in (4, 8):
        with pytest.raises(Exception):
            A.set_spmv(4, L)
    for L in (1, 2):
        A.set_spmv(4, L)
        y = A * x
        assert np.abs(y - yo).max() <= 1e-14 * scale, L
        assert np.array_equal(y, A * x), L
        assert np.all(y.reshape(-1, B)[lens == 0] == 0)
        y32 = A.spmv(x, precision=yb.PREC_MIXED).numpy()
        assert np.abs(y32 - yo32).max() <= 1e-14 * scale, L
        yc = A.spmv(x, precision=yb.SPMV_MIXED_CORRECTED).numpy()
        assert np.abs(yc - yoc).max() <= 1e-14 * scale, L
        assert np.array_equal(yc, A.spmv(x, precision=yb.SPMV_MIXED_CORRECTED).numpy()), L
    for nb in (1, 3, 31, 33, 700):
        rp3 = np.arange(nb + 1, dtype=np.int64)
        col3 = np.arange(nb, dtype=np.int64)
        v3 = rng.standard_normal(nb * B * B)
        A3 = yb.sparse_bcsr.from_bcsr(B, rp3, col3, v3)
        x3 = rng.standard_normal(nb * B)
        y3o = bcsr_to_oracle_csr(rp3, col3, v3, B).spmv(x3)
        for L in (1, 2, 4, 8):
            A3.set_spmv(4, L)
            assert np.abs(A3 * x3 - y3o).max() <= 1e-14 * np.abs(v3).max() * np.abs(x3).max() * B, (nb, L)


@pytest.mark.parametrize("lanes", [1, 2])
def test_whole_row_in_solvers(ctx, lanes):
    """The whole-row SpMV inside FP64 and mixed-precision Jacobi-PCG (fused p.Ap
    partial sums; FP32 values gathering the FP32 copy of the direction, with the
    row-sum correction) and inside BiCGSTAB (fused dot pairs) reaches the FP64
    true relative residual of 1e-10 and agrees with the warp-per-row kernel."""
    from yafel_b200 import meshgen
    dm = O.dofmanager(meshgen.structured_hex(5, 5, 5, order="ccw"), 2)
    K, _ = O.assemble(dm, 3, 3, O.ELASTICITY, [1.0, 0.5769230769230769, 0.3846153846153846])
    X = dm.nodes
    n = K.nrows
    b = np.random.Generator(np.random.PCG64(2)).standard_normal(n)
    mask = np.zeros(n, np.uint8)
    clamp = np.nonzero(X[:, 0] < 1e-9)[0]
    for c in range(3):
        mask[clamp * 3 + c] = 1
    O.dirichlet_apply(K, b, mask, np.zeros(n))
    Bm = O.bcsr_from_triplets(3, *O.csr_to_triplets(K))
    A = yb.sparse_bcsr.from_bcsr(3, Bm["brow_ptr"], Bm["bcol"], Bm["val"])
    M = yb.JacobiPreconditioner(A)
    A.set_spmv(2, 4)
    x2, s2 = yb.solve(A, b, M=M, tol=1e-10)
    A.set_spmv(4, lanes)
    for prec in (yb.PREC_FP64, yb.PREC_MIXED, yb.PREC_MIXED_IR):
        x4, s4 = yb.solve(A, b, M=M, tol=1e-10, precision=prec)
        assert s4.status == 0 and s4.rel_residual <= 1e-10, prec
        assert O.true_relres(K, b, x4.numpy()) <= 1e-10, prec
        assert np.linalg.norm(x4.numpy() - x2.numpy()) <= 1e-8 * np.linalg.norm(x2.numpy()), prec
    xb, sb = yb.solve(A, b, M=M, method="bicgstab", tol=1e-10)
    assert sb.status == 0 and O.true_relres(K, b, xb.numpy()) <= 1e-10


def test_spmv_choice_per_precision(ctx):
    """yg_matrix_set_spmv_for pins the kernel of one value precision and leaves
    the other alone; the autotuner is not a choice it takes; both kernels give
    the oracle's product."""
    rp, col, val = random_block_matrix(1500, 3, 20, seed=77)
    A = yb.sparse_bcsr.from_bcsr(3, rp, col, val)
    x = np.random.Generator(np.random.PCG64(8)).standard_normal(A.cols())
    A.set_spmv(0, 8)
    A.set_spmv_for(yb.PREC_MIXED, 4, 1)
    assert A.get_spmv(yb.PREC_FP64) == (0, 8) and A.get_spmv(yb.PREC_MIXED) == (4, 1)
    A.set_spmv_for(yb.PREC_FP64, 2, 4)
    assert A.get_spmv(yb.PREC_FP64) == (2, 4) and A.get_spmv(yb.PREC_MIXED) == (4, 1)
    with pytest.raises(Exception):
        A.set_spmv_for(yb.PREC_FP64, -1, 32)
    yo = bcsr_to_oracle_csr(rp, col, val, 3).spmv(x)
    assert np.abs(A * x - yo).max() <= 1e-13 * np.abs(yo).max()
    yo32 = bcsr_to_oracle_csr(rp, col, val.astype(np.float32).astype(np.float64), 3).spmv(x)
    assert np.abs(A.spmv(x, precision=yb.PREC_MIXED).numpy() - yo32).max() <= 1e-13 * np.abs(yo32).max()


@pytest.mark.parametrize("B", [1, 3])
def test_spmv_mixed_precision(ctx, B):
    rp, col, val = random_block_matrix(2000, B, 20, seed=3 + B)
    A = yb.sparse_bcsr.from_bcsr(B, rp, col, val) if B > 1 else yb.sparse_csr.from_csr(rp, col, val)
    x = np.random.Generator(np.random.PCG64(9)).standard_normal(A.cols())
    y32 = A.spmv(x, precision=yb.PREC_MIXED).numpy()
    Ao = bcsr_to_oracle_csr(rp, col, val.astype(np.float32).astype(np.float64), B)
    yo = Ao.spmv(x)
    assert np.abs(y32 - yo).max() <= 1e-13 * np.abs(yo).max()


def test_sparse_csr_from_triplets_matches_reference(ctx):
    g = gold("linalg.npz")
    for key in ("dup", "rand"):
        r, c, v = g[key + "_in"]
        A = yb.sparse_csr((r.astype(np.uint64), c.astype(np.uint64), v))
        rp, col, val = A.arrays()
        assert np.array_equal(rp, g[key + "_rp"])
        assert np.array_equal(col, g[key + "_col"])
        assert np.array_equal(val, g[key + "_val"])
    # test_sparse_csr.cpp test_1/test_3 sizes
    A = yb.sparse_csr([(9, 9, 1.0), (0, 0, 1.0)] * 10)
    assert A.rows() == 10 and A.cols() == 10 and A.nnz() == 2


def test_sparse_bcsr_from_triplets_matches_reference(ctx):
    g = gold("linalg.npz")
    ii, jj = np.meshgrid(np.arange(60), np.arange(60), indexing="ij")
    A = yb.sparse_bcsr(3, (ii.ravel().astype(np.uint64), jj.ravel().astype(np.uint64),
                           (ii * 60 + jj).ravel().astype(float)))
    rp, col, val = A.arrays()
    assert np.array_equal(rp, g["bcsr60_rp"]) and np.array_equal(col, g["bcsr60_col"])
    assert np.array_equal(val, g["bcsr60_val"])
    y = A * g["bcsr60_x"]
    assert np.allclose(y, g["bcsr60_y"], rtol=1e-14, atol=1e-10)
    # sparse_bcsr.hpp: rows rounded to whole blocks (test_sparse_bcsr.cpp test_2/test_3)
    B = yb.sparse_bcsr(3, [(59, 59, 1.0), (0, 0, 1.0)] * 60)
    assert B.rows() == 60 and B.cols() == 60
    rp, col, val = B.arrays()
    assert val[0] == 60.0 and val[-1] == 60.0


def test_cg_reference_tests(ctx):
    g = gold("linalg.npz")
    # test_cg_solve.cpp test_1: identity matrix returns the rhs exactly
    I = yb.sparse_csr((np.arange(10, dtype=np.uint64), np.arange(10, dtype=np.uint64), np.ones(10)))
    x = yb.cg_solve(I, g["ident_b"])
    assert np.array_equal(x, g["ident_b"])
    # test_2: tridiag(1,-2,1), ||x - x_ref||^2 < 1e-10
    r, c, v = g["lap_in"]
    A = yb.sparse_csr((r.astype(np.uint64), c.astype(np.uint64), v))
    x = yb.cg_solve(A, g["lap_b"])
    assert np.sum((x - np.arange(10)) ** 2) < 1e-10
    assert np.allclose(x, g["lap_cg"], rtol=1e-10, atol=1e-10)
    x = yb.bicgstab_solve(A, g["lap_b"])
    assert np.sum((x - np.arange(10)) ** 2) < 1e-10


def test_pcg_jacobi_ilu_match_reference_on_poisson(ctx):
    g = gold("poisson8.npz")
    A = yb.sparse_csr.from_csr(g["rp"], g["col"], g["val"])
    M = yb.JacobiPreconditioner(A)
    x = yb.pcg_solve(A, g["b"], M, np.zeros(A.rows()), 1e-20)
    assert np.abs(x - g["pcg_jacobi"]).max() <= 1e-12 * np.abs(g["pcg_jacobi"]).max()
    x = yb.cg_solve(A, g["b"], np.zeros(A.rows()), 1e-20)
    assert np.abs(x - g["cg"]).max() <= 1e-12 * np.abs(g["cg"]).max()
    L = yb.ILUPreconditioner(A)
    x = yb.pcg_solve(A, g["b"], L, np.zeros(A.rows()), 1e-20)
    assert np.abs(x - g["pcg_ilu"]).max() <= 1e-12 * np.abs(g["pcg_ilu"]).max()


def test_ilu_apply_matches_reference(ctx):
    g = gold("linalg.npz")
    r, c, v = g["ilu5_in"]
    A = yb.sparse_csr((r.astype(np.uint64), c.astype(np.uint64), v))
    L = yb.ILUPreconditioner(A)
    z = g["ilu5_z"].copy()
    L.solve(z)
    assert np.allclose(z, g["ilu5_apply"], rtol=1e-13, atol=1e-14)
    assert L.zero_pivots == 0
    # dependency levels of the sweeps: at least 1, at most one per row; none for Jacobi
    lo, up = L.levels
    assert 1 <= lo <= A.rows() and 1 <= up <= A.rows()
    assert yb.JacobiPreconditioner(A).levels == (0, 0)
    # a diagonal matrix: every row is independent, one level each way
    D = yb.sparse_csr([(i, i, 1.0 + i) for i in range(7)])
    assert yb.ILUPreconditioner(D).levels == (1, 1)
    # a bidiagonal (lower) chain: each row waits for the previous one
    Lc = yb.sparse_csr([(i, i, 2.0) for i in range(6)] + [(i + 1, i, 1.0) for i in range(5)])
    assert yb.ILUPreconditioner(Lc).levels[0] == 6


def test_jacobi_zero_diagonal_gives_inf_like_reference(ctx):
    A = yb.sparse_csr([(0, 0, 2.0), (1, 1, 0.0), (0, 1, 1.0)])
    M = yb.JacobiPreconditioner(A)
    assert M.zero_pivots == 1
    z = np.array([1.0, 1.0])
    M.solve(z)
    assert z[0] == 0.5 and np.isinf(z[1])


@pytest.mark.parametrize("precond", [None, "jacobi", "ilu"])
def test_relres_solve_reaches_1e10_and_matches_oracle(ctx, precond):
    from yafel_b200 import meshgen
    dm = O.dofmanager(meshgen.structured_quad(24, 24, order="tensor"), 1)
    K, R = O.assemble(dm, 1, 2, O.POISSON, [1.0, 1.0])
    X = dm.nodes
    mask = ((X[:, 0] < 1e-9) | (X[:, 0] > 1 - 1e-9) | (X[:, 1] < 1e-9) | (X[:, 1] > 1 - 1e-9)).astype(np.uint8)
    O.dirichlet_apply(K, R, mask, np.zeros(K.nrows))
    A = yb.sparse_csr.from_csr(K.row_ptr, K.col, K.val)
    M = None if precond is None else (yb.JacobiPreconditioner(A) if precond == "jacobi" else yb.ILUPreconditioner(A))
    x, st = yb.solve(A, R, M=M, tol=1e-10)
    assert st.status == 0 and st.rel_residual <= 1e-10
    xs = x.numpy()
    assert O.true_relres(K, R, xs) <= 1e-10
    xo, _, _ = O.cg(K, R, precond={None: 0, "jacobi": 1, "ilu": 2}[precond], tol=1e-12)
    assert np.linalg.norm(xs - xo) <= 1e-8 * np.linalg.norm(xo)


def test_mixed_precision_refinement_reaches_1e10(ctx):
    from yafel_b200 import meshgen
    dm = O.dofmanager(meshgen.structured_hex(6, 6, 6, order="ccw"), 2)
    K, _ = O.assemble(dm, 3, 3, O.ELASTICITY, [1.0, 0.5769230769230769, 0.3846153846153846])
    X = dm.nodes
    n = K.nrows
    rng = np.random.Generator(np.random.PCG64(1))
    b = rng.standard_normal(n)
    mask = np.zeros(n, np.uint8)
    clamp = np.nonzero(X[:, 0] < 1e-9)[0]
    for c in range(3):
        mask[clamp * 3 + c] = 1
    O.dirichlet_apply(K, b, mask, np.zeros(n))
    Bm = O.bcsr_from_triplets(3, *O.csr_to_triplets(K))
    A = yb.sparse_bcsr.from_bcsr(3, Bm["brow_ptr"], Bm["bcol"], Bm["val"])
    M = yb.JacobiPreconditioner(A)
    x64, s64 = yb.solve(A, b, M=M, tol=1e-10)
    xmx, smx = yb.solve(A, b, M=M, tol=1e-10, precision=yb.PREC_MIXED)
    assert s64.status == 0 and smx.status == 0
    assert s64.rel_residual <= 1e-10 and smx.rel_residual <= 1e-10
    assert O.true_relres(K, b, xmx.numpy()) <= 1e-10
    assert smx.refinements >= 1


def test_bicgstab_relres_nonsymmetric(ctx):
    from yafel_b200 import meshgen
    dm = O.dofmanager(meshgen.structured_quad(20, 20, order="tensor"), 1)
    K, R = O.assemble(dm, 1, 2, O.SUPG, [0.01, 0.05, 1.0, 0.0])
    X = dm.nodes
    b = np.sin(3 * X[:, 0]) + X[:, 1]
    mask = ((X[:, 0] < 1e-9) | (X[:, 1] < 1e-9) | (X[:, 1] > 1 - 1e-9)).astype(np.uint8)
    O.dirichlet_apply(K, b, mask, np.zeros(K.nrows))
    A = yb.sparse_csr.from_csr(K.row_ptr, K.col, K.val)
    for M in (None, yb.JacobiPreconditioner(A)):
        x, st = yb.solve(A, b, M=M, method="bicgstab", tol=1e-10)
        assert st.status == 0 and st.rel_residual <= 1e-10
        assert O.true_relres(K, b, x.numpy()) <= 1e-10
