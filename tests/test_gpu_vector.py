"""Vector<double> operations on the device against FP64 host arithmetic.

dot (VectorExpression.hpp:33-54, operator* of two vectors) and the axpy update
y += a*x of the solvers (cg_solve.hpp:44-52) through yg_vector_dot and
yg_vector_axpy, compared with numpy and with the exactly rounded sum
math.fsum.  The device sum runs short sequential runs per thread, then trees
within warps and blocks, then a second pass over the block partials; the test's
bound, (log2 n + 16) eps sum|a_i b_i|, covers every one of those roundings.
"""
import math

import numpy as np
import pytest

import yafel_b200 as yb

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


@pytest.mark.parametrize("n", [0, 1, 7, 257, 100_003, (1 << 21) + 5])
def test_dot_matches_exact_sum(ctx, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n)
    b = rng.standard_normal(n) * np.exp(rng.uniform(-5, 5, n))
    A, B = yb.DeviceVector(a, ctx), yb.DeviceVector(b, ctx)
    got = A.dot(B)
    prods = a * b
    exact = math.fsum(prods.tolist()) if n else 0.0
    bound = (math.log2(max(n, 2)) + 16) * EPS * float(np.abs(prods).sum())
    assert abs(got - exact) <= bound, (got, exact, bound)
    assert abs(got - float(np.dot(a, b))) <= 2 * bound


def test_dot_is_deterministic_and_symmetric(ctx):
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal(300_001), rng.standard_normal(300_001)
    A, B = yb.DeviceVector(a, ctx), yb.DeviceVector(b, ctx)
    vals = {A.dot(B) for _ in range(20)} | {B.dot(A) for _ in range(20)}
    assert len(vals) == 1


def test_dot_size_mismatch_is_an_error(ctx):
    with pytest.raises(yb.YafelError):
        yb.DeviceVector(np.ones(5), ctx).dot(yb.DeviceVector(np.ones(6), ctx))


@pytest.mark.parametrize("n", [1, 1000, (1 << 20) + 3])
@pytest.mark.parametrize("alpha", [2.5, -1.0, 0.0, 1e-300])
def test_axpy_matches_host(ctx, n, alpha):
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    X, Y = yb.DeviceVector(x, ctx), yb.DeviceVector(y, ctx)
    Y.axpy(alpha, X)
    got = Y.numpy()
    # one rounding (fused multiply-add) or two (numpy): within one ulp of the larger term
    want = y + alpha * x
    scale = np.maximum(np.abs(alpha * x), np.abs(y))
    assert np.all(np.abs(got - want) <= 2 * EPS * scale)
    assert np.array_equal(X.numpy(), x)  # x untouched


def test_axpy_size_mismatch_is_an_error(ctx):
    with pytest.raises(yb.YafelError):
        yb.DeviceVector(np.ones(5), ctx).axpy(1.0, yb.DeviceVector(np.ones(6), ctx))
