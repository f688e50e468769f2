"""yg_dot_static_scratch, the dot product that allocates nothing, against
yg_vector_dot on the same data and against an exactly rounded host sum
(math.fsum of the products): two calls in a row each agree within
1e-12 * sum|x_i y_i| (fixed-order FP64 sums that differ only in order).  Calls
go through the C ABI with device buffers that the test owns."""
import ctypes as C
import math

import numpy as np
import pytest
import torch

import yafel_b200 as yb
from yafel_b200._lib import YG_BAD_ARG, YG_OK, lib

pytestmark = pytest.mark.gpu

MAX_N = 8192 * 8192
TOL = 1e-12


def static_dot(x, y, n, out, stream):
    return lib().yg_dot_static_scratch(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), n,
                                       C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))


def vector_dot(a, b, ctx):
    va, vb = yb.DeviceVector(a, ctx), yb.DeviceVector(b, ctx)
    r = C.c_double()
    assert lib().yg_vector_dot(va.h, vb.h, C.byref(r)) == YG_OK
    return r.value


@pytest.mark.parametrize("n", [0, 1, 1000, 8192 * 3 + 5, 5_314_683])
def test_static_scratch_dot_matches_vector_dot(ctx, n):
    rng = np.random.Generator(np.random.PCG64(n + 11))
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    expect = vector_dot(a, b, ctx)
    exact = math.fsum(a * b)
    scale = float(np.abs(a * b).sum())
    assert abs(expect - exact) <= TOL * scale
    x = torch.from_numpy(a).to("cuda:0")
    y = torch.from_numpy(b).to("cuda:0")
    out = torch.full((2,), np.nan, dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream(0)
    assert static_dot(x, y, n, out[0:1], stream) == YG_OK
    assert static_dot(x, y, n, out[1:2], stream) == YG_OK
    torch.cuda.synchronize(0)
    got = out.cpu().numpy()
    for g in got:
        assert abs(g - expect) <= TOL * scale, (n, g, expect)
        assert abs(g - exact) <= TOL * scale, (n, g, exact)
    assert got[0] == got[1]


def test_static_scratch_dot_rejects_sizes_beyond_its_limit(ctx):
    x = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    # rejected on the host before anything is launched
    assert static_dot(x, x, MAX_N + 1, out, torch.cuda.current_stream(0)) == YG_BAD_ARG
    assert b"exceeds the static scratch limit" in lib().yg_last_error()
