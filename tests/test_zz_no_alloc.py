"""GPU test of the allocation-free inner product (lfx_dot_noalloc).

Callers that cannot allocate device memory where they need a dot product (a
pool owned by another runtime, a loop that must not synchronise) use
lfx_dot_noalloc, whose reduction scratch is a fixed array inside the library.
This checks it through the C ABI against the allocating entry point,
lfx_vec_dot, on two calls in a row (the second reuses the scratch the first
left behind): the header promises the same bits, and the parity tests'
relative tolerance is checked as well. An empty input gives 0.0, and an
oversized one is refused before any work is queued. The file is named to run
after the other tests.
"""
import numpy as np
import pytest

from lfric_core_b200 import lfx

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # the relative tolerance of the solver parity tests


def test_dot_noalloc_matches_vec_dot_on_two_calls(ctx):
    L = lfx.load_library()
    n = 3_000_017
    rng = np.random.default_rng(2024)
    X = lfx.FieldVector.from_array(ctx, rng.standard_normal(n))
    Y = lfx.FieldVector.from_array(ctx, rng.standard_normal(n))
    R = lfx.FieldVector(ctx, [1])
    R.set_scalar(0.0)
    results = []
    for call in range(2):
        if call == 1:
            Y.aypx(-0.75, X)  # different data for the second call
        want = Y.dot(X)
        rc = L.lfx_dot_noalloc(X.device_ptr(), Y.device_ptr(), n, R.device_ptr(), ctx.stream)
        assert rc == 0, L.lfx_noalloc_last_error().decode()
        ctx.synchronize()
        got = R.export_field()[0]
        assert abs(got - want) <= REL_TOL * abs(want), (call, got, want)
        assert np.float64(got).view(np.int64) == np.float64(want).view(np.int64), (call, got, want)
        results.append(float(got))
    assert results[0] != results[1]


def test_dot_noalloc_empty_input_gives_zero(ctx):
    L = lfx.load_library()
    X = lfx.FieldVector(ctx, [4])
    R = lfx.FieldVector(ctx, [1])
    R.set_scalar(7.0)
    rc = L.lfx_dot_noalloc(X.device_ptr(), X.device_ptr(), 0, R.device_ptr(), ctx.stream)
    assert rc == 0, L.lfx_noalloc_last_error().decode()
    ctx.synchronize()
    assert R.export_field()[0] == 0.0


def test_dot_noalloc_rejects_oversized_input(ctx):
    L = lfx.load_library()
    X = lfx.FieldVector(ctx, [16])
    R = lfx.FieldVector(ctx, [1])
    too_big = L.lfx_dot_noalloc_max_n() + 1
    rc = L.lfx_dot_noalloc(X.device_ptr(), X.device_ptr(), too_big, R.device_ptr(), ctx.stream)
    assert rc == 4
    assert b"exceeds the maximum" in L.lfx_noalloc_last_error()
