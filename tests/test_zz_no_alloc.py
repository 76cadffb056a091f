"""mtlgpu_dot_noalloc: the dot product for callers that cannot allocate.

Callers whose device memory is owned by someone else (a host application's
pool, another runtime) cannot create the context that mtlgpu_dot needs; this
entry point computes the same product with scratch kept inside the library.
The test calls it through the C ABI twice in a row (the scratch keeps the
previous call's contents, so the second call checks that it starts clean)
and compares each result with mtlgpu_dot on the same vectors, within the
tolerance the other dot-product tests use (1e-13 relative).  It lives in a
file of its own, collected last, and passes both alone in a fresh process
and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_dot(M, ctx, dx, dy, dres):
    L = M.lib()
    L.mtlgpu_dot_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    st = L.mtlgpu_dot_noalloc(dx.n, dx.ptr, dy.ptr, dres.ptr, ctx.stream)
    assert st == M.OK, st
    ctx.synchronize()
    return float(dres.download()[0])


@pytest.mark.parametrize("n", [1, 9, 100003, 2097152])
def test_dot_noalloc_matches_dot(M, ctx, n):
    dres = ctx.array(1)
    for call, seeds in enumerate([(61, 62), (63, 64)]):
        x, y = M.uniform(n, seeds[0]), M.uniform(n, seeds[1])
        dx, dy = ctx.to_device(x), ctx.to_device(y)
        got = _noalloc_dot(M, ctx, dx, dy, dres)
        ref = ctx.dot(dx, dy)
        assert abs(got - ref) <= 1e-13 * max(1.0, abs(ref)), (call, got, ref)


def test_dot_noalloc_known_answer_and_arguments(M, ctx):
    u = ctx.to_device(np.arange(1.0, 10.0))     # dot_test.cpp: 1..9 -> 285
    dres = ctx.array(1)
    assert _noalloc_dot(M, ctx, u, u, dres) == 285.0
    assert _noalloc_dot(M, ctx, u, u, dres) == 285.0
    L = M.lib()
    assert L.mtlgpu_dot_noalloc(-1, u.ptr, u.ptr, dres.ptr, ctx.stream) == M.INVALID_ARG
    assert L.mtlgpu_dot_noalloc(9, u.ptr, u.ptr, None, ctx.stream) == M.INVALID_ARG
