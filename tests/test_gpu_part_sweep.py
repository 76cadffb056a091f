"""The partitioned triangular sweep (MTLGPU_SWEEP=part; chosen automatically
for factors with narrow levels) against the level-ordered ticket sweep
(MTLGPU_SWEEP=ticket) and the oracle: all three follow the
reference's per-row operation order (lower_trisolve.hpp:173-209,
upper_trisolve.hpp:160-176) with separately rounded operations, so their
results are bit-identical.  Also: a bounded wait that runs out inside the
partitioned sweep ends with MTLGPU_TIMEOUT and leaves the context usable."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def sweep_context(M, mode):
    old = os.environ.get("MTLGPU_SWEEP")
    os.environ["MTLGPU_SWEEP"] = mode
    try:
        return M.Context(0)
    finally:
        if old is None:
            del os.environ["MTLGPU_SWEEP"]
        else:
            os.environ["MTLGPU_SWEEP"] = old


def part_context(M):
    return sweep_context(M, "part")


@pytest.mark.parametrize("A_fn", [lambda M: M.laplacian2d(160, 160), lambda M: M.fv2d(128),
                                  lambda M: M.laplacian3d(32)])
@pytest.mark.parametrize("kind", ["ic0", "ilu0"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_part_sweep_bit_exact_with_default(M, restate, A_fn, kind, prec):
    A = A_fn(M)
    n = A[0]
    p = M.FP32 if prec == "fp32" else M.FP64
    dt = np.float32 if prec == "fp32" else np.float64
    pc = part_context(M)
    ctx = sweep_context(M, "ticket")
    try:
        dA0, dA1 = M.Csr(ctx, *A[1:]), M.Csr(pc, *A[1:])
        P0, P1 = M.Pc(dA0, kind, p), M.Pc(dA1, kind, p)
        for which in (M.LOWER, M.UPPER):
            assert P0.sweep_kind(which, p) == 0
            assert P1.sweep_kind(which, p) == 1
            r = M.uniform(n, 3 + which).astype(dt)
            a0, z0 = ctx.to_device(r), ctx.array(n, dt)
            a1, z1 = pc.to_device(r), pc.array(n, dt)
            P0.sweep(which, a0, z0)
            P1.sweep(which, a1, z1)
            assert np.array_equal(z0.download(), z1.download()), which
            if prec == "fp64":
                L, U = getattr(restate, kind)(A)
                name = {(M.LOWER, "ic0"): "lower_invdiag_last", (M.LOWER, "ilu0"): "lower_unit"}
                ref = restate.sweep(name.get((which, kind), "upper_invdiag_first"),
                                    L if which == M.LOWER else U, r)
                assert np.array_equal(z1.download(), ref), which
        P1.close()
        dA1.close()
        P0.close()
        dA0.close()
    finally:
        pc.close()
        ctx.close()


def test_automatic_sweep_choice(M, ctx):
    # narrow levels (2-D grid): partitioned; wide levels (3-D grid): ticket
    P2 = M.Pc(M.Csr(ctx, *M.laplacian2d(200, 200)[1:]), "ic0")
    assert P2.sweep_kind(M.LOWER) == 1 and P2.sweep_kind(M.UPPER) == 1
    P3 = M.Pc(M.Csr(ctx, *M.laplacian3d(64)[1:]), "ic0")
    assert P3.sweep_kind(M.LOWER) == 0
    # long factor rows (27-point ILU(0), 13 off-diagonal entries a row): ticket
    P4 = M.Pc(M.Csr(ctx, *M.convdiff27(48, 2)[1:]), "ilu0")
    assert P4.sweep_kind(M.LOWER) == 0 and P4.sweep_kind(M.UPPER) == 0


def test_part_sweep_timeout_leaves_context_usable(M, ctx):
    A = M.laplacian2d(160, 160)
    n = A[0]
    pc = part_context(M)
    try:
        dA = M.Csr(pc, *A[1:])
        P = M.Pc(dA, "ic0")
        assert P.sweep_kind(M.LOWER) == 1
        dr, dz = pc.to_device(np.ones(n)), pc.array(n)
        pc.set_spin_limit(1)
        statuses = []
        for _ in range(5):
            try:
                P.apply(dr, dz)
                statuses.append(M.OK)
            except M.MtlgpuError as e:
                statuses.append(e.status)
        assert M.TIMEOUT in statuses
        pc.set_spin_limit(1 << 22)
        P.apply(dr, dz)
        got = dz.download()
        tc = sweep_context(M, "ticket")
        dA0 = M.Csr(tc, *A[1:])
        P0 = M.Pc(dA0, "ic0")
        assert P0.sweep_kind(M.LOWER) == 0
        d0, z0 = tc.to_device(np.ones(n)), tc.array(n)
        P0.apply(d0, z0)
        assert np.array_equal(got, z0.download())
        P0.close()
        dA0.close()
        tc.close()
    finally:
        pc.close()


def test_spmv_needs_no_bounded_wait(M, restate):
    # the SpMV kernels never wait on another thread: with a spin limit of one
    # poll they still give the reference's products
    A = M.laplacian3d(48)
    n = A[0]
    c = M.Context(0)
    try:
        dA = M.Csr(c, *A[1:])
        x = M.uniform(n, 3)
        dx, dy = c.to_device(x), c.array(n)
        c.set_spin_limit(1)
        dA.spmv(dx, dy)
        c.synchronize()
        assert np.array_equal(dy.download(), restate.spmv(A, x))
    finally:
        c.close()
