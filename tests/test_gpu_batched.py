"""Batched PCG (mtlgpu_solve_batched) against the oracle, system by system.

The workload is the batched one at small sizes: random-graph Laplacians of
log-uniform size with a diagonal shift, b ~ N(0,1).  Each system of the batch
must match the oracle's own itl::cg run on that system alone: iteration count
within +-2, final true relative residual at the tolerance (<= 3x, as for the
single-system solves), and the solution close to the oracle's."""
import numpy as np
import pytest

from helpers import rel_err


def test_batch_assembly_is_block_diagonal(M):
    systems, (n, rp, ci, v, off) = M.graph_batch(5, 100, 1500, seed=7)
    assert off[0] == 0 and off[-1] == n == sum(s[0] for s in systems)
    for s, (ns, srp, sci, sv) in enumerate(systems):
        a, b = off[s], off[s + 1]
        assert np.array_equal(rp[a:b + 1] - rp[a], srp)
        assert np.array_equal(ci[rp[a]:rp[b]] - a, sci)
        assert ci[rp[a]:rp[b]].min() >= a and ci[rp[a]:rp[b]].max() < b


@pytest.mark.gpu
@pytest.mark.parametrize("pc", ["identity", "diagonal", "ic0"])
def test_batched_cg_matches_each_system(M, ctx, restate, pc):
    systems, (n, rp, ci, v, off) = M.graph_batch(12, 100, 2000, 8.0, 32.0, 1e-2, seed=3)
    b = M.normal(n, 5)
    dA = M.Csr(ctx, rp, ci, v)
    P = None if pc == "identity" else M.Pc(dA, pc)
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    st, res = M.solve_batched(dA, P, off, dx, db, rtol=1e-8, max_iter=2000)
    assert st == M.OK
    x = dx.download()
    for s, A_s in enumerate(systems):
        a, e = off[s], off[s + 1]
        ref = restate.solve("cg", pc, A_s, b[a:e], rtol=1e-8, max_iter=2000)
        assert res[s].error == 0 and ref["err"] == 0
        assert abs(res[s].iterations - ref["iterations"]) <= 2, (s, res[s].iterations,
                                                                ref["iterations"])
        tr = np.linalg.norm(b[a:e] - M.csr_mult(A_s, x[a:e])) / np.linalg.norm(b[a:e])
        assert tr <= 3e-8, (s, tr)
        assert abs(res[s].true_resid / np.linalg.norm(b[a:e]) - tr) <= 1e-9
        assert rel_err(x[a:e], ref["x"]) <= 1e-6


@pytest.mark.gpu
def test_batched_max_iter_and_arguments(M, ctx):
    systems, (n, rp, ci, v, off) = M.graph_batch(4, 200, 800, seed=11)
    dA = M.Csr(ctx, rp, ci, v)
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(M.normal(n, 1))
    st, res = M.solve_batched(dA, None, off, dx, db, rtol=1e-14, max_iter=3)
    assert st == M.MAX_ITER and all(r.error == 1 and r.iterations == 3 for r in res)
    # offsets that do not cover the matrix, or a block boundary crossed by an entry
    st, _ = M.solve_batched(dA, None, off[:-1], dx, db)
    assert st == M.INCOMPATIBLE_SIZE
    bad = off.copy()
    bad[1] += 1
    st, _ = M.solve_batched(dA, None, bad, dx, db)
    assert st == M.INVALID_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("pc", ["diagonal", "ic0"])
def test_batched_mixed_refinement_reaches_fp64_tolerance(M, ctx, pc):
    # FP32 inner batched PCG, FP64 refinement per system, to 1e-8 true residual
    systems, (n, rp, ci, v, off) = M.graph_batch(10, 200, 3000, 8.0, 32.0, 1e-2, seed=5)
    b = M.normal(n, 6)
    dA = M.Csr(ctx, rp, ci, v)
    P = M.Pc(dA, pc, M.FP32)
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    st, res = M.solve_batched(dA, P, off, dx, db, rtol=1e-8, max_iter=4000, mode=M.SOLVE_MIXED)
    assert st == M.OK
    x = dx.download()
    for s, A_s in enumerate(systems):
        a, e = off[s], off[s + 1]
        tr = np.linalg.norm(b[a:e] - M.csr_mult(A_s, x[a:e])) / np.linalg.norm(b[a:e])
        assert res[s].error == 0 and res[s].outer_iterations >= 1
        assert tr <= 1e-8, (s, tr)
        assert abs(res[s].true_resid / np.linalg.norm(b[a:e]) - tr) <= 1e-10


def _batch_env(shape):
    import os
    old = os.environ.get("MTLGPU_BATCH_SHAPE")
    os.environ["MTLGPU_BATCH_SHAPE"] = shape
    return old


def _restore(old):
    import os
    if old is None:
        os.environ.pop("MTLGPU_BATCH_SHAPE", None)
    else:
        os.environ["MTLGPU_BATCH_SHAPE"] = old


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["1,8", "2,4", "4,16", "8,32", "8,8,0", "4,8,1500",
                                   "8,16,100000", "4,1", "8,1,0", "2,1,1500", "1,1"])
def test_batched_cluster_shapes_match_each_system(M, ctx, restate, shape):
    # every (CTAs per system, lanes per row, rows below which one CTA solves
    # a system) shape of the persistent launch gives each system the
    # reference's iteration count
    systems, (n, rp, ci, v, off) = M.graph_batch(9, 100, 3000, 8.0, 32.0, 1e-2, seed=9)
    b = M.normal(n, 2)
    dA = M.Csr(ctx, rp, ci, v)
    P = M.Pc(dA, "diagonal")
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    old = _batch_env(shape)
    try:
        st, res = M.solve_batched(dA, P, off, dx, db, rtol=1e-8, max_iter=2000)
    finally:
        _restore(old)
    assert st == M.OK
    x = dx.download()
    for s, A_s in enumerate(systems):
        a, e = off[s], off[s + 1]
        ref = restate.solve("cg", "diagonal", A_s, b[a:e], rtol=1e-8, max_iter=2000)
        assert abs(res[s].iterations - ref["iterations"]) <= 2, (s, res[s].iterations,
                                                                ref["iterations"])
        tr = np.linalg.norm(b[a:e] - M.csr_mult(A_s, x[a:e])) / np.linalg.norm(b[a:e])
        assert tr <= 3e-8 and rel_err(x[a:e], ref["x"]) <= 1e-6
        assert res[s].kernel_launches == 1


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("pc", ["ic0", "ilu0"])
def test_batched_jacobi_applied_factors(M, ctx, mode, pc):
    # factors applied by Jacobi iterations: the persistent launch, FP64 or FP32
    # inner solves with FP64 refinement; each system reaches 1e-8 (true residual)
    systems, (n, rp, ci, v, off) = M.graph_batch(10, 200, 4000, 8.0, 32.0, 1e-2, seed=4)
    b = M.normal(n, 3)
    dA = M.Csr(ctx, rp, ci, v)
    P = M.Pc(dA, pc, M.FP32 if mode == "mixed" else M.FP64)
    P.set_jacobi_sweeps(2)
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    kw = dict(rtol=1e-8, max_iter=4000)
    if mode == "mixed":
        kw["mode"] = M.SOLVE_MIXED
    st, res = M.solve_batched(dA, P, off, dx, db, **kw)
    assert st == M.OK
    x = dx.download()
    for s, A_s in enumerate(systems):
        a, e = off[s], off[s + 1]
        tr = np.linalg.norm(b[a:e] - M.csr_mult(A_s, x[a:e])) / np.linalg.norm(b[a:e])
        assert res[s].error == 0 and tr <= (1e-8 if mode == "mixed" else 3e-8), (s, tr)


@pytest.mark.gpu
def test_batched_autotune(M, ctx, restate):
    systems, (n, rp, ci, v, off) = M.graph_batch(12, 500, 6000, 8.0, 32.0, 1e-2, seed=6)
    b = M.normal(n, 4)
    dA = M.Csr(ctx, rp, ci, v)
    P = M.Pc(dA, "diagonal")
    x0 = M.uniform(n, 8)
    dx, db = ctx.to_device(x0), ctx.to_device(b)
    choice = M.batched_autotune(dA, P, off, dx, db, rtol=1e-8, max_iter=2000)
    assert choice // 1000 in (0, 8192, 32768)
    # lanes per row 1: the CSR-stream SpMV shape
    assert (choice % 1000) // 100 in (4, 8) and choice % 100 in (1, 4, 8, 16)
    assert np.array_equal(dx.download(), x0)      # the caller's x is not touched
    dx.upload(np.zeros(n))
    st, res = M.solve_batched(dA, P, off, dx, db, rtol=1e-8, max_iter=2000)
    assert st == M.OK
    for s, A_s in enumerate(systems):
        a, e = off[s], off[s + 1]
        ref = restate.solve("cg", "diagonal", A_s, b[a:e], rtol=1e-8, max_iter=2000)
        assert abs(res[s].iterations - ref["iterations"]) <= 2


@pytest.mark.gpu
@pytest.mark.parametrize("A_fn", [lambda M: M.laplacian3d(40), lambda M: M.random_graph(20000, 20.0, 1e-2, 2)])
def test_spmv_autotune_keeps_results(M, ctx, restate, A_fn):
    A = A_fn(M)
    dA = M.Csr(ctx, *A[1:])
    choice = dA.autotune()
    assert choice in (0, 2)
    x = M.uniform(A[0], 3)
    dx, dy = ctx.to_device(x), ctx.array(A[0])
    dA.spmv(dx, dy)
    assert np.array_equal(dy.download(), restate.spmv(A, x))
