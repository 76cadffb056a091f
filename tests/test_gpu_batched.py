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
