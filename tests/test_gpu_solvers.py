"""itl::cg / itl::bicgstab on the device against the reference.

Bar: FP64 iteration counts within +-2 of the reference's, final true
relative residual at the requested tolerance (a recurrence-residual solve may
drift above it by a small factor, tolerated here as <= 3x, as the reference's
own run shows the same drift), MIXED_REFINED reaching the tolerance in true
FP64 residual."""
import threading
import time

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


def true_rel(M, A, x, b):
    return np.linalg.norm(b - M.csr_mult(A, x)) / np.linalg.norm(b)


def run(M, ctx, A, b, method, kind, prec=None, x0=None, **kw):
    dA = M.Csr(ctx, *A[1:])
    P = None if kind is None else M.Pc(dA, kind, prec if prec is not None else M.FP64)
    dx = ctx.to_device(np.zeros(A[0]) if x0 is None else x0)
    db = ctx.to_device(b)
    st, res, hist = M.solve(method, dA, P, dx, db, **kw)
    return st, res, hist, dx.download()


def test_config1_cg_ic0_matches_golden(M, ctx, golden):
    A = M.laplacian2d(100, 100)
    b = golden["cfg1_b"]
    st, res, hist, x = run(M, ctx, A, b, "cg", "ic0", rtol=1e-10, max_iter=1000)
    ref_it, ref_err = golden["cfg1_iters"]
    assert st == M.OK and res.error == ref_err == 0
    assert abs(res.iterations - ref_it) <= 2
    assert true_rel(M, A, x, b) <= 3e-10
    assert rel_err(x, golden["cfg1_x"]) <= 1e-8
    # residual history follows the reference's (both are recurrence residuals)
    m = min(len(hist), len(golden["cfg1_hist"]))
    assert np.allclose(hist[:m], golden["cfg1_hist"][:m], rtol=1e-6)


@pytest.mark.parametrize("pc", ["identity", "diagonal", "ilu0"])
def test_config1_cg_other_pcs(M, ctx, golden, pc):
    A = M.laplacian2d(100, 100)
    b = golden["cfg1_b"]
    st, res, hist, x = run(M, ctx, A, b, "cg", pc, rtol=1e-10, max_iter=1000)
    assert st == M.OK
    assert abs(res.iterations - golden[f"cfg1_{pc}_iters"][0]) <= 2
    assert true_rel(M, A, x, b) <= 3e-10


def test_lap3d_16_pcg(M, ctx, golden):
    A = M.laplacian3d(16)
    st, res, hist, x = run(M, ctx, A, golden["lap16_b"], "cg", "ic0", rtol=1e-10, max_iter=2000)
    assert st == M.OK and abs(res.iterations - golden["lap16_iters"][0]) <= 2
    assert true_rel(M, A, x, golden["lap16_b"]) <= 3e-10


def test_convdiff_bicgstab_ilu0(M, ctx, golden):
    A = M.convdiff27(8, 2)
    b = golden["cd8_b"]
    st, res, hist, x = run(M, ctx, A, b, "bicgstab", "ilu0", rtol=1e-10, max_iter=1000)
    assert st == M.OK and abs(res.iterations - golden["cd8_iters"][0]) <= 2
    assert true_rel(M, A, x, b) <= 3e-10
    st, res, hist, x = run(M, ctx, A, b, "bicgstab", "diagonal", rtol=1e-10, max_iter=1000)
    assert st == M.OK and abs(res.iterations - golden["cd8_diag_iters"][0]) <= 2


@pytest.mark.parametrize("pc", ["ic0", "diagonal"])
def test_random_graph_cg(M, ctx, golden, pc):
    A = M.random_graph(600, 12.0, 1e-2, 3)
    st, res, hist, x = run(M, ctx, A, golden["rg_b"], "cg", pc, rtol=1e-8, max_iter=1000)
    assert st == M.OK and abs(res.iterations - golden[f"rg_{pc}_iters"][0]) <= 2


def test_fv2d_cg(M, ctx, golden):
    A = M.fv2d(32, 1.0, 8.0, 4)
    st, res, hist, x = run(M, ctx, A, golden["fv32_b"], "cg", "ic0", rtol=1e-10, max_iter=1000)
    assert st == M.OK and abs(res.iterations - golden["fv32_iters"][0]) <= 2


@pytest.mark.parametrize("method,pc", [("cg", "ic0"), ("cg", "ilu0"), ("cg", "identity"),
                                       ("bicgstab", "ilu0"), ("bicgstab", "diagonal")])
def test_against_reference_live(M, ctx, reference, method, pc):
    A = M.laplacian3d(10) if method == "cg" else M.convdiff27(7, 2)
    b = reference.spmv(A, M.uniform(A[0], 1))
    r = reference.solve(method, pc, A, b, rtol=1e-10, max_iter=1000)
    st, res, hist, x = run(M, ctx, A, b, method, pc, rtol=1e-10, max_iter=1000)
    assert st == M.OK and abs(res.iterations - r["iterations"]) <= 2


def test_small_known_answer_solvers(M, ctx):
    # ilu_0_cg_test.cpp:30-33: <= 4 iterations on the 3x3 grid, tol 1e-6
    A = M.laplacian2d(3, 3)
    b = M.csr_mult(A, np.ones(9))
    st, res, _, _ = run(M, ctx, A, b, "cg", "ilu0", rtol=1e-6, max_iter=9)
    assert st == M.OK and res.iterations <= 4
    # absolut_termination_criterion_test.cpp: ||b - A x|| <= 1e-6 with atol
    A = M.laplacian2d(4, 4)
    b = M.csr_mult(A, np.ones(16))
    st, res, _, x = run(M, ctx, A, b, "cg", "diagonal", rtol=0.0, atol=1e-6, max_iter=500)
    assert st == M.OK and np.linalg.norm(b - M.csr_mult(A, x)) <= 1e-6
    # cg_test.cpp / bicgstab_test.cpp converge
    A = M.laplacian2d(10, 10)
    b = M.csr_mult(A, np.ones(100))
    assert run(M, ctx, A, b, "cg", "identity", rtol=1e-11, max_iter=100)[0] == M.OK
    assert run(M, ctx, A, b, "bicgstab", "diagonal", rtol=1e-6, max_iter=500)[0] == M.OK


def test_max_iter_and_zero_rhs(M, ctx):
    A = M.laplacian2d(10, 10)
    b = M.csr_mult(A, np.ones(100))
    st, res, _, _ = run(M, ctx, A, b, "cg", "identity", rtol=1e-14, max_iter=3)
    assert st == M.MAX_ITER and res.error == 1 and res.iterations == 3
    # b = 0, x0 = 0: converged before the first iteration (norm_r0 = 0, atol 0)
    st, res, _, x = run(M, ctx, A, np.zeros(100), "cg", "ic0", rtol=1e-10, max_iter=10)
    assert st == M.OK and res.iterations == 0 and np.all(x == 0)


def test_warm_start(M, ctx, golden):
    A = M.laplacian2d(100, 100)
    b = golden["cfg1_b"]
    st, res, _, x = run(M, ctx, A, b, "cg", "ic0", rtol=1e-10, max_iter=1000)
    st2, res2, _, x2 = run(M, ctx, A, b, "cg", "ic0", x0=x, rtol=1e-10, max_iter=1000)
    assert st2 == M.OK and res2.iterations <= 2


def test_host_buffers(M, ctx, golden):
    A = M.laplacian2d(100, 100)
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, "ic0")
    x = np.zeros(A[0])
    st, res, x = M.solve_host("cg", dA, P, x, golden["cfg1_b"], rtol=1e-10, max_iter=1000)
    assert st == M.OK and rel_err(x, golden["cfg1_x"]) <= 1e-8


def test_breakdown(M, ctx):
    # rtilde . r == 0 at the first iteration: b orthogonal to itself is
    # impossible, so use a skew matrix where gamma = rtilde . A r = 0
    rp = np.array([0, 2, 4], np.int32)
    ci = np.array([0, 1, 0, 1], np.int32)
    v = np.array([0.0, 1.0, -1.0, 0.0])
    A = (2, rp, ci, v)
    st, res, _, _ = run(M, ctx, A, np.array([1.0, 1.0]), "bicgstab", None, rtol=1e-10, max_iter=10)
    assert st == M.BREAKDOWN


def test_interrupt_flag(M, ctx):
    # interrupted_cg_test.cpp:21-55: a host thread raises the flag mid-solve
    A = M.laplacian2d(300, 300)
    b = M.csr_mult(A, np.ones(A[0]))
    dA = M.Csr(ctx, *A[1:])
    dx, db = ctx.to_device(np.zeros(A[0])), ctx.to_device(b)
    flag = np.zeros(1, np.int32)
    t = threading.Timer(0.05, lambda: flag.__setitem__(0, 1))
    t.start()
    st, res, _ = M.solve("cg", dA, None, dx, db, rtol=0.0, atol=0.0, max_iter=100000,
                         interrupt=flag)
    t.join()
    assert st == M.INTERRUPTED and 0 < res.iterations < 100000


def test_timeout_is_reported_not_hung(M):
    # A bounded wait that runs out ends with MTLGPU_TIMEOUT and the context
    # stays usable: spin limit 1 makes any wait on a not-yet-final value give up.
    c = M.Context(0)
    try:
        A = M.laplacian3d(24)
        dA = M.Csr(c, *A[1:])
        c.set_spin_limit(1)
        try:
            P = M.Pc(dA, "ic0")
            dr, dz = c.to_device(np.ones(A[0])), c.array(A[0])
            statuses = []
            for _ in range(5):
                try:
                    P.apply(dr, dz)
                    statuses.append(M.OK)
                except M.MtlgpuError as e:
                    statuses.append(e.status)
        except M.MtlgpuError as e:
            statuses = [e.status]
        assert M.TIMEOUT in statuses
        c.set_spin_limit(1 << 22)
        P = M.Pc(dA, "ic0")
        dr, dz = c.to_device(np.ones(A[0])), c.array(A[0])
        P.apply(dr, dz)
        assert np.all(np.isfinite(dz.download()))
    finally:
        c.close()


@pytest.mark.parametrize("method,pc,A_fn", [
    ("cg", "ic0", lambda M: M.laplacian3d(24)),
    ("bicgstab", "ilu0", lambda M: M.convdiff27(12, 2)),
])
def test_mixed_refined_reaches_fp64_tolerance(M, ctx, method, pc, A_fn):
    A = A_fn(M)
    b = M.csr_mult(A, M.uniform(A[0], 1))
    st, res, _, x = run(M, ctx, A, b, method, pc, prec=M.FP32, rtol=1e-10, max_iter=5000,
                        mode=M.SOLVE_MIXED)
    assert st == M.OK, (st, res.iterations, res.outer_iterations, res.resid)
    assert true_rel(M, A, x, b) <= 1e-10
    assert res.outer_iterations >= 2


def test_config2_full_pcg_fp64_and_mixed(M, ctx, golden):
    # 128^3 7-point Laplacian, x_true ~ U[-1,1] seed 1, PCG-IC(0) to 1e-10
    A = M.laplacian3d(128)
    b = M.csr_mult(A, M.uniform(A[0], 1))
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, "ic0")
    dx, db = ctx.to_device(np.zeros(A[0])), ctx.to_device(b)
    st, res, hist = M.solve("cg", dA, P, dx, db, rtol=1e-10, max_iter=2000)
    assert st == M.OK and abs(res.iterations - golden["cfg2_iters"][0]) <= 2
    x = dx.download()
    assert true_rel(M, A, x, b) <= 3e-10
    P32 = M.Pc(dA, "ic0", M.FP32)
    dx.upload(np.zeros(A[0]))
    st, res, _ = M.solve("cg", dA, P32, dx, db, rtol=1e-10, max_iter=4000, mode=M.SOLVE_MIXED)
    assert st == M.OK and true_rel(M, A, dx.download(), b) <= 1e-10


@pytest.mark.parametrize("method,pc,A_fn,kw", [
    ("cg", "ic0", lambda M: M.laplacian3d(20), {}),
    ("bicgstab", "ilu0", lambda M: M.convdiff27(12, 2), {}),
    ("cg", "ic0", lambda M: M.laplacian3d(24), {"jacobi": 1}),
    ("cg", "identity", lambda M: M.laplacian2d(40, 40), {"max_iter": 37}),
])
def test_device_loop_matches_host_loop(M, ctx, method, pc, A_fn, kw):
    # Without an interrupt flag the iterations repeat in a device-side graph
    # loop; with one (held at 0) the host relaunches the graph and polls the
    # flag between launches.  Both run the same recorded kernels in the same
    # order: the same iterations, residual history and solution, bit for bit,
    # including a solve stopped by its iteration limit in mid-graph.
    A = A_fn(M)
    n = A[0]
    b = M.csr_mult(A, M.uniform(n, 1))
    dA = M.Csr(ctx, *A[1:])
    P = None if pc == "identity" else M.Pc(dA, pc)
    if kw.get("jacobi"):
        P.set_jacobi_sweeps(kw["jacobi"])
    max_iter = kw.get("max_iter", 2000)
    out = []
    for flag in (None, np.zeros(1, np.int32)):
        dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
        st, res, hist = M.solve(method, dA, P, dx, db, rtol=1e-10, max_iter=max_iter,
                                interrupt=flag)
        out.append((st, res.iterations, np.array(hist), dx.download()))
    (s0, i0, h0, x0), (s1, i1, h1, x1) = out
    assert s0 == s1 and i0 == i1
    assert np.array_equal(h0, h1) and np.array_equal(x0, x1)
    if "max_iter" in kw:
        assert s0 == M.MAX_ITER and i0 == max_iter
    else:
        assert s0 == M.OK


@pytest.mark.parametrize("method,pc", [("cg", "ic0"), ("bicgstab", "ilu0"), ("cg", None)])
@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("jacobi", [0, 1])
def test_empty_and_one_row_systems(M, ctx, method, pc, mixed, jacobi):
    # n = 0: ||b|| = 0, so basic_iteration converges before the first
    # iteration (basic_iteration.hpp:85-93), as the reference's solvers do on
    # an empty system.  n = 1: the 1 x 1 system 4 x = 8.
    if pc is None and jacobi:
        pytest.skip("Jacobi iterations apply factors")
    kw = dict(mode=M.SOLVE_MIXED, inner_rtol=1e-5) if mixed else {}
    prec = M.FP32 if mixed else M.FP64
    dA = M.Csr(ctx, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    P = M.Pc(dA, pc, prec) if pc else None
    if P and jacobi:
        P.set_jacobi_sweeps(jacobi)
    dx, db = ctx.array(0), ctx.array(0)
    st, res, _ = M.solve(method, dA, P, dx, db, rtol=1e-10, max_iter=10, **kw)
    assert st == M.OK and res.iterations == 0
    if P:
        P.close()
    dA.close()
    dA = M.Csr(ctx, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([4.0]))
    P = M.Pc(dA, pc, prec) if pc else None
    if P and jacobi:
        P.set_jacobi_sweeps(jacobi)
    dx, db = ctx.to_device(np.zeros(1)), ctx.to_device(np.array([8.0]))
    st, res, _ = M.solve(method, dA, P, dx, db, rtol=1e-10, max_iter=10, **kw)
    assert st == M.OK and abs(dx.download()[0] - 2.0) <= 1e-12
    if P:
        P.close()
    dA.close()
