"""The other ITL Krylov methods on the device (mtlgpu_solve_krylov, through the
C ABI) against the reference's runs (golden fixtures made by the reference
compiled from its headers): bicg, cgs, bicgstab_2, bicgstab_ell, tfqmr, qmr,
idr_s and gmres with left and right preconditioners.

Bars: the reference's error code; iteration count within +-2 (gmres: one
restart cycle); the solution within 1e-4 relative of the reference's for
converged runs (both stop somewhere below rtol 1e-8) and 1e-6 for runs the
iteration limit stops; the first residuals within 1e-6 relative.  Runs whose
course rounding alone changes (the numpy restatement parts from the
reference there too) are checked for a converged solve only, and gmres /
idr_s are also checked cut after a few cycles / steps, where the device
follows the reference to 1e-9."""
import numpy as np
import pytest

from golden_krylov import CASES, ROUNDING_SENSITIVE, STEP_CUTS, iter_tol, krylov_problem, \
    max_iter_of, param_of, x_tol
from helpers import rel_err

pytestmark = pytest.mark.gpu


def run(M, ctx, A, b, meth, pl, pr, param, max_iter, rtol=1e-8, x0=None):
    n = A[0]
    dA = M.Csr(ctx, *A[1:])
    L = M.Pc(dA, pl) if pl != "identity" else None
    R = M.Pc(dA, pr) if pr != "identity" else None
    dx = ctx.to_device(np.zeros(n) if x0 is None else x0)
    db = ctx.to_device(b)
    st, res, hist = M.solve_krylov(meth, dA, L, dx, db, R=R, param=param, max_iter=max_iter,
                                   rtol=rtol)
    return st, res, hist, dx.download()


@pytest.mark.parametrize("case", CASES, ids=["_".join(c) for c in CASES])
def test_krylov_matches_reference(M, ctx, golden, case):
    name, meth, pl, pr = case
    A, b = krylov_problem(M, golden, name)
    key = f"kry_{name}_{meth}_{pl}_{pr}"
    it_ref, err_ref = (int(v) for v in golden[key + "_iters"])
    st, res, hist, x = run(M, ctx, A, b, meth, pl, pr, param_of(meth), max_iter_of(meth))
    assert st in (M.OK, M.MAX_ITER, M.BREAKDOWN), st
    nb = np.linalg.norm(b)
    if case in ROUNDING_SENSITIVE:
        if res.error == 0:
            assert res.resid <= 1e-8 * res.norm_r0
        return
    assert res.error == err_ref, (res.error, err_ref, res.iterations, it_ref)
    assert abs(res.iterations - it_ref) <= iter_tol(meth, it_ref), (res.iterations, it_ref)
    assert rel_err(x, golden[key + "_x"]) <= x_tol(err_ref)
    # the true residual of the device's x is as small as that of the reference's
    xr = golden[key + "_x"]
    tr_ref = np.linalg.norm(b - M.csr_mult(A, xr))
    assert res.true_resid <= 10 * tr_ref + 1e-12 * nb, (res.true_resid, tr_ref)
    hr = golden[key + "_hist"]
    m = min(len(hist), len(hr), 8)
    if meth not in ("idr_s", "gmres"):
        assert np.allclose(hist[:m], hr[:m], rtol=1e-6, atol=0), (hist[:m], hr[:m])


@pytest.mark.parametrize("meth", ["gmres", "idr_s"])
def test_krylov_cut_runs(M, ctx, golden, meth):
    A, b = krylov_problem(M, golden, "cd6")
    for k in STEP_CUTS[meth]:
        st, res, _, x = run(M, ctx, A, b, meth, "identity", "identity", param_of(meth), k)
        ref = golden[f"kry_cut_{meth}_{k}_x"]
        assert res.iterations == int(golden[f"kry_cut_{meth}_{k}_resid"][1])
        assert rel_err(x, ref) <= 1e-9, (k, rel_err(x, ref))


@pytest.mark.parametrize("meth,param", [("cgs", 0), ("bicgstab_2", 0), ("bicgstab_ell", 4),
                                        ("tfqmr", 0), ("gmres", 30), ("idr_s", 2),
                                        ("bicg", 0), ("qmr", 0)])
def test_krylov_larger_unsymmetric(M, ctx, restate, meth, param):
    # 27-point convection-diffusion 24^3 (n = 13,824), ILU(0) on the left:
    # every method reaches rtol 1e-8 on its own residual, and the true residual
    # of the returned x is small
    A = M.convdiff27(24, 2)
    b = restate.spmv(A, M.uniform(A[0], 1))
    pl = "identity" if meth in ("bicg", "qmr", "idr_s") else "ilu0"
    st, res, _, x = run(M, ctx, A, b, meth, pl, "identity", param,
                        120 if meth == "qmr" else 2000)
    tr = np.linalg.norm(b - restate.spmv(A, x)) / np.linalg.norm(b)
    if meth == "qmr":  # runs to the limit (its test is on the Lanczos norm)
        assert st == M.MAX_ITER and tr <= 1e-8
    else:
        assert st == M.OK, (st, res.iterations)
        assert tr <= 1e-6, tr


def test_krylov_warm_start_and_right_pc_shift(M, ctx, golden):
    # bicgstab_ell and tfqmr with a nonzero initial guess and a right
    # preconditioner: the reference's shift (x0, solve(R, x)) at both ends
    import oracle
    ref = oracle.available_reference()
    if ref is None:
        pytest.skip("reference build not available")
    A = M.convdiff27(6, 2)
    b = golden["kry_cd6_b"]
    x0 = M.uniform(A[0], 9)
    for meth, pl, pr in (("bicgstab_ell", "ilu0", "diagonal"), ("tfqmr", "diagonal", "ilu0"),
                         ("qmr", "ic0", "diagonal")):
        r = ref.solve_krylov(meth, pl, A, b, pc_right=pr, param=param_of(meth), x0=x0,
                             max_iter=max_iter_of(meth), rtol=1e-8)
        st, res, _, x = run(M, ctx, A, b, meth, pl, pr, param_of(meth), max_iter_of(meth),
                            x0=x0)
        assert res.error == r["err"], meth
        assert abs(res.iterations - r["iterations"]) <= iter_tol(meth, r["iterations"]), meth
        assert rel_err(x, r["x"]) <= x_tol(r["err"]), meth
    # gmres from x0 with both preconditioners, cut after two restart cycles
    r = ref.solve_krylov("gmres", "ilu0", A, b, pc_right="diagonal", param=8, x0=x0,
                         max_iter=16, rtol=1e-8)
    st, res, _, x = run(M, ctx, A, b, "gmres", "ilu0", "diagonal", 8, 16, x0=x0)
    assert res.iterations == r["iterations"] == 16
    assert rel_err(x, r["x"]) <= 1e-9


def test_krylov_argument_errors(M, ctx):
    A = M.laplacian2d(6, 6)
    dA = M.Csr(ctx, *A[1:])
    dx, db = ctx.to_device(np.zeros(A[0])), ctx.to_device(np.ones(A[0]))
    st, _, _ = M.solve_krylov("idr_s", dA, None, dx, db, param=16)
    assert st == M.INVALID_ARG
    st, _, _ = M.solve_krylov("gmres", dA, None, dx, db, param=65)
    assert st == M.INVALID_ARG
    st, _, _ = M.solve_krylov("tfqmr", dA, None, dx, db, mode=M.SOLVE_MIXED)
    assert st == M.NOT_SUPPORTED
    B = M.Csr(ctx, *M.laplacian2d(6, 6)[1:])
    P = M.Pc(B, "diagonal")
    st, _, _ = M.solve_krylov("cgs", dA, P, dx, db)
    assert st == M.INVALID_ARG
    # max_iter 0: the reference's loops stop at once with error 1
    for meth in ("bicg", "cgs", "bicgstab_ell", "tfqmr", "qmr", "gmres"):
        st, res, _ = M.solve_krylov(meth, dA, None, dx, db, max_iter=0)
        assert st == M.MAX_ITER and res.error == 1 and res.iterations == 0, meth
    # the solver path still works after the rejected calls
    st, res, _ = M.solve_krylov("cgs", dA, None, dx, db)
    assert st == M.OK
