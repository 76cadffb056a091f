"""Preconditioners applied with Jacobi iterations (mtlgpu_pc_set_jacobi_sweeps),
and the mixed-precision solves that use them, through the C ABI.

The apply is checked against the same polynomial evaluated in numpy on the
oracle's factors (the C restatement of ic_0 / ilu_0): relative error
<= 1e-12 (the device sums each row's products in its own order).  Solves are
checked on their FP64 true relative residual (<= the requested 1e-10); their
iteration counts are not the reference's (the preconditioner is an
approximation of the exact triangular solves)."""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import rel_err

pytestmark = pytest.mark.gpu


def split(F, diag):
    """(N, d): off-diagonal part and stored diagonal of a factor; diag is
    'last', 'first' or None (unit diagonal)."""
    n, rp, ci, v = F
    S = sp.csr_matrix((v, ci, rp), shape=(n, n))
    if diag is None:
        return S, np.ones(n)
    d = S.diagonal().copy()
    return (S - sp.diags(d)).tocsr(), d


def jacobi(N, d, v, k):
    w = d * v
    for _ in range(k):
        w = d * (v - N @ w)
    return w


def oracle_apply(restate, kind, A, r, k, as_float=False):
    if kind == "ic0":
        L, U = restate.ic0(A, as_float)
        (LN, Ld), (UN, Ud) = split(L, "last"), split(U, "first")
    else:
        L, U = restate.ilu0(A, as_float)
        (LN, Ld), (UN, Ud) = split(L, None), split(U, "first")
    if as_float:
        f = lambda a: a.astype(np.float32).astype(np.float64)  # noqa: E731
        LN.data, UN.data, Ld, Ud = f(LN.data), f(UN.data), f(Ld), f(Ud)
    return jacobi(UN, Ud, jacobi(LN, Ld, r, k), k)


CASES = [("ic0", lambda M: M.laplacian3d(20)), ("ic0", lambda M: M.fv2d(64)),
         ("ic0", lambda M: M.random_graph(3000, 16.0, 1e-2, 3)),
         ("ilu0", lambda M: M.convdiff27(12, 2)), ("ilu0", lambda M: M.laplacian2d(50, 70))]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("k", [1, 2, 3])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_jacobi_apply_matches_polynomial(M, ctx, restate, case, k, prec):
    kind, A_fn = CASES[case]
    A = A_fn(M)
    n = A[0]
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, kind, M.FP32 if prec == "fp32" else M.FP64)
    P.set_jacobi_sweeps(k)
    assert P.sweep_kind(M.LOWER) == 2
    r = M.uniform(n, 11)
    dr, dz = ctx.to_device(r), ctx.array(n)
    P.apply(dr, dz)
    ref = oracle_apply(restate, kind, A, r, k, as_float=(prec == "fp32"))
    assert rel_err(dz.download(), ref) <= 1e-12
    # back to the exact sweeps: the reference's solve(P, r)
    P.set_jacobi_sweeps(0)
    assert P.sweep_kind(M.LOWER) != 2
    P.apply(dr, dz)
    name = kind + "_float" if prec == "fp32" else kind
    assert rel_err(dz.download(), restate.pc_apply(name, A, r)) <= 1e-12


def test_jacobi_ic0_operator_is_symmetric(M, ctx):
    # P(L)^T P(L): u . (M^-1 v) == v . (M^-1 u)
    A = M.laplacian3d(16)
    n = A[0]
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, "ic0")
    P.set_jacobi_sweeps(3)
    u, v = M.uniform(n, 1), M.uniform(n, 2)
    du, dv, dz = ctx.to_device(u), ctx.to_device(v), ctx.array(n)
    P.apply(dv, dz)
    a = u @ dz.download()
    P.apply(du, dz)
    b = v @ dz.download()
    assert abs(a - b) <= 1e-12 * max(abs(a), 1.0)
    # IC(0)'s adjoint apply is the apply itself
    P.adjoint_apply(dv, dz)
    z1 = dz.download()
    P.apply(dv, dz)
    assert np.array_equal(z1, dz.download())


def test_jacobi_ilu0_adjoint_not_supported(M, ctx):
    A = M.convdiff27(6, 2)
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, "ilu0")
    P.set_jacobi_sweeps(2)
    dr, dz = ctx.to_device(np.ones(A[0])), ctx.array(A[0])
    with pytest.raises(M.MtlgpuError) as e:
        P.adjoint_apply(dr, dz)
    assert e.value.status == M.NOT_SUPPORTED
    with pytest.raises(M.MtlgpuError):
        P.set_jacobi_sweeps(-1)


def true_rel(M, A, x, b):
    return np.linalg.norm(b - M.csr_mult(A, x)) / np.linalg.norm(b)


@pytest.mark.parametrize("method,pc,A_fn", [
    ("cg", "ic0", lambda M: M.laplacian3d(32)),
    ("cg", "ic0", lambda M: M.fv2d(96)),
    ("bicgstab", "ilu0", lambda M: M.convdiff27(16, 2)),
])
@pytest.mark.parametrize("k", [1, 2])
def test_mixed_solve_with_jacobi_sweeps(M, ctx, method, pc, A_fn, k):
    A = A_fn(M)
    n = A[0]
    b = M.csr_mult(A, M.uniform(n, 1))
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, pc, M.FP32)
    P.set_jacobi_sweeps(k)
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    st, res, _ = M.solve(method, dA, P, dx, db, rtol=1e-10, max_iter=20000,
                         mode=M.SOLVE_MIXED, inner_rtol=1e-5)
    assert st == M.OK, (st, res.iterations, res.outer_iterations)
    assert true_rel(M, A, dx.download(), b) <= 1e-10
    assert res.true_resid <= 1e-10 * np.linalg.norm(b)


def test_fp64_solve_with_jacobi_sweeps(M, ctx):
    A = M.laplacian3d(32)
    n = A[0]
    b = M.csr_mult(A, M.uniform(n, 1))
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, "ic0")
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    st, exact, _ = M.solve("cg", dA, P, dx, db, rtol=1e-10, max_iter=2000)
    assert st == M.OK
    P.set_jacobi_sweeps(3)
    dx.upload(np.zeros(n))
    st, res, _ = M.solve("cg", dA, P, dx, db, rtol=1e-10, max_iter=2000)
    assert st == M.OK and true_rel(M, A, dx.download(), b) <= 3e-10
    # switching back re-records the solver graph with the exact sweeps
    P.set_jacobi_sweeps(0)
    dx.upload(np.zeros(n))
    st, again, _ = M.solve("cg", dA, P, dx, db, rtol=1e-10, max_iter=2000)
    assert st == M.OK and again.iterations == exact.iterations


def test_config2_mixed_jacobi_full_size(M, ctx):
    # 128^3 7-point Laplacian (x_true ~ U[-1,1] seed 1): FP32 inner PCG with
    # IC(0) applied by 2 Jacobi iterations per triangle, FP64 refinement to a
    # true relative residual of 1e-10
    A = M.laplacian3d(128)
    n = A[0]
    b = M.csr_mult(A, M.uniform(n, 1))
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, "ic0", M.FP32)
    P.set_jacobi_sweeps(2)
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    st, res, _ = M.solve("cg", dA, P, dx, db, rtol=1e-10, max_iter=4000, mode=M.SOLVE_MIXED,
                         inner_rtol=1e-5)
    assert st == M.OK
    assert true_rel(M, A, dx.download(), b) <= 1e-10
    assert res.outer_iterations >= 2


@pytest.mark.parametrize("method,prec,pc,k,A_fn", [
    ("cg", "fp32", "ic0", 1, lambda M: M.laplacian3d(40)),
    ("cg", "fp32", "ic0", 2, lambda M: M.fv2d(96)),
    ("cg", "fp32", "ilu0", 3, lambda M: M.laplacian2d(80, 60)),
    ("cg", "fp64", "ic0", 1, lambda M: M.laplacian3d(24)),
    ("cg", "fp64", "ic0", 2, lambda M: M.fv2d(80)),
    ("bicgstab", "fp32", "ilu0", 1, lambda M: M.convdiff27(20, 2)),
    ("bicgstab", "fp64", "ilu0", 2, lambda M: M.convdiff27(16, 2)),
])
def test_fused_cg_matches_five_kernel_recording(M, ctx, monkeypatch, method, prec, pc, k, A_fn):
    # CG with Jacobi-applied factors is recorded as three kernels per
    # iteration (x/r update fused into the first L pass, p update into the
    # product); BiCGSTAB's t = A shat carries omega's two dots.  Against the
    # unfused recording (MTLGPU_CG_FUSED=0, read when the solver's workspace
    # is made): the same arithmetic up to the blocking of the dot products
    # that moved, so the iteration counts agree to one,
    # both solutions meet the tolerance and agree to 1e-6 (the condition
    # number times the tolerance bounds their distance), and fewer kernels
    # run.
    A = A_fn(M)
    n = A[0]
    b = M.csr_mult(A, M.uniform(n, 1))
    out = {}
    for fused in (False, True):
        if not fused:
            monkeypatch.setenv("MTLGPU_CG_FUSED", "0")
        else:
            monkeypatch.delenv("MTLGPU_CG_FUSED")
        dA = M.Csr(ctx, *A[1:])
        P = M.Pc(dA, pc, M.FP32 if prec == "fp32" else M.FP64)
        P.set_jacobi_sweeps(k)
        dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
        kw = dict(mode=M.SOLVE_MIXED, inner_rtol=1e-5) if prec == "fp32" else {}
        st, res, _ = M.solve(method, dA, P, dx, db, rtol=1e-10, max_iter=20000, **kw)
        assert st == M.OK, (fused, st, res.iterations)
        x = dx.download()
        assert true_rel(M, A, x, b) <= (1e-10 if prec == "fp32" else 3e-10)
        out[fused] = (res.iterations, res.kernel_launches, x)
        P.close()
        dA.close()
    (i0, l0, x0), (i1, l1, x1) = out[False], out[True]
    assert abs(i0 - i1) <= 1, (i0, i1)
    assert l1 < l0, (l0, l1)
    assert rel_err(x1, x0) <= 1e-6
