"""Adjoint of the solve x = A^{-1} b on the device against an FP64 CPU adjoint.

The workload is the differentiable-solve one at a small size: the 2-D
finite-volume operator with a log-normal coefficient field, b a Gaussian
source, L = 1/2 ||x - x_target||^2 with x_target = x + 0.01 N(0,1).  The CPU
side runs the oracle's itl::cg + ic_0 twice (forward and adjoint) in FP64 and
forms -lambda_i x_j on A's pattern; the device side uses mtlgpu_solve for both
solves and mtlgpu_csr_values_grad.  (The finite-difference check of the same
gradients runs through the C++ linear_solve object in test_cpp_layer.py.)"""
import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


def bump(N):
    c = (np.arange(N) + 0.5) / N - 0.5
    X, Y = np.meshgrid(c, c, indexing="ij")
    return np.exp(-(X ** 2 + Y ** 2) / (2 * 0.1 ** 2)).ravel()


def test_values_grad_matches_cpu_adjoint(M, ctx, restate):
    N = 48
    A = M.fv2d(N, 1.0, 8.0, 4)
    n, rp, ci, v = A
    b = bump(N)
    dA = M.Csr(ctx, rp, ci, v)
    P = M.Pc(dA, "ic0")
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    st, res, _ = M.solve("cg", dA, P, dx, db, rtol=1e-13, max_iter=5000)
    assert st == M.OK
    x = dx.download()
    xt = x + 0.01 * M.normal(n, 44)
    dl = x - xt
    dlam, dg = ctx.to_device(np.zeros(n)), ctx.to_device(dl)
    st, res, _ = M.solve("cg", dA, P, dlam, dg, rtol=1e-13, max_iter=5000)
    assert st == M.OK
    grad = ctx.array(len(ci))
    dA.values_grad(dlam, dx, grad)
    g = grad.download()

    xc = restate.solve("cg", "ic0", A, b, rtol=1e-13, max_iter=5000)["x"]
    lc = restate.solve("cg", "ic0", A, xc - xt, rtol=1e-13, max_iter=5000)["x"]
    rows = np.repeat(np.arange(n), np.diff(rp))
    gc = -lc[rows] * xc[ci]
    assert rel_err(dlam.download(), lc) <= 1e-8
    assert rel_err(g, gc) <= 1e-8
    # exact identity on the pattern: the kernel forms -lambda_i x_j
    lam = dlam.download()
    assert np.array_equal(g, -(lam[rows] * x[ci]))


def test_transposed_adjoint_unsymmetric(M, ctx):
    # A^T lambda = g for the unsymmetric 27-point operator through the
    # transposed handle and BiCGSTAB + ILU(0) on it
    A = M.convdiff27(10, 2)
    n, rp, ci, v = A
    dA = M.Csr(ctx, rp, ci, v)
    dT = dA.transpose()
    P = M.Pc(dT, "ilu0")
    g = M.normal(n, 9)
    dlam, dg = ctx.to_device(np.zeros(n)), ctx.to_device(g)
    st, res, _ = M.solve("bicgstab", dT, P, dlam, dg, rtol=1e-12, max_iter=2000)
    assert st == M.OK
    lam = dlam.download()
    # A^T lambda on the host from A's own arrays
    rows = np.repeat(np.arange(n), np.diff(rp))
    atl = np.zeros(n)
    np.add.at(atl, ci, v * lam[rows])
    assert np.linalg.norm(atl - g) <= 3e-12 * np.linalg.norm(g)
