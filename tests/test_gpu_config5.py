"""Config 5 at its stated size: the differentiable solve on the 512 x 512
finite-volume operator (n = 262,144, nnz = 1,308,672; log-normal kappa,
sigma 1, 8-cell correlation, seed 4), b the Gaussian source, L = 1/2
||x - x_target||^2 with x_target = x + 0.01 N(0,1) (seed 44).

The device computes x = A^{-1} b and the adjoint lambda = A^{-T} dL/dx
(mtlgpu_solve, PCG with IC(0), FP64, rtol 1e-13), dL/db = lambda and
dL/dvals = -lambda_i x_j on A's pattern (mtlgpu_csr_values_grad).  Checked:

* against the FP64 CPU adjoint of the MTL4 reference itself (tests/golden,
  make_golden.py --cfg5): projections on 64 seeded directions within 1e-8 of
  the gradient's norm, sampled entries within 1e-8 relative;
* against central finite differences with h = 1e-6 along 64 random unit
  directions in b and 64 in the stored values: each perturbed solve x(b +- h d)
  or x(A +- h E) is warm-started at x and iterated until its own residual has
  dropped 1e-10 (CG for b; BiCGSTAB for the values, A +- h E being
  unsymmetric), preconditioned by IC(0) of A applied with 2 Jacobi iterations
  per triangle.  L is quadratic in b, so the central difference has no
  truncation error there; the bar is 1e-5 of the gradient's norm per
  direction."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 512
H = 1e-6
DIRECTIONS = 64


def fv_source(N):
    c = (np.arange(N) + 0.5) / N - 0.5
    X, Y = np.meshgrid(c, c, indexing="ij")
    return np.exp(-(X ** 2 + Y ** 2) / (2 * 0.1 ** 2)).ravel()


@pytest.fixture(scope="module")
def cfg5(M, ctx):
    A = M.fv2d(N, 1.0, 8.0, 4)
    n, rp, ci, v = A
    assert n == 262144 and len(ci) == 1308672
    b = fv_source(N)
    dA = M.Csr(ctx, rp, ci, v)
    P = M.Pc(dA, "ic0")
    dx, db = ctx.to_device(np.zeros(n)), ctx.to_device(b)
    st, rf, _ = M.solve("cg", dA, P, dx, db, rtol=1e-13, max_iter=20000)
    assert st == M.OK
    x = dx.download()
    g = -0.01 * M.normal(n, 44)              # dL/dx at the solution
    dlam, dg = ctx.to_device(np.zeros(n)), ctx.to_device(g)
    st, ra, _ = M.solve("cg", dA, P, dlam, dg, rtol=1e-13, max_iter=20000)
    assert st == M.OK
    grad = ctx.array(len(ci))
    dA.values_grad(dlam, dx, grad)
    data = dict(A=A, b=b, x=x, lam=dlam.download(), G=grad.download(), x_target=x - g,
                iters=(rf.iterations, ra.iterations))
    yield data, dA, P
    P.close()
    dA.close()


def test_config5_gradients_match_reference_cpu_adjoint(M, golden, cfg5):
    data, _, _ = cfg5
    n, lam, G = data["A"][0], data["lam"], data["G"]
    nnz = len(G)
    nl, nG, nx = golden["cfg5_norms"]
    for m in range(DIRECTIONS):
        db = M.normal(n, 1000 + m)
        dv = M.normal(nnz, 2000 + m)
        assert abs(lam @ db - golden["cfg5_proj_b"][m]) <= 1e-8 * nl * np.linalg.norm(db), m
        assert abs(G @ dv - golden["cfg5_proj_vals"][m]) <= 1e-8 * nG * np.linalg.norm(dv), m
    ib, iv = golden["cfg5_idx_b"], golden["cfg5_idx_vals"]
    ref_l, ref_g = golden["cfg5_lambda_sample"], golden["cfg5_grad_vals_sample"]
    assert np.linalg.norm(lam[ib] - ref_l) <= 1e-8 * np.linalg.norm(ref_l)
    assert np.linalg.norm(G[iv] - ref_g) <= 1e-8 * np.linalg.norm(ref_g)
    assert np.linalg.norm(data["x"][ib] - golden["cfg5_x_sample"]) <= \
        1e-8 * np.linalg.norm(golden["cfg5_x_sample"])
    assert abs(np.linalg.norm(lam) - nl) <= 1e-8 * nl
    assert abs(np.linalg.norm(G) - nG) <= 1e-8 * nG


def _loss(x, x_target):
    r = x - x_target
    return 0.5 * (r @ r)


def test_config5_dL_db_central_differences(M, ctx, cfg5):
    data, dA, P = cfg5
    n, b, x, xt, lam = data["A"][0], data["b"], data["x"], data["x_target"], data["lam"]
    P.set_jacobi_sweeps(2)
    try:
        dx, db = ctx.array(n), ctx.array(n)
        fd, an = np.zeros(DIRECTIONS), np.zeros(DIRECTIONS)
        for m in range(DIRECTIONS):
            d = M.normal(n, 3000 + m)
            d /= np.linalg.norm(d)
            L = []
            for sgn in (1.0, -1.0):
                bp = b + sgn * H * d
                r0 = np.linalg.norm(bp - M.csr_mult(data["A"], x))
                dx.upload(x)
                db.upload(bp)
                st, res, _ = M.solve("cg", dA, P, dx, db, rtol=1e-10, norm_r0=r0, max_iter=20000)
                assert st == M.OK, (m, st)
                L.append(_loss(dx.download(), xt))
            fd[m] = (L[0] - L[1]) / (2 * H)
            an[m] = lam @ d
        assert np.max(np.abs(fd - an)) <= 1e-5 * np.linalg.norm(lam), np.max(np.abs(fd - an))
    finally:
        P.set_jacobi_sweeps(0)


def test_config5_dL_dvals_central_differences(M, ctx, cfg5):
    data, dA, P = cfg5
    A, b, x, xt, G = data["A"], data["b"], data["x"], data["x_target"], data["G"]
    n, rp, ci, v = A
    P.set_jacobi_sweeps(2)
    try:
        dx, db = ctx.array(n), ctx.to_device(b)
        fd, an = np.zeros(DIRECTIONS), np.zeros(DIRECTIONS)
        for m in range(DIRECTIONS):
            E = M.normal(len(ci), 4000 + m)
            E /= np.linalg.norm(E)
            L = []
            for sgn in (1.0, -1.0):
                vp = v + sgn * H * E
                dA.set_values(vp)
                r0 = np.linalg.norm(b - M.csr_mult((n, rp, ci, vp), x))
                dx.upload(x)
                st, res, _ = M.solve("bicgstab", dA, P, dx, db, rtol=1e-10, norm_r0=r0,
                                     max_iter=20000)
                assert st == M.OK, (m, st)
                L.append(_loss(dx.download(), xt))
            fd[m] = (L[0] - L[1]) / (2 * H)
            an[m] = G @ E
        assert np.max(np.abs(fd - an)) <= 1e-5 * np.linalg.norm(G), np.max(np.abs(fd - an))
    finally:
        dA.set_values(v)
        P.set_jacobi_sweeps(0)
