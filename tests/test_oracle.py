"""The CPU oracle pinned against the reference's own known-answer tests, and
the restatement pinned bit-for-bit against the reference compiled from its
unmodified headers.  CPU only."""
import numpy as np
import pytest

from helpers import csr_eq, dense, dense_ic0, dense_ilu0, from_dense, ilu_test_matrix


# --- known answers quoted from the reference's tests ------------------------

def test_ic0_float_solve_iota(restate):
    # libs/numeric/itl/test/ic_0_test.cpp:20-36: 3x3 grid, ic_0<M, float>,
    # y = solve(P, iota(9)), compared with 9 values, two_norm(y - yc) <= 1e-3
    yc = np.array([1.03194, 1.60198, 1.45357, 2.5258, 3.55386, 3.16, 2.91787, 4.09338, 3.81335])
    A = restate.laplacian_setup(3, 3)
    y = restate.pc_apply("ic0_float", A, np.arange(9.0))
    assert np.linalg.norm(y - yc) <= 1e-3


def test_matrix_vector_product_stencil(restate):
    # libs/numeric/mtl/test/matrix_vector_product_test.cpp:43-89 (5x5 grid, v = row 12)
    A = restate.laplacian_setup(5, 5)
    v = dense(A)[12].copy()
    w = restate.spmv(A, v)
    assert (w[12], w[13], w[14], w[15], w[17], w[18], w[22]) == (20, -8, 1, 0, -8, 2, 1)
    w = restate.spmv(A, v, w, mode=1)
    assert w[12] == 40 and w[18] == 4
    w = restate.spmv(A, v, w, mode=2)
    assert w[12] == 20 and w[18] == 2


def test_dot_285(restate):
    # libs/numeric/mtl/test/dot_test.cpp:21-45: u = v = 1..9 -> 285
    u = np.arange(1.0, 10.0)
    assert restate.dot(u, u) == 285.0


def test_laplacian_setup_structure(restate):
    # libs/numeric/mtl/test/laplacian_setup_test.cpp:27-44
    A = restate.laplacian_setup(4, 5)
    D = dense(A)
    assert D.shape == (20, 20)
    assert np.all(np.diag(D) == 4)
    assert D[0, 1] == -1 and D[0, 5] == -1 and D[6, 1] == -1 and D[4, 5] == 0
    assert np.array_equal(D, D.T)


def test_trisolve_5x5(restate):
    # libs/numeric/mtl/test/trisolve_test.cpp:21-62: upper matrix with
    # (0,0)=7 (1,1)=8 (1,3)=2 (1,4)=3 (2,2)=2 (3,3)=4 (4,4)=9, x = 1..5.  The
    # sweep restatements take the inverted diagonal (upper v3 / lower v6).
    Ud = np.zeros((5, 5))
    for (i, j, a) in [(0, 0, 7), (1, 1, 8), (1, 3, 2), (1, 4, 3), (2, 2, 2), (3, 3, 4), (4, 4, 9)]:
        Ud[i, j] = a
    x = np.arange(1.0, 6.0)
    b = Ud @ x
    inv = Ud.copy()
    np.fill_diagonal(inv, 1.0 / np.diag(Ud))
    assert np.allclose(restate.sweep("upper_invdiag_first", from_dense(inv), b), x, atol=1e-4)
    Ld = Ud.T.copy()
    invl = Ld.copy()
    np.fill_diagonal(invl, 1.0 / np.diag(Ld))
    assert np.allclose(restate.sweep("lower_invdiag_last", from_dense(invl), Ld @ x), x, atol=1e-4)


def test_ilu0_against_dense(restate):
    # libs/numeric/itl/test/ilu_0_test.cpp:31-118: glibc rand() 3x3 matrix;
    # L[2][1] and 1/U[2][2] against dense ILU(0), then solve round trips.
    D = ilu_test_matrix(3)
    A = from_dense(D)
    L, U = restate.ilu0(A)
    LU = dense_ilu0(D)
    Ld, Ud = dense(L), dense(U)
    assert abs(LU[2, 1] - Ld[2, 1]) <= 1e-3
    assert abs(LU[2, 2] - 1.0 / Ud[2, 2]) <= 1e-3
    x = np.full(3, 3.0)
    U_true = np.triu(Ud, 1) + np.diag(1.0 / np.diag(Ud))
    Px = (Ld + np.eye(3)) @ (U_true @ x)
    assert np.linalg.norm(restate.pc_apply("ilu0", A, Px) - x) <= 0.01
    PTx = ((Ld + np.eye(3)) @ U_true).T @ x
    assert np.linalg.norm(restate.pc_apply("ilu0", A, PTx, adjoint=True) - x) <= 0.01


def test_ic0_against_dense(restate):
    # libs/numeric/itl/test/ic_0_cg_test.cpp:17-40 (3x3 grid): U[2][3], 1/U[3][3]
    A = restate.laplacian_setup(3, 3)
    _, U = restate.ic0(A)
    Ud = dense(U)
    Uref = dense_ic0(dense(A))
    assert abs(Uref[2, 3] - Ud[2, 3]) <= 1e-3
    assert abs(Uref[3, 3] - 1.0 / Ud[3, 3]) <= 1e-3


def test_ilu0_bicgstab_factor(restate):
    # libs/numeric/itl/test/ilu_0_bicgstab_test.cpp:16-35: LU[3][2], 1/U[3][3]
    A = restate.laplacian_setup(3, 3)
    L, U = restate.ilu0(A)
    LU = dense_ilu0(dense(A))
    assert abs(LU[3, 2] - dense(L)[3, 2]) <= 1e-3
    assert abs(LU[3, 3] - 1.0 / dense(U)[3, 3]) <= 1e-3


def test_ilu0_cg_iterations(restate):
    # libs/numeric/itl/test/ilu_0_cg_test.cpp:18-34: <= 4 iterations (3x3 grid, 1e-6)
    A = restate.laplacian_setup(3, 3)
    b = restate.spmv(A, np.ones(9))
    r = restate.solve("cg", "ilu0", A, b, rtol=1e-6, max_iter=9)
    assert r["err"] == 0 and r["iterations"] <= 4


def test_absolute_termination(restate):
    # libs/numeric/itl/test/absolut_termination_criterion_test.cpp:17-42
    A = restate.laplacian_setup(4, 4)
    b = restate.spmv(A, np.ones(16))
    r = restate.solve("cg", "diagonal", A, b, rtol=0.0, atol=1e-6, max_iter=500)
    assert np.linalg.norm(b - restate.spmv(A, r["x"])) <= 1e-6


@pytest.mark.parametrize("method,pc,tol,maxit", [("cg", "identity", 1e-11, 100),
                                                 ("bicgstab", "diagonal", 1e-6, 500)])
def test_solver_tests_converge(restate, method, pc, tol, maxit):
    # cg_test.cpp:18-38, bicgstab_test.cpp:17-36 (10x10 grid)
    A = restate.laplacian_setup(10, 10)
    b = restate.spmv(A, np.ones(100))
    r = restate.solve(method, pc, A, b, rtol=tol, max_iter=maxit)
    assert r["err"] == 0


def test_max_iter_error_code(restate):
    # basic_iteration.hpp:43-48: error 1 "Too many iterations"
    A = restate.laplacian_setup(10, 10)
    b = restate.spmv(A, np.ones(100))
    r = restate.solve("cg", "identity", A, b, rtol=1e-14, max_iter=3)
    assert r["err"] == 1 and r["iterations"] == 3


# --- restatement == reference, bit for bit -----------------------------------

def _cases(M):
    A = M.laplacian2d(20, 17)
    n, rp, ci, v = A
    rows = np.repeat(np.arange(n), np.diff(rp))
    rng = np.random.default_rng(0)
    v2 = v.copy()
    off = ci != rows
    v2[off] *= rng.uniform(0.2, 1.8, off.sum())
    return [A, (n, rp, ci, v2), M.laplacian3d(6), M.convdiff27(4, 2), M.random_graph(80, 8.0),
            M.fv2d(9)]


def test_restatement_matches_reference_kernels(M, restate, reference):
    rng = np.random.default_rng(1)
    for A in _cases(M):
        n = A[0]
        x, y = rng.standard_normal(n), rng.standard_normal(n)
        for mode in range(3):
            assert np.array_equal(reference.spmv(A, x, y, mode), restate.spmv(A, x, y, mode))
        assert reference.dot(x, y) == restate.dot(x, y)
        assert reference.two_norm(x) == restate.two_norm(x)
        assert reference.unary_dot(x) == restate.unary_dot(x)
        for fl in (False, True):
            for which in ("ic0", "ilu0"):
                a = getattr(reference, which)(A, fl)
                b = getattr(restate, which)(A, fl)
                assert csr_eq(a[0], b[0]) and csr_eq(a[1], b[1]), (which, fl)
        for pc in range(6):
            for adj in (False, True):
                assert np.array_equal(reference.pc_apply(pc, A, x, adj),
                                      restate.pc_apply(pc, A, x, adj)), (pc, adj)


def test_restatement_matches_reference_solvers(M, restate, reference):
    for A in _cases(M):
        b = reference.spmv(A, M.uniform(A[0], 7))
        for method in ("cg", "bicgstab"):
            for pc in range(6):
                r1 = reference.solve(method, pc, A, b, rtol=1e-10, max_iter=300)
                r2 = restate.solve(method, pc, A, b, rtol=1e-10, max_iter=300)
                assert r1["err"] == r2["err"] and r1["iterations"] == r2["iterations"]
                assert np.array_equal(r1["x"], r2["x"]) and np.array_equal(r1["history"],
                                                                           r2["history"])


# --- the restatement against the committed golden vectors --------------------

def test_golden_config1(M, restate, golden):
    A = M.laplacian2d(100, 100)
    assert np.array_equal(restate.spmv(A, M.uniform(A[0], 0)), golden["cfg1_b"])
    r = restate.solve("cg", "ic0", A, golden["cfg1_b"], rtol=1e-10, max_iter=1000)
    assert [r["iterations"], r["err"]] == list(golden["cfg1_iters"])
    assert np.array_equal(r["history"], golden["cfg1_hist"])
    assert np.array_equal(r["x"], golden["cfg1_x"])
    L, U = restate.ic0(A)
    assert np.array_equal(L[3], golden["cfg1_ic0_L_v"]) and np.array_equal(U[3], golden["cfg1_ic0_U_v"])


def test_golden_factors_and_levels(M, restate, golden):
    A = M.laplacian3d(16)
    L, U = restate.ic0(A)
    for key, F in (("lap16_ic0_L", L), ("lap16_ic0_U", U)):
        assert csr_eq(F, (F[0], golden[key + "_rp"], golden[key + "_ci"], golden[key + "_v"]))
    assert np.array_equal(restate.levels(L, True)[0], golden["lap16_ic0_L_lev"])
    assert np.array_equal(restate.levels(U, False)[0], golden["lap16_ic0_U_lev"])
    # wavefront structure of the 7-point stencil: level = i + j + k
    i, j, k = np.unravel_index(np.arange(16 ** 3), (16, 16, 16))
    assert np.array_equal(golden["lap16_ic0_L_lev"], i + j + k)
    C = M.convdiff27(8, 2)
    L, U = restate.ilu0(C)
    for key, F in (("cd8_ilu0_L", L), ("cd8_ilu0_U", U)):
        assert csr_eq(F, (F[0], golden[key + "_rp"], golden[key + "_ci"], golden[key + "_v"]))
    G = M.random_graph(600, 12.0, 1e-2, 3)
    L, U = restate.ic0(G)
    assert np.array_equal(L[3], golden["rg_ic0_L_v"]) and np.array_equal(U[3], golden["rg_ic0_U_v"])


def test_ic0_as_written_differs_from_textbook(M, restate):
    # IC(0) as the reference writes it applies only diagonal updates
    # (itl/pc/ic_0.hpp:170-182); on a random-graph pattern with triangles the
    # textbook update of U(j,i) would change off-diagonal entries.
    G = M.random_graph(60, 10.0, 1e-2, 5)
    _, U = restate.ic0(G)
    Ud = dense(U)
    A = dense(G)
    offd = np.triu(Ud, 1)
    inv = np.diag(Ud)
    # every off-diagonal entry is the original a_ki times the row's inverse diagonal
    assert np.allclose(offd, np.triu(A, 1) * inv[:, None], rtol=0, atol=0)


def test_fixture_spmv_matches_reference_spmv(M, reference):
    # b = A x_true: the GPU arm of the benchmark forms it with the generator
    # library's CSR product, the reference arm with the reference's own SpMV;
    # both sum each row in column order, so the right-hand sides are identical
    for A in (M.laplacian3d(24), M.convdiff27(12, 2)):
        x = M.uniform(A[0], 1)
        assert np.array_equal(M.csr_mult(A, x), reference.spmv(A, x))
