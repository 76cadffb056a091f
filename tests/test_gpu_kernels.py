"""GPU kernels against the oracle, through the C ABI.

Tolerances (stated per test): SpMV normwise relative error <= 1e-14 (FP64),
and bit-identical where every row is summed in the reference's order;
factor values, triangular sweeps and preconditioner applies bit-identical
(the device follows the reference's operation order with separate
roundings); level arrays bit-exact."""
import numpy as np
import pytest

from helpers import csr_eq, rel_err

pytestmark = pytest.mark.gpu


def matrices(M):
    return {
        "lap2d_100": M.laplacian2d(100, 100),
        "lap3d_20": M.laplacian3d(20),
        "cd27_10": M.convdiff27(10, 2),
        "graph_2000": M.random_graph(2000, 20.0, 1e-2, 3),
        "fv2d_64": M.fv2d(64),
    }


@pytest.mark.parametrize("name", ["lap2d_100", "lap3d_20", "cd27_10", "graph_2000", "fv2d_64"])
def test_spmv_modes(M, ctx, restate, name):
    A = matrices(M)[name]
    n = A[0]
    dA = M.Csr(ctx, *A[1:])
    x = M.uniform(n, 5)
    y0 = M.uniform(n, 6)
    dx, dy = ctx.to_device(x), ctx.to_device(y0)
    for mode, (alpha, beta) in enumerate([(1.0, 0.0), (1.0, 1.0), (-1.0, 1.0)]):
        dy.upload(y0)
        dA.spmv(dx, dy, alpha, beta)
        ref = restate.spmv(A, x, y0, mode)
        got = dy.download()
        assert rel_err(got, ref) <= 1e-14, (name, mode)
        # the CSR-stream kernel sums each row in the reference's order with
        # separately rounded products: the result is bit-identical
        assert np.array_equal(got, ref), (name, mode)


def test_spmv_stencil_known_answer(M, ctx):
    # matrix_vector_product_test.cpp:43-89 on the device
    A = M.laplacian2d(5, 5)
    n, rp, ci, v = A
    row12 = np.zeros(25)
    row12[ci[rp[12]:rp[13]]] = v[rp[12]:rp[13]]
    dA = M.Csr(ctx, rp, ci, v)
    dv, dw = ctx.to_device(row12), ctx.array(25)
    dA.spmv(dv, dw)
    w = dw.download()
    assert (w[12], w[13], w[14], w[15], w[17], w[18], w[22]) == (20, -8, 1, 0, -8, 2, 1)
    dA.spmv(dv, dw, 1.0, 1.0)
    w = dw.download()
    assert w[12] == 40 and w[18] == 4
    dA.spmv(dv, dw, -1.0, 1.0)
    w = dw.download()
    assert w[12] == 20 and w[18] == 2


def test_spmv_binned_rows(M, ctx, restate):
    # rows of very different lengths exercise the row bins, including a
    # CTA-per-row bin (rows longer than 1024 entries)
    rng = np.random.default_rng(3)
    n = 3000
    lens = rng.integers(0, 12, n)
    lens[::97] = rng.integers(40, 300, len(lens[::97]))
    lens[5] = 2500
    lens[1700] = 1400
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    v = rng.standard_normal(len(ci))
    A = (n, rp, ci, v)
    dA = M.Csr(ctx, rp, ci, v)
    x = rng.standard_normal(n)
    dx, dy = ctx.to_device(x), ctx.array(n)
    dA.spmv(dx, dy)
    ref = restate.spmv(A, x)
    got = dy.download()
    assert rel_err(got, ref) <= 1e-14
    # rows of up to 256 entries are summed in the reference's order (bit-exact);
    # longer rows are reduced across a warp (tolerance above)
    short = np.diff(rp) <= 256
    assert np.array_equal(got[short], ref[short])


def test_spmv_config_sizes(M, ctx, restate):
    # full-size configurations: 128^3 7-point and 96^3 27-point; every row is
    # summed in the reference's order, so the products are bit-identical
    for A in (M.laplacian3d(128), M.convdiff27(96, 2)):
        n = A[0]
        dA = M.Csr(ctx, *A[1:])
        x = M.uniform(n, 13)
        dx, dy = ctx.to_device(x), ctx.array(n)
        dA.spmv(dx, dy)
        ref = restate.spmv(A, x)
        got = dy.download()
        assert rel_err(got, ref) <= 1e-14
        assert np.array_equal(got, ref)
        dA.close()


def banded(n, offsets, seed):
    """CSR of an n x n matrix with entries on the given diagonals (sorted)."""
    rng = np.random.default_rng(seed)
    offsets = sorted(offsets)
    rows, cols = [], []
    for r in range(n):
        for o in offsets:
            if 0 <= r + o < n:
                rows.append(r)
                cols.append(r + o)
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, np.asarray(rows) + 1, 1)
    return n, np.cumsum(rp).astype(np.int32), np.asarray(cols, np.int32), rng.standard_normal(len(cols))


@pytest.mark.parametrize("far", [32767, 32768])
def test_spmv_sell_index_widths(M, ctx, restate, monkeypatch, far):
    # The SELL-32 copy stores column indices as 16-bit offsets from the row
    # when every entry lies within 32,767 of its row (far = 32767: the
    # largest offset that fits), else as 32-bit indices (far = 32768).  Both
    # sum each row in the reference's order: bit-identical products.  With
    # MTLGPU_SELL_INDEX=32 the 16-bit copy is not built; the products agree.
    A = banded(70000, [-far, -1, 0, 1, 5, far], 7)
    n = A[0]
    x = M.uniform(n, 5)
    ref = restate.spmv(A, x)
    got = []
    for env in (None, "32"):
        if env:
            monkeypatch.setenv("MTLGPU_SELL_INDEX", env)
        dA = M.Csr(ctx, *A[1:])
        dx, dy = ctx.to_device(x), ctx.array(n)
        dA.spmv(dx, dy)
        got.append(dy.download())
        dA.close()
    assert np.array_equal(got[0], ref) and np.array_equal(got[1], ref)


@pytest.mark.parametrize("A_fn", [lambda M: M.convdiff27(6, 2), lambda M: M.convdiff27(20, 2),
                                  lambda M: M.random_graph(1500, 12.0, 1e-2, 5)])
def test_spmv_transposed(M, ctx, restate, A_fn):
    # trans(A) * x (transposed_sparse_matrix_vector_product_test.cpp:32)
    # against the oracle's SpMV with the oracle's CSR transpose
    A = A_fn(M)
    n = A[0]
    x = M.uniform(n, 9)
    dA = M.Csr(ctx, *A[1:])
    dx, dy = ctx.to_device(x), ctx.array(n)
    dA.spmv_transposed(dx, dy)
    ref = restate.spmv(restate.transpose(A), x)
    assert rel_err(dy.download(), ref) <= 1e-14


def test_csr_validation(M, ctx):
    A = M.laplacian2d(4, 4)
    n, rp, ci, v = A
    bad = ci.copy()
    bad[3], bad[4] = bad[4], bad[3]
    with pytest.raises(M.MtlgpuError) as e:
        M.Csr(ctx, rp, bad, v)
    assert e.value.status == M.NOT_SORTED
    bad = ci.copy()
    bad[-1] = 99
    with pytest.raises(M.MtlgpuError) as e:
        M.Csr(ctx, rp, bad, v)
    assert e.value.status == M.INDEX_RANGE
    # empty matrix
    E = M.Csr(ctx, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    E.close()


@pytest.mark.parametrize("n", [1, 3, 4, 7, 9, 1000, 100003, 2097152])
def test_blas1(M, ctx, restate, n):
    x, y = M.uniform(n, 21), M.uniform(n, 22)
    dx, dy = ctx.to_device(x), ctx.to_device(y)
    assert abs(ctx.dot(dx, dy) - restate.dot(x, y)) <= 1e-13 * max(1.0, abs(restate.dot(x, y)))
    assert abs(ctx.two_norm(dx) - restate.two_norm(x)) <= 1e-14 * restate.two_norm(x)
    ctx.axpy(0.5, dx, dy)
    assert np.allclose(dy.download(), y + 0.5 * x, rtol=0, atol=1e-15)
    dy.upload(y)
    ctx.xpay(dx, -2.0, dy)
    assert np.allclose(dy.download(), x - 2.0 * y, rtol=0, atol=1e-15)
    # determinism: same bits on every call
    assert ctx.dot(dx, dx) == ctx.dot(dx, dx)


def test_dot_known_answer(M, ctx):
    u = ctx.to_device(np.arange(1.0, 10.0))
    assert ctx.dot(u, u) == 285.0


FACTOR_CASES = ["lap3d_20", "cd27_10", "graph_2000", "fv2d_64", "lap2d_100"]


@pytest.mark.parametrize("name", FACTOR_CASES)
@pytest.mark.parametrize("kind", ["ic0", "ilu0"])
def test_factors_bit_exact(M, ctx, restate, name, kind):
    A = matrices(M)[name]
    if kind == "ic0" and name == "cd27_10":
        A = M.random_graph(1500, 9.0, 1e-2, 8)   # IC(0) needs a symmetric matrix
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, kind)
    L, U = getattr(restate, kind)(A)
    gL, gU = P.factor(M.LOWER), P.factor(M.UPPER)
    assert csr_eq(gL, L), "L pattern/values differ"
    assert csr_eq(gU, U), "U pattern/values differ"
    # level arrays: bit-exact with the levels of the reference's patterns
    assert np.array_equal(P.levels(M.LOWER), restate.levels(L, True)[0])
    assert np.array_equal(P.levels(M.UPPER), restate.levels(U, False)[0])
    nnzL, nlevL = P.factor_info(M.LOWER)
    assert nnzL == len(L[2]) and nlevL == restate.levels(L, True)[1]


def test_factors_against_golden(M, ctx, golden):
    A = M.laplacian3d(16)
    P = M.Pc(M.Csr(ctx, *A[1:]), "ic0")
    for which, key in ((M.LOWER, "lap16_ic0_L"), (M.UPPER, "lap16_ic0_U")):
        F = P.factor(which)
        assert csr_eq(F, (F[0], golden[key + "_rp"], golden[key + "_ci"], golden[key + "_v"]))
    assert np.array_equal(P.levels(M.LOWER), golden["lap16_ic0_L_lev"])
    assert np.array_equal(P.levels(M.UPPER), golden["lap16_ic0_U_lev"])
    Pf = M.Pc(M.Csr(ctx, *A[1:]), "ic0", M.FP32)
    assert np.array_equal(Pf.factor(M.UPPER)[3], golden["lap16_ic0f_U_v"])
    C = M.convdiff27(8, 2)
    P = M.Pc(M.Csr(ctx, *C[1:]), "ilu0")
    for which, key in ((M.LOWER, "cd8_ilu0_L"), (M.UPPER, "cd8_ilu0_U")):
        F = P.factor(which)
        assert csr_eq(F, (F[0], golden[key + "_rp"], golden[key + "_ci"], golden[key + "_v"]))
    assert np.array_equal(P.levels(M.LOWER), golden["cd8_ilu0_L_lev"])
    G = M.random_graph(600, 12.0, 1e-2, 3)
    P = M.Pc(M.Csr(ctx, *G[1:]), "ic0")
    assert np.array_equal(P.factor(M.LOWER)[3], golden["rg_ic0_L_v"])
    assert np.array_equal(P.factor(M.UPPER)[3], golden["rg_ic0_U_v"])


@pytest.mark.parametrize("name", FACTOR_CASES)
@pytest.mark.parametrize("kind", ["ic0", "ilu0", "diagonal", "identity"])
def test_pc_apply(M, ctx, restate, name, kind):
    A = matrices(M)[name]
    if kind == "ic0" and name == "cd27_10":
        A = M.random_graph(1500, 9.0, 1e-2, 8)
    n = A[0]
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, kind)
    r = M.uniform(n, 31)
    dr, dz = ctx.to_device(r), ctx.array(n)
    P.apply(dr, dz)
    ref = restate.pc_apply(kind, A, r)
    assert rel_err(dz.download(), ref) <= 1e-12
    assert np.array_equal(dz.download(), ref)
    P.adjoint_apply(dr, dz)
    ref = restate.pc_apply(kind, A, r, adjoint=True)
    assert rel_err(dz.download(), ref) <= 1e-12
    assert np.array_equal(dz.download(), ref)
    # a second apply reuses the plans and must give the same bits
    z1 = dz.download()
    P.adjoint_apply(dr, dz)
    assert np.array_equal(z1, dz.download())


def test_pc_apply_golden(M, ctx, golden):
    A = M.laplacian3d(16)
    P = M.Pc(M.Csr(ctx, *A[1:]), "ic0")
    db, dz = ctx.to_device(golden["lap16_b"]), ctx.array(A[0])
    P.apply(db, dz)
    assert np.array_equal(dz.download(), golden["lap16_pc_ic0_apply"])
    C = M.convdiff27(8, 2)
    P = M.Pc(M.Csr(ctx, *C[1:]), "ilu0")
    db, dz = ctx.to_device(golden["cd8_b"]), ctx.array(C[0])
    P.apply(db, dz)
    assert np.array_equal(dz.download(), golden["cd8_pc_ilu0_apply"])
    P.adjoint_apply(db, dz)
    assert np.array_equal(dz.download(), golden["cd8_pc_ilu0_adjoint"])


@pytest.mark.parametrize("A_fn", [lambda M: M.laplacian3d(12), lambda M: M.fv2d(40),
                                  lambda M: M.random_graph(2500, 24.0, 1e-2, 6)])
def test_single_sweeps(M, ctx, restate, A_fn):
    # one triangular sweep, bit-identical with the reference's loops (the
    # random graph has rows long enough for several passes of a lane group)
    A = A_fn(M)
    n = A[0]
    P = M.Pc(M.Csr(ctx, *A[1:]), "ic0")
    L, U = restate.ic0(A)
    r = M.uniform(n, 41)
    dr, dy = ctx.to_device(r), ctx.array(n)
    P.sweep(M.LOWER, dr, dy)
    assert np.array_equal(dy.download(), restate.sweep("lower_invdiag_last", L, r))
    P.sweep(M.UPPER, dr, dy)
    assert np.array_equal(dy.download(), restate.sweep("upper_invdiag_first", U, r))
    C = M.convdiff27(6, 2)
    Q = M.Pc(M.Csr(ctx, *C[1:]), "ilu0")
    L, U = restate.ilu0(C)
    r = M.uniform(C[0], 42)
    dr, dy = ctx.to_device(r), ctx.array(C[0])
    Q.sweep(M.LOWER, dr, dy)
    assert np.array_equal(dy.download(), restate.sweep("lower_unit", L, r))
    Q.sweep(M.UPPER, dr, dy)
    assert np.array_equal(dy.download(), restate.sweep("upper_invdiag_first", U, r))


def test_single_sweeps_fp32(M, ctx, restate):
    # the FP32 sweep of the mixed solves: float factors, float vectors,
    # separately rounded float products and differences in the reference's
    # order (the restatement run in float arithmetic, through numpy)
    A = M.laplacian3d(10)
    n = A[0]
    P = M.Pc(M.Csr(ctx, *A[1:]), "ic0", M.FP32)
    L, _ = restate.ic0(A, as_float=True)
    _, rp, ci, v = L
    v32 = v.astype(np.float32)
    r = M.uniform(n, 43).astype(np.float32)
    ref = np.zeros(n, np.float32)
    for i in range(n):
        rr = r[i]
        for j in range(rp[i], rp[i + 1] - 1):
            rr = np.float32(rr - np.float32(v32[j] * ref[ci[j]]))
        ref[i] = np.float32(rr * v32[rp[i + 1] - 1])
    dr, dy = ctx.to_device(r), ctx.array(n, np.float32)
    P.sweep(M.LOWER, dr, dy)
    assert np.array_equal(dy.download(), ref)


def test_missing_diagonal(M, ctx):
    A = M.laplacian2d(4, 4)
    n, rp, ci, v = A
    keep = np.ones(len(ci), bool)
    keep[rp[5] + 2] = False  # drop the diagonal of row 5 (5-point order: -n, -1, diag)
    assert ci[rp[5] + 2] == 5
    rp2 = np.concatenate([[0], np.cumsum([keep[rp[i]:rp[i + 1]].sum() for i in range(n)])])
    dA = M.Csr(ctx, rp2.astype(np.int32), ci[keep], v[keep])
    for kind in ("ic0", "ilu0"):
        with pytest.raises(M.MtlgpuError) as e:
            M.Pc(dA, kind)
        assert e.value.status == M.MISSING_DIAGONAL


def test_zero_pivot_reported(M, ctx):
    # a singular 2x2 block: the factor is still produced (inf), status ZERO_PIVOT
    rp = np.array([0, 2, 4], np.int32)
    ci = np.array([0, 1, 0, 1], np.int32)
    v = np.array([1.0, 1.0, 1.0, 1.0])
    P = M.Pc(M.Csr(ctx, rp, ci, v), "ilu0")
    assert P.status == M.ZERO_PIVOT
    Q = M.Pc(M.Csr(ctx, rp, ci, v), "ic0")
    assert Q.status == M.ZERO_PIVOT


@pytest.mark.parametrize("A_fn", [lambda M: M.laplacian3d(24), lambda M: M.convdiff27(12, 2)])
def test_cg_direction_product(M, ctx, restate, A_fn):
    # p' = z + beta p, q = A p', p'.q in one kernel (mtlgpu_cg_direction_product).
    # FP64: p' within one rounding of z + beta p (the kernel rounds once, by
    # fma), q bit-identical to the oracle's product of p', p'.q to 1e-14;
    # p = None gives p' = z.  FP32: q and p'.q against FP64 arithmetic on the
    # float-rounded values, 1e-6.
    A = A_fn(M)
    n, rp, ci, v = A
    dA = M.Csr(ctx, rp, ci, v)
    z, p, beta = M.uniform(n, 3), M.uniform(n, 4), 0.37
    for first in (False, True):
        dz, dp, dpo, dq, dpq = (ctx.to_device(z), ctx.to_device(p), ctx.array(n), ctx.array(n),
                                ctx.array(1))
        dA.cg_direction_product(M.FP64, dz, 0.0 if first else beta, None if first else dp,
                                dpo, dq, dpq)
        po, q, pq = dpo.download(), dq.download(), dpq.download()[0]
        want = z if first else z + beta * p
        assert rel_err(po, want) <= 2e-16 * 4
        if first:
            assert np.array_equal(po, z)
        assert np.array_equal(q, restate.spmv(A, po))
        assert abs(pq - np.dot(po, q)) <= 1e-14 * abs(np.dot(po, q))
    f = lambda a: a.astype(np.float32)  # noqa: E731
    dz, dp, dpo, dq, dpq = (ctx.to_device(f(z)), ctx.to_device(f(p)), ctx.array(n, np.float32),
                            ctx.array(n, np.float32), ctx.array(1))
    dA.cg_direction_product(M.FP32, dz, beta, dp, dpo, dq, dpq)
    po, q, pq = dpo.download().astype(np.float64), dq.download().astype(np.float64), \
        dpq.download()[0]
    b32 = float(np.float32(beta))
    assert rel_err(po, f(z).astype(np.float64) + b32 * f(p).astype(np.float64)) <= 1e-7
    A32 = (n, rp, ci, f(v).astype(np.float64))
    q64 = restate.spmv(A32, po)
    assert rel_err(q, q64) <= 1e-6
    assert abs(pq - np.dot(po, q)) <= 1e-6 * abs(np.dot(po, q))
    dA.close()


@pytest.mark.parametrize("kind", ["ic0", "ilu0"])
def test_factors_bit_exact_full_size(M, ctx, restate, kind):
    # The configurations' own factorisations: IC(0) of the 128^3 7-point
    # Laplacian (n = 2,097,152) and ILU(0) of the 96^3 27-point
    # convection-diffusion operator (n = 884,736, seed 2), bit-identical to
    # the C restatement of the reference's factorisations, with the same
    # level arrays (the level analysis takes rows in chunks, and ILU(0)
    # keeps short rows in registers: both must leave the results unchanged).
    A = M.laplacian3d(128) if kind == "ic0" else M.convdiff27(96, 2)
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, kind)
    L, U = getattr(restate, kind)(A)
    assert csr_eq(P.factor(M.LOWER), L), "L pattern/values differ"
    assert csr_eq(P.factor(M.UPPER), U), "U pattern/values differ"
    lv, nl = restate.levels(L, True)
    uv, nu = restate.levels(U, False)
    assert np.array_equal(P.levels(M.LOWER), lv)
    assert np.array_equal(P.levels(M.UPPER), uv)
    assert P.factor_info(M.LOWER)[1] == nl and P.factor_info(M.UPPER)[1] == nu
    P.close()
    dA.close()
