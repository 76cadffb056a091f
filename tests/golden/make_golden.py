"""Generates tests/golden/golden.npz from the MTL4 reference itself.

Run in a checkout where the reference tree is present (it is compiled by
``make -C oracle``; the library it produces is ``oracle/_ref/libmtlref.so``):

    python tests/golden/make_golden.py            # small cases (seconds)
    python tests/golden/make_golden.py --cfg2     # + the 128^3 solve (about a minute)
    python tests/golden/make_golden.py --cfg3     # + the 96^3 27-point BiCGSTAB solve
    python tests/golden/make_golden.py --cfg5     # + the 512^2 CPU adjoint (gradients)
    REFERENCE_ROOT=<MTL4 tree> python tests/golden/make_golden.py --mtx
                                                  # + the reference's Matrix Market fixtures

Every array stored here is an output of the reference's own code path
(laplacian_setup, compressed2D SpMV, the compressed2D inserter, ic_0 /
ilu_0 factors, solve(P, x), the other ITL Krylov methods,
itl::cg / itl::bicgstab with basic_iteration), except the level arrays,
which the reference does not compute: those come from the restatement
(oracle/restate.c, or_levels_lower/upper) applied to the reference's own
factor patterns.  Inputs come from the library's seeded generators
(include/mtlgpu_fixtures.h).
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "mtl4-mirror_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import mtlgpu as M  # noqa: E402
import oracle as O  # noqa: E402


def put_csr(out, key, A):
    out[key + "_rp"], out[key + "_ci"], out[key + "_v"] = A[1], A[2], A[3]


def fv_source(N):
    """The Gaussian source of the differentiable-solve workload."""
    c = (np.arange(N) + 0.5) / N - 0.5
    X, Y = np.meshgrid(c, c, indexing="ij")
    return np.exp(-(X ** 2 + Y ** 2) / (2 * 0.1 ** 2)).ravel()


CFG5_DIRECTIONS = 64


def cfg5(R, out):
    """Config 5: the FP64 CPU adjoint by the reference itself.  512 x 512
    finite-volume operator (sigma 1, 8-cell correlation, seed 4), b the
    Gaussian source, L = 1/2 ||x - x_target||^2 with x_target = x + 0.01 N(0,1)
    (seed 44), so dL/dx = -0.01 N(0,1) at the solution.  itl::cg + ic_0 to
    1e-13 for x = A^-1 b and for lambda = A^-T dL/dx; dL/db = lambda and
    dL/dvals = -lambda_i x_j on A's pattern.  Stored: their projections on
    64 seeded random directions (N(0,1), seeds 1000 + m for b, 2000 + m for
    the values), their norms, and 1024 sampled entries."""
    A = M.fv2d(512, 1.0, 8.0, 4)
    n, rp, ci, v = A
    b = fv_source(512)
    rf = R.solve("cg", "ic0", A, b, rtol=1e-13, max_iter=20000)
    g = -0.01 * M.normal(n, 44)
    ra = R.solve("cg", "ic0", A, g, rtol=1e-13, max_iter=20000)
    assert rf["err"] == 0 and ra["err"] == 0, (rf["err"], ra["err"])
    x, lam = rf["x"], ra["x"]
    rows = np.repeat(np.arange(n), np.diff(rp))
    G = -lam[rows] * x[ci]
    pb = np.array([lam @ M.normal(n, 1000 + m) for m in range(CFG5_DIRECTIONS)])
    pv = np.array([G @ M.normal(len(ci), 2000 + m) for m in range(CFG5_DIRECTIONS)])
    rng = np.random.default_rng(5)
    ib = rng.choice(n, 1024, replace=False)
    iv = rng.choice(len(ci), 1024, replace=False)
    out["cfg5_proj_b"], out["cfg5_proj_vals"] = pb, pv
    out["cfg5_norms"] = np.array([np.linalg.norm(lam), np.linalg.norm(G), np.linalg.norm(x)])
    out["cfg5_idx_b"], out["cfg5_lambda_sample"] = ib.astype(np.int64), lam[ib]
    out["cfg5_idx_vals"], out["cfg5_grad_vals_sample"] = iv.astype(np.int64), G[iv]
    out["cfg5_x_sample"] = x[ib]
    out["cfg5_iters"] = np.array([rf["iterations"], ra["iterations"]])


MTX_FIXTURES = ("bcsstk01", "bcspwr02", "jgl009", "plskz362", "dense_read")


def mtx_fixtures(R, S, out):
    """The real-valued Matrix Market files among the reference's test
    fixtures (libs/numeric/mtl/test/matrix_market/): each is read by the
    reference's own reader and by <mtlgpu/matrix_market.hpp> (tests/cpp/
    mm_parity, which fails unless both give the same CSR arrays); stored are
    the arrays and the reference's results on them: the SpMV of a seeded x
    for every file, and for the SPD stiffness matrix bcsstk01 its IC(0) and
    ILU(0) factors and its solves.  (mhd1280b is complex Hermitian and
    outside the real-valued path; obstacle_small and square3 are not Matrix
    Market files.)"""
    import json
    import subprocess
    root = os.environ.get("REFERENCE_ROOT")
    if not root:
        raise SystemExit("--mtx needs REFERENCE_ROOT (the MTL4 tree)")
    d = os.path.join(root, "libs", "numeric", "mtl", "test", "matrix_market")
    exe = os.path.join(ROOT, "tests", "cpp", "_build", "mm_parity")
    for name in MTX_FIXTURES:
        p = subprocess.run([exe, os.path.join(d, name + ".mtx")], capture_output=True, text=True)
        rec = json.loads(p.stdout.splitlines()[-1])
        assert p.returncode == 0 and rec["same"] == 1, name
        rp = np.array(rec["starts"], np.int32)
        ci = np.array(rec["indices"], np.int32)
        v = np.array(rec["data"], np.float64)
        rows, cols = rec["rows"], rec["cols"]
        key = "mtx_" + name
        out[key + "_rp"], out[key + "_ci"], out[key + "_v"] = rp, ci, v
        out[key + "_shape"] = np.array([rows, cols])
        x = M.uniform(cols, 7)
        A = (rows, rp, ci, v)
        out[key + "_x"] = x
        out[key + "_spmv"] = R.spmv(A, x) if rows == cols else S.spmv(A, x)
    # bcsstk01: factors and solves by the reference
    A = (48, out["mtx_bcsstk01_rp"], out["mtx_bcsstk01_ci"], out["mtx_bcsstk01_v"])
    L, U = R.ic0(A)
    out["mtx_bcsstk01_ic0_L_v"], out["mtx_bcsstk01_ic0_U_v"] = L[3], U[3]
    L, U = R.ilu0(A)
    out["mtx_bcsstk01_ilu0_L_v"], out["mtx_bcsstk01_ilu0_U_v"] = L[3], U[3]
    b = R.spmv(A, M.uniform(48, 1))
    out["mtx_bcsstk01_b"] = b
    its = []
    for method, pc in (("cg", "ic0"), ("cg", "diagonal"), ("bicgstab", "ilu0")):
        r = R.solve(method, pc, A, b, rtol=1e-10, max_iter=1000)
        its.append([r["iterations"], r["err"]])
    out["mtx_bcsstk01_iters"] = np.array(its)


def assembly_cases(R, out):
    """mtl::mat::inserter runs of the reference on seeded triplets with many
    duplicates (rows and columns drawn from small ranges), stored with their
    inputs: 'asm_u<k>' inserts with `<<` and class updater k (store, plus,
    minus, times) into an empty 300 x 250 matrix; 'asm_mix' mixes `=`, `+=`
    and `<<` (class updater plus) on top of a base matrix with entries."""
    rng = np.random.default_rng(7)
    nr, nc, cnt = 300, 250, 6000
    rows = rng.integers(0, nr, cnt).astype(np.int32)
    cols = (rows.astype(np.int64) * 7 + rng.integers(0, 12, cnt)) % nc
    cols = cols.astype(np.int32)
    vals = rng.normal(size=cnt)
    out["asm_rows"], out["asm_cols"], out["asm_vals"] = rows, cols, vals
    out["asm_shape"] = np.array([nr, nc])
    for u in range(4):
        rp, ci, v = R.assemble(nr, nc, rows, cols, vals, updater=u)
        out[f"asm_u{u}_rp"], out[f"asm_u{u}_ci"], out[f"asm_u{u}_v"] = rp, ci, v
    # base matrix: 2 seeded entries per row (sorted, distinct columns)
    brows = np.repeat(np.arange(nr, dtype=np.int32), 2)
    bcols = np.sort(np.stack([rng.choice(nc, 2, replace=False) for _ in range(nr)]), axis=1)
    bcols = bcols.ravel().astype(np.int32)
    bvals = rng.normal(size=2 * nr)
    base = R.assemble(nr, nc, brows, bcols, bvals)
    out["asm_base_rp"], out["asm_base_ci"], out["asm_base_v"] = base
    syntax = rng.integers(0, 3, cnt).astype(np.uint8)
    out["asm_mix_syntax"] = syntax
    rp, ci, v = R.assemble(nr, nc, rows, cols, vals, updater=1, base=base, syntax=syntax)
    out["asm_mix_rp"], out["asm_mix_ci"], out["asm_mix_v"] = rp, ci, v


KRYLOV_METHODS = ["bicg", "cgs", "bicgstab_2", "bicgstab_ell", "tfqmr", "qmr", "idr_s", "gmres"]
KRYLOV_PCS = [("identity", "identity"), ("ilu0", "identity"), ("diagonal", "ilu0"),
              ("ic0", "diagonal")]


def krylov_problems():
    """The small systems the other Krylov methods are pinned on: 27-point
    convection-diffusion 6^3 (unsymmetric), the 12 x 12 Laplacian and the
    16 x 16 finite-volume operator; b = A x_true, x_true ~ U[-1,1] seed 1."""
    return [("cd6", M.convdiff27(6, 2)), ("lap12", M.laplacian2d(12, 12)),
            ("fv16", M.fv2d(16, 1.0, 8.0, 4))]


def krylov_param(method):
    return {"bicgstab_ell": 4, "idr_s": 2, "gmres": 8}.get(method, 0)


def krylov_max_iter(method):
    return 60 if method == "qmr" else 400


def krylov_cases(R, out):
    """The reference's bicg, cgs, bicgstab_2, bicgstab_ell (l = 4), tfqmr, qmr
    (60 iterations: its test on the Lanczos norm never stops it earlier),
    idr_s (s = 2) and gmres (restart 8) with left / right preconditioners, to
    rtol 1e-8: [iterations, error], the last residual tested, x, and the
    first 64 residuals recorded."""
    for name, A in krylov_problems():
        b = R.spmv(A, M.uniform(A[0], 1))
        out[f"kry_{name}_b"] = b
        for meth in KRYLOV_METHODS:
            for pl, pr in KRYLOV_PCS:
                r = R.solve_krylov(meth, pl, A, b, pc_right=pr, param=krylov_param(meth),
                                   max_iter=krylov_max_iter(meth), rtol=1e-8)
                key = f"kry_{name}_{meth}_{pl}_{pr}"
                out[key + "_iters"] = np.array([r["iterations"], r["err"]])
                out[key + "_resid"] = np.array([r["resid"], r["norm_r0"]])
                out[key + "_x"] = r["x"]
                out[key + "_hist"] = r["history"][:64]
    # gmres and idr_s cut after a few cycles / steps on cd6 (no preconditioner)
    A = M.convdiff27(6, 2)
    b = out["kry_cd6_b"]
    for meth, cuts in (("gmres", (8, 16, 24, 32)), ("idr_s", (1, 2, 3, 5, 8, 13))):
        for k in cuts:
            r = R.solve_krylov(meth, "identity", A, b, param=krylov_param(meth), max_iter=k,
                               rtol=1e-8)
            out[f"kry_cut_{meth}_{k}_x"] = r["x"]
            out[f"kry_cut_{meth}_{k}_resid"] = np.array([r["resid"], r["iterations"]])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cfg2", action="store_true")
    ap.add_argument("--cfg3", action="store_true")
    ap.add_argument("--cfg5", action="store_true")
    ap.add_argument("--mtx", action="store_true")
    args = ap.parse_args()
    R = O.Reference()
    S = O.Restatement()
    out = {}

    # ic_0_test.cpp: 3x3 grid, ic_0<M, float>, y = solve(P, iota)
    A3 = R.laplacian_setup(3, 3)
    out["kat_ic0_float_iota"] = R.pc_apply("ic0_float", A3, np.arange(9.0))

    # config 1: 100x100 Laplacian, x_true ~ U[-1,1] seed 0, cg + ic_0 to 1e-10
    A1 = R.laplacian_setup(100, 100)
    xt = M.uniform(A1[0], 0)
    b1 = R.spmv(A1, xt)
    r = R.solve("cg", "ic0", A1, b1, rtol=1e-10, max_iter=1000)
    out["cfg1_b"], out["cfg1_x"], out["cfg1_hist"] = b1, r["x"], r["history"]
    out["cfg1_iters"] = np.array([r["iterations"], r["err"]])
    for pc in ("identity", "diagonal", "ilu0"):
        rr = R.solve("cg", pc, A1, b1, rtol=1e-10, max_iter=1000)
        out[f"cfg1_{pc}_iters"] = np.array([rr["iterations"], rr["err"]])
        out[f"cfg1_{pc}_hist"] = rr["history"]
    L, U = R.ic0(A1)
    out["cfg1_ic0_L_v"], out["cfg1_ic0_U_v"] = L[3], U[3]
    out["cfg1_ic0_L_lev"] = S.levels(L, True)[0]
    out["cfg1_ic0_U_lev"] = S.levels(U, False)[0]

    # 3-D 7-point, 16^3 (x_true seed 1)
    A = M.laplacian3d(16)
    xt = M.uniform(A[0], 1)
    b = R.spmv(A, xt)
    r = R.solve("cg", "ic0", A, b, rtol=1e-10, max_iter=2000)
    out["lap16_b"], out["lap16_hist"] = b, r["history"]
    out["lap16_iters"] = np.array([r["iterations"], r["err"]])
    L, U = R.ic0(A)
    put_csr(out, "lap16_ic0_L", L)
    put_csr(out, "lap16_ic0_U", U)
    out["lap16_ic0_L_lev"] = S.levels(L, True)[0]
    out["lap16_ic0_U_lev"] = S.levels(U, False)[0]
    Lf, Uf = R.ic0(A, as_float=True)
    out["lap16_ic0f_U_v"] = Uf[3]
    out["lap16_pc_ic0_apply"] = R.pc_apply("ic0", A, b)

    # 27-point convection-diffusion, 8^3 (seed 2): bicgstab + ilu_0
    A = M.convdiff27(8, 2)
    xt = M.uniform(A[0], 1)
    b = R.spmv(A, xt)
    r = R.solve("bicgstab", "ilu0", A, b, rtol=1e-10, max_iter=1000)
    out["cd8_b"], out["cd8_hist"], out["cd8_x"] = b, r["history"], r["x"]
    out["cd8_iters"] = np.array([r["iterations"], r["err"]])
    L, U = R.ilu0(A)
    put_csr(out, "cd8_ilu0_L", L)
    put_csr(out, "cd8_ilu0_U", U)
    out["cd8_ilu0_L_lev"] = S.levels(L, True)[0]
    out["cd8_ilu0_U_lev"] = S.levels(U, False)[0]
    out["cd8_pc_ilu0_apply"] = R.pc_apply("ilu0", A, b)
    out["cd8_pc_ilu0_adjoint"] = R.pc_apply("ilu0", A, b, adjoint=True)
    rr = R.solve("bicgstab", "diagonal", A, b, rtol=1e-10, max_iter=1000)
    out["cd8_diag_iters"] = np.array([rr["iterations"], rr["err"]])

    # random-graph Laplacian (n = 600, degree 12, seed 3): IC(0) as written
    A = M.random_graph(600, 12.0, 1e-2, 3)
    b = M.normal(A[0], 3)
    L, U = R.ic0(A)
    put_csr(out, "rg_ic0_L", L)
    put_csr(out, "rg_ic0_U", U)
    out["rg_ic0_L_lev"] = S.levels(L, True)[0]
    out["rg_ic0_U_lev"] = S.levels(U, False)[0]
    out["rg_b"] = b
    for pc in ("ic0", "diagonal"):
        rr = R.solve("cg", pc, A, b, rtol=1e-8, max_iter=1000)
        out[f"rg_{pc}_iters"] = np.array([rr["iterations"], rr["err"]])
        out[f"rg_{pc}_hist"] = rr["history"]

    assembly_cases(R, out)
    krylov_cases(R, out)

    # 2-D finite volume, 32^2 (seed 4)
    A = M.fv2d(32, 1.0, 8.0, 4)
    b = M.normal(A[0], 4)
    rr = R.solve("cg", "ic0", A, b, rtol=1e-10, max_iter=1000)
    out["fv32_b"] = b
    out["fv32_iters"] = np.array([rr["iterations"], rr["err"]])
    out["fv32_hist"] = rr["history"]

    if args.cfg2:
        A = M.laplacian3d(128)
        xt = M.uniform(A[0], 1)
        b = M.csr_mult(A, xt)
        rr = R.solve("cg", "ic0", A, b, rtol=1e-10, max_iter=2000)
        out["cfg2_iters"] = np.array([rr["iterations"], rr["err"]])
        out["cfg2_hist"] = rr["history"]
    if args.cfg3:
        # 27-point convection-diffusion 96^3 (seed 2), x_true ~ U[-1,1] seed 1,
        # b = A x_true by the reference's SpMV; FP64 bicgstab + ilu_0 to 1e-10
        A = M.convdiff27(96, 2)
        xt = M.uniform(A[0], 1)
        b = R.spmv(A, xt)
        rr = R.solve("bicgstab", "ilu0", A, b, rtol=1e-10, max_iter=2000)
        out["cfg3_iters"] = np.array([rr["iterations"], rr["err"]])
        out["cfg3_hist"] = rr["history"]
        out["cfg3_b_sum"] = np.array([b.sum(), np.linalg.norm(b)])
    if args.cfg5:
        cfg5(R, out)
    if args.mtx:
        mtx_fixtures(R, S, out)
    old = os.path.join(HERE, "golden.npz")
    if os.path.exists(old):
        prev = np.load(old)
        for k in prev.files:
            if k.startswith(("cfg2_", "cfg3_", "cfg5_", "mtx_")) and k not in out:
                out[k] = prev[k]

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
