"""Device assembly (mtlgpu_csr_assemble) and device Laplacian generation
against the reference's inserter: bit-identical CSR arrays (row starts,
column indices and the 64-bit patterns of the values), through the C ABI."""
import numpy as np
import pytest

from test_assembly import ops_from_syntax, same, triplets

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["u0", "u1", "u2", "u3", "mix"])
def test_assemble_matches_reference_golden(M, ctx, golden, case):
    nr, nc = (int(x) for x in golden["asm_shape"])
    rows, cols, vals = golden["asm_rows"], golden["asm_cols"], golden["asm_vals"]
    if case == "mix":
        base = M.Csr(ctx, golden["asm_base_rp"], golden["asm_base_ci"], golden["asm_base_v"],
                     n_cols=nc)
        A = M.Csr.assemble(ctx, nr, nc, rows, cols, vals, updater=M.UPDATE_PLUS, base=base,
                           ops=ops_from_syntax(golden["asm_mix_syntax"], 1))
    else:
        A = M.Csr.assemble(ctx, nr, nc, rows, cols, vals, updater=int(case[1]))
    ref = (golden[f"asm_{case}_rp"], golden[f"asm_{case}_ci"], golden[f"asm_{case}_v"])
    assert same(A.download(), ref)


@pytest.mark.parametrize("nr,nc,cnt,spread,seed", [
    (1, 1, 1, 1, 1),             # one entry
    (1, 5000, 20000, 5000, 2),   # one long row, heavy duplication
    (5000, 3, 30000, 3, 3),      # narrow rectangle
    (70000, 70000, 400000, 40, 4),  # keys wider than 32 bits, several tiles
    (3000, 3000, 2049, 2, 5),    # a tile boundary plus one
])
def test_assemble_matches_restatement(M, ctx, restate, nr, nc, cnt, spread, seed):
    rng, rows, cols, vals = triplets(seed, nr, nc, cnt, spread)
    for u in range(4):
        ops = rng.integers(0, 4, cnt).astype(np.uint8)
        for o in (None, ops):
            A = M.Csr.assemble(ctx, nr, nc, rows, cols, vals, updater=u, ops=o)
            ref = restate.assemble(nr, nc, rows, cols, vals, updater=u, ops=o)
            assert same(A.download(), ref), (u, o is None)


def test_assemble_into_base_twice(M, ctx, restate):
    # the result of one assembly is the base of the next (inserter on a matrix
    # that already holds entries, twice)
    rng, rows, cols, vals = triplets(9, 4000, 4000, 50000, 11)
    A = M.Csr.assemble(ctx, 4000, 4000, rows[:20000], cols[:20000], vals[:20000],
                       updater=M.UPDATE_PLUS)
    B = M.Csr.assemble(ctx, 4000, 4000, rows[20000:], cols[20000:], vals[20000:],
                       updater=M.UPDATE_MINUS, base=A)
    ra = restate.assemble(4000, 4000, rows[:20000], cols[:20000], vals[:20000], updater=1)
    rb = restate.assemble(4000, 4000, rows[20000:], cols[20000:], vals[20000:], updater=2,
                          base=ra)
    assert same(A.download(), ra)
    assert same(B.download(), rb)


def test_assemble_edge_cases(M, ctx, restate):
    for nr, nc, rows, cols, vals in [(5, 5, [], [], []), (0, 0, [], [], []),
                                     (4, 4, [3, 3, 3], [3, 3, 3], [0.0, 0.0, 0.0])]:
        A = M.Csr.assemble(ctx, nr, nc, np.array(rows, np.int32), np.array(cols, np.int32),
                           np.array(vals, np.float64))
        assert same(A.download(), restate.assemble(nr, nc, rows, cols, vals)), (nr, nc)
    for r, c in [([0, 4], [0, 0]), ([0, 1], [0, -1]), ([-1], [2])]:
        with pytest.raises(M.MtlgpuError) as e:
            M.Csr.assemble(ctx, 4, 4, np.array(r, np.int32), np.array(c, np.int32),
                           np.ones(len(r)))
        assert e.value.status == M.INDEX_RANGE
    # the context stays usable after a rejected assembly
    A = M.Csr.assemble(ctx, 2, 2, np.array([1, 0], np.int32), np.array([0, 1], np.int32),
                       np.array([2.0, 3.0]))
    assert same(A.download(), (np.array([0, 1, 2]), np.array([1, 0]), np.array([3.0, 2.0])))


def test_assemble_shuffled_stencil_128(M, ctx):
    # size-independent property at the headline size: the 128^3 7-point
    # Laplacian's 14.6M entries inserted in a seeded random order, each value
    # split into two exactly representable halves added with `+=`, assemble
    # to the generator's matrix bit for bit.
    n, rp, ci, v = M.laplacian3d(128)
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
    perm = np.random.default_rng(12).permutation(2 * len(ci))
    r2 = np.concatenate([rows, rows])[perm]
    c2 = np.concatenate([ci, ci])[perm]
    v2 = np.concatenate([0.5 * v, 0.5 * v])[perm]
    A = M.Csr.assemble(ctx, n, n, r2, c2, v2, updater=M.UPDATE_PLUS)
    got = A.download()
    assert same(got, (rp, ci, v))


@pytest.mark.parametrize("m,n", [(1, 1), (1, 7), (7, 1), (100, 100), (33, 65)])
def test_device_laplacian2d_matches_reference(M, ctx, restate, m, n):
    A = M.Csr.laplacian2d(ctx, m, n)
    L = restate.laplacian_setup(m, n)
    assert same(A.download(), L[1:])


@pytest.mark.parametrize("N", [1, 2, 16, 128])
def test_device_laplacian3d_matches_generator(M, ctx, N):
    A = M.Csr.laplacian3d(ctx, N)
    n, rp, ci, v = M.laplacian3d(N)
    assert same(A.download(), (rp, ci, v))
