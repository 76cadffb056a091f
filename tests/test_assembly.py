"""The assembly oracle: the C restatement of mtl::mat::inserter (or_assemble)
pinned bit-for-bit against the reference's own inserter (compressed2D.hpp:
662-1151) compiled from its headers, and against the golden runs of it.
CPU only."""
import numpy as np
import pytest

SYNTAX_TO_OP = {0: 0, 1: 1}  # ins = v -> store, ins += v -> plus; `<<` -> class updater


def ops_from_syntax(syntax, updater):
    return np.array([SYNTAX_TO_OP.get(int(s), updater) for s in syntax], np.uint8)


def triplets(seed, nr, nc, cnt, spread):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, nr, cnt).astype(np.int32)
    cols = ((rows.astype(np.int64) * 5 + rng.integers(0, spread, cnt)) % nc).astype(np.int32)
    return rng, rows, cols, rng.normal(size=cnt)


def same(a, b):
    return (np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
            and np.array_equal(np.asarray(a[2]).view(np.uint64), np.asarray(b[2]).view(np.uint64)))


@pytest.mark.parametrize("updater", [0, 1, 2, 3])
@pytest.mark.parametrize("slot", [0, 1, 3])
def test_restatement_matches_reference_inserter(restate, reference, updater, slot):
    # slot sizes 1 and 3 push most entries through the inserter's spare map
    _, rows, cols, vals = triplets(11 + updater, 120, 90, 3000, 9)
    ref = reference.assemble(120, 90, rows, cols, vals, updater=updater, slot_size=slot)
    got = restate.assemble(120, 90, rows, cols, vals, updater=updater)
    assert same(got, ref)


def test_restatement_mixed_syntax_on_base(restate, reference):
    rng, rows, cols, vals = triplets(5, 200, 200, 5000, 7)
    base = reference.assemble(200, 200, rows[:600], cols[:600], vals[:600])
    syntax = rng.integers(0, 3, len(rows)).astype(np.uint8)
    for u in range(4):
        ref = reference.assemble(200, 200, rows, cols, vals, updater=u, base=base, syntax=syntax)
        got = restate.assemble(200, 200, rows, cols, vals, updater=u, base=base,
                               ops=ops_from_syntax(syntax, u))
        assert same(got, ref), u


def test_restatement_edge_cases(restate, reference):
    # no triplets, an empty matrix, a single row, explicit zeros kept
    for nr, nc, rows, cols, vals in [
            (5, 5, [], [], []),
            (0, 0, [], [], []),
            (1, 8, [0, 0, 0, 0], [7, 0, 7, 3], [1.0, 2.0, 3.0, 0.0]),
            (4, 4, [3, 3, 3], [3, 3, 3], [0.0, 0.0, 0.0])]:
        for u in range(4):
            ref = reference.assemble(nr, nc, rows, cols, vals, updater=u)
            got = restate.assemble(nr, nc, rows, cols, vals, updater=u)
            assert same(got, ref), (nr, nc, u)


def test_restatement_rejects_out_of_range(restate):
    with pytest.raises(IndexError):
        restate.assemble(4, 4, [0, 4], [0, 0], [1.0, 1.0])
    with pytest.raises(IndexError):
        restate.assemble(4, 4, [0, 1], [0, -1], [1.0, 1.0])


def test_restatement_laplacian_by_insertion(restate, reference):
    # laplacian_setup.hpp:30-41 inserts diagonal first, then the neighbours
    m, n = 13, 17
    rows, cols, vals = [], [], []
    for i in range(m):
        for j in range(n):
            r = i * n + j
            ent = [(r, 4.0)]
            if j < n - 1:
                ent.append((r + 1, -1.0))
            if i < m - 1:
                ent.append((r + n, -1.0))
            if j > 0:
                ent.append((r - 1, -1.0))
            if i > 0:
                ent.append((r - n, -1.0))
            for c, w in ent:
                rows.append(r), cols.append(c), vals.append(w)
    got = restate.assemble(m * n, m * n, rows, cols, vals)
    L = reference.laplacian_setup(m, n)
    assert same(got, L[1:])


@pytest.mark.parametrize("case", ["u0", "u1", "u2", "u3", "mix"])
def test_restatement_matches_golden(restate, golden, case):
    nr, nc = (int(x) for x in golden["asm_shape"])
    rows, cols, vals = golden["asm_rows"], golden["asm_cols"], golden["asm_vals"]
    if case == "mix":
        base = (golden["asm_base_rp"], golden["asm_base_ci"], golden["asm_base_v"])
        got = restate.assemble(nr, nc, rows, cols, vals, updater=1, base=base,
                               ops=ops_from_syntax(golden["asm_mix_syntax"], 1))
    else:
        got = restate.assemble(nr, nc, rows, cols, vals, updater=int(case[1]))
    ref = (golden[f"asm_{case}_rp"], golden[f"asm_{case}_ci"], golden[f"asm_{case}_v"])
    assert same(got, ref)
