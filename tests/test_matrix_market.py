"""Matrix Market input (<mtlgpu/matrix_market.hpp>, after mtl/io/matrix_market.hpp).

CPU: the reader on its own (symmetric expansion, skew signs, pattern zeros,
last-wins duplicates, column-major arrays, rejected input) and, where it was
built, the program that runs the reference's own reader on the same inputs.
GPU: a matrix read from a Matrix Market file solved with CG + IC(0) against
the oracle."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "cpp", "_build")


def read(path):
    exe = os.path.join(BUILD, "mm_read")
    if not os.path.exists(exe):
        subprocess.run(["make", "-C", os.path.join(ROOT, "tests", "cpp")], check=True,
                       capture_output=True)
    p = subprocess.run([exe, str(path)], capture_output=True, text=True)
    return p.returncode, (json.loads(p.stdout) if p.returncode == 0 else p.stderr)


def write(tmp_path, name, text):
    f = tmp_path / name
    f.write_text(text)
    return f


def test_symmetric_skew_pattern_duplicates_array(tmp_path):
    rc, A = read(write(tmp_path, "s.mtx", "%%MatrixMarket matrix coordinate real symmetric\n"
                                          "% comment\n3 3 3\n1 1 4\n3 1 -1\n2 2 5\n"))
    assert rc == 0 and A["starts"] == [0, 2, 3, 4] and A["indices"] == [0, 2, 1, 0]
    assert A["data"] == [4, -1, 5, -1]
    rc, A = read(write(tmp_path, "k.mtx", "%%MatrixMarket matrix coordinate real skew-symmetric\n"
                                          "2 2 1\n2 1 1.5\n"))
    assert A["indices"] == [1, 0] and A["data"] == [-1.5, 1.5]
    rc, A = read(write(tmp_path, "p.mtx", "%%MatrixMarket matrix coordinate pattern general\n"
                                          "2 2 2\n1 2\n2 1\n"))
    assert A["data"] == [0, 0] and A["indices"] == [1, 0]
    rc, A = read(write(tmp_path, "d.mtx", "%%MatrixMarket matrix coordinate real general\n"
                                          "2 2 3\n1 1 1\n1 1 3\n2 2 5\n"))
    assert A["data"] == [3, 5]
    rc, A = read(write(tmp_path, "a.mtx", "%%MatrixMarket matrix array real general\n"
                                          "2 2\n1\n2\n3\n4\n"))
    assert A["starts"] == [0, 2, 4] and A["data"] == [1, 3, 2, 4]


def test_rejected_input(tmp_path):
    # rejected as the reference's reader rejects them (the header's object and
    # field are compared as written; there is no 'double' field)
    for text in ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n",
                 "%%NotMarket matrix coordinate real general\n1 1 1\n1 1 1\n",
                 "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n",
                 "%%MatrixMarket matrix coordinate double general\n1 1 1\n1 1 1\n",
                 "%%MatrixMarket Matrix coordinate real general\n1 1 1\n1 1 1\n",
                 "%%MatrixMarket matrix coordinate Real general\n1 1 1\n1 1 1\n"):
        rc, err = read(write(tmp_path, "bad.mtx", text))
        assert rc == 1 and err


def test_integer_entries_read_as_integers(tmp_path):
    # "1.5" in an integer file: 1 is read, and the reader stops at ".5"
    rc, A = read(write(tmp_path, "i.mtx", "%%MatrixMarket matrix coordinate integer general\n"
                                          "2 2 2\n1 1 1.5\n2 2 3\n"))
    assert rc == 0 and A["starts"] == [0, 1, 1] and A["data"] == [1]


def test_same_as_reference_reader():
    exe = os.path.join(BUILD, "mm_parity")
    if not os.path.exists(exe):
        pytest.skip("built only where the MTL4 headers are present")
    p = subprocess.run([exe], capture_output=True, text=True)
    lines = [json.loads(l) for l in p.stdout.splitlines()]
    assert p.returncode == 0 and len(lines) == 12 and all(l["same"] for l in lines), lines


@pytest.mark.gpu
def test_solve_matrix_read_from_file(M, ctx, restate, tmp_path):
    n0, rp, ci, v = M.laplacian2d(30, 30)
    rows = np.repeat(np.arange(n0), np.diff(rp))
    low = ci <= rows       # lower triangle, written as a symmetric file
    text = "%%MatrixMarket matrix coordinate real symmetric\n"
    text += "{} {} {}\n".format(n0, n0, int(low.sum()))
    text += "".join("%d %d %.17g\n" % (r + 1, c + 1, x)
                    for r, c, x in zip(rows[low], ci[low], v[low]))
    rc, A = read(write(tmp_path, "lap.mtx", text))
    assert rc == 0
    assert np.array_equal(A["starts"], rp) and np.array_equal(A["indices"], ci)
    assert np.array_equal(A["data"], v)
    b = M.csr_mult((n0, rp, ci, v), M.uniform(n0, 2))
    dA = M.Csr(ctx, np.array(A["starts"], np.int32), np.array(A["indices"], np.int32),
               np.array(A["data"]))
    P = M.Pc(dA, "ic0")
    dx, db = ctx.to_device(np.zeros(n0)), ctx.to_device(b)
    st, res, _ = M.solve("cg", dA, P, dx, db, rtol=1e-10, max_iter=1000)
    ref = restate.solve("cg", "ic0", (n0, rp, ci, v), b, rtol=1e-10, max_iter=1000)
    assert st == M.OK and abs(res.iterations - ref["iterations"]) <= 2


def test_reference_fixtures_match_golden(golden):
    # the arrays stored in tests/golden are what the reader gives on the
    # reference's own fixture files (checked where the MTL4 tree is present)
    root = os.environ.get("REFERENCE_ROOT", "")
    d = os.path.join(root, "libs", "numeric", "mtl", "test", "matrix_market")
    if not root or not os.path.isdir(d):
        pytest.skip("REFERENCE_ROOT does not name the MTL4 tree here")
    for name in ("bcsstk01", "bcspwr02", "jgl009", "plskz362", "dense_read"):
        rc, A = read(os.path.join(d, name + ".mtx"))
        assert rc == 0, name
        k = "mtx_" + name
        assert np.array_equal(A["starts"], golden[k + "_rp"]), name
        assert np.array_equal(A["indices"], golden[k + "_ci"]), name
        assert np.array_equal(np.array(A["data"]), golden[k + "_v"]), name
