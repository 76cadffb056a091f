"""The C-ABI library loads and exports every entry point its headers declare
(no compute calls: runs without a GPU); fixture generators behave as
documented."""
import ctypes
import os
import re
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mtl4-mirror_b200", "lib", "libmtlgpu.so")


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b(mtlgpu_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB)
    lib = ctypes.CDLL(LIB)
    exported = set(re.findall(r" T (mtlgpu_\w+)", subprocess.run(["nm", "-D", LIB],
                                                                 capture_output=True,
                                                                 text=True).stdout))
    declared = declared_symbols()
    assert len(declared) > 40
    missing = sorted(declared - exported)
    assert not missing, missing
    for name in declared:
        assert hasattr(lib, name)


def test_no_hidden_extra_exports():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    ours = [l.split()[-1] for l in out.splitlines() if " T " in l]
    assert all(n.startswith("mtlgpu_") for n in ours if not n.startswith("_")), ours[:10]


def test_status_strings(M):
    L = M.lib()
    assert L.mtlgpu_status_string(1) == b"too many iterations"
    assert L.mtlgpu_abi_version() == 1


def test_iter_params_default(M):
    p = M.IterParams()
    M.lib().mtlgpu_iter_params_default(ctypes.byref(p))
    assert p.max_iter == 1000 and p.rtol == 1e-10 and p.norm_r0 == -1.0


def test_laplacian2d_matches_reference(M, reference):
    for (m, n) in [(3, 3), (5, 5), (100, 100), (7, 13), (1, 4)]:
        a = M.laplacian2d(m, n)
        b = reference.laplacian_setup(m, n)
        assert all(np.array_equal(x, y) for x, y in zip(a[1:], b[1:]))


def test_fixture_sizes_and_properties(M):
    A = M.laplacian3d(9)
    assert len(A[2]) == 7 * 9 ** 3 - 6 * 9 ** 2
    C = M.convdiff27(7, 2)
    n, rp, ci, v = C
    assert len(ci) == (3 * 7 - 2) ** 3
    rows = np.repeat(np.arange(n), np.diff(rp))
    diag = v[ci == rows]
    offsum = np.bincount(rows[ci != rows], np.abs(v[ci != rows]), minlength=n)
    assert np.all(diag > offsum)                  # strictly diagonally dominant
    D = np.zeros((n, n))
    D[rows, ci] = v
    assert not np.allclose(D, D.T)                # unsymmetric
    G = M.random_graph(300, 10.0, 1e-2, 3)
    n, rp, ci, v = G
    rows = np.repeat(np.arange(n), np.diff(rp))
    D = np.zeros((n, n))
    D[rows, ci] = v
    assert np.allclose(D, D.T) and np.all(np.linalg.eigvalsh(D) > 0)
    F = M.fv2d(20)
    assert len(F[2]) == 5 * 400 - 4 * 20
    for X in (A, C, G, F):
        n, rp, ci, _ = X
        for i in range(0, n, max(1, n // 50)):
            row = ci[rp[i]:rp[i + 1]]
            assert np.all(np.diff(row) > 0) and i in row


def test_generators_are_deterministic(M):
    assert np.array_equal(M.uniform(100, 1), M.uniform(100, 1))
    assert not np.array_equal(M.uniform(100, 1), M.uniform(100, 2))
    u = M.uniform(200000, 11)
    assert u.min() >= -1 and u.max() <= 1 and abs(u.mean()) < 0.01
    g = M.normal(200000, 12)
    assert abs(g.mean()) < 0.01 and abs(g.std() - 1) < 0.01
