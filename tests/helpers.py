"""Small helpers shared by the tests."""
import numpy as np


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def csr_eq(A, B):
    """Bit-exact equality of two (n, rp, ci, v) CSR tuples."""
    return (A[0] == B[0] and np.array_equal(A[1], B[1]) and np.array_equal(A[2], B[2])
            and np.array_equal(np.asarray(A[3]).view(np.uint64), np.asarray(B[3]).view(np.uint64)))


def dense(A):
    n, rp, ci, v = A
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(rp[i], rp[i + 1]):
            D[i, ci[j]] = v[j]
    return D


def from_dense(D):
    n = D.shape[0]
    rp, ci, v = [0], [], []
    for i in range(n):
        for j in range(n):
            if D[i, j] != 0:
                ci.append(j)
                v.append(D[i, j])
        rp.append(len(ci))
    return (n, np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.float64))


def glibc_rand_sequence(count):
    """The first `count` values of glibc rand() with the default seed (1), as
    the reference's ilu_0 tests draw them (unseeded rand())."""
    import ctypes
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1)
    return [libc.rand() for _ in range(count)]


def ilu_test_matrix(n=3):
    """setup() of libs/numeric/itl/test/ilu_0_test.cpp:16-28: A = I, then 2n
    draws r = rand()%n, c = rand()%n with A[r][c] += -1, A[r][r] += 1."""
    seq = glibc_rand_sequence(4 * n)
    D = np.eye(n)
    k = 0
    for _ in range(2 * n):
        r = seq[k] % n
        c = seq[k + 1] % n
        k += 2
        D[r, c] += -1
        D[r, r] += 1
    return D


def dense_ilu0(D):
    """dense_ilu_0 of the reference tests (ilu_0_test.cpp:31-49)."""
    LU = D.copy()
    n = LU.shape[0]
    for i in range(1, n):
        for k in range(i):
            LU[i, k] /= LU[k, k]
            for j in range(k + 1, n):
                if LU[i, j] != 0:
                    LU[i, j] -= LU[i, k] * LU[k, j]
    return LU


def dense_ic0(D):
    """dense_ic_0 of ic_0_cg_test.cpp:17-40 (textbook IC(0) on upper(A))."""
    U = np.triu(D).copy()
    n = U.shape[0]
    for k in range(n):
        dia = U[k, k] = np.sqrt(U[k, k])
        for i in range(k + 1, n):
            d = U[k, i] = U[k, i] / dia
            for j in range(k + 1, i + 1):
                if U[j, i] != 0.0:
                    U[j, i] -= d * U[k, j]
    return U
