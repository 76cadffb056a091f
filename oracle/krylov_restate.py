"""Restatement of the other ITL Krylov methods in numpy.  TEST INFRASTRUCTURE ONLY.

bicg, cgs, bicgstab_2, bicgstab_ell, tfqmr, qmr, idr_s and gmres, each
following the reference loop it names (file:line inside the MTL4 tree), with
basic_iteration's termination test (itl/iteration/basic_iteration.hpp:51-93).
The matrix product and the preconditioners come from the C restatement
(oracle/restate.c: or_spmv, or_pc_apply); the small dense algebra (the
orthogonalisation factors of bicgstab_ell, the LU solves of idr_s and gmres,
gmres's Givens rotations) is restated here.  Vector arithmetic is numpy's, so
results agree with the reference to rounding, not bit for bit;
tests/test_krylov_oracle.py pins iteration counts, error codes, residual
histories and solutions against the reference compiled from its headers.

Only the tests import this module.
"""
from __future__ import annotations

import ctypes

import numpy as np

import oracle as _oracle


class Singular(Exception):
    """mtl::matrix_singular (mtl/utility/exception.hpp)."""


class Iteration:
    """basic_iteration(norm_r0, max_iter, rtol, atol); records every residual
    passed to finished()."""

    def __init__(self, norm_r0, max_iter, rtol, atol=0.0):
        self.error, self.i = 0, 0
        self.norm_r0, self.max_iter, self.rtol, self.atol = norm_r0, max_iter, rtol, atol
        self.resid = 0.0
        self.is_finished = False
        self.history = []

    def converged(self, r):
        self.resid = r
        if self.norm_r0 == 0:
            return r <= self.atol
        return r <= self.rtol * self.norm_r0 or r <= self.atol

    def check_max(self):
        if self.i >= self.max_iter:
            self.error, self.is_finished = 1, True
        return self.is_finished

    def finished(self, r):
        """finished(r) for a vector (two_norm) or a scalar residual."""
        r = float(np.sqrt(np.dot(r, r))) if isinstance(r, np.ndarray) else float(r)
        self.history.append(r)
        if self.converged(r):
            self.is_finished = True
            return True
        return self.check_max()

    def first(self):
        return self.i <= 1

    def fail(self, code):
        self.error = code
        return code


def glibc_rand_columns(count, length):
    """mtl::mat::random on a multi_vector of `count` vectors of `length`
    (mtl/operation/random.hpp:27-37, 45-50, 70-75, 105-110): the matrix-level
    seed object takes srand(17), then each vector k creates its own and is
    filled from srand(17 * (k + 2)) and rand() -- in a process whose seed
    counter starts at 0."""
    libc = ctypes.CDLL("libc.so.6")
    out = np.empty((count, length))
    for k in range(count):
        libc.srand(17 * (k + 2))
        out[k] = [libc.rand() for _ in range(length)]
    return out


def lu_solve(Mat, b):
    """lu_solve (mtl/operation/lu.hpp:58-84, 121-138): LU with partial pivoting
    (the first largest magnitude in the column), matrix_singular for a zero
    pivot before the last row, then the two triangular solves."""
    A = np.array(Mat, dtype=np.float64, copy=True)
    n = A.shape[0]
    P = np.arange(n)
    for i in range(n - 1):
        rmax = i + int(np.argmax(np.abs(A[i:, i])))
        A[[i, rmax]] = A[[rmax, i]]
        P[[i, rmax]] = P[[rmax, i]]
        if abs(A[i, i]) <= 0:
            raise Singular()
        A[i + 1:, i] /= A[i, i]
        A[i + 1:, i + 1:] -= np.outer(A[i + 1:, i], A[i, i + 1:])
    y = np.array(b, dtype=np.float64)[P]
    for r in range(n):                       # unit lower
        y[r] -= np.dot(A[r, :r], y[:r])
    x = np.zeros(n)
    for r in range(n - 1, -1, -1):           # upper
        x[r] = (y[r] - np.dot(A[r, r + 1:], x[r + 1:])) / A[r, r]
    return x


class Krylov:
    """The methods on CSR A = (n, rp, ci, v) with left / right
    preconditioners named as in oracle.PC_NAMES."""

    def __init__(self, A, pc_left="identity", pc_right="identity"):
        self.A = A
        self.S = _oracle.Restatement()
        self.pl, self.pr = pc_left, pc_right
        n, rp, ci, v = A
        At = self.S.transpose((n, rp, ci, v))
        self.AT = (n,) + tuple(At[1:]) if len(At) == 4 else At

    def mv(self, x):
        return self.S.spmv(self.A, x)

    def mvT(self, x):
        return self.S.spmv(self.AT, x)

    def L(self, r, adjoint=False):
        return self.S.pc_apply(self.pl, self.A, r, adjoint)

    def R(self, r, adjoint=False):
        return self.S.pc_apply(self.pr, self.A, r, adjoint)

    # itl/krylov/bicg.hpp:22-63
    def bicg(self, x, b, it):
        r = b - self.mv(x)
        rt = r.copy()
        p = pt = None
        rho_2 = 0.0
        while not it.finished(r):
            it.i += 1
            z = self.L(r)
            zt = self.L(rt, True)
            rho_1 = np.dot(zt, z)
            if rho_1 == 0.0:
                return it.fail(2)
            if it.first():
                p, pt = z.copy(), zt.copy()
            else:
                beta = rho_1 / rho_2
                p = z + beta * p
                pt = zt + beta * pt
            q = self.mv(p)
            qt = self.mvT(pt)
            alpha = rho_1 / np.dot(pt, q)
            x += alpha * p
            r -= alpha * q
            rt -= alpha * qt
            rho_2 = rho_1
        return it.error

    # itl/krylov/cgs.hpp:23-65
    def cgs(self, x, b, it):
        r = b - self.mv(x)
        rtilde = r.copy()
        p = q = u = None
        rho_2 = 0.0
        while not it.finished(r):
            it.i += 1
            rho_1 = np.dot(rtilde, r)
            if rho_1 == 0.0:
                it.fail(2)             # no return: the reference carries on
            if it.first():
                u = r.copy()
                p = r.copy()
            else:
                beta = rho_1 / rho_2
                u = r + beta * q
                p = u + beta * (q + beta * p)
            vhat = self.mv(self.L(p))
            alpha = rho_1 / np.dot(rtilde, vhat)
            q = u - alpha * vhat
            u = u + q
            uhat = self.L(u)
            x += alpha * uhat
            qhat = self.mv(uhat)
            r -= alpha * qhat
            rho_2 = rho_1
        return it.error

    # itl/krylov/bicgstab_ell.hpp:37-132 (right=True) and bicgstab_2.hpp:33-131
    def bicgstab_ell(self, x, b, it, l, right=True):
        if len(b) == 0:
            raise ValueError("empty rhs vector")
        Rs = self.R if right else (lambda v, adjoint=False: v.copy())
        x0 = np.zeros_like(x)
        rh = [None] * (l + 1)
        uh = [np.zeros_like(x) for _ in range(l + 1)]
        rh[0] = b.copy()
        if np.sqrt(np.dot(x, x)) != 0.0:
            rh[0] -= self.mv(x)
            x0 = x.copy()
            x[:] = 0.0
        r0t = rh[0] / np.sqrt(np.dot(rh[0], rh[0]))
        rh[0] = self.L(rh[0])
        for k in range(1, l + 1):
            rh[k] = np.zeros_like(x)
        rho_0, alpha, omega = 1.0, 0.0, 1.0
        tau = np.zeros((l + 1, l + 1))
        gamma, gamma_a, gamma_aa = np.zeros(l + 1), np.zeros(l + 1), np.zeros(l + 1)

        def done():
            xs = Rs(x)
            x[:] = xs + x0
            return it.error

        while not it.finished(rh[0]):
            it.i += 1
            rho_0 = -omega * rho_0
            for j in range(l):
                rho_1 = np.dot(r0t, rh[j])
                beta = alpha * rho_1 / rho_0
                rho_0 = rho_1
                for i in range(j + 1):
                    uh[i] = rh[i] - beta * uh[i]
                y = self.mv(Rs(uh[j]))
                uh[j + 1] = self.L(y)
                Gamma = np.dot(r0t, uh[j + 1])
                alpha = rho_0 / Gamma
                for i in range(j + 1):
                    rh[i] = rh[i] - alpha * uh[i + 1]
                if it.finished(rh[j]):
                    return done()
                rh[j + 1] = Rs(rh[j])
                y = self.mv(rh[j + 1])
                rh[j + 1] = self.L(y)
                x += alpha * uh[0]
            # orthogonalize_factors(r_hat[1..l]) (mtl/operation/orth.hpp:53-88)
            tail = rh[1:]
            tau[1:, 1:] = 0.0
            tau[1, 1] = np.dot(tail[0], tail[0])
            for jj in range(1, l):
                for ii in range(jj):
                    t = np.dot(tail[ii], tail[jj]) / tau[ii + 1, ii + 1]
                    tau[ii + 1, jj + 1] = t
                    tail[jj] = tail[jj] - t * tail[ii]
                tau[jj + 1, jj + 1] = np.dot(tail[jj], tail[jj])
            rh[1:] = tail
            for j in range(1, l + 1):
                gamma_a[j] = np.dot(rh[j], rh[0]) / tau[j, j]
            gamma[l] = gamma_a[l]
            omega = gamma[l]
            if omega == 0.0:
                it.fail(3)
                return it.error
            for j in range(l - 1, 0, -1):
                s = 0.0
                for i in range(j + 1, l + 1):
                    s += tau[j, i] * gamma[i]
                gamma[j] = gamma_a[j] - s
            for a in range(l - 1):           # strict_upper(tau[1..l-1][1..l-1]) * gamma[2..l] + gamma[2..l]
                s = 0.0
                for bb in range(a + 1, l - 1):
                    s += tau[1 + a, 1 + bb] * gamma[2 + bb]
                gamma_aa[1 + a] = s + gamma[2 + a]
            x += gamma[1] * rh[0]
            rh[0] = rh[0] - gamma_a[l] * rh[l]
            uh[0] = uh[0] - gamma[l] * uh[l]
            for j in range(1, l):
                uh[0] = uh[0] - gamma[j] * uh[j]
                x += gamma_aa[j] * rh[j]
                rh[0] = rh[0] - gamma_a[j] * rh[j]
        return done()

    # itl/krylov/tfqmr.hpp:26-100
    def tfqmr(self, x, b, it):
        if len(b) == 0:
            raise ValueError("empty rhs vector")
        theta = eta = 0.0
        rt = b - self.mv(self.R(x))
        r = self.L(rt)
        d = np.zeros_like(x)
        if it.finished(rt):
            return it.error
        y1 = r.copy()
        w = r.copy()
        rt = self.mv(self.R(y1))
        u1 = self.L(rt)
        v = u1.copy()
        tau = np.sqrt(np.dot(r, r))
        rho = tau * tau
        u2 = y2 = None
        while not it.finished(tau):
            it.i += 1
            sigma = np.dot(r, v)
            if sigma == 0.0:
                return it.fail(1)
            alpha = rho / sigma
            for j in (1, 2):
                if j == 1:
                    w = w - alpha * u1
                    d = y1 + (theta * theta * eta / alpha) * d
                else:
                    y2 = y1 - alpha * v
                    rt = self.mv(self.R(y2))
                    u2 = self.L(rt)
                    w = w - alpha * u2
                    d = y2 + (theta * theta * eta / alpha) * d
                theta = np.sqrt(np.dot(w, w)) / tau
                c = 1.0 / np.sqrt(1.0 + theta * theta)
                tau *= theta * c
                eta = c * c * alpha
                x += eta * d
            if rho == 0.0:
                return it.fail(1)
            rhon = np.dot(r, w)
            beta = rhon / rho
            rho = rhon
            y1 = w + beta * y2
            rt = self.mv(self.R(y1))
            u1 = self.L(rt)
            v = u1 + beta * (u2 + beta * v)
        x[:] = self.R(x)
        return it.error

    # itl/krylov/qmr.hpp:24-109
    def qmr(self, x, b, it):
        if len(b) == 0:
            raise ValueError("empty rhs vector")
        gamma, eta, ep, theta = 1.0, -1.0, 1.0, 0.0
        r = b - self.mv(x)
        v_tld = r.copy()
        y = self.L(v_tld)
        w_tld = r.copy()
        z = self.R(w_tld, True)
        if it.finished(r):
            return it.error
        rho = np.sqrt(np.dot(y, y))
        xi = np.sqrt(np.dot(z, z))
        p = q = d = s = None
        while not it.finished(rho):
            it.i += 1
            if rho == 0.0:
                return it.fail(1)
            if xi == 0.0:
                return it.fail(2)
            v = v_tld / rho
            y = y / rho
            w = w_tld / xi
            z = z / xi
            delta = np.dot(z, y)
            if delta == 0.0:
                return it.fail(3)
            y_tld = self.R(y)
            z_tld = self.L(z, True)
            if it.first():
                p, q = y_tld.copy(), z_tld.copy()
            else:
                p = y_tld - ((xi * delta) / ep) * p
                q = z_tld - ((rho * delta) / ep) * q
            p_tld = self.mv(p)
            ep = np.dot(q, p_tld)
            if ep == 0.0:
                return it.fail(4)
            beta = ep / delta
            if beta == 0.0:
                return it.fail(5)
            v_tld = p_tld - beta * v
            y = self.L(v_tld)
            rho_1 = rho
            rho = np.sqrt(np.dot(y, y))
            w_tld = self.mvT(q) - beta * w
            z = self.R(w_tld, True)
            xi = np.sqrt(np.dot(z, z))
            gamma_1, theta_1 = gamma, theta
            theta = rho / (gamma_1 * beta)
            gamma = 1.0 / np.sqrt(1.0 + theta * theta)
            if gamma == 0.0:
                return it.fail(6)
            eta = -eta * rho_1 * gamma * gamma / (beta * gamma_1 * gamma_1)
            if it.first():
                d = eta * p
                s = eta * p_tld
            else:
                d = eta * p + (theta_1 * theta_1 * gamma * gamma) * d
                s = eta * p_tld + (theta_1 * theta_1 * gamma * gamma) * s
            x += d
            r -= s
        return it.error

    # itl/krylov/idr_s.hpp:30-105 (both preconditioners ignored)
    def idr_s(self, x, b, it, s):
        if len(b) == 0:
            raise ValueError("empty rhs vector")
        s = max(1, s)
        n = len(b)
        r = b - self.mv(x)
        dR, dX = np.zeros((s, n)), np.zeros((s, n))
        P = glibc_rand_columns(s, n)
        P[0] = r
        for j in range(s):                   # orth(P): Gram-Schmidt, then normalise
            for i in range(j):
                P[j] = P[j] - np.dot(P[i], P[j]) * P[i]
            P[j] = P[j] / np.sqrt(np.dot(P[j], P[j]))
        Mm = np.zeros((s, s))
        for k in range(s):
            v = self.mv(r)
            omega = np.dot(v, r) / np.dot(v, v)
            dX[k] = omega * r
            dR[k] = -omega * v
            x += dX[k]
            r = r + dR[k]
            it.i += 1
            if it.finished(r):
                return it.error
            Mm[:, k] = P @ dR[k]
        oldest = 0
        m = P @ r
        omega = 0.0
        while not it.finished(r):
            for k in range(s):
                c = lu_solve(Mm, m)
                q = -(c @ dR)
                v = r + q
                if k == 0:
                    t = self.mv(v)
                    omega = np.dot(t, v) / np.dot(t, t)
                    dR[oldest] = q - omega * t
                    dX[oldest] = omega * v - c @ dX
                else:
                    dX[oldest] = omega * v - c @ dX
                    dR[oldest] = self.mv(-dX[oldest])
                r = r + dR[oldest]
                x += dX[oldest]
                it.i += 1
                if it.finished(r):
                    return it.error
                dm = P @ dR[oldest]
                Mm[:, oldest] = dm
                m = m + dm
                oldest = (oldest + 1) % s
        return it.error

    # itl/krylov/gmres.hpp:34-119 (gmres_full) and 121-135 (restarts)
    def _givens_rows_cols(self, H, a, b, k):
        """mat::givens(H, a, b).trafo(k) (mtl/operation/givens.hpp:33-82):
        rows k, k+1 by G^T, then columns k, k+1 by G."""
        if b == 0.0:
            c, s = 1.0, 0.0
        elif abs(b) > abs(a):
            t = -a / b
            s = 1.0 / np.sqrt(1.0 + t * t)
            c = s * t
        else:
            t = -b / a
            c = 1.0 / np.sqrt(1.0 + t * t)
            s = c * t
        G = np.array([[c, s], [-s, c]])
        H[k:k + 2, :] = G.T @ H[k:k + 2, :]
        H[:, k:k + 2] = H[:, k:k + 2] @ G

    def gmres_full(self, x, b, it):
        n = len(b)
        if n == 0:
            raise ValueError("empty rhs vector")
        kmax = min(n, it.max_iter - it.i)
        r0 = b - self.mv(x)
        r = self.L(r0)
        V = np.zeros((kmax + 1, n))
        s_, c_, g = np.zeros(kmax + 1), np.zeros(kmax + 1), np.zeros(kmax + 1)
        H = np.zeros((kmax + 1, kmax))
        rho = g[0] = np.sqrt(np.dot(r, r))
        if it.finished(rho):
            return it.error
        V[0] = r / rho
        k = 0
        while k < kmax:
            va0 = self.mv(self.R(V[k]))
            V[k + 1] = self.L(va0)
            for j in range(k + 1):
                H[j, k] = np.dot(V[j], V[k + 1])
                V[k + 1] = V[k + 1] - H[j, k] * V[j]
            H[k + 1, k] = np.sqrt(np.dot(V[k + 1], V[k + 1]))
            for j in range(k + 1):
                hr = np.dot(V[k + 1], V[j])
                H[j, k] += hr
                V[k + 1] = V[k + 1] - hr * V[j]
            H[k + 1, k] = np.sqrt(np.dot(V[k + 1], V[k + 1]))
            if H[k + 1, k] != 0.0:
                V[k + 1] = V[k + 1] * (1.0 / H[k + 1, k])
            for i in range(k):
                self._givens_rows_cols(H, H[i, k - 1], H[i + 1, k - 1], i)
            nu = np.sqrt(H[k, k] * H[k, k] + H[k + 1, k] * H[k + 1, k])
            if nu != 0.0:
                c_[k] = H[k, k] / nu
                s_[k] = -H[k + 1, k] / nu
                H[k, k] = c_[k] * H[k, k] - s_[k] * H[k + 1, k]
                H[k + 1, k] = 0.0
                w1 = c_[k] * g[k] - s_[k] * g[k + 1]
                w2 = s_[k] * g[k] + c_[k] * g[k + 1]
                g[k], g[k + 1] = w1, w2
            rho = abs(g[k + 1])
            k += 1
            it.i += 1
        while k > 0 and abs(g[k - 1]) <= it.atol:
            k -= 1
        rng = k
        y = None
        while rng > 0:
            try:
                y = lu_solve(H[:rng, :rng], g[:rng])
            except Singular:
                rng -= 1
                continue
            break
        if rng == 0:
            return it.fail(2)
        x += self.R(y @ V[:rng])
        r = b - self.mv(x)
        it.finished(r)
        return it.error

    def gmres(self, x, b, it, restart):
        while True:
            inner = Iteration(it.norm_r0, min(it.i + restart, it.max_iter), it.rtol, it.atol)
            inner.i, inner.error, inner.resid = it.i, it.error, it.resid
            inner.history = it.history
            self.gmres_full(x, b, inner)
            it.i, it.resid = inner.i, inner.resid
            if inner.error > 1:
                it.error = inner.error
                it.is_finished = True
            else:
                if it.converged(it.resid):
                    it.is_finished = True
                else:
                    it.check_max()
            if it.is_finished:
                return it.error


def solve(method, A, b, pc_left="identity", pc_right="identity", param=0, x0=None,
          max_iter=1000, rtol=1e-10, atol=0.0, norm_r0=-1.0):
    """Same result dict as oracle.Reference.solve_krylov."""
    b = np.asarray(b, np.float64)
    x = np.zeros(len(b)) if x0 is None else np.array(x0, np.float64, copy=True)
    nr0 = float(np.sqrt(np.dot(b, b))) if norm_r0 < 0 else norm_r0
    it = Iteration(nr0, max_iter, rtol, atol)
    K = Krylov(A, pc_left, pc_right)
    if method == "bicg":
        err = K.bicg(x, b, it)
    elif method == "cgs":
        err = K.cgs(x, b, it)
    elif method == "bicgstab_2":
        err = K.bicgstab_ell(x, b, it, 2, right=False)
    elif method == "bicgstab_ell":
        err = K.bicgstab_ell(x, b, it, param or 8)
    elif method == "tfqmr":
        err = K.tfqmr(x, b, it)
    elif method == "qmr":
        err = K.qmr(x, b, it)
    elif method == "idr_s":
        err = K.idr_s(x, b, it, param or 8)
    elif method == "gmres":
        err = K.gmres(x, b, it, param or 8)
    else:
        raise ValueError(method)
    return dict(err=err, x=x, iterations=it.i, resid=it.resid, norm_r0=nr0,
                history=np.array(it.history))
