"""ctypes binding of libmtlgpu's C ABI (include/mtlgpu.h, include/mtlgpu_fixtures.h).

This is the binding a Python caller of the library uses; the tests and the
benchmark drive the library through it, so every call crosses the same C
boundary a C, C++ or FFI user crosses.  Device buffers are ``DeviceArray``
objects (memory from ``mtlgpu_malloc``); numpy arrays are host buffers.

The library must be built (``make -C mtl4-mirror_b200``); loading fails
loudly otherwise -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libmtlgpu.so")
FIX_PATH = os.path.join(PKG, "lib", "libmtlgpu_fixtures.so")

OK, MAX_ITER, INVALID_ARG, NOT_SQUARE, MISSING_DIAGONAL, ZERO_PIVOT, BREAKDOWN, TIMEOUT, \
    INTERRUPTED, CUDA_ERROR, NOT_SORTED, INDEX_RANGE, OUT_OF_MEMORY, INCOMPATIBLE_SIZE, \
    NOT_SUPPORTED = range(15)
FP64, FP32 = 0, 1
PC_IDENTITY, PC_DIAGONAL, PC_ILU0, PC_IC0 = range(4)
PC_KINDS = {"identity": PC_IDENTITY, "diagonal": PC_DIAGONAL, "ilu0": PC_ILU0, "ic0": PC_IC0}
CG, BICGSTAB, BICG, CGS, BICGSTAB_2, BICGSTAB_ELL, TFQMR, QMR, IDR_S, GMRES = range(10)
METHODS = {"cg": CG, "bicgstab": BICGSTAB, "bicg": BICG, "cgs": CGS, "bicgstab_2": BICGSTAB_2,
           "bicgstab_ell": BICGSTAB_ELL, "tfqmr": TFQMR, "qmr": QMR, "idr_s": IDR_S,
           "gmres": GMRES}
SOLVE_FP64, SOLVE_MIXED = 0, 1
LOWER, UPPER = 0, 1
UPDATE_STORE, UPDATE_PLUS, UPDATE_MINUS, UPDATE_TIMES = range(4)

_vp = C.c_void_p


class MtlgpuError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = _lib().mtlgpu_status_string(status).decode() if _LIB else str(status)
        super().__init__(f"{what}: {msg} ({status})" if what else f"{msg} ({status})")


class IterParams(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("rtol", C.c_double), ("atol", C.c_double),
                ("norm_r0", C.c_double), ("mode", C.c_int), ("inner_rtol", C.c_double),
                ("inner_max_iter", C.c_int), ("max_outer", C.c_int),
                ("h_resid_history", C.POINTER(C.c_double)), ("history_cap", C.c_int),
                ("h_interrupt", C.POINTER(C.c_int))]


class IterResult(C.Structure):
    _fields_ = [("error", C.c_int), ("status", C.c_int), ("iterations", C.c_int),
                ("outer_iterations", C.c_int), ("resid", C.c_double), ("norm_r0", C.c_double),
                ("true_resid", C.c_double), ("history_len", C.c_int),
                ("kernel_launches", C.c_longlong)]


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libmtlgpu not built: {LIB_PATH} missing (make -C mtl4-mirror_b200)")
        L = C.CDLL(LIB_PATH)
        L.mtlgpu_status_string.restype = C.c_char_p
        L.mtlgpu_last_error.restype = C.c_char_p
        L.mtlgpu_ctx_stream.restype = _vp
        L.mtlgpu_ctx_set_spin_limit.argtypes = [_vp, C.c_longlong]
        L.mtlgpu_malloc.argtypes = [_vp, C.c_size_t, C.POINTER(_vp)]
        L.mtlgpu_free.argtypes = [_vp, _vp]
        L.mtlgpu_memcpy_h2d.argtypes = [_vp, _vp, _vp, C.c_size_t]
        L.mtlgpu_memcpy_d2h.argtypes = [_vp, _vp, _vp, C.c_size_t]
        L.mtlgpu_spmv.argtypes = [_vp, _vp, _vp, C.c_double, C.c_double]
        L.mtlgpu_cg_direction_product.argtypes = [_vp, C.c_int, _vp, C.c_double, _vp, _vp, _vp,
                                                  _vp]
        L.mtlgpu_axpy.argtypes = [_vp, C.c_int, C.c_double, _vp, _vp]
        L.mtlgpu_xpay.argtypes = [_vp, C.c_int, _vp, C.c_double, _vp]
        L.mtlgpu_dot.argtypes = [_vp, C.c_int, _vp, _vp, C.POINTER(C.c_double)]
        L.mtlgpu_two_norm.argtypes = [_vp, C.c_int, _vp, C.POINTER(C.c_double)]
        L.mtlgpu_unary_dot.argtypes = [_vp, C.c_int, _vp, C.POINTER(C.c_double)]
        L.mtlgpu_csr_assemble.argtypes = [_vp, _vp, C.c_int, C.c_int, C.c_longlong, _vp, _vp,
                                          _vp, _vp, C.c_int, C.POINTER(_vp)]
        L.mtlgpu_csr_laplacian2d.argtypes = [_vp, C.c_int, C.c_int, C.POINTER(_vp)]
        L.mtlgpu_csr_laplacian3d.argtypes = [_vp, C.c_int, C.POINTER(_vp)]
        _LIB = L
    return _LIB


_FIX = None


def _fix():
    """libmtlgpu_fixtures: the seeded generators alone (include/mtlgpu_fixtures.h,
    no CUDA), so that building inputs never maps the solver library."""
    global _FIX
    if _FIX is None:
        if not os.path.exists(FIX_PATH):
            raise OSError(f"libmtlgpu_fixtures not built: {FIX_PATH} missing "
                          "(make -C mtl4-mirror_b200)")
        L = C.CDLL(FIX_PATH)
        for name in ("mtlgpu_gen_laplacian2d", "mtlgpu_gen_laplacian3d", "mtlgpu_gen_convdiff27",
                     "mtlgpu_gen_random_graph", "mtlgpu_gen_fv2d", "mtlgpu_gen_graph_batch"):
            getattr(L, name).restype = C.c_longlong
        L.mtlgpu_gen_convdiff27.argtypes = [C.c_int, C.c_uint64, _vp, _vp, _vp]
        L.mtlgpu_gen_random_graph.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64, _vp,
                                              _vp, _vp]
        L.mtlgpu_gen_fv2d.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64, _vp, _vp, _vp]
        L.mtlgpu_gen_graph_batch.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                             C.c_double, C.c_uint64, _vp, _vp, _vp, _vp]
        L.mtlgpu_gen_uniform.argtypes = [C.c_longlong, C.c_uint64, C.c_double, C.c_double, _vp]
        L.mtlgpu_gen_normal.argtypes = [C.c_longlong, C.c_uint64, _vp]
        _FIX = L
    return _FIX


def lib():
    return _lib()


def check(status, what=""):
    if status != OK:
        raise MtlgpuError(status, what)


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


# ---------------------------------------------------------------------------
class Context:
    def __init__(self, device=0, stream=None):
        self.h = _vp()
        if stream is None:
            check(_lib().mtlgpu_ctx_create(device, C.byref(self.h)), "ctx_create")
        else:
            check(_lib().mtlgpu_ctx_create_on_stream(device, _vp(stream), C.byref(self.h)),
                  "ctx_create_on_stream")

    @property
    def stream(self):
        return _lib().mtlgpu_ctx_stream(self.h)

    def synchronize(self):
        check(_lib().mtlgpu_ctx_synchronize(self.h))

    def set_spin_limit(self, polls):
        check(_lib().mtlgpu_ctx_set_spin_limit(self.h, int(polls)))

    def last_error(self):
        return _lib().mtlgpu_last_error(self.h).decode()

    def close(self):
        if self.h:
            _lib().mtlgpu_ctx_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # device memory -------------------------------------------------------
    def array(self, n, dtype=np.float64):
        return DeviceArray(self, n, dtype)

    def to_device(self, a):
        a = np.ascontiguousarray(a)
        d = DeviceArray(self, a.size, a.dtype)
        d.upload(a)
        return d

    def dot(self, x, y):
        r = C.c_double()
        check(_lib().mtlgpu_dot(self.h, x.n, x.ptr, y.ptr, C.byref(r)), "dot")
        return r.value

    def two_norm(self, x):
        r = C.c_double()
        check(_lib().mtlgpu_two_norm(self.h, x.n, x.ptr, C.byref(r)), "two_norm")
        return r.value

    def unary_dot(self, x):
        r = C.c_double()
        check(_lib().mtlgpu_unary_dot(self.h, x.n, x.ptr, C.byref(r)), "unary_dot")
        return r.value

    def axpy(self, alpha, x, y):
        check(_lib().mtlgpu_axpy(self.h, x.n, float(alpha), x.ptr, y.ptr), "axpy")

    def xpay(self, x, beta, y):
        check(_lib().mtlgpu_xpay(self.h, x.n, x.ptr, float(beta), y.ptr), "xpay")


class DeviceArray:
    def __init__(self, ctx, n, dtype=np.float64):
        self.ctx = ctx
        self.n = int(n)
        self.dtype = np.dtype(dtype)
        self.ptr = _vp()
        check(_lib().mtlgpu_malloc(ctx.h, max(1, self.n) * self.dtype.itemsize,
                                   C.byref(self.ptr)), "malloc")

    @property
    def nbytes(self):
        return self.n * self.dtype.itemsize

    def upload(self, a):
        a = np.ascontiguousarray(a, self.dtype)
        assert a.size == self.n
        check(_lib().mtlgpu_memcpy_h2d(self.ctx.h, self.ptr, _p(a), self.nbytes), "h2d")

    def download(self, out=None):
        out = np.empty(self.n, self.dtype) if out is None else out
        check(_lib().mtlgpu_memcpy_d2h(self.ctx.h, _p(out), self.ptr, self.nbytes), "d2h")
        return out

    def free(self):
        if self.ptr:
            _lib().mtlgpu_free(self.ctx.h, self.ptr)
            self.ptr = _vp()

    def __del__(self):
        try:
            if self.ctx.h:
                self.free()
        except Exception:
            pass


class Csr:
    """Device CSR handle (replaces compressed2D on the solve path)."""

    def __init__(self, ctx, rp, ci, v, n_cols=None):
        self.ctx = ctx
        rp = np.ascontiguousarray(rp, np.int32)
        ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        self.n = len(rp) - 1
        self.n_cols = self.n if n_cols is None else n_cols
        self.nnz = len(ci)
        self.h = _vp()
        st = _lib().mtlgpu_csr_create(ctx.h, self.n, self.n_cols, self.nnz, _p(rp), _p(ci), _p(v),
                                      C.byref(self.h))
        check(st, "csr_create")

    @classmethod
    def _adopt(cls, ctx, h):
        A = cls.__new__(cls)
        A.ctx, A.h = ctx, h
        n, m, nnz = C.c_int(), C.c_int(), C.c_int()
        check(_lib().mtlgpu_csr_info(h, C.byref(n), C.byref(m), C.byref(nnz)), "csr_info")
        A.n, A.n_cols, A.nnz = n.value, m.value, nnz.value
        return A

    @classmethod
    def assemble(cls, ctx, n_rows, n_cols, rows, cols, vals, ops=None, updater=UPDATE_STORE,
                 base=None):
        """mtl::mat::inserter on the device (mtlgpu_csr_assemble): triplets
        (device arrays, or numpy arrays uploaded here) inserted in order into
        an empty n_rows x n_cols matrix, or into a copy of `base`."""
        keep = []

        def dev(a, dt):
            if a is None or isinstance(a, DeviceArray):
                return a
            d = ctx.to_device(np.ascontiguousarray(a, dt))
            keep.append(d)
            return d
        r, c, v, o = dev(rows, np.int32), dev(cols, np.int32), dev(vals, np.float64), \
            dev(ops, np.uint8)
        count = r.n if r is not None else 0
        h = _vp()
        check(_lib().mtlgpu_csr_assemble(ctx.h, base.h if base is not None else None, n_rows,
                                         n_cols, count, r.ptr if count else None,
                                         c.ptr if count else None, v.ptr if count else None,
                                         o.ptr if o is not None else None, int(updater),
                                         C.byref(h)), "csr_assemble")
        return cls._adopt(ctx, h)

    @classmethod
    def laplacian2d(cls, ctx, m, n):
        """laplacian_setup(A, m, n) built on the device."""
        h = _vp()
        check(_lib().mtlgpu_csr_laplacian2d(ctx.h, m, n, C.byref(h)), "csr_laplacian2d")
        return cls._adopt(ctx, h)

    @classmethod
    def laplacian3d(cls, ctx, N):
        """The 3-D 7-point Laplacian on an N^3 grid built on the device."""
        h = _vp()
        check(_lib().mtlgpu_csr_laplacian3d(ctx.h, N, C.byref(h)), "csr_laplacian3d")
        return cls._adopt(ctx, h)

    def download(self):
        """(rp, ci, v) host copies of the CSR arrays."""
        rp_, ci_, v_ = _vp(), _vp(), _vp()
        check(_lib().mtlgpu_csr_device_arrays(self.h, C.byref(rp_), C.byref(ci_), C.byref(v_)),
              "csr_device_arrays")
        rp = np.empty(self.n + 1, np.int32)
        ci = np.empty(self.nnz, np.int32)
        v = np.empty(self.nnz, np.float64)
        L = _lib()
        check(L.mtlgpu_memcpy_d2h(self.ctx.h, _p(rp), rp_, rp.nbytes), "d2h")
        if self.nnz:
            check(L.mtlgpu_memcpy_d2h(self.ctx.h, _p(ci), ci_, ci.nbytes), "d2h")
            check(L.mtlgpu_memcpy_d2h(self.ctx.h, _p(v), v_, v.nbytes), "d2h")
        return rp, ci, v

    def set_values(self, v):
        v = np.ascontiguousarray(v, np.float64)
        check(_lib().mtlgpu_csr_set_values(self.h, _p(v), None), "csr_set_values")

    def transpose(self):
        """A^T as a new handle (mtlgpu_csr_create_transpose)."""
        T = Csr.__new__(Csr)
        T.ctx, T.n, T.n_cols, T.nnz = self.ctx, self.n_cols, self.n, self.nnz
        T.h = _vp()
        check(_lib().mtlgpu_csr_create_transpose(self.h, C.byref(T.h)), "csr_create_transpose")
        return T

    def values_grad(self, lam, x, grad):
        """grad[k] = -lam[i] x[j] for the k-th stored entry (i, j)."""
        check(_lib().mtlgpu_csr_values_grad(self.h, lam.ptr, x.ptr, grad.ptr), "csr_values_grad")

    def spmv(self, x, y, alpha=1.0, beta=0.0):
        check(_lib().mtlgpu_spmv(self.h, x.ptr, y.ptr, float(alpha), float(beta)), "spmv")

    def spmv_f32(self, x, y):
        check(_lib().mtlgpu_spmv_f32(self.h, x.ptr, y.ptr), "spmv_f32")

    def cg_direction_product(self, prec, z, beta, p, p_out, q, pq):
        """p_out = z + beta p (p = None: p_out = z), q = A p_out, pq[0] = p_out . q
        (pq: a device array of at least one double)."""
        check(_lib().mtlgpu_cg_direction_product(self.h, prec, z.ptr, beta,
                                                 p.ptr if p is not None else None, p_out.ptr,
                                                 q.ptr, pq.ptr), "cg_direction_product")

    def spmv_transposed(self, x, y):
        check(_lib().mtlgpu_spmv_transposed(self.h, x.ptr, y.ptr), "spmv_transposed")

    def autotune(self):
        c = C.c_int()
        check(_lib().mtlgpu_csr_autotune(self.h, C.byref(c)), "autotune")
        return c.value

    def close(self):
        if self.h:
            _lib().mtlgpu_csr_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            if self.ctx.h:
                self.close()
        except Exception:
            pass


class Pc:
    """Preconditioner handle (itl::pc::identity / diagonal / ilu_0 / ic_0)."""

    def __init__(self, A, kind, prec=FP64, allow_pivot=True):
        self.A = A
        self.kind = PC_KINDS.get(kind, kind)
        self.prec = prec
        self.h = _vp()
        st = _lib().mtlgpu_pc_create(A.h, self.kind, prec, C.byref(self.h))
        self.status = st
        if st != OK and not (allow_pivot and st == ZERO_PIVOT and self.h):
            raise MtlgpuError(st, "pc_create")

    def apply(self, r, z):
        check(_lib().mtlgpu_pc_apply(self.h, r.ptr, z.ptr), "pc_apply")

    def apply_f32(self, r, z):
        """FP32 apply (asynchronous; errors surface at ctx.synchronize())."""
        check(_lib().mtlgpu_pc_apply_f32(self.h, r.ptr, z.ptr), "pc_apply_f32")

    def adjoint_apply(self, r, z):
        check(_lib().mtlgpu_pc_adjoint_apply(self.h, r.ptr, z.ptr), "pc_adjoint_apply")

    def sweep(self, which, x, y):
        if x.dtype == np.float32:
            check(_lib().mtlgpu_pc_sweep_f32(self.h, which, x.ptr, y.ptr), "pc_sweep_f32")
        else:
            check(_lib().mtlgpu_pc_sweep(self.h, which, x.ptr, y.ptr), "pc_sweep")

    def set_jacobi_sweeps(self, iters):
        """Apply the triangular factors with `iters` Jacobi iterations per
        triangle (0: the exact sweeps)."""
        check(_lib().mtlgpu_pc_set_jacobi_sweeps(self.h, int(iters)), "pc_set_jacobi_sweeps")

    def sweep_kind(self, which, prec=FP64):
        """0: level-ordered sweep, 1: partitioned sweep, 2: Jacobi iterations."""
        k = C.c_int()
        check(_lib().mtlgpu_pc_sweep_kind(self.h, which, prec, C.byref(k)), "pc_sweep_kind")
        return k.value

    def factor_info(self, which):
        nnz, lev = C.c_int(), C.c_int()
        check(_lib().mtlgpu_pc_factor_info(self.h, which, C.byref(nnz), C.byref(lev)))
        return nnz.value, lev.value

    def factor(self, which):
        nnz, _ = self.factor_info(which)
        n = self.A.n
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(max(nnz, 1), np.int32)
        v = np.zeros(max(nnz, 1))
        check(_lib().mtlgpu_pc_get_factor(self.h, which, _p(rp), _p(ci), _p(v)), "get_factor")
        return (n, rp, ci[:nnz], v[:nnz])

    def levels(self, which):
        lev = np.zeros(self.A.n, np.int32)
        check(_lib().mtlgpu_pc_get_levels(self.h, which, _p(lev)), "get_levels")
        return lev

    def close(self):
        if self.h:
            _lib().mtlgpu_pc_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            if self.A.ctx.h and self.A.h:
                self.close()
        except Exception:
            pass


def make_params(max_iter=1000, rtol=1e-10, atol=0.0, norm_r0=-1.0, mode=SOLVE_FP64,
                inner_rtol=0.0, inner_max_iter=0, max_outer=0, history=None, interrupt=None):
    p = IterParams()
    _lib().mtlgpu_iter_params_default(C.byref(p))
    p.max_iter, p.rtol, p.atol, p.norm_r0, p.mode = max_iter, rtol, atol, norm_r0, mode
    p.inner_rtol, p.inner_max_iter, p.max_outer = inner_rtol, inner_max_iter, max_outer
    if history is not None:
        p.h_resid_history = history.ctypes.data_as(C.POINTER(C.c_double))
        p.history_cap = len(history)
    if interrupt is not None:
        p.h_interrupt = interrupt.ctypes.data_as(C.POINTER(C.c_int))
    return p


def solve(method, A, P, x, b, **kw):
    """itl::cg / itl::bicgstab on device arrays; returns (status, IterResult, history)."""
    hist = np.zeros(2 * kw.get("max_iter", 1000) + 8)
    prm = make_params(history=hist, **kw)
    res = IterResult()
    st = _lib().mtlgpu_solve(METHODS.get(method, method), A.h, P.h if P else None, x.ptr, b.ptr,
                             C.byref(prm), C.byref(res))
    return st, res, hist[:min(res.history_len, len(hist))].copy()


def solve_krylov(method, A, L, x, b, R=None, param=0, **kw):
    """mtlgpu_solve_krylov: bicg / cgs / bicgstab_2 / bicgstab_ell / tfqmr /
    qmr / idr_s / gmres with left preconditioner L and right preconditioner R
    (None: identity) on device arrays; returns (status, IterResult, history)."""
    max_iter = kw.get("max_iter", 1000)
    hist = np.zeros((max(param, 2) + 3) * (max_iter + 2) + 16)
    prm = make_params(history=hist, **kw)
    res = IterResult()
    st = _lib().mtlgpu_solve_krylov(METHODS.get(method, method), A.h, L.h if L else None,
                                    R.h if R else None, int(param), x.ptr, b.ptr, C.byref(prm),
                                    C.byref(res))
    return st, res, hist[:min(res.history_len, len(hist))].copy()


def solve_batched(A, P, offsets, x, b, **kw):
    """Batched itl::cg over the diagonal blocks [offsets[s], offsets[s+1]) of the
    block-diagonal device matrix A; returns (status, list of IterResult)."""
    off = np.ascontiguousarray(offsets, np.int32)
    count = len(off) - 1
    prm = make_params(**kw)
    res = (IterResult * count)()
    st = _lib().mtlgpu_solve_batched(METHODS["cg"], A.h, P.h if P else None, count, _p(off),
                                     x.ptr, b.ptr, C.byref(prm), res)
    return st, list(res)


def batched_autotune(A, P, offsets, x, b, **kw):
    """mtlgpu_batched_autotune: times the batched kernel's shapes on these
    systems and keeps the fastest on A; returns 1000 * (rows below which one
    CTA solves a system) + 100 * (CTAs per larger system) + lanes per row."""
    off = np.ascontiguousarray(offsets, np.int32)
    prm = make_params(**kw)
    c = C.c_int()
    check(_lib().mtlgpu_batched_autotune(A.h, P.h if P else None, len(off) - 1, _p(off), x.ptr,
                                         b.ptr, C.byref(prm), C.byref(c)), "batched_autotune")
    return c.value


def solve_host(method, A, P, x, b, **kw):
    """Same with host numpy x (updated in place) and b."""
    hist = np.zeros(2 * kw.get("max_iter", 1000) + 8)
    prm = make_params(history=hist, **kw)
    res = IterResult()
    x = np.ascontiguousarray(x, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    st = _lib().mtlgpu_solve_host(METHODS.get(method, method), A.h, P.h if P else None, _p(x),
                                  _p(b), C.byref(prm), C.byref(res))
    return st, res, x


def solve_host_ptrs(method, A, P, x_ptr, b_ptr, **kw):
    """mtlgpu_solve_host on raw host pointers (e.g. pinned buffers)."""
    prm = make_params(**kw)
    res = IterResult()
    st = _lib().mtlgpu_solve_host(METHODS.get(method, method), A.h, P.h if P else None,
                                  _vp(x_ptr), _vp(b_ptr), C.byref(prm), C.byref(res))
    return st, res


# ---------------------------------------------------------------------------
# fixtures (host generators)
def laplacian2d(m, n):
    L = _fix()
    nnz = L.mtlgpu_gen_laplacian2d(m, n, None, None, None)
    rp, ci, v = np.zeros(m * n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.mtlgpu_gen_laplacian2d(m, n, _p(rp), _p(ci), _p(v))
    return (m * n, rp, ci, v)


def laplacian3d(N):
    L = _fix()
    nnz = L.mtlgpu_gen_laplacian3d(N, None, None, None)
    rp, ci, v = np.zeros(N ** 3 + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.mtlgpu_gen_laplacian3d(N, _p(rp), _p(ci), _p(v))
    return (N ** 3, rp, ci, v)


def convdiff27(N, seed=2):
    L = _fix()
    nnz = L.mtlgpu_gen_convdiff27(N, seed, None, None, None)
    rp, ci, v = np.zeros(N ** 3 + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.mtlgpu_gen_convdiff27(N, seed, _p(rp), _p(ci), _p(v))
    return (N ** 3, rp, ci, v)


def random_graph(n, avg_deg, shift_frac=1e-2, seed=3):
    L = _fix()
    nnz = L.mtlgpu_gen_random_graph(n, avg_deg, shift_frac, seed, None, None, None)
    rp, ci, v = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.mtlgpu_gen_random_graph(n, avg_deg, shift_frac, seed, _p(rp), _p(ci), _p(v))
    return (n, rp, ci, v)


def graph_batch(count, n_min=1000, n_max=65536, deg_min=8.0, deg_max=32.0, shift_frac=1e-2,
                seed=3):
    """`count` random-graph Laplacians of log-uniform sizes (the batched-PCG
    workload): returns (systems, blockdiag) with systems a list of
    (n, rp, ci, v) and blockdiag = (n_total, rp, ci, v, offsets)."""
    L = _fix()
    sizes = np.zeros(2 * count, np.int64)
    total = L.mtlgpu_gen_graph_batch(count, n_min, n_max, deg_min, deg_max, shift_frac, seed,
                                     _p(sizes), None, None, None)
    ns, nz = sizes[0::2], sizes[1::2]
    rp = np.zeros(int(ns.sum() + count), np.int32)
    ci, v = np.zeros(total, np.int32), np.zeros(total)
    L.mtlgpu_gen_graph_batch(count, n_min, n_max, deg_min, deg_max, shift_frac, seed, _p(sizes),
                             _p(rp), _p(ci), _p(v))
    systems, ro, eo = [], 0, 0
    for s in range(count):
        n, m = int(ns[s]), int(nz[s])
        systems.append((n, rp[ro:ro + n + 1].copy(), ci[eo:eo + m].copy(), v[eo:eo + m].copy()))
        ro, eo = ro + n + 1, eo + m
    offsets = np.concatenate([[0], np.cumsum(ns)]).astype(np.int32)
    brp = np.zeros(int(offsets[-1]) + 1, np.int32)
    bci = np.zeros(total, np.int32)
    e = 0
    for s, (n, srp, sci, sv) in enumerate(systems):
        brp[offsets[s] + 1:offsets[s + 1] + 1] = srp[1:] + e
        bci[e:e + len(sci)] = sci + offsets[s]
        e += len(sci)
    return systems, (int(offsets[-1]), brp, bci, v, offsets)


def fv2d(N, sigma=1.0, corr=8.0, seed=4):
    L = _fix()
    nnz = L.mtlgpu_gen_fv2d(N, sigma, corr, seed, None, None, None)
    rp, ci, v = np.zeros(N * N + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.mtlgpu_gen_fv2d(N, sigma, corr, seed, _p(rp), _p(ci), _p(v))
    return (N * N, rp, ci, v)


def uniform(n, seed, a=-1.0, b=1.0):
    out = np.zeros(n)
    _fix().mtlgpu_gen_uniform(n, seed, a, b, _p(out))
    return out


def normal(n, seed):
    out = np.zeros(n)
    _fix().mtlgpu_gen_normal(n, seed, _p(out))
    return out


def csr_mult(A, x):
    n, rp, ci, v = A
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(n)
    _fix().mtlgpu_gen_csr_mult(n, _p(rp), _p(ci), _p(v), _p(x), _p(y))
    return y
