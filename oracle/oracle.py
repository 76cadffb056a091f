"""ctypes access to the CPU oracles.  TEST INFRASTRUCTURE ONLY.

Two implementations with the same call signatures:

* ``Restatement`` -- ``oracle/_build/liboracle.so``, the plain-C restatement of
  the reference loops (``oracle/restate.c``);
* ``Reference``   -- ``oracle/_ref/libmtlref.so`` (or ``libmtlref_omp.so``),
  the MTL4/ITL reference itself compiled from its unmodified headers
  (``oracle/ref_driver.cpp``).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  CSR matrices are passed as
``(n, rp, ci, v)`` numpy arrays (int32, int32, float64).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = C.c_void_p

PC_IDENTITY, PC_DIAGONAL, PC_ILU0, PC_IC0, PC_ILU0_FLOAT, PC_IC0_FLOAT = range(6)
PC_NAMES = {"identity": PC_IDENTITY, "diagonal": PC_DIAGONAL, "ilu0": PC_ILU0, "ic0": PC_IC0,
            "ilu0_float": PC_ILU0_FLOAT, "ic0_float": PC_IC0_FLOAT}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


class _Base:
    prefix = ""

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library {path} not built (make -C oracle)")
        self.path = path
        self.lib = C.CDLL(path)
        p = self.prefix
        L = self.lib
        getattr(L, p + "spmv").restype = C.c_int
        getattr(L, p + "dot").restype = C.c_double
        getattr(L, p + "two_norm").restype = C.c_double
        getattr(L, p + "unary_dot").restype = C.c_double
        getattr(L, p + "solve").restype = C.c_int
        getattr(L, p + "pc_apply").restype = C.c_int
        getattr(L, p + "laplacian_setup").restype = C.c_int
        getattr(L, p + "assemble").restype = C.c_int

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    # --- matrices ---------------------------------------------------------
    def laplacian_setup(self, m, n):
        f = self._f("laplacian_setup")
        nnz = f(C.c_uint(m), C.c_uint(n), None, None, None)
        rp = np.zeros(m * n + 1, np.int32)
        ci = np.zeros(nnz, np.int32)
        v = np.zeros(nnz, np.float64)
        f(C.c_uint(m), C.c_uint(n), _ptr(rp), _ptr(ci), _ptr(v))
        return (m * n, rp, ci, v)

    def assemble(self, n_rows, n_cols, rows, cols, vals, ops=None, updater=0, base=None,
                 syntax=None, slot_size=0):
        """The matrix mtl::mat::inserter leaves after the triplets (see
        or_assemble / ref_assemble): returns (rp, ci, v), or raises
        IndexError for an index out of range.  The restatement takes `ops`
        (updater per triplet); the reference takes `syntax` (0: ins = v,
        1: ins += v, 2: ins << v with the class updater)."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        if base is not None:
            brp, bci, bv = (np.ascontiguousarray(base[0], np.int32),
                            np.ascontiguousarray(base[1], np.int32),
                            np.ascontiguousarray(base[2], np.float64))
            bn = len(bci)
        else:
            brp = bci = bv = None
            bn = 0
        cap = max(1, bn + len(rows))
        rp = np.zeros(n_rows + 1, np.int32)
        ci = np.zeros(cap, np.int32)
        v = np.zeros(cap, np.float64)
        if self.prefix == "ref_":
            sx = None if syntax is None else np.ascontiguousarray(syntax, np.uint8)
            secs = C.c_double()
            nnz = self._f("assemble")(C.c_int(n_rows), C.c_int(n_cols), C.c_int(bn), _ptr(brp),
                                      _ptr(bci), _ptr(bv), C.c_longlong(len(rows)), _ptr(rows),
                                      _ptr(cols), _ptr(vals), _ptr(sx), C.c_int(updater),
                                      C.c_int(slot_size), _ptr(rp), _ptr(ci), _ptr(v),
                                      C.byref(secs))
            self.last_seconds = secs.value
        else:
            o = None if ops is None else np.ascontiguousarray(ops, np.uint8)
            nnz = self._f("assemble")(C.c_int(n_rows), C.c_int(n_cols), C.c_int(bn), _ptr(brp),
                                      _ptr(bci), _ptr(bv), C.c_longlong(len(rows)), _ptr(rows),
                                      _ptr(cols), _ptr(vals), _ptr(o), C.c_int(updater),
                                      _ptr(rp), _ptr(ci), _ptr(v))
        if nnz == -1:
            raise IndexError("Index is out of range!")
        if nnz < 0:
            raise RuntimeError(f"assemble failed ({nnz})")
        return rp, ci[:nnz].copy(), v[:nnz].copy()

    def spmv(self, A, x, y=None, mode=0):
        n, rp, ci, v = A
        y = np.zeros(n) if y is None else np.array(y, np.float64, copy=True)
        x = np.ascontiguousarray(x, np.float64)
        if self.prefix == "ref_":
            self._f("spmv")(C.c_int(n), C.c_int(len(ci)), _ptr(rp), _ptr(ci), _ptr(v), _ptr(x),
                            _ptr(y), C.c_int(mode))
        else:
            self._f("spmv")(C.c_int(n), _ptr(rp), _ptr(ci), _ptr(v), _ptr(x), _ptr(y),
                            C.c_int(mode))
        return y

    def dot(self, x, y):
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        return self._f("dot")(C.c_int(len(x)), _ptr(x), _ptr(y))

    def two_norm(self, x):
        x = np.ascontiguousarray(x, np.float64)
        return self._f("two_norm")(C.c_int(len(x)), _ptr(x))

    def unary_dot(self, x):
        x = np.ascontiguousarray(x, np.float64)
        return self._f("unary_dot")(C.c_int(len(x)), _ptr(x))

    # --- preconditioners ---------------------------------------------------
    def pc_apply(self, pc, A, r, adjoint=False):
        n, rp, ci, v = A
        pc = PC_NAMES.get(pc, pc)
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros(n)
        if self.prefix == "ref_":
            st = self._f("pc_apply")(C.c_int(pc), C.c_int(n), C.c_int(len(ci)), _ptr(rp), _ptr(ci),
                                     _ptr(v), _ptr(r), _ptr(z), C.c_int(int(adjoint)))
        else:
            st = self._f("pc_apply")(C.c_int(pc), C.c_int(n), _ptr(rp), _ptr(ci), _ptr(v),
                                     _ptr(r), _ptr(z), C.c_int(int(adjoint)))
        if st:
            raise RuntimeError(f"pc_apply failed with {st}")
        return z

    # --- solvers -----------------------------------------------------------
    def solve(self, method, pc, A, b, x0=None, max_iter=1000, rtol=1e-10, atol=0.0,
              norm_r0=-1.0, hist_cap=None):
        """Returns dict(err, x, iterations, resid, norm_r0, t_factor, t_solve, history)."""
        n, rp, ci, v = A
        method = {"cg": 0, "bicgstab": 1}.get(method, method)
        pc = PC_NAMES.get(pc, pc)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(n) if x0 is None else np.array(x0, np.float64, copy=True)
        cap = (2 * max_iter + 4) if hist_cap is None else hist_cap
        hist = np.zeros(max(cap, 1))
        out = np.zeros(6)
        if self.prefix == "ref_":
            err = self._f("solve")(C.c_int(method), C.c_int(pc), C.c_int(n), C.c_int(len(ci)),
                                   _ptr(rp), _ptr(ci), _ptr(v), _ptr(b), _ptr(x),
                                   C.c_int(max_iter), C.c_double(rtol), C.c_double(atol),
                                   C.c_double(norm_r0), _ptr(hist), C.c_int(cap), _ptr(out))
        else:
            err = self._f("solve")(C.c_int(method), C.c_int(pc), C.c_int(n), _ptr(rp), _ptr(ci),
                                   _ptr(v), _ptr(b), _ptr(x), C.c_int(max_iter),
                                   C.c_double(rtol), C.c_double(atol), C.c_double(norm_r0),
                                   _ptr(hist), C.c_int(cap), _ptr(out))
        cnt = int(out[5])
        return dict(err=err, x=x, iterations=int(out[0]), resid=float(out[1]),
                    norm_r0=float(out[2]), t_factor=float(out[3]), t_solve=float(out[4]),
                    history=hist[:min(cnt, cap)].copy())


KRYLOV = {"bicg": 2, "cgs": 3, "bicgstab_2": 4, "bicgstab_ell": 5, "tfqmr": 6, "qmr": 7,
          "idr_s": 8, "gmres": 9}


class Restatement(_Base):
    prefix = "or_"

    def __init__(self, path=None):
        super().__init__(path or os.path.join(HERE, "_build", "liboracle.so"))
        L = self.lib
        for name in ("ic0", "ilu0", "upper_nnz", "strict_lower_nnz", "levels_lower",
                     "levels_upper"):
            getattr(L, "or_" + name).restype = C.c_int

    def ic0(self, A, as_float=False):
        n, rp, ci, v = A
        nu = self.lib.or_upper_nnz(C.c_int(n), _ptr(rp), _ptr(ci))
        Lrp, Urp = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
        Lci, Uci = np.zeros(nu, np.int32), np.zeros(nu, np.int32)
        Lv, Uv = np.zeros(nu), np.zeros(nu)
        st = self.lib.or_ic0(C.c_int(n), _ptr(rp), _ptr(ci), _ptr(v), C.c_int(int(as_float)),
                             _ptr(Lrp), _ptr(Lci), _ptr(Lv), _ptr(Urp), _ptr(Uci), _ptr(Uv))
        if st:
            raise RuntimeError(f"IC(0): missing diagonal in row {-st - 1}")
        return (n, Lrp, Lci, Lv), (n, Urp, Uci, Uv)

    def ilu0(self, A, as_float=False):
        n, rp, ci, v = A
        nl = self.lib.or_strict_lower_nnz(C.c_int(n), _ptr(rp), _ptr(ci))
        nu = self.lib.or_upper_nnz(C.c_int(n), _ptr(rp), _ptr(ci))
        Lrp, Urp = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
        Lci, Uci = np.zeros(max(nl, 1), np.int32), np.zeros(max(nu, 1), np.int32)
        Lv, Uv = np.zeros(max(nl, 1)), np.zeros(max(nu, 1))
        st = self.lib.or_ilu0(C.c_int(n), _ptr(rp), _ptr(ci), _ptr(v), C.c_int(int(as_float)),
                              _ptr(Lrp), _ptr(Lci), _ptr(Lv), _ptr(Urp), _ptr(Uci), _ptr(Uv))
        if st:
            raise RuntimeError(f"ILU(0): missing diagonal in row {-st - 1}")
        return (n, Lrp, Lci[:nl], Lv[:nl]), (n, Urp, Uci[:nu], Uv[:nu])

    def levels(self, F, lower):
        n, rp, ci, _ = F
        lev = np.zeros(n, np.int32)
        f = self.lib.or_levels_lower if lower else self.lib.or_levels_upper
        nlev = f(C.c_int(n), _ptr(rp), _ptr(ci), _ptr(lev))
        return lev, nlev

    def sweep(self, kind, F, rhs):
        """kind: 'lower_unit' | 'lower_invdiag_last' | 'upper_invdiag_first'."""
        n, rp, ci, v = F
        rhs = np.ascontiguousarray(rhs, np.float64)
        out = np.zeros(n)
        getattr(self.lib, "or_" + kind)(C.c_int(n), _ptr(rp), _ptr(ci), _ptr(v), _ptr(rhs),
                                        _ptr(out))
        return out

    def transpose(self, F):
        n, rp, ci, v = F
        trp = np.zeros(n + 1, np.int32)
        tci = np.zeros(max(len(ci), 1), np.int32)
        tv = np.zeros(max(len(ci), 1))
        self.lib.or_transpose(C.c_int(n), _ptr(rp), _ptr(ci), _ptr(v), _ptr(trp), _ptr(tci),
                              _ptr(tv))
        return (n, trp, tci[:len(ci)], tv[:len(ci)])


class Reference(_Base):
    prefix = "ref_"

    FLAVOURS = {"parity": "libmtlref.so", "omp": "libmtlref_omp.so",
                "serial": "libmtlref_serial.so"}

    def __init__(self, path=None, openmp=False, flavour=None):
        """flavour: 'parity' (-O2, no FMA contraction: the bit-comparable
        oracle), 'omp' (-O3 -march=x86-64-v3 with OpenMP: the timed CPU
        baseline on all cores), 'serial' (the same without OpenMP, CG's fused
        loops active).  openmp=True is flavour 'omp'."""
        flavour = flavour or ("omp" if openmp else "parity")
        self.flavour = flavour
        super().__init__(path or os.path.join(HERE, "_ref", self.FLAVOURS[flavour]))
        L = self.lib
        L.ref_spmv_time.restype = C.c_double
        L.ref_build_info.restype = C.c_char_p
        L.ref_omp_threads.restype = C.c_int
        L.ref_ic0.restype = C.c_int
        L.ref_ilu0.restype = C.c_int

    def build_info(self):
        return self.lib.ref_build_info().decode()

    def threads(self):
        return int(self.lib.ref_omp_threads())

    def solve_krylov(self, method, pc_left, A, b, pc_right="identity", param=0, x0=None,
                     max_iter=1000, rtol=1e-10, atol=0.0, norm_r0=-1.0, hist_cap=None):
        """The reference's bicg / cgs / bicgstab_2 / bicgstab_ell / tfqmr / qmr /
        idr_s / gmres (ref_solve_krylov).  Same result dict as solve()."""
        n, rp, ci, v = A
        method = KRYLOV.get(method, method)
        pl, pr = PC_NAMES.get(pc_left, pc_left), PC_NAMES.get(pc_right, pc_right)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(n) if x0 is None else np.array(x0, np.float64, copy=True)
        cap = (4 * max_iter + 16) if hist_cap is None else hist_cap
        hist = np.zeros(max(cap, 1))
        out = np.zeros(6)
        f = self._f("solve_krylov")
        f.restype = C.c_int
        err = f(C.c_int(method), C.c_int(pl), C.c_int(pr), C.c_int(param), C.c_int(n),
                C.c_int(len(ci)), _ptr(rp), _ptr(ci), _ptr(v), _ptr(b), _ptr(x),
                C.c_int(max_iter), C.c_double(rtol), C.c_double(atol), C.c_double(norm_r0),
                _ptr(hist), C.c_int(cap), _ptr(out))
        cnt = int(out[5])
        return dict(err=err, x=x, iterations=int(out[0]), resid=float(out[1]),
                    norm_r0=float(out[2]), t_factor=float(out[3]), t_solve=float(out[4]),
                    history=hist[:min(cnt, cap)].copy())

    def spmv_time(self, A, x, reps):
        n, rp, ci, v = A
        x = np.ascontiguousarray(x, np.float64)
        return self.lib.ref_spmv_time(C.c_int(n), C.c_int(len(ci)), _ptr(rp), _ptr(ci), _ptr(v),
                                      _ptr(x), C.c_int(reps))

    def ic0(self, A, as_float=False):
        n, rp, ci, v = A
        nu = int(np.count_nonzero(ci >= np.repeat(np.arange(n), np.diff(rp))))
        Lrp, Urp = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
        Lci, Uci = np.zeros(max(nu, 1), np.int32), np.zeros(max(nu, 1), np.int32)
        Lv, Uv = np.zeros(max(nu, 1)), np.zeros(max(nu, 1))
        self.lib.ref_ic0(C.c_int(n), C.c_int(len(ci)), _ptr(rp), _ptr(ci), _ptr(v),
                         C.c_int(int(as_float)), _ptr(Lrp), _ptr(Lci), _ptr(Lv), _ptr(Urp),
                         _ptr(Uci), _ptr(Uv))
        return (n, Lrp, Lci[:nu], Lv[:nu]), (n, Urp, Uci[:nu], Uv[:nu])

    def ilu0(self, A, as_float=False):
        n, rp, ci, v = A
        rows = np.repeat(np.arange(n), np.diff(rp))
        nl = int(np.count_nonzero(ci < rows))
        nu = len(ci) - nl
        Lrp, Urp = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
        Lci, Uci = np.zeros(max(nl, 1), np.int32), np.zeros(max(nu, 1), np.int32)
        Lv, Uv = np.zeros(max(nl, 1)), np.zeros(max(nu, 1))
        nnz = np.zeros(2, np.int32)
        self.lib.ref_ilu0(C.c_int(n), C.c_int(len(ci)), _ptr(rp), _ptr(ci), _ptr(v),
                          C.c_int(int(as_float)), _ptr(nnz), _ptr(Lrp), _ptr(Lci), _ptr(Lv),
                          _ptr(Urp), _ptr(Uci), _ptr(Uv))
        return (n, Lrp, Lci[:nl], Lv[:nl]), (n, Urp, Uci[:nu], Uv[:nu])


def available_reference(openmp=False, flavour=None):
    """Reference() if its library was built (it is compiled where the
    reference tree exists and shipped prebuilt elsewhere), else None."""
    try:
        return Reference(openmp=openmp, flavour=flavour)
    except (FileNotFoundError, OSError):
        return None
