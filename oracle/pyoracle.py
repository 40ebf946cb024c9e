"""ctypes bindings for the CPU oracle (test infrastructure only).

Two libraries share one interface:

* ``Oracle``   -- oracle/libpgmg_oracle.so, the C restatement of the
  reference hot path (oracle/pgmg_oracle.c);
* ``Reference`` -- oracle/_ref/libpgmg_ref.so, the reference's own sources
  (buffer.cc common.cc geometry.cc region.cc region_tr.cc multigrid.cc)
  compiled with a single-rank MPI shim (oracle/Makefile).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
bench.py import this module; it is the checker, never the product.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libpgmg_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpgmg_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def _bind(lib, prefix: str):
    P = C.c_void_p
    sig = {
        "destroy": (None, [P]),
        "nlevels": (C.c_int, [P]),
        "level_dims": (None, [P, C.c_int, _ip]),
        "lu_enabled": (C.c_int, [P]),
        "get_x": (None, [P, C.c_int, _dp]),
        "set_x": (None, [P, C.c_int, _dp]),
        "get_r": (None, [P, C.c_int, _dp]),
        "set_r": (None, [P, C.c_int, _dp]),
        "get_S": (None, [P, C.c_int, _ip]),
        "gauss_seidel": (None, [P, C.c_int, C.c_int]),
        "restriction": (None, [P, C.c_int]),
        "interpolation": (None, [P, C.c_int]),
        "solve_exact": (None, [P, C.c_int]),
        "v_cycle": (None, [P, C.c_int]),
        "l2_error_all": (C.c_double, [P, C.c_int]),
        "rhs_l2norm": (C.c_double, [P, C.c_int]),
        "solve_v_cycles": (C.c_int, [P, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_long)]),
        "setup_test": (None, [P, C.c_int, C.c_int, C.c_int]),
        "clear_x": (None, [P, C.c_int]),
        "guide_pred_iters": (C.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = args
    return lib


class _Base:
    prefix = ""

    def __init__(self, lib, handle, m, n, o):
        self.lib = lib
        self.h = handle
        self.m, self.n, self.o = m, n, o

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nlevels(self) -> int:
        return self._f("nlevels")(self.h)

    def dims(self, l: int):
        d = np.zeros(3, np.int32)
        self._f("level_dims")(self.h, l, d)
        return tuple(int(v) for v in d)

    def npts(self, l):
        m, n, o = self.dims(l)
        return m * n * o

    @property
    def lu_enabled(self) -> bool:
        return bool(self._f("lu_enabled")(self.h))

    def get_x(self, l=0):
        out = np.zeros(self.npts(l))
        self._f("get_x")(self.h, l, out)
        return out

    def set_x(self, l, x):
        self._f("set_x")(self.h, l, np.ascontiguousarray(x, np.float64))

    def get_r(self, l=0):
        out = np.zeros(self.npts(l))
        self._f("get_r")(self.h, l, out)
        return out

    def set_r(self, l, r):
        self._f("set_r")(self.h, l, np.ascontiguousarray(r, np.float64))

    def get_S(self, l):
        out = np.zeros(6 * self.npts(l), np.int32)
        self._f("get_S")(self.h, l, out)
        return out.reshape(-1, 6)

    def get_A27(self, l):
        out = np.zeros(27 * self.npts(l))
        bad = self._f("get_A27")(self.h, l, out)
        if bad:
            raise ValueError(f"{bad} stencil boxes exceed the 27-point neighbourhood")
        return out.reshape(-1, 27)

    def gauss_seidel(self, mode=0, level=0):
        self._f("gauss_seidel")(self.h, mode, level)

    def restriction(self, level):
        self._f("restriction")(self.h, level)

    def interpolation(self, level):
        self._f("interpolation")(self.h, level)

    def solve_exact(self, level):
        self._f("solve_exact")(self.h, level)

    def v_cycle(self, mode=0):
        self._f("v_cycle")(self.h, mode)

    def l2_error_all(self, level=0) -> float:
        return self._f("l2_error_all")(self.h, level)

    def rhs_l2norm(self, level=0) -> float:
        return self._f("rhs_l2norm")(self.h, level)

    def solve_v_cycles(self, p_scale: float):
        res = C.c_double(0)
        sw = C.c_long(0)
        st = self._f("solve_v_cycles")(self.h, p_scale, C.byref(res), C.byref(sw))
        return st, res.value, sw.value

    def setup_test(self, ca, xfield, level):
        self._f("setup_test")(self.h, ca, int(xfield), level)

    def clear_x(self, level):
        self._f("clear_x")(self.h, level)

    def guide_pred_iters(self):
        return self._f("guide_pred_iters")(self.h)


_oracle_lib = None
_ref_lib = None


def oracle_lib():
    global _oracle_lib
    if _oracle_lib is None:
        lib = C.CDLL(ORACLE_SO)
        _bind(lib, "orc_")
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.c_int] * 3 + [_ip, _dp, C.c_void_p, C.c_void_p, C.c_int]
        lib.orc_get_A27.restype = None
        lib.orc_get_A27.argtypes = [C.c_void_p, C.c_int, _dp]
        lib.orc_gauss_seidel_mc8.restype = None
        lib.orc_gauss_seidel_mc8.argtypes = [C.c_void_p, C.c_int, C.c_int]
        lib.orc_set_slab_budget.restype = None
        lib.orc_set_slab_budget.argtypes = [C.c_void_p, C.c_longlong]
        lib.orc_set_smoother.restype = None
        lib.orc_set_smoother.argtypes = [C.c_void_p, C.c_int]
        lib.orc_dgetrf.restype = C.c_int
        lib.orc_dgetrf.argtypes = [C.c_int, _dp, _ip]
        lib.orc_dgetrs.restype = None
        lib.orc_dgetrs.argtypes = [C.c_int, _dp, _ip, _dp]
        _oracle_lib = lib
    return _oracle_lib


def _input_lib():
    lib = oracle_lib()
    if not getattr(lib, "_inputs_bound", False):
        u64 = C.c_uint64
        lib.orc_input_gauss.restype = C.c_int
        lib.orc_input_gauss.argtypes = [C.c_int] * 3 + [u64, C.c_double, _dp]
        lib.orc_input_kappa.restype = C.c_int
        lib.orc_input_kappa.argtypes = [C.c_int] * 3 + [C.c_double, u64, C.c_double, _dp]
        lib.orc_input_q1.restype = C.c_int
        lib.orc_input_q1.argtypes = [C.c_int] * 3 + [C.c_void_p, _dp, _ip]
        lib.orc_input_rhs.restype = C.c_int
        lib.orc_input_rhs.argtypes = [C.c_int] * 3 + [u64, _dp]
        lib._inputs_bound = True
    return lib


def input_gauss(m, n, o, seed, width=8.0):
    """The normalised Gaussian cell field, (m-1)(n-1)(o-1) values."""
    out = np.empty((m - 1) * (n - 1) * (o - 1))
    if _input_lib().orc_input_gauss(m, n, o, seed, width, out):
        raise ValueError("orc_input_gauss")
    return out


def input_kappa(m, n, o, sigma, seed, width=8.0):
    """kappa = exp(sigma g) per cell."""
    out = np.empty((m - 1) * (n - 1) * (o - 1))
    if _input_lib().orc_input_kappa(m, n, o, sigma, seed, width, out):
        raise ValueError("orc_input_kappa")
    return out


def input_q1(m, n, o, kappa=None):
    """Q1 stencils (27 slots per point) and boxes (6 ints per point)."""
    c = np.empty(27 * m * n * o)
    S = np.empty(6 * m * n * o, np.int32)
    kp = None if kappa is None else np.ascontiguousarray(kappa, np.float64)
    if _input_lib().orc_input_q1(m, n, o, _ptr(kp), c, S):
        raise ValueError("orc_input_q1")
    return c, S


def input_rhs(m, n, o, seed):
    """Uniform[-1,1] interior source, zero on the boundary."""
    out = np.empty(m * n * o)
    if _input_lib().orc_input_rhs(m, n, o, seed, out):
        raise ValueError("orc_input_rhs")
    return out


def benchmark_problem(m, n, o, sigma, seed, width=8.0):
    """Stencils, boxes and source of a seeded variable-kappa Q1 problem, from
    the oracle library only (the same arrays as the product's generators)."""
    kap = input_kappa(m, n, o, sigma, seed, width)
    coef, S = input_q1(m, n, o, kap)
    del kap
    return coef, S, input_rhs(m, n, o, seed)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        lib = C.CDLL(REF_SO)
        _bind(lib, "ref_")
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_int] * 6 + [_ip, _dp, C.c_void_p, C.c_void_p]
        lib.ref_get_A27.restype = C.c_int
        lib.ref_get_A27.argtypes = [C.c_void_p, C.c_int, _dp]
        lib.ref_gs_count.restype = C.c_long
        lib.ref_fmg_cycle.restype = None
        lib.ref_fmg_cycle.argtypes = [C.c_void_p]
        for name in ("ref_compute_residual",):
            getattr(lib, name).restype = None
            getattr(lib, name).argtypes = [C.c_void_p, _dp]
        for name in ("ref_Ax", "ref_unpadded_Ax"):
            getattr(lib, name).restype = None
            getattr(lib, name).argtypes = [C.c_void_p, _dp, _dp]
        lib.ref_source_soln_dot.restype = C.c_double
        lib.ref_source_soln_dot.argtypes = [C.c_void_p]
        lib.ref_soln_diff.restype = C.c_double
        lib.ref_soln_diff.argtypes = [C.c_void_p, _dp]
        lib.ref_copy_rhs_to_soln.restype = None
        lib.ref_copy_rhs_to_soln.argtypes = [C.c_void_p]
        lib.ref_l0_error_all.restype = C.c_double
        lib.ref_l0_error_all.argtypes = [C.c_void_p, C.c_int]
        _ref_lib = lib
    return _ref_lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle(_Base):
    """The C restatement.  ``coarse``: True = LU on the bottom level (with the
    reference's conditioning fallback), False = 24 Gauss-Seidel sweeps."""

    prefix = "orc_"

    def __init__(self, m, n, o, S6, c27, r=None, x=None, coarse=True):
        lib = oracle_lib()
        S6 = np.ascontiguousarray(S6, np.int32).reshape(-1)
        c27 = np.ascontiguousarray(c27, np.float64).reshape(-1)
        r = None if r is None else np.ascontiguousarray(r, np.float64)
        x = None if x is None else np.ascontiguousarray(x, np.float64)
        h = lib.orc_create(m, n, o, S6, c27, _ptr(r), _ptr(x), int(coarse))
        super().__init__(lib, h, m, n, o)
        self._keep = (S6, c27, r, x)

    def get_A27(self, l):
        out = np.zeros(27 * self.npts(l))
        self.lib.orc_get_A27(self.h, l, out)
        return out.reshape(-1, 27)

    def gauss_seidel_mc8(self, mode=0, level=0):
        self.lib.orc_gauss_seidel_mc8(self.h, mode, level)

    def set_smoother(self, mc8: bool):
        self.lib.orc_set_smoother(self.h, int(mc8))

    def set_slab_budget(self, nbytes: int):
        self.lib.orc_set_slab_budget(self.h, int(nbytes))


class Reference(_Base):
    """The reference multigrid itself (non-periodic unless flags given)."""

    prefix = "ref_"

    def __init__(self, m, n, o, S6, c27, r=None, x=None, prd=(False, False, False)):
        lib = ref_lib()
        S6 = np.ascontiguousarray(S6, np.int32).reshape(-1)
        c27 = np.ascontiguousarray(c27, np.float64).reshape(-1)
        r = None if r is None else np.ascontiguousarray(r, np.float64)
        x = None if x is None else np.ascontiguousarray(x, np.float64)
        # S6 and c27 are read during construction only; r and x are copied.
        h = lib.ref_create(m, n, o, int(prd[0]), int(prd[1]), int(prd[2]), S6, c27, _ptr(r), _ptr(x))
        super().__init__(lib, h, m, n, o)

    def fmg_cycle(self):
        """multigrid::fmg_cycle (multigrid.cc:109-134)."""
        self.lib.ref_fmg_cycle(self.h)

    # PCG helpers of level 0 (region.cc:1848-1940, multigrid.hh:222-251).
    def compute_residual(self):
        out = np.zeros(self.npts(0))
        self.lib.ref_compute_residual(self.h, out)
        return out

    def Ax(self, v, unpadded=False):
        out = np.zeros(self.npts(0))
        f = self.lib.ref_unpadded_Ax if unpadded else self.lib.ref_Ax
        f(self.h, np.ascontiguousarray(v, np.float64), out)
        return out

    def source_soln_dot(self):
        return self.lib.ref_source_soln_dot(self.h)

    def soln_diff(self, ext_x):
        return self.lib.ref_soln_diff(self.h, np.ascontiguousarray(ext_x, np.float64).copy())

    def copy_rhs_to_soln(self):
        self.lib.ref_copy_rhs_to_soln(self.h)

    def l0_error_all(self, level=0):
        return self.lib.ref_l0_error_all(self.h, level)

    @staticmethod
    def gs_count() -> int:
        return ref_lib().ref_gs_count()
