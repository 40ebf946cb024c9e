"""Python binding of libpgmg_b200.so (the C ABI in include/pgmg_dev.h).

``Multigrid`` mirrors the reference's ``multigrid`` class (multigrid.hh:20-276)
for a single process: construct with the grid size, ``setup_matrices`` with
the level-0 stencils, ``setup_fields`` with the source, then ``v_cycle``,
``solve_v_cycles``, per-level ``gauss_seidel`` / ``restriction`` /
``interpolation`` / ``solve_exact`` and the norms.  All work runs in the
CUDA library; there is no CPU fallback -- constructing a ``Multigrid`` without
the built library or without a GPU raises ``PgmgError``.

The host problem generators (``problem_kappa``, ``problem_q1``,
``problem_rhs``) run on the CPU and need no GPU.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpgmg_b200.so")

FP64, MIXED = 0, 1
SMOOTH_MC8, SMOOTH_LEX = 0, 1
COARSE_LU, COARSE_GS, COARSE_LU_EXACT = 0, 1, 2
FIELD_X, FIELD_R, FIELD_RES = 0, 1, 2
OPT_GRAPHS, OPT_CLUSTER_FIRST, OPT_CLUSTER_SIZE, OPT_SLAB_BUDGET = 1, 2, 3, 4
OPT_V_DOWN, OPT_V_UP, OPT_V_BOTTOM = 5, 6, 7
OPT_PDL = 8
OPT_GS_BLOCK = 9
OPT_GRID_MAX = 10
OPT_CHECK_EVERY = 11
OPT_GS_VECTOR = 12
OPT_INNER_DIGITS = 13
OPT_GS_ALTERNATE = 14
OPT_GS_PREFETCH = 15
OPT_COARSE_SHARED = 16
OPT_FUSED_RESTRICT = 17
OPT_LU_WINDOW = 18
OPT_GS_TMA = 19
OPT_RAT_TILE = 20
OPT_GS_L2_PREFETCH = 21
OPT_LU_INVERSE_BAND = 22
OPT_GS_BLOCK_LEVELS = 23

_STATUS = {
    0: "ok", 1: "file error", 2: "memory error", 3: "internal error", 4: "multigrid error",
    5: "math error", 6: "setup error", 7: "bad argument", 8: "CUDA error", 9: "timeout",
    10: "admission rejected", 11: "unsupported", 12: "no CUDA device",
}


class PgmgError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {_STATUS.get(status, status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class Dims(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("o", C.c_int),
                ("x_prd", C.c_int), ("y_prd", C.c_int), ("z_prd", C.c_int),
                ("precision", C.c_int), ("coarse", C.c_int), ("smoother", C.c_int),
                ("device", C.c_int)]


_lib = None
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_VP = C.c_void_p

# (name, restype, argtypes) of every exported function.
SIGNATURES = [
    ("pgmg_dev_create", C.c_int, [C.POINTER(Dims), C.POINTER(C.c_void_p)]),
    ("pgmg_dev_destroy", C.c_int, [_VP]),
    ("pgmg_dev_set_stream", C.c_int, [_VP, _VP]),
    ("pgmg_dev_sync", C.c_int, [_VP]),
    ("pgmg_dev_last_error", C.c_char_p, [_VP]),
    ("pgmg_dev_launch_count", C.c_int, [_VP, C.POINTER(C.c_longlong)]),
    ("pgmg_dev_set_smoother", C.c_int, [_VP, C.c_int]),
    ("pgmg_dev_set_option", C.c_int, [_VP, C.c_int, C.c_longlong]),
    ("pgmg_dev_get_option", C.c_int, [_VP, C.c_int, C.POINTER(C.c_longlong)]),
    ("pgmg_dev_autotune", C.c_int, [_VP, C.c_int, C.POINTER(C.c_double)]),
    ("pgmg_dev_grid_check", C.c_int, [_VP, C.c_int, C.c_int]),
    ("pgmg_dev_num_levels", C.c_int, [_VP, C.POINTER(C.c_int)]),
    ("pgmg_dev_level_dims", C.c_int, [_VP, C.c_int, _ip]),
    ("pgmg_dev_memory", C.c_int, [_VP, C.POINTER(C.c_size_t)]),
    ("pgmg_dev_plan_bytes", C.c_int, [C.POINTER(Dims), C.POINTER(C.c_size_t)]),
    ("pgmg_dev_upload_level0", C.c_int, [_VP, _VP, _VP]),
    ("pgmg_dev_build_rat", C.c_int, [_VP]),
    ("pgmg_dev_lu_enabled", C.c_int, [_VP, C.POINTER(C.c_int)]),
    ("pgmg_dev_get_coef", C.c_int, [_VP, C.c_int, _VP]),
    ("pgmg_dev_get_boxes", C.c_int, [_VP, C.c_int, _VP]),
    ("pgmg_dev_set_field", C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    ("pgmg_dev_get_field", C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    ("pgmg_dev_apply", C.c_int, [_VP, C.c_int, _VP, _VP]),
    ("pgmg_dev_clear_x", C.c_int, [_VP, C.c_int]),
    ("pgmg_dev_setup_test", C.c_int, [_VP, C.c_int, C.c_int, C.c_int]),
    ("pgmg_dev_gs", C.c_int, [_VP, C.c_int, C.c_int, C.c_int]),
    ("pgmg_dev_restrict", C.c_int, [_VP, C.c_int]),
    ("pgmg_dev_interp", C.c_int, [_VP, C.c_int]),
    ("pgmg_dev_coarse_solve", C.c_int, [_VP]),
    ("pgmg_dev_vcycle", C.c_int, [_VP, C.c_int, C.c_int]),
    ("pgmg_dev_fmg_cycle", C.c_int, [_VP, C.c_int]),
    ("pgmg_dev_profile_vcycle", C.c_int, [_VP, C.c_int, _dp, C.c_int, C.POINTER(C.c_int)]),
    ("pgmg_dev_tma_check", C.c_int, [_VP, C.c_int, C.c_int]),
    ("pgmg_dev_source_soln_dot", C.c_int, [_VP, C.c_int, C.POINTER(C.c_double)]),
    ("pgmg_dev_soln_diff", C.c_int, [_VP, C.c_int, _VP, C.POINTER(C.c_double)]),
    ("pgmg_dev_l0_error", C.c_int, [_VP, C.c_int, C.POINTER(C.c_double)]),
    ("pgmg_dev_copy_r_to_x", C.c_int, [_VP, C.c_int]),
    ("pgmg_dev_norms", C.c_int, [_VP, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("pgmg_dev_solve_v_cycles", C.c_int, [_VP, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    ("pgmg_dev_solve_relres", C.c_int, [_VP, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    ("pgmg_dev_solve_io", C.c_int, [_VP, _VP, _VP, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int),
                                    C.POINTER(C.c_double)]),
    ("pgmg_batch_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("pgmg_batch_destroy", C.c_int, [_VP]),
    ("pgmg_batch_last_error", C.c_char_p, [_VP]),
    ("pgmg_batch_attach", C.c_int, [_VP, C.c_int, _VP]),
    ("pgmg_batch_detach", C.c_int, [_VP, C.c_int]),
    ("pgmg_batch_solve", C.c_int, [_VP, C.c_double, C.c_int, _VP, _VP]),
    ("pgmg_batch_launch_count", C.c_int, [_VP, C.POINTER(C.c_longlong)]),
    ("pgmg_batch_begin", C.c_int, [_VP, C.c_int]),
    ("pgmg_batch_step", C.c_int, [_VP, C.c_double, C.c_int, C.POINTER(C.c_int)]),
    ("pgmg_batch_poll", C.c_int, [_VP, _VP, _VP, _VP]),
    ("pgmg_batch_set_graphs", C.c_int, [_VP, C.c_int]),
    ("pgmg_batch_set_option", C.c_int, [_VP, C.c_int, C.c_longlong]),
    ("pgmg_dev_create_in", C.c_int, [C.POINTER(Dims), _VP, C.c_size_t, C.POINTER(C.c_void_p)]),
    ("pgmg_dev_assemble_q1", C.c_int, [_VP, _VP, C.c_int, C.c_double]),
    ("pgmg_dev_rhs_uniform", C.c_int, [_VP, C.c_uint64]),
    ("pgmg_residual_norms_noalloc", C.c_int, [C.c_int, C.c_int, C.c_int, _VP, _VP, _VP, _VP, _VP]),
    ("pgmg_problem_gauss", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_double, _dp]),
    ("pgmg_problem_kappa", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint64, C.c_double, _dp]),
    ("pgmg_problem_q1", C.c_int, [C.c_int, C.c_int, C.c_int, _VP, _dp, _VP]),
    ("pgmg_problem_rhs", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint64, _dp]),
]


def lib():
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PgmgError(3, "load", f"{LIB_PATH} not built; run python -m pgmg_b200.build")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- generators

def problem_kappa(m: int, n: int, o: int, sigma: float, seed: int, width: float = 8.0) -> np.ndarray:
    """Cell-centred kappa = exp(sigma*g), (m-1)(n-1)(o-1) cells."""
    out = np.empty((m - 1) * (n - 1) * (o - 1))
    st = lib().pgmg_problem_kappa(m, n, o, float(sigma), int(seed), float(width), out)
    if st:
        raise PgmgError(st, "pgmg_problem_kappa")
    return out


def problem_gauss(m: int, n: int, o: int, seed: int, width: float = 8.0) -> np.ndarray:
    """The normalised smoothed Gaussian cell field g (kappa = exp(sigma*g))."""
    out = np.empty((m - 1) * (n - 1) * (o - 1))
    st = lib().pgmg_problem_gauss(m, n, o, int(seed), float(width), out)
    if st:
        raise PgmgError(st, "pgmg_problem_gauss")
    return out


def problem_q1(m: int, n: int, o: int, kappa: np.ndarray | None = None):
    """Q1 FEM stencils (27 slots per point) and boxes (6 ints per point)."""
    coef = np.empty(27 * m * n * o)
    S = np.empty(6 * m * n * o, np.int32)
    kp = None
    if kappa is not None:
        kappa = np.ascontiguousarray(kappa, np.float64)
        kp = _ptr(kappa)
    st = lib().pgmg_problem_q1(m, n, o, kp, coef, _ptr(S))
    if st:
        raise PgmgError(st, "pgmg_problem_q1")
    return coef, S


def problem_rhs(m: int, n: int, o: int, seed: int) -> np.ndarray:
    out = np.empty(m * n * o)
    st = lib().pgmg_problem_rhs(m, n, o, int(seed), out)
    if st:
        raise PgmgError(st, "pgmg_problem_rhs")
    return out


def residual_norms_noalloc(m: int, n: int, o: int, coef27_ptr: int, x_ptr: int, r_ptr: int, out_ptr: int,
                           stream_ptr: int | None = None) -> None:
    """sum (r - A x)^2 and sum r^2 into out (2 device doubles) from
    caller-owned device arrays, without allocating device memory (for callers
    whose framework owns all device memory, or whose loops must not stall in
    an allocation); at most 16,777,216 points; see pgmg_dev.h."""
    st = lib().pgmg_residual_norms_noalloc(m, n, o, coef27_ptr, x_ptr, r_ptr, out_ptr, stream_ptr)
    if st:
        raise PgmgError(st, "pgmg_residual_norms_noalloc")


def plan_bytes(m, n, o, precision=FP64) -> int:
    d = Dims(m, n, o, 0, 0, 0, precision, COARSE_LU, SMOOTH_MC8, -1)
    b = C.c_size_t(0)
    st = lib().pgmg_dev_plan_bytes(C.byref(d), C.byref(b))
    if st:
        raise PgmgError(st, "pgmg_dev_plan_bytes")
    return b.value


# ---------------------------------------------------------------- solver

class Multigrid:
    """One multigrid hierarchy on one GPU (see module docstring)."""

    def __init__(self, m: int, n: int, o: int, precision: int = FP64, coarse: int = COARSE_LU,
                 smoother: int = SMOOTH_MC8, device: int = -1, prd=(False, False, False), mem=None):
        """mem: optional (device pointer, bytes) the handle lives in (no
        device allocation of its own; see pgmg_dev_create_in)."""
        self.m, self.n, self.o = m, n, o
        self.precision, self.coarse, self.smoother = precision, coarse, smoother
        self._h = None
        d = Dims(m, n, o, int(prd[0]), int(prd[1]), int(prd[2]), precision, coarse, smoother, device)
        h = C.c_void_p()
        if mem is None:
            st = lib().pgmg_dev_create(C.byref(d), C.byref(h))
        else:
            st = lib().pgmg_dev_create_in(C.byref(d), mem[0], mem[1], C.byref(h))
        if st:
            raise PgmgError(st, "pgmg_dev_create")
        self._h = h

    # -- plumbing
    def _ck(self, st, where):
        if st:
            detail = lib().pgmg_dev_last_error(self._h)
            raise PgmgError(st, where, detail.decode() if detail else "")

    def close(self):
        if self._h is not None:
            lib().pgmg_dev_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int | None):
        self._ck(lib().pgmg_dev_set_stream(self._h, stream_ptr), "set_stream")

    def sync(self):
        self._ck(lib().pgmg_dev_sync(self._h), "sync")

    @property
    def launches(self) -> int:
        v = C.c_longlong()
        self._ck(lib().pgmg_dev_launch_count(self._h, C.byref(v)), "launch_count")
        return v.value

    def set_option(self, key: int, value: int):
        self._ck(lib().pgmg_dev_set_option(self._h, key, int(value)), "set_option")

    def get_option(self, key: int) -> int:
        v = C.c_longlong()
        self._ck(lib().pgmg_dev_get_option(self._h, key, C.byref(v)), "get_option")
        return v.value

    # Result-neutral execution options the autotuner chooses among.
    TUNED_OPTIONS = {"gs_block": OPT_GS_BLOCK, "cluster_size": OPT_CLUSTER_SIZE, "cluster_first": OPT_CLUSTER_FIRST,
                     "pdl": OPT_PDL, "grid_max": OPT_GRID_MAX, "gs_vector": OPT_GS_VECTOR,
                     "gs_alternate": OPT_GS_ALTERNATE, "gs_prefetch": OPT_GS_PREFETCH,
                     "fused_restrict": OPT_FUSED_RESTRICT, "gs_tma": OPT_GS_TMA,
                     "gs_l2_prefetch": OPT_GS_L2_PREFETCH, "gs_block_levels": OPT_GS_BLOCK_LEVELS}

    def autotune(self, reps: int = 3, cache: str = None) -> dict:
        """Times V-cycles under the result-neutral execution options and keeps
        the fastest (pgmg_dev_autotune); returns the chosen options and the
        V-cycle time in ms.

        ``cache``: a JSON file of earlier choices, keyed by grid shape,
        precision, smoother and coarse solve.  A shape found there gets the
        stored options without timing (``"cached": True`` in the result);
        otherwise the choice made here is added to the file.  This lets a
        second process -- for instance the same program run under a
        profiler, where timings mean nothing -- use the options a plain run
        chose."""
        key = "%dx%dx%d/p%d/s%d/c%d" % (self.m, self.n, self.o, self.precision, self.smoother, self.coarse)
        if cache and os.path.exists(cache):
            with open(cache) as f:
                known = json.load(f)
            if key in known:
                for name, opt in self.TUNED_OPTIONS.items():
                    if name in known[key]:
                        self.set_option(opt, int(known[key][name]))
                return dict(known[key], cached=True)
        ms = C.c_double()
        self._ck(lib().pgmg_dev_autotune(self._h, int(reps), C.byref(ms)), "autotune")
        out = {name: self.get_option(opt) for name, opt in self.TUNED_OPTIONS.items()}
        out["vcycle_ms"] = ms.value
        if cache:
            known = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    known = json.load(f)
            known[key] = out
            with open(cache, "w") as f:
                json.dump(known, f, indent=1)
        return out

    def set_smoother(self, smoother: int):
        self._ck(lib().pgmg_dev_set_smoother(self._h, smoother), "set_smoother")
        self.smoother = smoother

    @property
    def nlevels(self) -> int:
        v = C.c_int()
        self._ck(lib().pgmg_dev_num_levels(self._h, C.byref(v)), "num_levels")
        return v.value

    def dims(self, level: int):
        d = np.zeros(3, np.int32)
        self._ck(lib().pgmg_dev_level_dims(self._h, level, d), "level_dims")
        return tuple(int(v) for v in d)

    def npts(self, level: int) -> int:
        m, n, o = self.dims(level)
        return m * n * o

    @property
    def memory_bytes(self) -> int:
        b = C.c_size_t()
        self._ck(lib().pgmg_dev_memory(self._h, C.byref(b)), "memory")
        return b.value

    # -- set-up
    def setup_matrices(self, coef27, S6=None):
        """Upload level-0 stencils and build every coarse operator (RAT + LU)."""
        c = coef27 if isinstance(coef27, int) else np.ascontiguousarray(coef27, np.float64)
        cp = c if isinstance(c, int) else _ptr(c)
        sp = None
        if S6 is not None:
            S6 = np.ascontiguousarray(S6, np.int32)
            sp = _ptr(S6)
        self._ck(lib().pgmg_dev_upload_level0(self._h, cp, sp), "upload_level0")
        self._ck(lib().pgmg_dev_build_rat(self._h), "build_rat")

    def assemble_q1(self, cells=None, from_log: bool = False, sigma: float = 1.0, build: bool = True):
        """Level-0 Q1 stencils assembled on the GPU from a cell field (kappa,
        or g with kappa = exp(sigma*g)); host array or device pointer."""
        if cells is None:
            cp = None
        elif isinstance(cells, int):
            cp = cells
        else:
            cells = np.ascontiguousarray(cells, np.float64)
            cp = _ptr(cells)
        self._ck(lib().pgmg_dev_assemble_q1(self._h, cp, int(from_log), float(sigma)), "assemble_q1")
        if build:
            self._ck(lib().pgmg_dev_build_rat(self._h), "build_rat")

    def rhs_uniform(self, seed: int):
        """Level-0 source = problem_rhs(m, n, o, seed), generated on the GPU."""
        self._ck(lib().pgmg_dev_rhs_uniform(self._h, int(seed)), "rhs_uniform")

    @property
    def lu_enabled(self) -> bool:
        v = C.c_int()
        self._ck(lib().pgmg_dev_lu_enabled(self._h, C.byref(v)), "lu_enabled")
        return bool(v.value)

    def get_coef(self, level: int) -> np.ndarray:
        out = np.empty(27 * self.npts(level))
        self._ck(lib().pgmg_dev_get_coef(self._h, level, _ptr(out)), "get_coef")
        return out.reshape(-1, 27)

    def get_boxes(self, level: int) -> np.ndarray:
        out = np.empty(6 * self.npts(level), np.int32)
        self._ck(lib().pgmg_dev_get_boxes(self._h, level, _ptr(out)), "get_boxes")
        return out.reshape(-1, 6)

    # -- fields
    def set_field(self, level: int, field: int, data):
        if isinstance(data, int):  # device pointer
            self._ck(lib().pgmg_dev_set_field(self._h, level, field, data), "set_field")
            return
        a = np.ascontiguousarray(data, np.float64)
        if a.size != self.npts(level):
            raise ValueError("field size does not match the level")
        self._ck(lib().pgmg_dev_set_field(self._h, level, field, _ptr(a)), "set_field")

    def get_field(self, level: int, field: int, out=None) -> np.ndarray:
        if isinstance(out, int):
            self._ck(lib().pgmg_dev_get_field(self._h, level, field, out), "get_field")
            return None
        if out is None:
            out = np.empty(self.npts(level))
        self._ck(lib().pgmg_dev_get_field(self._h, level, field, _ptr(out)), "get_field")
        return out

    def setup_fields(self, r, x=None):
        self.set_field(0, FIELD_R, r)
        if x is None:
            self.clear_x(0)
        else:
            self.set_field(0, FIELD_X, x)

    def get_x(self, level=0):
        return self.get_field(level, FIELD_X)

    def set_x(self, level, x):
        self.set_field(level, FIELD_X, x)

    def get_r(self, level=0):
        return self.get_field(level, FIELD_R)

    def set_r(self, level, r):
        self.set_field(level, FIELD_R, r)

    def get_residual(self, level=0):
        return self.get_field(level, FIELD_RES)

    def apply(self, level: int, vec) -> np.ndarray:
        """A @ vec on a level (natural order)."""
        a = np.ascontiguousarray(vec, np.float64)
        out = np.empty_like(a)
        self._ck(lib().pgmg_dev_apply(self._h, level, _ptr(a), _ptr(out)), "apply")
        return out

    def clear_x(self, level=0):
        self._ck(lib().pgmg_dev_clear_x(self._h, level), "clear_x")

    def setup_test(self, ca: int, xfield: bool, level: int = 0):
        self._ck(lib().pgmg_dev_setup_test(self._h, level, ca, int(xfield)), "setup_test")

    # -- hot path
    def gauss_seidel(self, mode: int = 0, level: int = 0, smoother: int | None = None):
        s = -1 if smoother is None else smoother
        self._ck(lib().pgmg_dev_gs(self._h, level, mode, s), "gauss_seidel")

    def restriction(self, level: int):
        self._ck(lib().pgmg_dev_restrict(self._h, level), "restriction")

    def interpolation(self, level: int):
        self._ck(lib().pgmg_dev_interp(self._h, level), "interpolation")

    def solve_exact(self):
        self._ck(lib().pgmg_dev_coarse_solve(self._h), "solve_exact")

    def v_cycle(self, mode: int = 0, smoother: int | None = None):
        s = -1 if smoother is None else smoother
        self._ck(lib().pgmg_dev_vcycle(self._h, mode, s), "v_cycle")

    def fmg_cycle(self, smoother: int | None = None):
        s = -1 if smoother is None else smoother
        self._ck(lib().pgmg_dev_fmg_cycle(self._h, s), "fmg_cycle")

    def source_soln_dot(self, level: int = 0) -> float:
        """sum x*r on a level (region::source_soln_dot)."""
        v = C.c_double(0)
        self._ck(lib().pgmg_dev_source_soln_dot(self._h, level, C.byref(v)), "source_soln_dot")
        return v.value

    def soln_diff(self, ext_x, level: int = 0) -> float:
        """sum (ext_x - x)^2 (region::soln_diff); ext_x natural order."""
        e = np.ascontiguousarray(ext_x, np.float64)
        v = C.c_double(0)
        self._ck(lib().pgmg_dev_soln_diff(self._h, level, e.ctypes.data, C.byref(v)), "soln_diff")
        return v.value

    def l0_error(self, level: int = 0) -> float:
        """max |r - A x| (region::l0_error_all)."""
        v = C.c_double(0)
        self._ck(lib().pgmg_dev_l0_error(self._h, level, C.byref(v)), "l0_error")
        return v.value

    def copy_rhs_to_soln(self, level: int = 0):
        """x = r (region::copy_rhs_to_soln)."""
        self._ck(lib().pgmg_dev_copy_r_to_x(self._h, level), "copy_r_to_x")

    def profile_vcycle(self, fp32: bool = False) -> dict:
        """Stage times (ms) of one V-cycle launched stage by stage: per level
        above the coarse part its pre-sweeps, residual+restriction,
        interpolation and post-sweeps, and the coarse part."""
        ms = np.zeros(4 * 16 + 1)
        fc = C.c_int(0)
        self._ck(lib().pgmg_dev_profile_vcycle(self._h, int(fp32), ms, len(ms), C.byref(fc)), "profile_vcycle")
        out = {"levels": [], "coarse_first": fc.value, "coarse_ms": float(ms[64])}
        for l in range(fc.value):
            out["levels"].append({"pre_ms": float(ms[4 * l]), "restrict_ms": float(ms[4 * l + 1]),
                                  "interp_ms": float(ms[4 * l + 2]), "post_ms": float(ms[4 * l + 3])})
        out["total_ms"] = float(ms.sum())
        return out

    def norms(self, level: int = 0):
        a, b = C.c_double(), C.c_double()
        self._ck(lib().pgmg_dev_norms(self._h, level, C.byref(a), C.byref(b)), "norms")
        return a.value, b.value

    def l2_error_all(self, level: int = 0) -> float:
        return self.norms(level)[0]

    def rhs_l2norm(self, level: int = 0) -> float:
        return self.norms(level)[1]

    def solve_v_cycles(self, p_scale: float = 0.0):
        res = C.c_double()
        st = C.c_int()
        cyc = C.c_int()
        self._ck(lib().pgmg_dev_solve_v_cycles(self._h, p_scale, C.byref(st), C.byref(res), C.byref(cyc)),
                 "solve_v_cycles")
        return st.value, res.value, cyc.value

    def solve(self, tol: float = 1e-10, max_cycles: int = 100, check_every: int = 1):
        cyc = C.c_int()
        rr = C.c_double()
        self._ck(lib().pgmg_dev_solve_relres(self._h, tol, max_cycles, check_every, C.byref(cyc), C.byref(rr)),
                 "solve")
        return cyc.value, rr.value

    def solve_io(self, r, x_out, tol: float = 1e-10, max_cycles: int = 100, check_every: int = 1):
        """The whole solve from caller arrays (pgmg_dev_solve_io): source r in,
        solution written to x_out (natural order; numpy arrays or pointers,
        host or device), x starting from zero."""
        n = self.npts(0)
        if not isinstance(r, int):
            r = np.ascontiguousarray(r, np.float64)
            if r.size != n:
                raise ValueError("source size does not match level 0")
        if not isinstance(x_out, int):
            if x_out.dtype != np.float64 or not x_out.flags.c_contiguous or x_out.size != n:
                raise ValueError("x_out must be a contiguous float64 array of level 0's size")
        cyc = C.c_int()
        rr = C.c_double()
        self._ck(lib().pgmg_dev_solve_io(self._h, r if isinstance(r, int) else _ptr(r),
                                         x_out if isinstance(x_out, int) else _ptr(x_out), tol, max_cycles,
                                         check_every, C.byref(cyc), C.byref(rr)), "solve_io")
        return cyc.value, rr.value


class Batch:
    """Slots of set-up ``Multigrid`` objects solved together (one launch per
    level/colour across all problems; see pgmg_batch_* in pgmg_dev.h)."""

    def __init__(self, max_slots: int, precision: int = MIXED, device: int = -1):
        self.max_slots = max_slots
        self._b = None
        b = C.c_void_p()
        st = lib().pgmg_batch_create(max_slots, precision, device, C.byref(b))
        if st:
            raise PgmgError(st, "pgmg_batch_create")
        self._b = b
        self._members = {}

    def _ck(self, st, where):
        if st:
            detail = lib().pgmg_batch_last_error(self._b)
            raise PgmgError(st, where, detail.decode() if detail else "")

    def attach(self, slot: int, mg: "Multigrid"):
        self._ck(lib().pgmg_batch_attach(self._b, slot, mg.handle), "batch_attach")
        self._members[slot] = mg

    def detach(self, slot: int):
        self._ck(lib().pgmg_batch_detach(self._b, slot), "batch_detach")
        self._members.pop(slot, None)

    def solve(self, tol: float = 1e-10, max_cycles: int = 100):
        cyc = np.zeros(self.max_slots, np.int32)
        rr = np.zeros(self.max_slots)
        self._ck(lib().pgmg_batch_solve(self._b, tol, max_cycles, _ptr(cyc), _ptr(rr)), "batch_solve")
        return cyc, rr

    def begin(self, slot: int):
        self._ck(lib().pgmg_batch_begin(self._b, slot), "batch_begin")

    def step(self, tol: float = 1e-10, max_cycles: int = 100) -> int:
        n = C.c_int()
        self._ck(lib().pgmg_batch_step(self._b, tol, max_cycles, C.byref(n)), "batch_step")
        return n.value

    def poll(self):
        act = np.zeros(self.max_slots, np.int32)
        cyc = np.zeros(self.max_slots, np.int32)
        rr = np.zeros(self.max_slots)
        self._ck(lib().pgmg_batch_poll(self._b, _ptr(act), _ptr(cyc), _ptr(rr)), "batch_poll")
        return act, cyc, rr

    def set_graphs(self, on: bool):
        self._ck(lib().pgmg_batch_set_graphs(self._b, int(on)), "batch_set_graphs")

    def set_option(self, key: int, value: int):
        """OPT_GRAPHS or OPT_PDL for the batch's step launches, OPT_CHECK_EVERY
        for its residual-check schedule (1 = every cycle, 0 = adaptive)."""
        self._ck(lib().pgmg_batch_set_option(self._b, int(key), int(value)), "batch_set_option")

    @property
    def launches(self) -> int:
        v = C.c_longlong()
        self._ck(lib().pgmg_batch_launch_count(self._b, C.byref(v)), "batch_launch_count")
        return v.value

    def close(self):
        if self._b is not None:
            lib().pgmg_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
