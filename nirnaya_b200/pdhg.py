"""Python mirror of the reference's PDHG interface over the C ABI.

The reference's path is `sov::PdhgSolver::solve(const Model&, const
Options&, const Deadline&) -> PdhgResult` (src/gpu/pdhg_solver.hpp:14-25).
This module keeps those names and meanings:

  * `Options.threads`, `Options.simplex_iter_limit` and `Options.time_limit`
    mean what they mean in src/core/options.hpp:10-32; the iteration cap is
    max(5000, simplex_iter_limit // 10) as at src/gpu/pdhg_solver.hpp:60;
  * `Deadline` mirrors src/core/timer.hpp:34-46 (wall limit plus a stop flag
    that another thread may set, like Solver::interrupt);
  * `PdhgResult` has the reference's fields (status, objective, x, y,
    iterations) plus the engine's diagnostics.

Everything runs in libnir_pdhg.so on the GPU.  There is no CPU fallback:
if the library or a CUDA device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .lp import LP, NirLpView
from .mps import VerifyReport, report_dict

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnir_pdhg.so")

# sov::Status (src/core/status.hpp:7-24)
OPTIMAL, TIME_LIMIT, ITERATION_LIMIT, INTERRUPTED, NUMERICAL_TROUBLE, INPUT_ERROR, INTERNAL_ERROR = 0, 4, 6, 10, 11, 12, 14
STATUS_NAMES = {0: "optimal", 4: "time_limit", 6: "iteration_limit", 10: "interrupted", 11: "numerical_trouble",
                12: "input_error", 14: "internal_error"}

ALGO_REFERENCE, ALGO_PDHG, ALGO_PDLP = 0, 1, 2
PREC_FP64, PREC_MIXED, PREC_FP32 = 0, 1, 2


class Params(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int32), ("precision", C.c_int32), ("tol", C.c_double), ("feas_tol", C.c_double),
        ("max_iters", C.c_int64), ("time_limit", C.c_double), ("check_every", C.c_int32),
        ("ruiz_iters", C.c_int32), ("pock_chambolle", C.c_int32), ("reflection", C.c_double),
        ("restart_sufficient", C.c_double), ("restart_necessary", C.c_double),
        ("restart_artificial", C.c_double), ("primal_weight_smoothing", C.c_double),
        ("step_factor", C.c_double), ("power_iters", C.c_int32), ("polish_stall_checks", C.c_int32),
        ("polish_switch_kkt", C.c_double), ("spmv_block_nnz", C.c_int32), ("use_graphs", C.c_int32),
        ("verbose", C.c_int32), ("restart_anchor", C.c_int32), ("polish_fresh", C.c_int32),
        ("x_init", C.POINTER(C.c_double)), ("y_init", C.POINTER(C.c_double)),
        ("omega_init", C.c_double), ("primal_weight_decades", C.c_double), ("persistent", C.c_int32),
        ("pad_", C.c_int32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("restarts", C.c_int32), ("iterations", C.c_int64),
        ("iterations_fp64", C.c_int64), ("objective", C.c_double), ("rel_kkt", C.c_double),
        ("rel_primal", C.c_double), ("rel_dual", C.c_double), ("rel_gap", C.c_double),
        ("max_rel_row_viol", C.c_double), ("primal_weight", C.c_double), ("step_size", C.c_double),
        ("setup_seconds", C.c_double), ("solve_seconds", C.c_double), ("time_to_fp64_seconds", C.c_double),
        ("kernel_launches", C.c_int32), ("parallel_groups", C.c_int32), ("iterations_to_tol", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class KernelTime(C.Structure):
    """Mean event times of the fused kernels; index 0 = FP32 chunks, 1 = FP64."""
    _fields_ = [("primal_us", C.c_double * 2), ("dual_us", C.c_double * 2), ("iter_us", C.c_double * 2),
                ("samples", C.c_int64 * 2)]


class Layout(C.Structure):
    _fields_ = [("nrow", C.c_int32), ("ncol", C.c_int32), ("nnz", C.c_int64), ("blocks_a", C.c_int32),
                ("blocks_at", C.c_int32), ("block_nnz", C.c_int32), ("device_bytes", C.c_int64),
                ("block_nnz_at", C.c_int32), ("pad_", C.c_int32)]


POLL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)

EXPORTED = [
    "nir_pdhg_default_params", "nir_pdhg_create", "nir_pdhg_update_vectors", "nir_pdhg_solve",
    "nir_pdhg_solve_lp", "nir_pdhg_free", "nir_pdhg_last_error", "nir_pdhg_spmv", "nir_pdhg_time_spmv",
    "nir_pdhg_set_profiling", "nir_pdhg_kernel_times", "nir_pdhg_get_layout", "nir_pdhg_history",
    "nir_pdhg_reference_solve_noalloc", "nir_pdhg_batch_create", "nir_pdhg_batch_solve", "nir_pdhg_batch_free",
    "nir_pdhg_verify", "nir_pdhg_batch_verify", "nir_pdhg_spmv_kernel", "nir_pdhg_time_kernel",
    "nir_pdhg_time_iteration", "nir_pdhg_parallel_groups",
]

# Kernel kinds of nir_pdhg_spmv_kernel / nir_pdhg_time_kernel.
K_REF, K_WARP64, K_WARP32, K_CTA64, K_CTA32, K_CTA_MIXED = 0, 1, 2, 3, 4, 5
K_CEIL_GATHER64, K_CEIL_GATHER32, K_CEIL_STREAM64, K_CEIL_STREAM32 = 6, 7, 8, 9

_lib = None


def lib():
    """Loads libnir_pdhg.so (raises if it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m nirnaya_b200.build`")
        L = C.CDLL(LIB_PATH)
        VP = C.POINTER(NirLpView)
        D = C.POINTER(C.c_double)
        L.nir_pdhg_default_params.argtypes = [C.POINTER(Params)]
        L.nir_pdhg_create.argtypes = [VP, C.c_int, C.POINTER(C.c_void_p)]
        L.nir_pdhg_update_vectors.argtypes = [C.c_void_p, D, D, D, D, D]
        L.nir_pdhg_solve.argtypes = [C.c_void_p, C.POINTER(Params), POLL_FN, C.c_void_p, D, D, C.POINTER(Info)]
        L.nir_pdhg_solve_lp.argtypes = [VP, C.c_int, C.POINTER(Params), POLL_FN, C.c_void_p, D, D, C.POINTER(Info)]
        L.nir_pdhg_free.argtypes = [C.c_void_p]
        L.nir_pdhg_last_error.restype = C.c_char_p
        L.nir_pdhg_spmv.argtypes = [C.c_void_p, C.c_int, C.c_int, D, D]
        L.nir_pdhg_time_spmv.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, D]
        L.nir_pdhg_spmv_kernel.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, D, D]
        L.nir_pdhg_time_kernel.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, D]
        L.nir_pdhg_time_iteration.argtypes = [C.c_void_p, C.c_int, C.c_int, D, D, D]
        L.nir_pdhg_parallel_groups.argtypes = [VP, C.POINTER(C.c_int32), D, C.POINTER(C.c_int32)]
        L.nir_pdhg_set_profiling.argtypes = [C.c_void_p, C.c_int]
        L.nir_pdhg_kernel_times.argtypes = [C.c_void_p, C.POINTER(KernelTime)]
        L.nir_pdhg_get_layout.argtypes = [C.c_void_p, C.POINTER(Layout)]
        L.nir_pdhg_history.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
        L.nir_pdhg_verify.argtypes = [C.c_void_p, D, C.POINTER(C.c_int8), C.c_double, C.c_double,
                                      C.POINTER(VerifyReport)]
        _lib = L
    return _lib


def last_error() -> str:
    return lib().nir_pdhg_last_error().decode()


def default_params(**overrides) -> Params:
    p = Params()
    lib().nir_pdhg_default_params(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def parallel_groups(lp: LP):
    """(rep_of, lam, groups): the parallel-column groups the engine
    re-expresses before a PDHG / PDLP solve (nir_pdhg_parallel_groups;
    host only)."""
    rep = np.zeros(lp.ncol, np.int32)
    lam = np.zeros(lp.ncol)
    g = C.c_int32()
    rc = lib().nir_pdhg_parallel_groups(C.byref(lp.view()), rep.ctypes.data_as(C.POINTER(C.c_int32)),
                                        lam.ctypes.data_as(C.POINTER(C.c_double)), C.byref(g))
    if rc != 0:
        raise RuntimeError(last_error())
    return rep, lam, g.value


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _start_ptr(v, keep):
    """A starting vector for nir_pdhg_solve: a device address (int) as is,
    else a contiguous FP64 host copy kept alive in keep."""
    if isinstance(v, (int, np.integer)) and not isinstance(v, bool):
        return C.cast(C.c_void_p(int(v)), C.POINTER(C.c_double))
    a = np.ascontiguousarray(v, np.float64)
    keep.append(a)
    return _dptr(a)


class Engine:
    """One LP resident on one GPU (nir_pdhg_create ... nir_pdhg_free)."""

    def __init__(self, lp: LP, device: int = 0):
        self.lp = lp
        self._h = C.c_void_p()
        rc = lib().nir_pdhg_create(C.byref(lp.view()), device, C.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"nir_pdhg_create failed ({STATUS_NAMES.get(rc, rc)}): {last_error()}")

    def close(self):
        if self._h:
            lib().nir_pdhg_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def update_vectors(self, cost=None, collo=None, colup=None, rowlo=None, rowup=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (cost, collo, colup, rowlo, rowup)]
        ptrs = [None if a is None else _dptr(a) for a in arrs]
        rc = lib().nir_pdhg_update_vectors(self._h, *ptrs)
        if rc != 0:
            raise RuntimeError(last_error())
        for name, a in zip(("cost", "collo", "colup", "rowlo", "rowup"), arrs):
            if a is not None:
                setattr(self.lp, name, a)
        self.lp._view = None

    def solve(self, params: Params | None = None, poll=None, x_init=None, y_init=None, omega_init=None):
        """x_init / y_init: host arrays, or device addresses (int) of FP64
        vectors on this handle's device, complete before the call."""
        # a copy: the warm-start pointers must not outlive this call in the caller's params
        p = Params.from_buffer_copy(params) if params is not None else default_params()
        keep = []
        if x_init is not None:
            p.x_init = _start_ptr(x_init, keep)
        if y_init is not None:
            p.y_init = _start_ptr(y_init, keep)
        if omega_init is not None:
            p.omega_init = float(omega_init)
        x = np.zeros(self.lp.ncol)
        y = np.zeros(self.lp.nrow)
        info = Info()
        cb = POLL_FN(0) if poll is None else POLL_FN(lambda _ctx: 1 if poll() else 0)
        lib().nir_pdhg_solve(self._h, C.byref(p), cb, None, _dptr(x), _dptr(y), C.byref(info))
        if info.status in (INPUT_ERROR, INTERNAL_ERROR):
            raise RuntimeError(f"nir_pdhg_solve failed ({STATUS_NAMES[info.status]}): {last_error()}")
        return x, y, info

    def spmv(self, x, transpose: bool = False, kernel: int = 1):
        nout = self.lp.ncol if transpose else self.lp.nrow
        y = np.zeros(nout)
        rc = lib().nir_pdhg_spmv(self._h, int(transpose), kernel, _dptr(np.ascontiguousarray(x, np.float64)), _dptr(y))
        if rc != 0:
            raise RuntimeError(last_error())
        return y

    def time_spmv(self, transpose: bool, kernel: int, reps: int = 20, flush_l2: bool = True) -> float:
        us = C.c_double()
        rc = lib().nir_pdhg_time_spmv(self._h, int(transpose), kernel, reps, int(flush_l2), C.byref(us))
        if rc != 0:
            raise RuntimeError(last_error())
        return us.value

    def spmv_kernel(self, x, transpose: bool, kernel: int, block_nnz: int = 0):
        """One SpMV of the unscaled matrix with a chosen kernel kind (K_*)."""
        nout = self.lp.ncol if transpose else self.lp.nrow
        y = np.zeros(nout)
        rc = lib().nir_pdhg_spmv_kernel(self._h, int(transpose), kernel, block_nnz,
                                        _dptr(np.ascontiguousarray(x, np.float64)), _dptr(y))
        if rc != 0:
            raise RuntimeError(last_error())
        return y

    def time_kernel(self, transpose: bool, kernel: int, block_nnz: int = 0, reps: int = 20,
                    flush_l2: bool = True) -> float:
        """Mean CUDA-event time (us) of one launch of a kernel kind (K_*),
        including the row-less ceilings."""
        us = C.c_double()
        rc = lib().nir_pdhg_time_kernel(self._h, int(transpose), kernel, block_nnz, reps, int(flush_l2), C.byref(us))
        if rc != 0:
            raise RuntimeError(last_error())
        return us.value

    def time_iteration(self, precision: int, reps: int = 200):
        """(primal_us, dual_us, pair_us): steady-state event times of the
        fused iteration kernels after a solve (nir_pdhg_time_iteration)."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        rc = lib().nir_pdhg_time_iteration(self._h, precision, reps, C.byref(a), C.byref(b), C.byref(c))
        if rc != 0:
            raise RuntimeError(last_error())
        return a.value, b.value, c.value

    def set_profiling(self, on: bool):
        lib().nir_pdhg_set_profiling(self._h, int(on))

    def kernel_times(self) -> KernelTime:
        kt = KernelTime()
        lib().nir_pdhg_kernel_times(self._h, C.byref(kt))
        return kt

    def history(self, max_entries: int = 4096) -> np.ndarray:
        """(iteration, kkt, primal, dual, gap, residual, omega, phase) per check."""
        buf = np.zeros((max_entries, 8))
        cnt = lib().nir_pdhg_history(self._h, _dptr(buf), max_entries)
        if cnt < 0:
            raise RuntimeError(last_error())
        return buf[:cnt].copy()

    def verify(self, x, claimed_obj: float = float("nan"), tol: float = 1e-6, vartype=None, col_names=None,
               row_names=None) -> dict:
        """verify_solution (src/io/sol_io.hpp:25-106) on the GPU against
        this handle's LP (nir_pdhg_verify): the report mps.verify_solution
        gives on the host, bit for bit.  x None checks the point the last
        solve returned, where it still lies on the device."""
        xv = None
        if x is not None:
            xv = np.ascontiguousarray(x, np.float64)
            if xv.shape != (self.lp.ncol,):
                raise ValueError(f"x has {xv.size} values for {self.lp.ncol} columns")
        vt = None if vartype is None else np.ascontiguousarray(vartype, np.int8)
        if vt is not None and vt.shape != (self.lp.ncol,):
            raise ValueError(f"vartype has {vt.size} marks for {self.lp.ncol} columns")
        rep = VerifyReport()
        rc = lib().nir_pdhg_verify(self._h, None if xv is None else _dptr(xv),
                                   None if vt is None else vt.ctypes.data_as(C.POINTER(C.c_int8)),
                                   float(claimed_obj), float(tol), C.byref(rep))
        if rc != 0:
            raise RuntimeError(f"nir_pdhg_verify failed ({STATUS_NAMES.get(rc, rc)}): {last_error()}")
        return report_dict(rep, col_names, row_names)

    def layout(self) -> Layout:
        lo = Layout()
        lib().nir_pdhg_get_layout(self._h, C.byref(lo))
        return lo


# ------------------------------------------------------- reference-shaped API

@dataclass
class Options:
    """The fields of sov::Options (src/core/options.hpp:9-32) the path reads,
    plus the engine's knobs (defaults: include/nir_pdhg.h)."""
    time_limit: float = 600.0
    threads: int = 1
    simplex_iter_limit: int = 500000
    method: str = "pdhg"
    pdhg_algorithm: int = ALGO_PDLP
    pdhg_precision: int = PREC_MIXED
    pdhg_tol: float = 1e-6
    pdhg_feas_tol: float = 0.0
    pdhg_max_iters: int = 0            # 0 = the reference's max(5000, simplex_iter_limit // 10),
                                       # times 10 for the restarted methods (as the C++ drop-in)
    device: int = 0
    extra: dict = field(default_factory=dict)


class Deadline:
    """sov::Deadline (src/core/timer.hpp:34-46): wall limit + stop flag."""

    def __init__(self, wall_limit_sec: float = float("inf")):
        self.start = time.monotonic()
        self.wall_limit_sec = wall_limit_sec
        self._stop = threading.Event()

    def interrupt(self):
        self._stop.set()

    def expired(self) -> bool:
        return self._stop.is_set() or (time.monotonic() - self.start) >= self.wall_limit_sec


@dataclass
class PdhgResult:
    status: int
    objective: float
    x: np.ndarray
    y: np.ndarray
    iterations: int
    info: dict = field(default_factory=dict)


class PdhgSolver:
    """sov::PdhgSolver (src/gpu/pdhg_solver.hpp:23-108) on the GPU."""

    @staticmethod
    def params_from(options: Options) -> Params:
        ref_cap = max(5000, options.simplex_iter_limit // 10)
        cap = options.pdhg_max_iters or (ref_cap if options.pdhg_algorithm == ALGO_REFERENCE else 10 * ref_cap)
        p = default_params(algorithm=options.pdhg_algorithm, precision=options.pdhg_precision,
                           tol=options.pdhg_tol, feas_tol=options.pdhg_feas_tol, max_iters=cap)
        for k, v in options.extra.items():
            setattr(p, k, v)
        return p

    @staticmethod
    def solve(model: LP, options: Options | None = None, deadline: Deadline | None = None) -> PdhgResult:
        options = options or Options()
        deadline = deadline or Deadline(options.time_limit)
        p = PdhgSolver.params_from(options)
        with Engine(model, options.device) as eng:
            x, y, info = eng.solve(p, poll=deadline.expired)
        status = info.status
        # as the C++ drop-in: at the cap with only the row margin missing,
        # the point meets the PDHG criterion and is reported Optimal
        if status == ITERATION_LIMIT and p.feas_tol > 0.0 and info.rel_kkt <= p.tol:
            status = OPTIMAL
        return PdhgResult(status, info.objective, x, y, int(info.iterations), info.as_dict())
