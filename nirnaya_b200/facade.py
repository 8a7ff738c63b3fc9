"""Python binding of the presolve and scaling before the PDHG path
(libnir_facade.so, include/nir_facade.h).

`presolve(lp, vartype)` is sov::Presolver::presolve
(src/presolve/presolve.hpp:32-345) on the internal-minimisation LP, and
`scale(lp, vartype)` is sov::scale_model (src/model/scaling.hpp:56-154).
Solver::solve runs them in that order before PdhgSolver::solve
(include/sov/solver.hpp:155-181).  Both run in parallel on the host and
return what the reference returns, bit for bit.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from .lp import LP, NirLpView

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

EXPORTED = ["nir_presolve", "nir_presolved_status", "nir_presolved_reduced", "nir_presolved_maps",
            "nir_presolved_free", "nir_scale", "nir_facade_last_error"]

OPTIMAL, INFEASIBLE, UNBOUNDED = 0, 1, 2

_D = C.POINTER(C.c_double)


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libnir_facade.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m nirnaya_b200.build`")
        L = C.CDLL(path)
        L.nir_presolve.restype = C.c_int
        L.nir_presolve.argtypes = [C.POINTER(NirLpView), C.POINTER(C.c_int8), C.c_int32, C.c_int32,
                                   C.POINTER(C.c_void_p)]
        L.nir_presolved_status.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                           C.POINTER(C.c_int32)]
        L.nir_presolved_reduced.argtypes = [C.c_void_p, C.POINTER(NirLpView), C.POINTER(C.POINTER(C.c_int8))]
        L.nir_presolved_maps.argtypes = [C.c_void_p, C.POINTER(C.POINTER(C.c_int32)),
                                         C.POINTER(C.POINTER(C.c_int32)), C.POINTER(_D),
                                         C.POINTER(C.POINTER(C.c_uint8))]
        L.nir_presolved_free.restype = None
        L.nir_presolved_free.argtypes = [C.c_void_p]
        L.nir_scale.restype = C.c_int
        L.nir_scale.argtypes = [C.POINTER(NirLpView), C.POINTER(C.c_int8), C.c_int32, C.c_int64,
                                C.POINTER(C.c_int64), C.POINTER(C.c_int32), _D, C.c_int32, _D, _D,
                                C.POINTER(C.c_int32), _D, _D, _D, _D, _D, _D, _D]
        L.nir_facade_last_error.restype = C.c_char_p
        _LIB = L
    return _LIB


@dataclass
class Presolved:
    status: int                 # OPTIMAL (continue / solved), INFEASIBLE or UNBOUNDED
    solved_in_presolve: bool
    rows_removed: int
    cols_removed: int
    bound_tightenings: int
    reduced: LP                 # empty when presolve stopped early
    vartype: np.ndarray         # int8[reduced.ncol]
    orig_col_map: np.ndarray    # int32[reduced.ncol]
    orig_row_map: np.ndarray    # int32[reduced.nrow]
    fixed_x: np.ndarray         # float64[original ncol]
    is_col_fixed: np.ndarray    # bool[original ncol]

    def postsolve(self, x_red) -> np.ndarray:
        """PresolveResult::postsolve (src/presolve/presolve.hpp:21-26)."""
        x = self.fixed_x.copy()
        k = min(len(self.orig_col_map), len(x_red))
        x[self.orig_col_map[:k]] = np.asarray(x_red, dtype=np.float64)[:k]
        return x


def _cp(p, n, dt):
    return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)


def _vt(vartype, n):
    if vartype is None:
        return None, None
    a = np.ascontiguousarray(vartype, np.int8)
    assert a.size == n
    return a, a.ctypes.data_as(C.POINTER(C.c_int8))


def presolve(lp: LP, vartype=None, max_rounds: int = 20, threads: int = 0) -> Presolved:
    L = lib()
    _, vtp = _vt(vartype, lp.ncol)
    h = C.c_void_p()
    st = L.nir_presolve(C.byref(lp.view()), vtp, int(max_rounds), int(threads), C.byref(h))
    if st != 0:
        raise RuntimeError(f"nir_presolve: status {st}: {L.nir_facade_last_error().decode()}")
    try:
        status, solved, cnt = C.c_int32(), C.c_int32(), (C.c_int32 * 3)()
        L.nir_presolved_status(h, C.byref(status), C.byref(solved), cnt)
        v = NirLpView()
        vt = C.POINTER(C.c_int8)()
        L.nir_presolved_reduced(h, C.byref(v), C.byref(vt))
        red = LP(v.nrow, v.ncol, _cp(v.col_start, v.ncol + 1, np.int64), _cp(v.row_index, v.nnz, np.int32),
                 _cp(v.value, v.nnz, np.float64), _cp(v.cost, v.ncol, np.float64), _cp(v.collo, v.ncol, np.float64),
                 _cp(v.colup, v.ncol, np.float64), _cp(v.rowlo, v.nrow, np.float64),
                 _cp(v.rowup, v.nrow, np.float64), v.obj_offset)
        cm, rm = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)()
        fx, isf = _D(), C.POINTER(C.c_uint8)()
        L.nir_presolved_maps(h, C.byref(cm), C.byref(rm), C.byref(fx), C.byref(isf))
        return Presolved(int(status.value), bool(solved.value), int(cnt[0]), int(cnt[1]), int(cnt[2]), red,
                         _cp(vt, v.ncol, np.int8), _cp(cm, v.ncol, np.int32), _cp(rm, v.nrow, np.int32),
                         _cp(fx, lp.ncol, np.float64), _cp(isf, lp.ncol, np.uint8).astype(bool))
    finally:
        L.nir_presolved_free(h)


@dataclass
class Scaled:
    active: bool
    R: np.ndarray   # row scales (powers of two)
    C: np.ndarray   # column scales
    lp: LP          # the scaled LP
    q_value: np.ndarray | None


def scale(lp: LP, vartype=None, enable: bool = True, q=None, threads: int = 0) -> Scaled:
    L = lib()
    _, vtp = _vt(vartype, lp.ncol)
    m, n = lp.nrow, lp.ncol
    R, Cs = np.ones(m), np.ones(n)
    out = {k: np.empty_like(getattr(lp, k)) for k in ("cost", "collo", "colup", "value", "rowlo", "rowup")}
    act = C.c_int32()
    if q is not None:
        qs, qi, qv = (np.ascontiguousarray(q[0], np.int64), np.ascontiguousarray(q[1], np.int32),
                      np.ascontiguousarray(q[2], np.float64))
        qo = np.empty_like(qv)
        qargs = (int(qs[-1]), qs.ctypes.data_as(C.POINTER(C.c_int64)), qi.ctypes.data_as(C.POINTER(C.c_int32)),
                 qv.ctypes.data_as(_D))
    else:
        qo, qargs = None, (0, None, None, None)
    dp = lambda a: a.ctypes.data_as(_D)  # noqa: E731
    st = L.nir_scale(C.byref(lp.view()), vtp, int(bool(enable)), *qargs, int(threads), dp(R), dp(Cs), C.byref(act),
                     dp(out["cost"]), dp(out["collo"]), dp(out["colup"]), dp(out["value"]), dp(out["rowlo"]),
                     dp(out["rowup"]), None if qo is None else dp(qo))
    if st != 0:
        raise RuntimeError(f"nir_scale: status {st}: {L.nir_facade_last_error().decode()}")
    slp = LP(m, n, lp.col_start, lp.row_index, out["value"], out["cost"], out["collo"], out["colup"], out["rowlo"],
             out["rowup"], lp.obj_offset)
    return Scaled(bool(act.value), R, Cs, slp, qo)
