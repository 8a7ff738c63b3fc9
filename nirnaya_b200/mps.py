"""Python binding of the multi-threaded MPS reader (libnir_mps.so, include/nir_mps.h).

`read_mps(path)` is sov::MpsReader::read (src/io/mps_reader.hpp:15-304)
followed by Model::validate (src/model/model.hpp:117-178): it returns the
model in the file's own objective sense, and `MpsModel.internal_min()`
applies Model::to_internal_min (src/model/model.hpp:101-110) -- the LP the
PDHG path solves.  Failures raise `MpsError` carrying the sov::Status code
(1 infeasible bounds, 12 input error) and the reference's message.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from .lp import LP, NirLpView

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

EXPORTED = ["nir_mps_read", "nir_mps_view", "nir_mps_vartypes", "nir_mps_quadratic", "nir_mps_timings",
            "nir_mps_free", "nir_mps_last_error"]

CONTINUOUS, INTEGER, BINARY = 0, 1, 2
TIMING_PHASES = ("file_read", "line_scan", "columns_parse", "columns_replay", "csc_build", "other")


class MpsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"status {status}: {message}")
        self.status = status
        self.message = message


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libnir_mps.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m nirnaya_b200.build`")
        L = C.CDLL(path)
        L.nir_mps_read.restype = C.c_int
        L.nir_mps_read.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p)]
        L.nir_mps_view.restype = C.c_int
        L.nir_mps_view.argtypes = [C.c_void_p, C.POINTER(NirLpView), C.POINTER(C.c_int32)]
        L.nir_mps_vartypes.restype = C.POINTER(C.c_int8)
        L.nir_mps_vartypes.argtypes = [C.c_void_p]
        L.nir_mps_quadratic.restype = C.c_int
        L.nir_mps_quadratic.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_int64)),
                                        C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_double))]
        L.nir_mps_timings.restype = C.c_int
        L.nir_mps_timings.argtypes = [C.POINTER(C.c_double)]
        L.nir_mps_free.restype = None
        L.nir_mps_free.argtypes = [C.c_void_p]
        L.nir_mps_last_error.restype = C.c_char_p
        L.nir_mps_last_error.argtypes = []
        _LIB = L
    return _LIB


@dataclass
class MpsModel:
    lp: LP                      # file sense: cost and offset as written
    sense: int                  # 1 minimise, -1 maximise
    vartype: np.ndarray         # int8[ncol]: 0 continuous, 1 integer, 2 binary
    q_start: np.ndarray         # int64[ncol+1], quadratic objective (upper triangle)
    q_index: np.ndarray         # int32[qnnz]
    q_value: np.ndarray         # float64[qnnz]
    timings: dict

    def internal_min(self) -> tuple[LP, np.ndarray]:
        """Model::to_internal_min: for MAX, cost, offset and Q negated.
        Returns (LP, Q values)."""
        if self.sense == 1:
            return self.lp, self.q_value
        lp = self.lp
        out = LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index, lp.value, -lp.cost, lp.collo, lp.colup, lp.rowlo,
                 lp.rowup, -lp.obj_offset)
        return out, -self.q_value


def _copy(p, n, dt):
    return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)


def read_mps(path: str, threads: int = 0) -> MpsModel:
    L = lib()
    h = C.c_void_p()
    st = L.nir_mps_read(os.fsencode(path), int(threads), C.byref(h))
    if st != 0:
        raise MpsError(st, L.nir_mps_last_error().decode(errors="replace"))
    try:
        v = NirLpView()
        sense = C.c_int32()
        L.nir_mps_view(h, C.byref(v), C.byref(sense))
        lp = LP(v.nrow, v.ncol, _copy(v.col_start, v.ncol + 1, np.int64), _copy(v.row_index, v.nnz, np.int32),
                _copy(v.value, v.nnz, np.float64), _copy(v.cost, v.ncol, np.float64),
                _copy(v.collo, v.ncol, np.float64), _copy(v.colup, v.ncol, np.float64),
                _copy(v.rowlo, v.nrow, np.float64), _copy(v.rowup, v.nrow, np.float64), v.obj_offset)
        vt = _copy(L.nir_mps_vartypes(h), v.ncol, np.int8)
        qn = C.c_int64()
        qs, qi, qv = C.POINTER(C.c_int64)(), C.POINTER(C.c_int32)(), C.POINTER(C.c_double)()
        L.nir_mps_quadratic(h, C.byref(qn), C.byref(qs), C.byref(qi), C.byref(qv))
        t = (C.c_double * 6)()
        L.nir_mps_timings(t)
        return MpsModel(lp, int(sense.value), vt, _copy(qs, v.ncol + 1, np.int64), _copy(qi, qn.value, np.int32),
                        _copy(qv, qn.value, np.float64), dict(zip(TIMING_PHASES, list(t))))
    finally:
        L.nir_mps_free(h)
