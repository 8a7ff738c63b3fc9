"""Python binding of the multi-threaded MPS reader (libnir_mps.so, include/nir_mps.h)
and of the SOL file I/O and solution check in the same library (include/nir_sol.h).

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

EXPORTED = ["nir_mps_read", "nir_mps_view", "nir_mps_vartypes", "nir_mps_model_name", "nir_mps_names",
            "nir_mps_quadratic", "nir_mps_timings", "nir_mps_free", "nir_mps_write", "nir_mps_last_error"]
EXPORTED_SOL = ["nir_sol_write", "nir_sol_read", "nir_sol_objective_token", "nir_eval_objective",
                "nir_verify_solution"]

# worst_kind of nir_verify_report -> the reference's worst_item prefix (src/io/sol_io.hpp:33-92)
WORST_ITEM = {0: "", 1: "Solution size mismatch", 2: "NaN/Inf in variable ", 3: "Lower bound on ",
              4: "Upper bound on ", 5: "Integrality on ", 6: "Row lower bound on ", 7: "Row upper bound on "}

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
        L.nir_mps_model_name.restype = C.c_char_p
        L.nir_mps_model_name.argtypes = [C.c_void_p]
        L.nir_mps_names.restype = C.c_int
        L.nir_mps_names.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.POINTER(C.c_char)),
                                    C.POINTER(C.POINTER(C.c_int64))]
        L.nir_mps_write.restype = C.c_int
        L.nir_mps_write.argtypes = [C.POINTER(NirLpView), C.POINTER(C.c_int8), C.c_int32, C.c_char_p,
                                    C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), C.c_int64,
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_int32,
                                    C.c_char_p]
        L.nir_mps_quadratic.restype = C.c_int
        L.nir_mps_quadratic.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_int64)),
                                        C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_double))]
        L.nir_mps_timings.restype = C.c_int
        L.nir_mps_timings.argtypes = [C.POINTER(C.c_double)]
        L.nir_mps_free.restype = None
        L.nir_mps_free.argtypes = [C.c_void_p]
        L.nir_mps_last_error.restype = C.c_char_p
        L.nir_mps_last_error.argtypes = []
        _D = C.POINTER(C.c_double)
        L.nir_sol_write.restype = C.c_int
        L.nir_sol_write.argtypes = [C.c_char_p, C.c_char_p, C.c_double, C.c_double, C.c_int32, _D, C.c_int64,
                                    C.POINTER(C.c_char_p), C.c_int64, C.c_int32]
        L.nir_sol_read.restype = C.c_int
        L.nir_sol_read.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_char_p), C.c_int32, _D, _D,
                                   C.POINTER(C.c_int32)]
        L.nir_sol_objective_token.restype = C.c_char_p
        L.nir_sol_objective_token.argtypes = [C.c_int32]
        L.nir_eval_objective.restype = C.c_double
        L.nir_eval_objective.argtypes = [C.POINTER(NirLpView), C.c_int64, C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int32), _D, _D]
        L.nir_verify_solution.restype = C.c_int
        L.nir_verify_solution.argtypes = [C.POINTER(NirLpView), C.POINTER(C.c_int8), C.c_int64,
                                          C.POINTER(C.c_int64), C.POINTER(C.c_int32), _D, _D, C.c_int64,
                                          C.c_double, C.c_double, C.c_int32, C.POINTER(VerifyReport)]
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
    name: str = "mps_model"
    col_names: list | None = None
    row_names: list | None = None

    def internal_min(self) -> tuple[LP, np.ndarray]:
        """Model::to_internal_min: for MAX, cost, offset and Q negated.
        Returns (LP, Q values)."""
        if self.sense == 1:
            return self.lp, self.q_value
        lp = self.lp
        out = LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index, lp.value, -lp.cost, lp.collo, lp.colup, lp.rowlo,
                 lp.rowup, -lp.obj_offset)
        return out, -self.q_value


class VerifyReport(C.Structure):
    _fields_ = [("passed", C.c_int32), ("worst_kind", C.c_int32), ("worst_index", C.c_int64),
                ("max_bound_viol", C.c_double), ("max_row_viol", C.c_double), ("max_int_viol", C.c_double),
                ("computed_obj", C.c_double), ("obj_rel_err", C.c_double)]


class _Handle:
    """Owns one nir_mps model; freed when the last array viewing it goes."""

    def __init__(self, h):
        self.h = h
        self._free = lib().nir_mps_free  # held so that teardown order does not matter

    def __del__(self):
        if self.h:
            self._free(self.h)
            self.h = None


class _View:
    """An array interface over memory the handle owns, keeping it alive."""

    def __init__(self, ptr, n, dt, owner):
        self.__array_interface__ = {"data": (C.cast(ptr, C.c_void_p).value or 0, True), "shape": (n,),
                                    "typestr": np.dtype(dt).str, "version": 3}
        self.owner = owner


def _view(p, n, dt, owner):
    if not n:
        return np.zeros(0, dt)
    return np.asarray(_View(p, n, dt, owner))


def _names(L, h, of_rows: int, n: int) -> list:
    chars, off = C.POINTER(C.c_char)(), C.POINTER(C.c_int64)()
    L.nir_mps_names(h, of_rows, C.byref(chars), C.byref(off))
    o = np.ctypeslib.as_array(off, shape=(n + 1,)).copy()
    blob = C.string_at(chars, int(o[-1])) if o[-1] else b""
    return [blob[o[i]:o[i + 1]].decode(errors="surrogateescape") for i in range(n)]


def read_mps(path: str, threads: int = 0, names: bool = False) -> MpsModel:
    """Reads an MPS file (threads <= 0: all hardware threads); names=True
    also returns the column and row names."""
    L = lib()
    h = C.c_void_p()
    st = L.nir_mps_read(os.fsencode(path), int(threads), C.byref(h))
    if st != 0:
        raise MpsError(st, L.nir_mps_last_error().decode(errors="replace"))
    owner = _Handle(h.value)
    v = NirLpView()
    sense = C.c_int32()
    L.nir_mps_view(h, C.byref(v), C.byref(sense))
    # the arrays are read-only views of the native model (no copy)
    lp = LP(v.nrow, v.ncol, _view(v.col_start, v.ncol + 1, np.int64, owner),
            _view(v.row_index, v.nnz, np.int32, owner), _view(v.value, v.nnz, np.float64, owner),
            _view(v.cost, v.ncol, np.float64, owner), _view(v.collo, v.ncol, np.float64, owner),
            _view(v.colup, v.ncol, np.float64, owner), _view(v.rowlo, v.nrow, np.float64, owner),
            _view(v.rowup, v.nrow, np.float64, owner), v.obj_offset)
    vt = _view(L.nir_mps_vartypes(h), v.ncol, np.int8, owner)
    qn = C.c_int64()
    qs, qi, qv = C.POINTER(C.c_int64)(), C.POINTER(C.c_int32)(), C.POINTER(C.c_double)()
    L.nir_mps_quadratic(h, C.byref(qn), C.byref(qs), C.byref(qi), C.byref(qv))
    t = (C.c_double * 6)()
    L.nir_mps_timings(t)
    model = MpsModel(lp, int(sense.value), vt, _view(qs, v.ncol + 1, np.int64, owner),
                     _view(qi, qn.value, np.int32, owner), _view(qv, qn.value, np.float64, owner),
                     dict(zip(TIMING_PHASES, list(t))), L.nir_mps_model_name(h).decode(errors="replace"))
    if names:
        model.col_names = _names(L, h, 0, v.ncol)
        model.row_names = _names(L, h, 1, v.nrow)
    return model


def write_mps(path: str, lp: LP, vartype=None, sense: int = 1, name: str = "", col_names=None, row_names=None,
              q=None, threads: int = 0) -> None:
    """MpsReader::write's bytes for the LP (file-sense cost and offset);
    q = (q_start, q_index, q_value) adds the QUADOBJ block."""
    L = lib()
    vt = None if vartype is None else np.ascontiguousarray(vartype, np.int8)

    def cnames(ns):
        if ns is None:
            return None
        arr = (C.c_char_p * len(ns))()
        arr[:] = [s.encode() for s in ns]
        return arr

    cn, rn = cnames(col_names), cnames(row_names)
    if q is not None:
        qs, qi, qv = (np.ascontiguousarray(q[0], np.int64), np.ascontiguousarray(q[1], np.int32),
                      np.ascontiguousarray(q[2], np.float64))
        qargs = (int(qs[-1]), qs.ctypes.data_as(C.POINTER(C.c_int64)), qi.ctypes.data_as(C.POINTER(C.c_int32)),
                 qv.ctypes.data_as(C.POINTER(C.c_double)))
    else:
        qargs = (0, None, None, None)
    st = L.nir_mps_write(C.byref(lp.view()), None if vt is None else vt.ctypes.data_as(C.POINTER(C.c_int8)),
                         int(sense), name.encode(), cn, rn, *qargs, int(threads), os.fsencode(path))
    if st != 0:
        raise MpsError(st, L.nir_mps_last_error().decode(errors="replace"))


def _name_array(names):
    if names is None:
        return None, 0
    arr = (C.c_char_p * len(names))()
    arr[:] = [n.encode() for n in names]
    return arr, len(names)


def write_sol(path: str, x, status: str = "optimal", objective: float = 0.0, gap: float = 0.0, col_names=None,
              ncol: int | None = None, threads: int = 0) -> None:
    """SolIo::write_sol's bytes (src/io/sol_io.hpp:110-132); status is the
    reference's status_to_string text."""
    L = lib()
    xv = np.ascontiguousarray(x, np.float64)
    names, nn = _name_array(col_names)
    st = L.nir_sol_write(os.fsencode(path), status.encode(), float(objective), float(gap),
                         int(len(xv) if ncol is None else ncol), xv.ctypes.data_as(C.POINTER(C.c_double)),
                         len(xv), names, nn, int(threads))
    if st != 0:
        raise MpsError(st, f"cannot write {path}")


def read_sol(path: str, col_names, threads: int = 0):
    """SolIo::read_sol (src/io/sol_io.hpp:134-170): (x, objective, the
    objective lines' tokens)."""
    L = lib()
    names, n = _name_array(col_names)
    x = np.zeros(n)
    obj = C.c_double()
    nobj = C.c_int32()
    st = L.nir_sol_read(os.fsencode(path), n, names, int(threads), x.ctypes.data_as(C.POINTER(C.c_double)),
                        C.byref(obj), C.byref(nobj))
    if st == 14:
        raise MpsError(st, f"cannot open {path}")
    tokens = [L.nir_sol_objective_token(k).decode() for k in range(nobj.value)]
    if st != 0:
        raise MpsError(st, f"objective token is not a number: {tokens}")
    return x, obj.value, tokens


def _q_args(q):
    if q is None:
        return (0, None, None, None), None
    qs, qi, qv = (np.ascontiguousarray(q[0], np.int64), np.ascontiguousarray(q[1], np.int32),
                  np.ascontiguousarray(q[2], np.float64))
    return (int(qs[-1]), qs.ctypes.data_as(C.POINTER(C.c_int64)), qi.ctypes.data_as(C.POINTER(C.c_int32)),
            qv.ctypes.data_as(C.POINTER(C.c_double))), (qs, qi, qv)


def eval_objective(lp: LP, x, q=None) -> float:
    """Model::eval_objective (src/model/model.hpp:73-98) in double-double."""
    qa, keep = _q_args(q)
    xv = np.ascontiguousarray(x, np.float64)
    return lib().nir_eval_objective(C.byref(lp.view()), *qa, xv.ctypes.data_as(C.POINTER(C.c_double)))


def verify_solution(lp: LP, x, claimed_obj: float, tol: float = 1e-6, vartype=None, col_names=None,
                    row_names=None, q=None, threads: int = 0) -> dict:
    """verify_solution (src/io/sol_io.hpp:25-106): the report's fields, with
    worst_item spelled as the reference spells it when names are given."""
    qa, keep = _q_args(q)
    xv = np.ascontiguousarray(x, np.float64)
    vt = None if vartype is None else np.ascontiguousarray(vartype, np.int8)
    rep = VerifyReport()
    lib().nir_verify_solution(C.byref(lp.view()), None if vt is None else vt.ctypes.data_as(C.POINTER(C.c_int8)),
                              *qa, xv.ctypes.data_as(C.POINTER(C.c_double)), len(xv), float(claimed_obj),
                              float(tol), int(threads), C.byref(rep))
    return report_dict(rep, col_names, row_names)


def report_dict(rep: VerifyReport, col_names=None, row_names=None) -> dict:
    """A nir_verify_report as the reference's VerificationReport fields
    (src/io/sol_io.hpp:14-22), worst_item spelled as the reference spells it
    (column or row index in place of a name when names are not given)."""
    item = WORST_ITEM[rep.worst_kind]
    if rep.worst_kind >= 2:
        names = row_names if rep.worst_kind >= 6 else col_names
        item += names[rep.worst_index] if names is not None else str(rep.worst_index)
    return dict(passed=bool(rep.passed), max_bound_viol=rep.max_bound_viol, max_row_viol=rep.max_row_viol,
                max_int_viol=rep.max_int_viol, computed_obj=rep.computed_obj, obj_rel_err=rep.obj_rel_err,
                worst_item=item)
