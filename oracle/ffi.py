"""ctypes bindings of the oracle (liboracle.so, our C restatement) and of the
reference compiled from source (_ref/libref_nirnaya.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from nirnaya_b200.lp import LP, NirLpView

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_nirnaya.so")

_VP = C.POINTER(NirLpView)
_D = C.POINTER(C.c_double)


class PdhgOut(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("stopped", C.c_int32), ("objective", C.c_double),
                ("tau", C.c_double), ("sigma", C.c_double), ("first_hit", C.c_int64),
                ("last_kkt", C.c_double)]


class VerifyReport(C.Structure):
    _fields_ = [("passed", C.c_int32), ("max_bound_viol", C.c_double), ("max_row_viol", C.c_double),
                ("computed_obj", C.c_double), ("obj_rel_err", C.c_double)]


class Kkt(C.Structure):
    _fields_ = [("rel_primal", C.c_double), ("rel_dual", C.c_double), ("rel_gap", C.c_double),
                ("rel_kkt", C.c_double), ("pobj", C.c_double), ("dobj", C.c_double),
                ("max_rel_row_viol", C.c_double)]


def _dptr(a):
    return a.ctypes.data_as(_D)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        lib = C.CDLL(ORACLE_SO)
        lib.or_dd_cancellation_probe.restype = C.c_double
        lib.or_dd_cancellation_probe.argtypes = [C.c_double] * 3
        lib.or_neumaier_probe.restype = C.c_double
        lib.or_neumaier_probe.argtypes = [C.c_double] * 3
        lib.or_spmv.argtypes = [_VP, _D, _D]
        lib.or_spmv_t.argtypes = [_VP, _D, _D]
        lib.or_csc_from_triplets.restype = C.c_int64
        lib.or_csc_from_triplets.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32), _D, C.POINTER(C.c_int64),
                                             C.POINTER(C.c_int32), _D]
        lib.or_ref_pdhg.argtypes = [_VP, C.c_int64, C.c_int64, C.c_double, C.c_int, _D, _D, C.POINTER(PdhgOut)]
        lib.or_eval_objective.restype = C.c_double
        lib.or_eval_objective.argtypes = [_VP, _D]
        lib.or_verify.argtypes = [_VP, _D, C.c_double, C.c_double, C.POINTER(VerifyReport)]
        lib.or_rel_kkt.argtypes = [_VP, _D, _D, C.POINTER(Kkt)]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"{REF_SO} is missing (built from the reference sources by oracle/Makefile)")
        lib = C.CDLL(REF_SO)
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_pdhg_solve.argtypes = [_VP, C.c_int, C.c_int, C.c_double, _D, _D, C.POINTER(C.c_int),
                                       _D, C.POINTER(C.c_int)]
        lib.ref_solver_solve.argtypes = [_VP, C.c_int, C.c_char_p, C.c_int, C.c_int, _D, C.POINTER(C.c_int),
                                         _D, C.POINTER(C.c_int)]
        lib.ref_verify.argtypes = [_VP, _D, C.c_double, C.c_double, C.POINTER(C.c_int), _D, _D, _D, _D]
        lib.ref_eval_objective.restype = C.c_double
        lib.ref_eval_objective.argtypes = [_VP, _D]
        lib.ref_spmv.argtypes = [_VP, _D, _D]
        lib.ref_spmv_t.argtypes = [_VP, _D, _D]
        lib.ref_from_triplets.restype = C.c_int64
        lib.ref_from_triplets.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32), _D, C.POINTER(C.c_int64),
                                          C.POINTER(C.c_int32), _D]
        lib.ref_dd_probe.argtypes = [C.c_double] * 3 + [_D, _D]
        lib.ref_read_mps.restype = C.c_void_p
        lib.ref_read_mps.argtypes = [C.c_char_p]
        lib.ref_model_view.argtypes = [C.c_void_p, _VP, C.POINTER(C.c_int)]
        lib.ref_model_free.argtypes = [C.c_void_p]
        lib.ref_last_status.restype = C.c_int
        lib.ref_model_vartypes.argtypes = [C.c_void_p, C.POINTER(C.c_int8)]
        lib.ref_model_qnnz.restype = C.c_int64
        lib.ref_model_qnnz.argtypes = [C.c_void_p]
        lib.ref_model_q.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32), _D]
        lib.ref_write_mps.argtypes = [_VP, C.POINTER(C.c_int8), C.c_int, C.c_char_p]
        lib.ref_mps_roundtrip.argtypes = [C.c_char_p, C.c_char_p]
        lib.ref_presolve.restype = C.c_void_p
        lib.ref_presolve.argtypes = [_VP, C.POINTER(C.c_int8), C.c_int, C.c_int]
        lib.ref_presolved_status.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                             C.POINTER(C.c_int)]
        lib.ref_presolved_reduced.argtypes = [C.c_void_p, _VP, C.POINTER(C.c_int8)]
        lib.ref_presolved_maps.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _D,
                                           C.POINTER(C.c_uint8)]
        lib.ref_presolved_map_sizes.restype = C.c_int64
        lib.ref_presolved_map_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        lib.ref_presolved_free.argtypes = [C.c_void_p]
        lib.ref_write_sol.argtypes = [_VP, C.POINTER(C.c_char_p), C.c_int, C.c_double, C.c_double, _D, C.c_int64,
                                      C.c_char_p]
        lib.ref_verify_full.argtypes = [_VP, C.POINTER(C.c_int8), C.POINTER(C.c_char_p), _D, C.c_int64, C.c_double,
                                        C.c_double, C.POINTER(C.c_int), _D, C.c_char_p, C.c_int]
        lib.ref_scale.argtypes = [_VP, C.POINTER(C.c_int8), C.c_int, C.c_int64, C.POINTER(C.c_int64),
                                  C.POINTER(C.c_int32), _D, _D, _D, C.POINTER(C.c_int)] + [_D] * 7
        _ref = lib
    return _ref


# ------------------------------------------------------------------ oracle

def spmv(lp: LP, x):
    y = np.zeros(lp.nrow)
    oracle_lib().or_spmv(C.byref(lp.view()), _dptr(np.ascontiguousarray(x, float)), _dptr(y))
    return y


def spmv_t(lp: LP, y):
    x = np.zeros(lp.ncol)
    oracle_lib().or_spmv_t(C.byref(lp.view()), _dptr(np.ascontiguousarray(y, float)), _dptr(x))
    return x


def ref_pdhg_restated(lp: LP, max_iters: int, probe_every: int = 0, probe_tol: float = 1e-6,
                      stop_at_probe: bool = False):
    """The reference PDHG loop restated in C (bit-identical arithmetic)."""
    x = np.zeros(lp.ncol)
    y = np.zeros(lp.nrow)
    out = PdhgOut()
    oracle_lib().or_ref_pdhg(C.byref(lp.view()), max_iters, probe_every, probe_tol, int(stop_at_probe),
                             _dptr(x), _dptr(y), C.byref(out))
    return x, y, out


def eval_objective(lp: LP, x) -> float:
    return oracle_lib().or_eval_objective(C.byref(lp.view()), _dptr(np.ascontiguousarray(x, float)))


def verify(lp: LP, x, claimed: float, tol: float = 1e-6) -> VerifyReport:
    r = VerifyReport()
    oracle_lib().or_verify(C.byref(lp.view()), _dptr(np.ascontiguousarray(x, float)), claimed, tol, C.byref(r))
    return r


def rel_kkt(lp: LP, x, y) -> Kkt:
    k = Kkt()
    oracle_lib().or_rel_kkt(C.byref(lp.view()), _dptr(np.ascontiguousarray(x, float)),
                            _dptr(np.ascontiguousarray(y, float)), C.byref(k))
    return k


def csc_from_triplets(nrow, ncol, rows, cols, vals, use_ref=False):
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    start = np.zeros(ncol + 1, np.int64)
    idx = np.zeros(max(1, len(rows)), np.int32)
    val = np.zeros(max(1, len(rows)), np.float64)
    lib = ref_lib() if use_ref else oracle_lib()
    fn = lib.ref_from_triplets if use_ref else lib.or_csc_from_triplets
    nnz = fn(nrow, ncol, len(rows), rows.ctypes.data_as(C.POINTER(C.c_int32)),
             cols.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(vals), start.ctypes.data_as(C.POINTER(C.c_int64)),
             idx.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(val))
    return start, idx[:nnz].copy(), val[:nnz].copy()


# --------------------------------------------------------------- reference

def ref_pdhg(lp: LP, threads: int = 1, simplex_iter_limit: int = 500000, time_limit: float = 1e30):
    """sov::PdhgSolver::solve, the reference's own compiled code."""
    lib = ref_lib()
    x = np.zeros(lp.ncol)
    y = np.zeros(lp.nrow)
    st, it = C.c_int(), C.c_int()
    obj = C.c_double()
    if lib.ref_pdhg_solve(C.byref(lp.view()), threads, simplex_iter_limit, time_limit, _dptr(x), _dptr(y),
                          C.byref(st), C.byref(obj), C.byref(it)) != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    return x, y, st.value, obj.value, it.value


def ref_solver(lp: LP, sense: int = 1, method: str = "auto", presolve: int = 2, scale: bool = True):
    """sov::Solver::solve (validate, presolve, scale, engine, postsolve, dd check)."""
    lib = ref_lib()
    x = np.zeros(lp.ncol)
    st, ver = C.c_int(), C.c_int()
    obj = C.c_double()
    if lib.ref_solver_solve(C.byref(lp.view()), sense, method.encode(), presolve, int(scale), _dptr(x),
                            C.byref(st), C.byref(obj), C.byref(ver)) != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    return x, st.value, obj.value, bool(ver.value)


def ref_spmv(lp: LP, x):
    y = np.zeros(lp.nrow)
    ref_lib().ref_spmv(C.byref(lp.view()), _dptr(np.ascontiguousarray(x, float)), _dptr(y))
    return y


def ref_spmv_t(lp: LP, y):
    x = np.zeros(lp.ncol)
    ref_lib().ref_spmv_t(C.byref(lp.view()), _dptr(np.ascontiguousarray(y, float)), _dptr(x))
    return x


def ref_verify(lp: LP, x, claimed, tol=1e-6):
    p = C.c_int()
    vals = [C.c_double() for _ in range(4)]
    ref_lib().ref_verify(C.byref(lp.view()), _dptr(np.ascontiguousarray(x, float)), claimed, tol, C.byref(p),
                         *[C.byref(v) for v in vals])
    return dict(passed=bool(p.value), max_bound_viol=vals[0].value, max_row_viol=vals[1].value,
                computed_obj=vals[2].value, obj_rel_err=vals[3].value)


def ref_dd_probe(a, b, c):
    d, nsum = C.c_double(), C.c_double()
    ref_lib().ref_dd_probe(a, b, c, C.byref(d), C.byref(nsum))
    return d.value, nsum.value


def _ref_model_lp(lib, h):
    v = NirLpView()
    sense = C.c_int()
    lib.ref_model_view(h, C.byref(v), C.byref(sense))

    def cp(p, n, dt):
        return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)

    lp = LP(v.nrow, v.ncol, cp(v.col_start, v.ncol + 1, np.int64), cp(v.row_index, v.nnz, np.int32),
            cp(v.value, v.nnz, np.float64), cp(v.cost, v.ncol, np.float64), cp(v.collo, v.ncol, np.float64),
            cp(v.colup, v.ncol, np.float64), cp(v.rowlo, v.nrow, np.float64), cp(v.rowup, v.nrow, np.float64),
            v.obj_offset)
    return lp, sense.value


def ref_read_mps(path: str):
    """MpsReader::read + to_internal_min; returns (LP, sense)."""
    lib = ref_lib()
    h = lib.ref_read_mps(path.encode())
    if not h:
        raise RuntimeError(lib.ref_last_error().decode())
    try:
        return _ref_model_lp(lib, h)
    finally:
        lib.ref_model_free(h)


class RefMpsError(RuntimeError):
    """A failed MpsReader::read: status is the sov::Status code, or -1 when
    the reader let an exception escape (std::stod on a bad number)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"status {status}: {message}")
        self.status = status
        self.message = message


def ref_read_mps_full(path: str):
    """MpsReader::read + to_internal_min: (LP, sense, vartype, (q_start,
    q_index, q_value)); raises RefMpsError on failure."""
    lib = ref_lib()
    h = lib.ref_read_mps(path.encode())
    if not h:
        raise RefMpsError(lib.ref_last_status(), lib.ref_last_error().decode(errors="replace"))
    try:
        lp, sense = _ref_model_lp(lib, h)
        vt = np.zeros(lp.ncol, np.int8)
        lib.ref_model_vartypes(h, vt.ctypes.data_as(C.POINTER(C.c_int8)))
        qn = lib.ref_model_qnnz(h)
        qs = np.zeros(lp.ncol + 1, np.int64)
        qi = np.zeros(qn, np.int32)
        qv = np.zeros(qn, np.float64)
        lib.ref_model_q(h, qs.ctypes.data_as(C.POINTER(C.c_int64)), qi.ctypes.data_as(C.POINTER(C.c_int32)),
                        _dptr(qv))
        return lp, sense, vt, (qs, qi, qv)
    finally:
        lib.ref_model_free(h)


def ref_write_mps(lp: LP, path: str, vartype=None, sense: int = 1) -> None:
    """MpsReader::write of an LP (names C<j> / R<i>, objective row OBJ)."""
    vt = None if vartype is None else np.ascontiguousarray(vartype, np.int8)
    rc = ref_lib().ref_write_mps(C.byref(lp.view()),
                                 None if vt is None else vt.ctypes.data_as(C.POINTER(C.c_int8)), int(sense),
                                 path.encode())
    if rc != 0:
        raise RuntimeError(f"MpsReader::write failed on {path}")


def ref_mps_roundtrip(src: str, dst: str) -> int:
    """MpsReader::read of src, then MpsReader::write of that model to dst."""
    return ref_lib().ref_mps_roundtrip(src.encode(), dst.encode())


def ref_presolve(lp: LP, vartype=None, level: int = 2, rounds: int = 20) -> dict:
    """Presolver::presolve on the LP (names C<j> / R<i>): status, counters,
    the reduced LP and vartypes, the maps, fixed_x and is_col_fixed."""
    lib = ref_lib()
    vt = None if vartype is None else np.ascontiguousarray(vartype, np.int8)
    h = lib.ref_presolve(C.byref(lp.view()), None if vt is None else vt.ctypes.data_as(C.POINTER(C.c_int8)),
                         level, rounds)
    try:
        st, solved, cnt = C.c_int(), C.c_int(), (C.c_int * 3)()
        lib.ref_presolved_status(h, C.byref(st), C.byref(solved), cnt)
        v = NirLpView()
        lib.ref_presolved_reduced(h, C.byref(v), None)
        rvt = np.zeros(v.ncol, np.int8)
        lib.ref_presolved_reduced(h, C.byref(v), rvt.ctypes.data_as(C.POINTER(C.c_int8)))

        def cp(p, n, dt):
            return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)

        red = LP(v.nrow, v.ncol, cp(v.col_start, v.ncol + 1, np.int64) if v.col_start else np.zeros(1, np.int64),
                 cp(v.row_index, v.nnz, np.int32), cp(v.value, v.nnz, np.float64), cp(v.cost, v.ncol, np.float64),
                 cp(v.collo, v.ncol, np.float64), cp(v.colup, v.ncol, np.float64), cp(v.rowlo, v.nrow, np.float64),
                 cp(v.rowup, v.nrow, np.float64), v.obj_offset)
        nc = C.c_int64()
        nr = lib.ref_presolved_map_sizes(h, C.byref(nc))
        cm, rm = np.zeros(nc.value, np.int32), np.zeros(nr, np.int32)
        fx, isf = np.zeros(lp.ncol), np.zeros(lp.ncol, np.uint8)
        lib.ref_presolved_maps(h, cm.ctypes.data_as(C.POINTER(C.c_int32)), rm.ctypes.data_as(C.POINTER(C.c_int32)),
                               _dptr(fx), isf.ctypes.data_as(C.POINTER(C.c_uint8)))
        return dict(status=st.value, solved_in_presolve=bool(solved.value), rows_removed=cnt[0],
                    cols_removed=cnt[1], bound_tightenings=cnt[2], reduced=red, vartype=rvt, orig_col_map=cm,
                    orig_row_map=rm, fixed_x=fx, is_col_fixed=isf.astype(bool))
    finally:
        lib.ref_presolved_free(h)


def ref_scale(lp: LP, vartype=None, enable: bool = True, q=None) -> dict:
    """scale_model: active, R, C and the scaled arrays."""
    lib = ref_lib()
    vt = None if vartype is None else np.ascontiguousarray(vartype, np.int8)
    R, Cs = np.zeros(lp.nrow), np.zeros(lp.ncol)
    out = {k: np.empty_like(getattr(lp, k)) for k in ("cost", "collo", "colup", "value", "rowlo", "rowup")}
    act = C.c_int()
    if q is not None:
        qs, qi, qv = (np.ascontiguousarray(q[0], np.int64), np.ascontiguousarray(q[1], np.int32),
                      np.ascontiguousarray(q[2], np.float64))
        qo = np.empty_like(qv)
        qargs = (int(qs[-1]), qs.ctypes.data_as(C.POINTER(C.c_int64)), qi.ctypes.data_as(C.POINTER(C.c_int32)),
                 _dptr(qv))
    else:
        qo, qargs = None, (0, None, None, None)
    lib.ref_scale(C.byref(lp.view()), None if vt is None else vt.ctypes.data_as(C.POINTER(C.c_int8)), int(enable),
                  *qargs, _dptr(R), _dptr(Cs), C.byref(act), _dptr(out["cost"]), _dptr(out["collo"]),
                  _dptr(out["colup"]), _dptr(out["value"]), _dptr(out["rowlo"]), _dptr(out["rowup"]),
                  None if qo is None else _dptr(qo))
    return dict(active=bool(act.value), R=R, C=Cs, q_value=qo, **out)


def _names(names):
    arr = (C.c_char_p * len(names))()
    arr[:] = [n.encode() for n in names]
    return arr


def ref_write_sol(lp: LP, names, status: int, obj: float, gap: float, x, path: str) -> int:
    """SolIo::write_sol for a model with these column names (None: C<j>)."""
    xv = np.ascontiguousarray(x, np.float64)
    return ref_lib().ref_write_sol(C.byref(lp.view()), None if names is None else _names(names), status, obj, gap,
                                   _dptr(xv), len(xv), path.encode())


REF_SOL_TOOL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "ref_sol_tool")


def ref_read_sol(model_mps: str, sol_path: str, ncol: int):
    """SolIo::read_sol of sol_path for the model in model_mps, run as its own
    process (oracle/_ref/ref_sol_tool): ("ok", x, objective), ("exception",
    what) or ("cannot-open",)."""
    import subprocess

    out = subprocess.run([REF_SOL_TOOL, model_mps, sol_path], capture_output=True, text=True, timeout=600)
    lines = out.stdout.splitlines()
    head = lines[0].split(" ", 1)
    if head[0] in ("exception", "cannot-open", "model-error"):
        return tuple(head)
    obj = float.fromhex(lines[1].split()[1])
    x = np.zeros(ncol)
    for ln in lines[2:]:
        j, v = ln.split()
        x[int(j)] = float.fromhex(v)
    return "ok", x, obj


def ref_verify_full(lp: LP, x, claimed: float, tol: float = 1e-6, vartype=None, names=None) -> dict:
    """verify_solution with every report field (names: C<j>/R<i> unless given)."""
    xv = np.ascontiguousarray(x, np.float64)
    vt = None if vartype is None else np.ascontiguousarray(vartype, np.int8)
    passed = C.c_int()
    out = np.zeros(5)
    worst = C.create_string_buffer(512)
    ref_lib().ref_verify_full(C.byref(lp.view()), None if vt is None else vt.ctypes.data_as(C.POINTER(C.c_int8)),
                              None if names is None else _names(names), _dptr(xv), len(xv), claimed, tol,
                              C.byref(passed), _dptr(out), worst, 512)
    return dict(passed=bool(passed.value), max_bound_viol=out[0], max_row_viol=out[1], max_int_viol=out[2],
                computed_obj=out[3], obj_rel_err=out[4], worst_item=worst.value.decode())
