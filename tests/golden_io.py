"""Loads tests/golden/pdhg_golden.json (made by tests/golden/make_golden.py)."""
import json
import os

import numpy as np

from nirnaya_b200.lp import LP

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pdhg_golden.json")


def load():
    with open(PATH) as f:
        return json.load(f)


def unhex(a):
    return np.array([float.fromhex(v) for v in a], dtype=np.float64)


def lp_from(d) -> LP:
    return LP(d["nrow"], d["ncol"], np.array(d["col_start"], np.int64), np.array(d["row_index"], np.int32),
              unhex(d["value"]), unhex(d["cost"]), unhex(d["collo"]), unhex(d["colup"]), unhex(d["rowlo"]),
              unhex(d["rowup"]), float.fromhex(d["obj_offset"]))


def bits(a):
    return np.asarray(a, np.float64).view(np.int64)


def highs_optimum(lp):
    """An independent optimum of an LP by HiGHS (scipy.optimize.linprog),
    objective offset included; for instances HiGHS solves in seconds."""
    import scipy.sparse as sp
    from scipy.optimize import linprog

    A = sp.csc_matrix((lp.value, lp.row_index, lp.col_start), shape=(lp.nrow, lp.ncol)).tocsr()
    fin = lambda v: np.isfinite(v) & (np.abs(v) < 1e20)  # noqa: E731  (src/core/types.hpp:49-51)
    eq = fin(lp.rowlo) & fin(lp.rowup) & (lp.rowlo == lp.rowup)
    fu = fin(lp.rowup) & ~eq
    fl = fin(lp.rowlo) & ~eq
    parts = []
    if fu.any():
        parts.append((A[fu], lp.rowup[fu]))
    if fl.any():
        parts.append((-A[fl], -lp.rowlo[fl]))
    A_ub = sp.vstack([q[0] for q in parts]) if parts else None
    b_ub = np.concatenate([q[1] for q in parts]) if parts else None
    bounds = np.stack([np.where(fin(lp.collo), lp.collo, -np.inf), np.where(fin(lp.colup), lp.colup, np.inf)], axis=1)
    r = linprog(lp.cost, A_ub=A_ub, b_ub=b_ub, A_eq=A[eq] if eq.any() else None,
                b_eq=lp.rowlo[eq] if eq.any() else None, bounds=bounds, method="highs")
    assert r.status == 0, r.message
    return r.fun + lp.obj_offset
