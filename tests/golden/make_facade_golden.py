"""Generates tests/golden/facade_golden.json from the reference's own code.

Run where the reference's sources are present (it builds oracle/_ref from
them through oracle/Makefile):

    python tests/golden/make_facade_golden.py [/path/to/reference]

Recorded, with doubles as hex strings so that bit-identity can be checked:
  - Presolver::presolve (src/presolve/presolve.hpp:32-345) on seeded
    instances from tests/test_facade.py (rich_instance, forcing_instance);
  - scale_model (src/model/scaling.hpp:56-154) on three of them;
  - SolIo::read_sol (src/io/sol_io.hpp:134-170) on a file of odd tokens
    (tests/test_sol.py's SOL_LINES) for a 30-column model;
  - verify_solution (src/io/sol_io.hpp:25-106) on seeded points.
The inputs are regenerated by the tests from the seeds; only the
reference's outputs are stored.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

PRESOLVE = [("rich", s, dict(m=60, n=100, int_frac=f)) for s, f in ((0, 0.0), (1, 0.3), (2, 0.6), (3, 0.0), (4, 0.3))]
PRESOLVE += [("forcing", s, {}) for s in range(4)]
SCALE = [("rich", 6, dict(m=60, n=100, int_frac=0.3)), ("rich", 7, dict(m=40, n=80, int_frac=0.0))]
VERIFY_SEEDS = [0, 1, 2, 3]


def hexs(a):
    return [float(v).hex() for v in np.asarray(a, dtype=np.float64).ravel()]


def instance(kind, seed, kw):
    from test_facade import forcing_instance, rich_instance

    return rich_instance(seed, **kw) if kind == "rich" else forcing_instance(seed)


def scale_input(seed, kw):
    """rich_instance with coefficients spread over decades (scaling active)."""
    from nirnaya_b200 import lp as L

    lp, vt = instance("rich", seed, kw)
    rng = np.random.default_rng([0x5CA, seed])
    lp = L.LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index, lp.value * 10.0 ** rng.uniform(-3, 3, lp.nnz), lp.cost,
              lp.collo, lp.colup, lp.rowlo, lp.rowup)
    return lp, vt


def verify_input(seed):
    """A generated LP, integer marks and a point with violations of each kind."""
    from nirnaya_b200 import lp as L

    rng = np.random.default_rng([0x7E5, seed])
    lp = L.generate(1, seed, m=50, n=120)
    vt = (rng.random(lp.ncol) < 0.3).astype(np.int8)
    x = rng.normal(size=lp.ncol) * 3
    if seed % 2 == 0:
        x = np.clip(x, lp.collo, lp.colup)
    x[rng.random(lp.ncol) < 0.2] = 0.0
    return lp, vt, x, float(rng.normal() * 10), [1e-9, 1e-6, 10.0][seed % 3]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else (os.environ.get("NIRNAYA_REF") or os.path.join(ROOT, os.pardir, "reference"))
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={ref}"], check=True)
    from nirnaya_b200 import build
    build.build_lpgen()
    build.build_mps()
    from test_sol import SOL_LINES

    from nirnaya_b200 import lp as L
    from nirnaya_b200 import mps
    from oracle import ffi

    out = {"presolve": [], "scale": [], "read_sol": None, "verify": []}
    for kind, seed, kw in PRESOLVE:
        lp, vt = instance(kind, seed, kw)
        b = ffi.ref_presolve(lp, vt, 2, 20)
        r = b["reduced"]
        out["presolve"].append({
            "kind": kind, "seed": seed, "kw": kw, "status": b["status"], "solved": b["solved_in_presolve"],
            "counters": [b["rows_removed"], b["cols_removed"], b["bound_tightenings"]],
            "nrow": r.nrow, "ncol": r.ncol, "col_start": r.col_start.tolist(), "row_index": r.row_index.tolist(),
            "value": hexs(r.value), "cost": hexs(r.cost), "collo": hexs(r.collo), "colup": hexs(r.colup),
            "rowlo": hexs(r.rowlo), "rowup": hexs(r.rowup), "obj_offset": float(r.obj_offset).hex(),
            "vartype": b["vartype"].tolist(), "orig_col_map": b["orig_col_map"].tolist(),
            "orig_row_map": b["orig_row_map"].tolist(), "fixed_x": hexs(b["fixed_x"]),
            "is_col_fixed": b["is_col_fixed"].astype(int).tolist()})
    for kind, seed, kw in SCALE:
        lp, vt = scale_input(seed, kw)
        s = ffi.ref_scale(lp, vt)
        out["scale"].append({"seed": seed, "kw": kw, "active": s["active"], "R": hexs(s["R"]), "C": hexs(s["C"]),
                             **{k: hexs(s[k]) for k in ("cost", "collo", "colup", "value", "rowlo", "rowup")}})
    with tempfile.TemporaryDirectory() as d:
        lp = L.generate(1, 0, m=5, n=30)
        lp.cost[lp.cost == 0.0] = 1.0
        names = [f"C{j}" for j in range(30)]
        model, sol = os.path.join(d, "m.mps"), os.path.join(d, "x.sol")
        mps.write_mps(model, lp, name="solmodel", col_names=names)
        with open(sol, "w", newline="") as f:
            f.write("\n".join(SOL_LINES) + "\n")
        res = ffi.ref_read_sol(model, sol, 30)
        out["read_sol"] = {"x": hexs(res[1]), "objective": float(res[2]).hex()}
    for seed in VERIFY_SEEDS:
        lp, vt, x, claimed, tol = verify_input(seed)
        rep = ffi.ref_verify_full(lp, x, claimed, tol, vartype=vt)
        out["verify"].append({"seed": seed, "passed": rep["passed"], "worst_item": rep["worst_item"],
                              **{k: float(rep[k]).hex() for k in ("max_bound_viol", "max_row_viol", "max_int_viol",
                                                                 "computed_obj", "obj_rel_err")}})
    path = os.path.join(HERE, "facade_golden.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
