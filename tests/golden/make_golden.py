"""Generates the golden fixtures of the PDHG path from the reference itself.

Run in a container where the reference's sources are present (it builds
oracle/_ref/libref_nirnaya.so from them through oracle/Makefile):

    python tests/golden/make_golden.py [/path/to/reference]

Every fixture records the LP (in the reference's internal-minimisation
layout), what the reference's own compiled code returns for it, and the
known answers its tests assert.  Doubles are stored as hex strings so that
bit-identity can be checked.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

INF = float("inf")


def hexs(a):
    return [float(v).hex() for v in np.asarray(a, dtype=np.float64).ravel()]


def lp_json(lp):
    return {
        "nrow": lp.nrow, "ncol": lp.ncol, "col_start": lp.col_start.tolist(), "row_index": lp.row_index.tolist(),
        "value": hexs(lp.value), "cost": hexs(lp.cost), "collo": hexs(lp.collo), "colup": hexs(lp.colup),
        "rowlo": hexs(lp.rowlo), "rowup": hexs(lp.rowup), "obj_offset": float(lp.obj_offset).hex(),
    }


def ref_pdhg_record(ffi, lp, simplex_iter_limit=500000):
    x, y, st, obj, it = ffi.ref_pdhg(lp, threads=1, simplex_iter_limit=simplex_iter_limit)
    return {"status": st, "objective": float(obj).hex(), "iterations": it, "x": hexs(x), "y": hexs(y),
            "max_iters": max(5000, simplex_iter_limit // 10)}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else (os.environ.get("NIRNAYA_REF") or os.path.join(ROOT, os.pardir, "reference"))
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={ref}"], check=True)
    from nirnaya_b200 import build
    build.build_lpgen()
    from nirnaya_b200 import lp as L
    from oracle import ffi

    out = {}

    # tests/unit_tests.cpp:29-42 -- dd_real and Neumaier cancellation
    d, nsum = ffi.ref_dd_probe(1e16, 1.0, -1e16)
    out["dd_probe"] = {"inputs": [1e16, 1.0, -1e16], "dd": d, "neumaier": nsum, "expected": 1.0}

    # tests/unit_tests.cpp:45-76 -- 2x2 CSC with a duplicate, SpMV known answer
    rows, cols, vals = [0, 0, 1, 0, 1], [0, 0, 0, 1, 1], [1.5, 0.5, -3.0, 4.0, 2.0]
    start, idx, val = ffi.csc_from_triplets(2, 2, rows, cols, vals, use_ref=True)
    out["spmv_2x2"] = {"triplets": {"row": rows, "col": cols, "val": vals}, "col_start": start.tolist(),
                       "row_index": idx.tolist(), "value": val.tolist(), "x": [2.0, 3.0], "y": [16.0, 0.0]}

    # tests/unit_tests.cpp:316-331 -- the PDHG unit-test LP
    lp = L.LP.from_rows(2, [([0, 1], [1.0, 1.0]), ([0, 1], [1.0, 3.0])], cost=[2.0, 3.0], collo=[0.0, 0.0],
                        colup=[20.0, 20.0], rowlo=[4.0, 6.0], rowup=[20.0, 30.0])
    _, st, obj, ver = ffi.ref_solver(lp, method="pdhg")
    out["unit_test_pdhg_lp"] = {"lp": lp_json(lp), "expected_objective": 9.0, "expected_tol": 1e-2,
                                "optimum_x": [3.0, 1.0], "solver_pdhg": {"status": st, "objective": obj, "verified": ver},
                                "ref_pdhg": ref_pdhg_record(ffi, lp)}

    # tools/bench_runner.cpp:24-39 -- Degenerate_Transport_LP (5x5 assignment)
    N = 5
    rws = []
    cost = []
    for i in range(N):
        for j in range(N):
            cost.append(float((i + 1) * (j + 2) % 7 + 1))
    for i in range(N):
        rws.append(([i * N + j for j in range(N)], [1.0] * N))
        rws.append(([r * N + i for r in range(N)], [1.0] * N))
    lp = L.LP.from_rows(N * N, rws, cost=cost, collo=[0.0] * 25, colup=[1.0] * 25, rowlo=[1.0] * 10, rowup=[1.0] * 10)
    _, st, obj, ver = ffi.ref_solver(lp, method="pdhg")
    _, st2, obj2, _ = ffi.ref_solver(lp, method="auto")
    out["degenerate_transport"] = {"lp": lp_json(lp), "expected_objective": 13.0,
                                   "solver_pdhg": {"status": st, "objective": obj, "verified": ver},
                                   "solver_simplex": {"status": st2, "objective": obj2},
                                   "ref_pdhg": ref_pdhg_record(ffi, lp)}

    # data/refinery/MRPL_Crude_Blending_LP.mps and .sol (maximisation)
    mps = os.path.join(ref, "data", "refinery", "MRPL_Crude_Blending_LP.mps")
    sol = os.path.join(ref, "data", "refinery", "MRPL_Crude_Blending_LP.sol")
    lp, sense = ffi.ref_read_mps(mps)
    sol_obj, sol_x = None, []
    with open(sol) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "#":
                if t[1] == "objective":
                    sol_obj = float(t[2])
                continue
            sol_x.append(float(t[1]))
    # Solver::solve with method=pdhg, on the user (maximisation) model
    user = L.LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index, lp.value, -lp.cost, lp.collo, lp.colup,
                lp.rowlo, lp.rowup, -lp.obj_offset)
    xs, st, obj, ver = ffi.ref_solver(user, sense=-1, method="pdhg")
    out["crude_blending"] = {"lp_internal_min": lp_json(lp), "sense": sense, "sol_objective": sol_obj,
                             "sol_x": sol_x, "solver_pdhg": {"status": st, "objective": obj, "verified": ver,
                                                             "x": xs.tolist()},
                             "ref_pdhg": ref_pdhg_record(ffi, lp)}

    # a generated instance: the reference PDHG on RANDOM_EQ m=200 n=500 seed 7
    lp = L.generate(L.RANDOM_EQ, 7, m=200, n=500)
    rec = ref_pdhg_record(ffi, lp, simplex_iter_limit=30000)
    out["random_eq_200x500_seed7"] = {"generator": {"kind": L.RANDOM_EQ, "seed": 7, "m": 200, "n": 500},
                                      "nnz": lp.nnz, "ref_pdhg": rec}

    path = os.path.join(HERE, "pdhg_golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
