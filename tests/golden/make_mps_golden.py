"""Generates tests/golden/mps_golden.json from the reference's own MPS reader.

Run in a container where the reference's sources are present (it builds
oracle/_ref/libref_nirnaya.so from them through oracle/Makefile):

    python tests/golden/make_mps_golden.py [/path/to/reference]

For every input of tests/mps_cases.py (the hand-written CASES and a few
seeded random layouts) it records what sov::MpsReader::read followed by
Model::to_internal_min returns -- status and message on failure, every
array (doubles as hex strings, so bit-identity can be checked) otherwise.
Status -1 marks an input on which the reference lets std::stod's exception
escape instead of returning a status.
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

RANDOM = [  # (generator kind, seed, sizes, sense) written by mps_cases.random_mps
    (1, 0, dict(m=60, n=150), 1),
    (2, 1, dict(m=200, n=500, target_nnz=3000), -1),
    (5, 2, dict(m=30, n=80), 1),
]


def hexs(a):
    return [float(v).hex() for v in np.asarray(a, dtype=np.float64).ravel()]


def record(ffi, path):
    try:
        lp, sense, vt, (qs, qi, qv) = ffi.ref_read_mps_full(path)
    except ffi.RefMpsError as e:
        return {"status": e.status, "message": e.message}
    return {"status": 0, "sense": sense, "nrow": lp.nrow, "ncol": lp.ncol, "col_start": lp.col_start.tolist(),
            "row_index": lp.row_index.tolist(), "value": hexs(lp.value), "cost": hexs(lp.cost),
            "collo": hexs(lp.collo), "colup": hexs(lp.colup), "rowlo": hexs(lp.rowlo), "rowup": hexs(lp.rowup),
            "obj_offset": float(lp.obj_offset).hex(), "vartype": vt.tolist(), "q_start": qs.tolist(),
            "q_index": qi.tolist(), "q_value": hexs(qv)}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else (os.environ.get("NIRNAYA_REF") or os.path.join(ROOT, os.pardir, "reference"))
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={ref}"], check=True)
    from nirnaya_b200 import build
    build.build_lpgen()
    from mps_cases import CASES, random_mps

    from nirnaya_b200 import lp as L
    from oracle import ffi

    out = {"cases": {}, "random": []}
    with tempfile.TemporaryDirectory() as d:
        for name, text in CASES.items():
            p = os.path.join(d, name + ".mps")
            with open(p, "w", newline="") as f:
                f.write(text)
            out["cases"][name] = record(ffi, p)
        for kind, seed, kw, sense in RANDOM:
            lp = L.generate(kind, seed, **kw)
            p = os.path.join(d, "random.mps")
            with open(p, "w", newline="") as f:
                f.write(random_mps(lp, seed, sense=sense))
            out["random"].append({"kind": kind, "seed": seed, "kw": kw, "sense": sense, "result": record(ffi, p)})
    path = os.path.join(HERE, "mps_golden.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
