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
