"""The optimal objectives of tests/golden/optima.json, on CPU.

  - Every entry still rebuilds from the seeded generator with the sizes it
    records, so the GPU tests compare against the LP that was solved.
  - An entry that a second algorithm re-solved (HiGHS's dual simplex,
    tests/golden/make_optima.py --confirm) agrees with the first solver's
    objective to 1e-9 relative.
"""
import json
import os

import pytest

from conftest import ROOT

OPT = json.load(open(os.path.join(ROOT, "tests", "golden", "optima.json")))


@pytest.mark.parametrize("name", sorted(OPT))
def test_each_optimum_rebuilds_its_lp(name):
    from nirnaya_b200 import lp as L

    e = OPT[name]
    lp = L.generate(e["kind"], e["seed"], **e["kw"])
    assert (lp.nrow, lp.ncol, lp.nnz) == (e["nrow"], e["ncol"], e["nnz"])
    assert float.fromhex(e["objective_hex"]) == pytest.approx(e["objective"], rel=1e-15)


def test_confirmed_optima_agree_across_algorithms():
    confirmed = {k: v for k, v in OPT.items() if "confirmed" in v}
    for name, e in confirmed.items():
        a = float.fromhex(e["objective_hex"])
        b = float.fromhex(e["confirmed"]["objective_hex"])
        assert e["confirmed"]["solver"] != e["solver"], name
        assert abs(a - b) / (1.0 + abs(a)) <= 1e-9, (name, a, b)
