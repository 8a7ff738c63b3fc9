"""Presolve, scaling, SOL reading and the solution check against fixtures
recorded from the reference's own code (tests/golden/facade_golden.json,
made by tests/golden/make_facade_golden.py).  These run without the
reference present: the inputs come from the seeds, the expected outputs
from the fixtures, bit for bit."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from nirnaya_b200 import facade
from nirnaya_b200 import lp as L
from nirnaya_b200 import mps

GOLDEN = os.path.join(ROOT, "tests", "golden", "facade_golden.json")


def _unhex(a):
    return np.array([float.fromhex(v) for v in a], dtype=np.float64)


def _bits(a):
    return np.atleast_1d(np.asarray(a, np.float64)).view(np.uint64)


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _instance(kind, seed, kw):
    from test_facade import forcing_instance, rich_instance

    return rich_instance(seed, **kw) if kind == "rich" else forcing_instance(seed)


def test_presolve_matches_the_fixtures(golden):
    for g in golden["presolve"]:
        lp, vt = _instance(g["kind"], g["seed"], g["kw"])
        for threads in (1, 3):
            a = facade.presolve(lp, vt, 20, threads)
            tag = (g["kind"], g["seed"], threads)
            assert (a.status, a.solved_in_presolve) == (g["status"], g["solved"]), tag
            assert [a.rows_removed, a.cols_removed, a.bound_tightenings] == g["counters"], tag
            r = a.reduced
            assert (r.nrow, r.ncol) == (g["nrow"], g["ncol"]), tag
            if r.ncol:
                assert r.col_start.tolist() == g["col_start"], tag
            assert r.row_index.tolist() == g["row_index"], tag
            for k in ("value", "cost", "collo", "colup", "rowlo", "rowup"):
                assert np.array_equal(_bits(getattr(r, k)), _bits(_unhex(g[k]))) if g[k] else getattr(r, k).size == 0, \
                    (tag, k)
            assert _bits(r.obj_offset) == _bits(float.fromhex(g["obj_offset"])), tag
            assert a.vartype.tolist() == g["vartype"], tag
            assert a.orig_col_map.tolist() == g["orig_col_map"] and a.orig_row_map.tolist() == g["orig_row_map"], tag
            assert np.array_equal(_bits(a.fixed_x), _bits(_unhex(g["fixed_x"]))), tag
            assert a.is_col_fixed.astype(int).tolist() == g["is_col_fixed"], tag


def test_scale_matches_the_fixtures(golden):
    from golden.make_facade_golden import scale_input

    for g in golden["scale"]:
        lp, vt = scale_input(g["seed"], g["kw"])
        s = facade.scale(lp, vt, threads=2)
        assert s.active == g["active"]
        assert np.array_equal(_bits(s.R), _bits(_unhex(g["R"]))) and np.array_equal(_bits(s.C), _bits(_unhex(g["C"])))
        for k in ("cost", "collo", "colup", "value", "rowlo", "rowup"):
            assert np.array_equal(_bits(getattr(s.lp, k)), _bits(_unhex(g[k]))), k


def test_read_sol_matches_the_fixture(golden, tmp_path):
    from test_sol import SOL_LINES

    sol = tmp_path / "x.sol"
    with open(sol, "w", newline="") as f:
        f.write("\n".join(SOL_LINES) + "\n")
    x, obj, _ = mps.read_sol(str(sol), [f"C{j}" for j in range(30)])
    assert np.array_equal(_bits(x), _bits(_unhex(golden["read_sol"]["x"])))
    assert _bits(obj) == _bits(float.fromhex(golden["read_sol"]["objective"]))


def test_verify_matches_the_fixtures(golden):
    from golden.make_facade_golden import verify_input

    for g in golden["verify"]:
        lp, vt, x, claimed, tol = verify_input(g["seed"])
        rep = mps.verify_solution(lp, x, claimed, tol, vartype=vt, col_names=[f"C{j}" for j in range(lp.ncol)],
                                  row_names=[f"R{i}" for i in range(lp.nrow)])
        assert rep["passed"] == g["passed"] and rep["worst_item"] == g["worst_item"], g["seed"]
        for k in ("max_bound_viol", "max_row_viol", "max_int_viol", "computed_obj", "obj_rel_err"):
            assert _bits(rep[k]) == _bits(float.fromhex(g[k])), (g["seed"], k)


def test_fixtures_cover_every_rule(golden):
    statuses = {g["status"] for g in golden["presolve"]}
    assert any(g["counters"][2] > 0 for g in golden["presolve"])  # tightenings
    assert any(g["counters"][0] > 0 and g["counters"][1] > 0 for g in golden["presolve"])
    assert statuses & {0}
    assert any(s["active"] for s in golden["scale"])
    assert {g["passed"] for g in golden["verify"]} == {True, False} or len(golden["verify"]) > 0
