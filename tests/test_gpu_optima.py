"""PDLP parity at the workload sizes, against independent optima.

The optimal objectives in tests/golden/optima.json were computed by HiGHS
(interior point with crossover) by tests/golden/make_optima.py: the full
2,000 x 5,000 random LP (config 1), a held-out member of the 20,000 x 50,000
blending family (config 4), eight instances of the multiperiod batch
(config 3) and the badly scaled construction at 5,000 x 12,000 (config 5,
reduced).  The reference's own simplex does not finish these sizes.

The reduced badly scaled LP does not reach 1e-6: its cost vector, after
the diagonal preconditioning, spans the eight decades of the column scales
(c_j = A_j'y0 + U(0,1) is not scaled with the column), and PDLP stalls at a
relative gap of ~3e-3 with or without its duplicated columns.  Those tests
are strict xfails that document the stall; the tests below them pin what
the engine does on it.

Every other solve runs to 1e-6 relative KKT with the default parameters, and
  - the status is Optimal;
  - the relative KKT error, evaluated independently by the oracle in
    double-double (oracle/ffi.rel_kkt), is at most 1e-6 (5% slack for the
    FP64 evaluation on the device);
  - the objective is the double-double c'x of Model::eval_objective
    (src/model/model.hpp:73-98), bit for bit;
  - it agrees with the optimum to 1e-6 relative, |obj - opt| / (1 + |opt|)
    (the relative objective error of src/io/sol_io.hpp:96-102).
"""
import json
import os

import pytest

from conftest import ROOT, has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

from nirnaya_b200 import batch as B  # noqa: E402
from nirnaya_b200 import lp as L  # noqa: E402
from nirnaya_b200 import pdhg  # noqa: E402
from oracle import ffi  # noqa: E402

OPT = json.load(open(os.path.join(ROOT, "tests", "golden", "optima.json")))
TOL = 1e-6


def _lp(name):
    e = OPT[name]
    lp = L.generate(e["kind"], e["seed"], **e["kw"])
    assert (lp.nrow, lp.ncol, lp.nnz) == (e["nrow"], e["ncol"], e["nnz"]), "the generator changed"
    return lp, float.fromhex(e["objective_hex"])


def _check(lp, x, y, info, opt):
    assert info.status == pdhg.OPTIMAL, (pdhg.STATUS_NAMES.get(info.status), info.rel_kkt)
    k = ffi.rel_kkt(lp, x, y)
    assert k.rel_kkt <= 1.05 * TOL, k.rel_kkt
    assert info.objective == ffi.eval_objective(lp, x)
    err = abs(info.objective - opt) / (1.0 + abs(opt))
    assert err <= TOL, (info.objective, opt, err)
    return err


C5_STALL = pytest.mark.xfail(strict=True, reason="PDLP stalls on the badly scaled cost (relative gap ~3e-3)")


@pytest.mark.parametrize("name", ["c1_random_eq_2000x5000", "c4_blend_member_900000",
                                  pytest.param("c5_badly_scaled_5000x12000", marks=C5_STALL)])
def test_default_solve_matches_the_optimum(name):
    lp, opt = _lp(name)
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(tol=TOL))
    _check(lp, x, y, info, opt)


@pytest.mark.parametrize("name", ["c1_random_eq_2000x5000",
                                  pytest.param("c5_badly_scaled_5000x12000", marks=C5_STALL)])
def test_fp64_solve_matches_the_optimum(name):
    lp, opt = _lp(name)
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(tol=TOL, precision=pdhg.PREC_FP64))
    _check(lp, x, y, info, opt)
    assert info.iterations_fp64 == info.iterations


def test_badly_scaled_lp_reports_its_original_kkt_and_gains_from_its_parallel_columns(monkeypatch):
    # half of its columns duplicate the other half up to a 1e-9 perturbation:
    # the engine re-expresses each pair (one group, one row per pair); the
    # status and the KKT error it reports are the original LP's, and the
    # re-expression lowers the error reached in a fixed budget
    lp, opt = _lp("c5_badly_scaled_5000x12000")
    budget = 200000
    res = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("NIR_PDHG_PARALLEL_COLUMNS", flag)
        with pdhg.Engine(lp) as eng:
            x, y, info = eng.solve(pdhg.default_params(tol=TOL, precision=pdhg.PREC_FP64, max_iters=budget))
        assert info.parallel_groups == (lp.ncol // 2 if flag == "1" else 0)
        k = ffi.rel_kkt(lp, x, y)
        assert info.rel_kkt == pytest.approx(k.rel_kkt, rel=0.05)
        assert info.objective == ffi.eval_objective(lp, x)
        assert (info.status == pdhg.OPTIMAL) == (k.rel_kkt <= TOL)
        res[flag] = k.rel_kkt
    assert res["1"] < 0.5 * res["0"], res


def test_batch_of_multiperiod_members_matches_their_optima():
    names = sorted(k for k in OPT if k.startswith("c3_multiperiod_"))
    assert len(names) == 8
    lps, opts = zip(*[_lp(n) for n in names])
    with B.BatchEngine(list(lps), 0) as eng:
        res, total = eng.solve(pdhg.default_params(tol=TOL))
    assert total.status == pdhg.OPTIMAL
    for lp, (x, y, info), opt in zip(lps, res, opts):
        _check(lp, x, y, info, opt)


def test_power_law_lp_at_full_size_is_confirmed_by_the_oracle():
    # C2, the headline workload (200,000 x 500,000, 5M nonzeros): no external
    # optimum finishes at this size, so the engine's report is checked
    # instead: the relative KKT error it claims is the oracle's double-double
    # one on the returned point, and its objective is the dd c'x bit for bit
    lp = L.generate(L.ZIPF, 1)
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(tol=TOL))
    assert info.status == pdhg.OPTIMAL, (pdhg.STATUS_NAMES.get(info.status), info.rel_kkt)
    k = ffi.rel_kkt(lp, x, y)
    assert k.rel_kkt <= 1.05 * TOL, k.rel_kkt
    assert info.rel_kkt == pytest.approx(k.rel_kkt, rel=0.05)
    assert info.objective == ffi.eval_objective(lp, x)
