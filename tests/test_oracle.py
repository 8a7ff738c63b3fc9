"""The oracle pinned against the reference's own known answers and outputs.

CPU only.  The oracle (oracle/nir_oracle.c) must reproduce:
  * the reference's unit-test known answers (tests/unit_tests.cpp:29-76,
    :316-331), tools/bench_runner.cpp's Degenerate_Transport_LP and the
    Crude_Blending_LP optimum (data/refinery/*.sol), via the committed
    fixtures in tests/golden/;
  * the reference's compiled PdhgSolver::solve bit for bit, both from the
    fixtures and live against oracle/_ref when it was built.
"""
import numpy as np
import pytest

import golden_io as G
from nirnaya_b200 import lp as L
from oracle import ffi

GOLD = G.load()


def test_dd_and_neumaier_cancellation():
    # tests/unit_tests.cpp:29-42
    assert ffi.oracle_lib().or_dd_cancellation_probe(1e16, 1.0, -1e16) == 1.0
    assert ffi.oracle_lib().or_neumaier_probe(1e16, 1.0, -1e16) == 1.0
    assert GOLD["dd_probe"]["dd"] == 1.0 and GOLD["dd_probe"]["neumaier"] == 1.0


def test_csc_merge_and_spmv_known_answer():
    # tests/unit_tests.cpp:45-76: duplicate (0,0) merged, y = (16, 0)
    g = GOLD["spmv_2x2"]
    t = g["triplets"]
    start, idx, val = ffi.csc_from_triplets(2, 2, t["row"], t["col"], t["val"])
    assert start.tolist() == g["col_start"] and idx.tolist() == g["row_index"] and val.tolist() == g["value"]
    lp = L.LP(2, 2, start, idx, val, [0, 0], [0, 0], [1, 1], [0, 0], [1, 1])
    assert ffi.spmv(lp, g["x"]).tolist() == g["y"]
    # transpose of the same matrix: (2*2 + -3*3, 4*2 + 2*3)
    assert ffi.spmv_t(lp, [2.0, 3.0]).tolist() == [2 * 2.0 - 3 * 3.0, 4 * 2.0 + 2 * 3.0]


def test_csc_from_triplets_drops_zeros_and_out_of_range():
    start, idx, val = ffi.csc_from_triplets(3, 2, [0, 5, 1, 1, 2], [0, 0, 1, 1, 1], [1.0, 2.0, 3.0, -3.0, 0.0])
    assert start.tolist() == [0, 1, 1] and idx.tolist() == [0] and val.tolist() == [1.0]


@pytest.mark.parametrize("name", ["unit_test_pdhg_lp", "degenerate_transport", "crude_blending"])
def test_oracle_reference_loop_matches_reference_fixture(name):
    g = GOLD[name]
    lp = G.lp_from(g.get("lp") or g["lp_internal_min"])
    r = g["ref_pdhg"]
    x, y, out = ffi.ref_pdhg_restated(lp, r["max_iters"])
    assert out.iterations == r["iterations"]
    assert np.array_equal(G.bits(x), G.bits(G.unhex(r["x"])))
    assert np.array_equal(G.bits(y), G.bits(G.unhex(r["y"])))
    assert out.objective == float.fromhex(r["objective"])


def test_known_answers_of_the_reference_tests():
    # tests/unit_tests.cpp:329-330: objective 9 within 1e-2
    g = GOLD["unit_test_pdhg_lp"]
    x, y, out = ffi.ref_pdhg_restated(G.lp_from(g["lp"]), g["ref_pdhg"]["max_iters"])
    assert out.stopped == 1 and abs(out.objective - 9.0) <= 1e-2
    # bench_runner: PDHG objective 13 on the degenerate assignment
    g = GOLD["degenerate_transport"]
    x, y, out = ffi.ref_pdhg_restated(G.lp_from(g["lp"]), g["ref_pdhg"]["max_iters"])
    assert abs(out.objective - 13.0) <= 1e-5
    assert ffi.verify(G.lp_from(g["lp"]), x, out.objective).passed
    # Crude blending (maximise): internal min objective is -22171.59777...
    g = GOLD["crude_blending"]
    lp = G.lp_from(g["lp_internal_min"])
    x, y, out = ffi.ref_pdhg_restated(lp, g["ref_pdhg"]["max_iters"])
    assert abs(-out.objective - g["sol_objective"]) / g["sol_objective"] <= 1e-6
    # the .sol optimum passes the dd checker and has a tiny KKT error
    xs = np.array(g["sol_x"])
    rep = ffi.verify(lp, xs, ffi.eval_objective(lp, xs))
    assert rep.passed and abs(-rep.computed_obj - g["sol_objective"]) <= 1e-9 * g["sol_objective"]


def test_oracle_generated_instance_fixture():
    g = GOLD["random_eq_200x500_seed7"]
    gen = g["generator"]
    lp = L.generate(gen["kind"], gen["seed"], m=gen["m"], n=gen["n"])
    assert lp.nnz == g["nnz"]
    r = g["ref_pdhg"]
    x, y, out = ffi.ref_pdhg_restated(lp, r["max_iters"])
    assert out.iterations == r["iterations"]
    assert np.array_equal(G.bits(x), G.bits(G.unhex(r["x"])))
    assert np.array_equal(G.bits(y), G.bits(G.unhex(r["y"])))


@pytest.mark.skipif(not ffi.ref_available(), reason="reference not built from source here")
@pytest.mark.parametrize("kind,kw,iters", [
    (L.RANDOM_EQ, dict(m=300, n=700), 5000),
    (L.ZIPF, dict(m=300, n=700, target_nnz=6000, zipf_cap=200), 5000),
    (L.MULTIPERIOD, dict(m=240), 5000),
    (L.BADLY_SCALED, dict(m=200, n=400, target_nnz=3000), 5000),
])
def test_oracle_bit_identical_to_compiled_reference(kind, kw, iters):
    lp = L.generate(kind, 11, **kw)
    xr, yr, st, obj, it = ffi.ref_pdhg(lp, threads=1, simplex_iter_limit=10 * iters)
    x, y, out = ffi.ref_pdhg_restated(lp, iters)
    assert it == out.iterations
    assert np.array_equal(G.bits(x), G.bits(xr)) and np.array_equal(G.bits(y), G.bits(yr))
    assert obj == out.objective
    # the reference's SpMV pair and checker, too
    v = np.linspace(-1, 1, lp.ncol)
    w = np.linspace(2, -1, lp.nrow)
    assert np.array_equal(G.bits(ffi.spmv(lp, v)), G.bits(ffi.ref_spmv(lp, v)))
    assert np.array_equal(G.bits(ffi.spmv_t(lp, w)), G.bits(ffi.ref_spmv_t(lp, w)))
    rep = ffi.verify(lp, x, obj)
    rr = ffi.ref_verify(lp, x, obj)
    assert rep.passed == rr["passed"] and rep.max_row_viol == rr["max_row_viol"]
    assert rep.computed_obj == rr["computed_obj"] and rep.max_bound_viol == rr["max_bound_viol"]


def test_rel_kkt_of_known_optimum_is_small():
    g = GOLD["unit_test_pdhg_lp"]
    lp = G.lp_from(g["lp"])
    # optimum x = (3, 1) with duals (1.5, 0.5) from tests/unit_tests.cpp:117-139
    k = ffi.rel_kkt(lp, np.array([3.0, 1.0]), np.array([1.5, 0.5]))
    assert k.rel_kkt <= 1e-15 and abs(k.pobj - 9.0) < 1e-15 and abs(k.dobj - 9.0) < 1e-15
    k = ffi.rel_kkt(lp, np.array([3.0, 1.0]), np.array([1.0, 0.5]))
    assert k.rel_kkt > 1e-3


def test_generator_is_deterministic_and_feasible():
    for kind, kw in [(L.RANDOM_EQ, {}), (L.ZIPF, dict(m=2000, n=5000, target_nnz=50000)),
                     (L.MULTIPERIOD, dict(m=600)), (L.BLEND_FAMILY, dict(m=2000, n=5000, target_nnz=40000)),
                     (L.BADLY_SCALED, dict(m=500, n=1200, target_nnz=10000))]:
        a = L.generate(kind, 3, **kw)
        b = L.generate(kind, 3, **kw)
        assert np.array_equal(a.value, b.value) and np.array_equal(a.row_index, b.row_index)
        assert np.array_equal(a.cost, b.cost)
        ax = ffi.spmv(a, a.x0)
        scale = 1 + np.abs(ax)
        assert np.all(ax >= a.rowlo - 1e-9 * scale) and np.all(ax <= a.rowup + 1e-9 * scale)
        assert np.all(a.x0 >= a.collo) and np.all(a.x0 <= a.colup)
    assert L.generate(L.RANDOM_EQ, 1).nnz == 40000


def test_blend_family_shares_matrix_and_perturbs_vectors():
    a = L.generate(L.BLEND_FAMILY, 1, m=2000, n=5000, target_nnz=40000)
    b = L.generate(L.BLEND_FAMILY, 2, m=2000, n=5000, target_nnz=40000)
    assert np.array_equal(a.value, b.value)
    assert not np.array_equal(a.cost, b.cost)
    nd = len(a.extra["demand_factors"])
    assert not np.array_equal(a.rowlo[:nd], b.rowlo[:nd]) and np.array_equal(a.rowup[nd:], b.rowup[nd:])
