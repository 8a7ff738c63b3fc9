"""GPU parity of the CUDA path against the oracle, through the C ABI.

  * SpMV: the reference-order kernel is bit-identical to the reference's
    CscMatrix::spmv / spmv_transpose (restated by the oracle); the
    CSR-adaptive FP64 and FP32 kernels agree within their rounding bounds.
  * NIR_ALGO_REFERENCE reproduces the reference PDHG loop bit for bit
    (iterates, iteration count, objective) on the golden fixtures, the
    generated instances and the full C1 workload.
  * PDHG/PDLP in FP64, FP32 and mixed precision reach the requested
    relative KKT as the oracle measures it (tolerance written in each test)
    and the objective agrees with an independent optimum.
  * Status behaviour: iteration cap, host stop, warm start, bad input.
"""
import time

import numpy as np
import pytest

import golden_io as G
from conftest import has_gpu
from nirnaya_b200 import lp as L
from nirnaya_b200 import pdhg
from oracle import ffi

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

GOLD = G.load()


def dense_row_lp(m=40, n=9000, seed=5):
    """Edge cases for the row-block layout: one row longer than any row
    block (9000 > 4096 nonzeros), empty rows and columns, a 1-entry row."""
    rng = np.random.default_rng(seed)
    rows = [(list(range(n)), rng.normal(size=n))]
    for i in range(1, m - 2):
        k = int(rng.integers(1, 60))
        cols = sorted(rng.choice(n - 10, size=k, replace=False).tolist())
        rows.append((cols, rng.normal(size=k)))
    rows.append(([], []))                      # empty row
    rows.append(([3], [2.5]))                  # single entry
    x0 = rng.uniform(0, 1, n)
    lp = L.LP.from_rows(n, rows, cost=np.zeros(n), collo=np.zeros(n), colup=np.ones(n),
                        rowlo=np.zeros(m), rowup=np.zeros(m))
    ax = ffi.spmv(lp, x0)
    lp.rowlo[:] = ax
    lp.rowup[:] = ax
    lp.cost[:] = ffi.spmv_t(lp, rng.normal(size=m)) + rng.uniform(0, 1, n)
    lp._view = None
    return lp


SPMV_CASES = [
    ("c1", lambda: L.generate(L.RANDOM_EQ, 1)),
    ("zipf", lambda: L.generate(L.ZIPF, 2, m=20000, n=50000, target_nnz=500000)),
    ("multiperiod", lambda: L.generate(L.MULTIPERIOD, 3, m=3000)),
    ("badly_scaled", lambda: L.generate(L.BADLY_SCALED, 4, m=2000, n=5000, target_nnz=40000)),
    ("dense_row", dense_row_lp),
]


@pytest.mark.parametrize("name,make", SPMV_CASES)
def test_spmv_parity(name, make):
    lp = make()
    rng = np.random.default_rng(0)
    x = rng.normal(size=lp.ncol)
    y = rng.normal(size=lp.nrow)
    with pdhg.Engine(lp) as eng:
        # reference order: bit-identical
        assert np.array_equal(G.bits(eng.spmv(x, False, 0)), G.bits(ffi.spmv(lp, x)))
        assert np.array_equal(G.bits(eng.spmv(y, True, 0)), G.bits(ffi.spmv_t(lp, y)))
        absA = L.LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index, np.abs(lp.value), lp.cost, lp.collo, lp.colup,
                    lp.rowlo, lp.rowup)
        for tr, v, ref in ((False, x, ffi.spmv(lp, x)), (True, y, ffi.spmv_t(lp, y))):
            mag = ffi.spmv_t(absA, np.abs(v)) if tr else ffi.spmv(absA, np.abs(v))
            # CSR-adaptive FP64: reordered sums, |err| <= ~len * eps * sum|a||x|
            got = eng.spmv(v, tr, 1)
            assert np.all(np.abs(got - ref) <= 1e-12 * mag + 1e-300)
            # FP32 values, inputs and accumulation: 1e-4 of sum|a||x|
            got32 = eng.spmv(v, tr, 2)
            assert np.all(np.abs(got32 - ref) <= 1e-4 * mag + 1e-30)


def _ref_loop_check(lp, max_iters, record=None):
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, max_iters=max_iters))
    xo, yo, out = ffi.ref_pdhg_restated(lp, max_iters)
    assert info.iterations == out.iterations
    assert np.array_equal(G.bits(x), G.bits(xo)), "x differs from the reference loop"
    assert np.array_equal(G.bits(y), G.bits(yo)), "y differs from the reference loop"
    assert info.objective == out.objective
    assert info.status == (pdhg.OPTIMAL if out.stopped else pdhg.ITERATION_LIMIT)
    if record is not None:
        assert info.iterations == record["iterations"]
        assert np.array_equal(G.bits(x), G.bits(G.unhex(record["x"])))
        assert info.objective == float.fromhex(record["objective"])
    return info


@pytest.mark.parametrize("name", ["unit_test_pdhg_lp", "degenerate_transport", "crude_blending"])
def test_reference_loop_bit_identical_on_fixtures(name):
    g = GOLD[name]
    lp = G.lp_from(g.get("lp") or g["lp_internal_min"])
    info = _ref_loop_check(lp, g["ref_pdhg"]["max_iters"], g["ref_pdhg"])
    assert info.status == pdhg.OPTIMAL  # these stop on the reference's own test


def test_reference_loop_known_answers():
    g = GOLD["unit_test_pdhg_lp"]
    with pdhg.Engine(G.lp_from(g["lp"])) as eng:
        _, _, info = eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, max_iters=50000))
    assert abs(info.objective - 9.0) <= 1e-2  # tests/unit_tests.cpp:329-330


@pytest.mark.parametrize("kind,kw,iters", [
    (L.RANDOM_EQ, dict(m=200, n=500), 5000),
    (L.ZIPF, dict(m=3000, n=7000, target_nnz=60000), 3000),
    (L.MULTIPERIOD, dict(m=1200), 3000),
    (L.BADLY_SCALED, dict(m=1000, n=2400, target_nnz=20000), 3000),
])
def test_reference_loop_bit_identical_generated(kind, kw, iters):
    _ref_loop_check(L.generate(kind, 7, **kw), iters)


@pytest.mark.slow
def test_reference_loop_bit_identical_c1_full():
    # the full C1 workload (2000 x 5000, 40000 nonzeros), the reference's
    # default cap of 50000 iterations
    lp = L.generate(L.RANDOM_EQ, 1)
    _ref_loop_check(lp, 50000)


def test_reference_loop_matches_compiled_reference():
    if not ffi.ref_available():
        pytest.skip("oracle/_ref not built")
    lp = L.generate(L.RANDOM_EQ, 1)
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, max_iters=5000))
    xr, yr, st, obj, it = ffi.ref_pdhg(lp, threads=1, simplex_iter_limit=50000)
    assert it == info.iterations and obj == info.objective
    assert np.array_equal(G.bits(x), G.bits(xr)) and np.array_equal(G.bits(y), G.bits(yr))


def _optimum(lp):
    return G.highs_optimum(lp)


PDLP_CASES = [
    ("c1_small", lambda: L.generate(L.RANDOM_EQ, 3, m=500, n=1250)),
    ("multiperiod", lambda: L.generate(L.MULTIPERIOD, 3, m=600)),
    ("blend", lambda: L.generate(L.BLEND_FAMILY, 3, m=1000, n=2500, target_nnz=20000)),
    ("crude_blending", lambda: G.lp_from(GOLD["crude_blending"]["lp_internal_min"])),
    ("degenerate_transport", lambda: G.lp_from(GOLD["degenerate_transport"]["lp"])),
]


@pytest.mark.parametrize("prec", [pdhg.PREC_FP64, pdhg.PREC_MIXED])
@pytest.mark.parametrize("name,make", PDLP_CASES)
def test_pdlp_reaches_tolerance(name, make, prec):
    lp = make()
    tol = 1e-6
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(precision=prec, tol=tol, max_iters=200000))
    assert info.status == pdhg.OPTIMAL, (pdhg.STATUS_NAMES.get(info.status), info.rel_kkt)
    k = ffi.rel_kkt(lp, x, y)
    # the device's FP64 KKT and the oracle's double-double KKT agree
    assert k.rel_kkt <= 1.05 * tol, k.rel_kkt
    assert abs(k.rel_kkt - info.rel_kkt) <= 1e-3 * tol + 1e-2 * k.rel_kkt
    # the objective is the dd_real evaluation of c'x, and it is near the optimum
    assert info.objective == ffi.eval_objective(lp, x)
    opt = _optimum(lp)
    # the relative objective error of src/io/sol_io.hpp:96-102, within the required 1e-6
    assert abs(info.objective - opt) / (1 + abs(opt)) <= 1e-6, (info.objective, opt)
    if prec == pdhg.PREC_FP64:
        assert info.iterations_fp64 == info.iterations


def test_crude_blending_objective_matches_sol_file():
    g = GOLD["crude_blending"]
    lp = G.lp_from(g["lp_internal_min"])
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(precision=pdhg.PREC_FP64, tol=1e-9, max_iters=200000))
    assert info.status == pdhg.OPTIMAL
    assert abs(-info.objective - g["sol_objective"]) / g["sol_objective"] <= 1e-8
    assert np.allclose(x, g["sol_x"], rtol=1e-6, atol=1e-5)
    assert ffi.verify(lp, x, info.objective).passed


def test_plain_pdhg_on_fast_kernels_tracks_reference_loop():
    # ALGO_PDHG in FP64 runs the reference iteration on the CSR-adaptive
    # kernels: it differs from the bit-exact loop only by summation order.
    lp = L.generate(L.RANDOM_EQ, 9, m=300, n=700)
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_PDHG, precision=pdhg.PREC_FP64, tol=0.0,
                                                   max_iters=640, check_every=64))
    xo, yo, out = ffi.ref_pdhg_restated(lp, 640)
    assert info.iterations == 640
    # x+ at the last check is the iterate after 640 steps
    assert np.max(np.abs(x - xo)) <= 1e-9 * (1 + np.max(np.abs(xo)))


def test_iteration_limit_and_host_stop():
    lp = L.generate(L.RANDOM_EQ, 5, m=500, n=1250)
    with pdhg.Engine(lp) as eng:
        _, _, info = eng.solve(pdhg.default_params(max_iters=128, tol=0.0))
        assert info.status == pdhg.ITERATION_LIMIT and info.iterations == 128
        _, _, info = eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, max_iters=100))
        assert info.iterations == 100
        calls = []

        def poll():
            calls.append(1)
            return len(calls) > 3

        _, _, info = eng.solve(pdhg.default_params(tol=0.0, max_iters=10 ** 7), poll=poll)
        assert info.status == pdhg.TIME_LIMIT and len(calls) >= 4
        t = time.time()
        _, _, info = eng.solve(pdhg.default_params(tol=0.0, max_iters=10 ** 8, time_limit=0.5))
        assert info.status == pdhg.TIME_LIMIT and time.time() - t < 10


def test_warm_start_from_solution_converges_at_once():
    lp = L.generate(L.RANDOM_EQ, 6, m=400, n=1000)
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(precision=pdhg.PREC_FP64, tol=1e-8, max_iters=200000))
        assert info.status == pdhg.OPTIMAL
        x2, y2, info2 = eng.solve(pdhg.default_params(precision=pdhg.PREC_FP64, tol=1e-7), x_init=x, y_init=y,
                                  omega_init=info.primal_weight)
        assert info2.status == pdhg.OPTIMAL and info2.iterations <= 128


def test_update_vectors_matches_fresh_handle():
    a = L.generate(L.BLEND_FAMILY, 1, m=1000, n=2500, target_nnz=20000)
    b = L.generate(L.BLEND_FAMILY, 2, m=1000, n=2500, target_nnz=20000)
    p = pdhg.default_params(precision=pdhg.PREC_FP64, tol=1e-7, max_iters=100000)
    with pdhg.Engine(a) as eng:
        eng.update_vectors(cost=b.cost, rowlo=b.rowlo, rowup=b.rowup, collo=b.collo, colup=b.colup)
        x1, _, i1 = eng.solve(p)
    with pdhg.Engine(b) as eng:
        x2, _, i2 = eng.solve(p)
    assert i1.iterations == i2.iterations and np.array_equal(x1, x2)


def test_bad_input_is_rejected():
    lp = L.generate(L.RANDOM_EQ, 1, m=20, n=50)
    bad = L.LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index.copy(), lp.value, lp.cost, lp.collo, lp.colup,
               lp.rowlo, lp.rowup)
    bad.row_index[3] = 999
    with pytest.raises(RuntimeError, match="input_error"):
        pdhg.Engine(bad)
    with pdhg.Engine(lp) as eng:
        with pytest.raises(RuntimeError, match="input_error"):
            eng.solve(pdhg.default_params(reflection=2.0))


def test_reference_shaped_api():
    g = GOLD["unit_test_pdhg_lp"]
    lp = G.lp_from(g["lp"])
    r = pdhg.PdhgSolver.solve(lp, pdhg.Options(threads=2), pdhg.Deadline(60.0))
    assert r.status == pdhg.OPTIMAL and abs(r.objective - 9.0) <= 1e-2
    assert r.x.shape == (2,) and r.y.shape == (2,) and r.iterations > 0
    d = pdhg.Deadline(60.0)
    d.interrupt()
    r = pdhg.PdhgSolver.solve(L.generate(L.RANDOM_EQ, 1), pdhg.Options(pdhg_tol=0.0), d)
    assert r.status == pdhg.TIME_LIMIT


def test_reference_loop_kkt_probe_matches_oracle():
    # the probe reads the iterates only (bit-identical loop) and finds the
    # first 32-iteration boundary at which the reference iterate has rel KKT
    # <= tol, as the oracle's restatement probing at the same interval does
    lp = L.generate(L.RANDOM_EQ, 5, m=200, n=500)
    tol = 1e-4
    cap = 60016  # the chunk that ends the loop is not probed; the one before is
    with pdhg.Engine(lp) as eng:
        x, y, info = eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, max_iters=cap, tol=tol))
    xo, yo, out = ffi.ref_pdhg_restated(lp, cap, probe_every=32, probe_tol=tol)
    assert np.array_equal(G.bits(x), G.bits(xo)) and info.iterations == out.iterations
    assert out.first_hit > 0
    assert info.iterations_to_tol == out.first_hit
    # same iterate at the last probe: FP64 device sums vs double-double
    assert abs(info.rel_kkt - out.last_kkt) <= 1e-9 * out.last_kkt
    with pdhg.Engine(lp) as eng:
        _, _, off = eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, max_iters=60000, tol=0.0))
    assert off.iterations_to_tol == -1 and np.isnan(off.rel_kkt)


@pytest.mark.parametrize("prec", [pdhg.PREC_FP64, pdhg.PREC_MIXED])
def test_persistent_chunks_are_bit_identical_to_two_kernel_path(prec):
    # one cooperative launch per chunk with grid barriers runs the same row
    # blocks in the same order as the per-iteration kernels
    # the third LP (a 9000-nonzero row, empty rows) exercises the long-row
    # path over a fixed number of iterations; the first two are solved
    cases = [(L.generate(L.RANDOM_EQ, 3, m=500, n=1250), 200000),
             (L.generate(L.BLEND_FAMILY, 3, m=1000, n=2500, target_nnz=20000), 200000),
             (dense_row_lp(), 3200)]
    for lp, cap in cases:
        with pdhg.Engine(lp) as eng:
            base = dict(precision=prec, tol=1e-6, max_iters=cap, spmv_block_nnz=256)
            x0, y0, i0 = eng.solve(pdhg.default_params(persistent=0, **base))
            x1, y1, i1 = eng.solve(pdhg.default_params(persistent=1, **base))
        assert i1.status == i0.status
        assert i0.status == (pdhg.OPTIMAL if cap > 3200 else pdhg.ITERATION_LIMIT)
        assert i1.iterations == i0.iterations
        assert np.array_equal(G.bits(x0), G.bits(x1)) and np.array_equal(G.bits(y0), G.bits(y1))
        assert i1.kernel_launches < i0.kernel_launches


def test_persistent_barrier_wait_is_bounded():
    # persistent=2 launches one CTA fewer than the barrier waits for: every
    # wait must give up after its bound, the solve must end with an internal
    # error, and the handle (and the CUDA context) must stay usable
    lp = L.generate(L.RANDOM_EQ, 4, m=300, n=700)
    with pdhg.Engine(lp) as eng:
        t = time.perf_counter()
        with pytest.raises(RuntimeError, match="internal_error"):
            eng.solve(pdhg.default_params(persistent=2, max_iters=5000))
        assert time.perf_counter() - t < 10.0
        x, y, info = eng.solve(pdhg.default_params(persistent=1))
        assert info.status == pdhg.OPTIMAL
        assert ffi.rel_kkt(lp, x, y).rel_kkt <= 1.05e-6
