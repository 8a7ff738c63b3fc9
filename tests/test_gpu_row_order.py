"""The engine's own row order (longest rows first on LPs with skewed row
lengths, nirnaya_b200/csrc/engine.cu row_order), checked through the C ABI
against the caller's order (NIR_PDHG_ROW_ORDER=0):
  - every row keeps its entries and their order, so the sequential SpMV,
    the reference loop (no probe) and the device solution check give the
    same bits in the caller's order; the row-block SpMV, whose summation
    tree depends on which rows share a block, agrees to rounding;
  - PDLP reaches the same tolerance, confirmed by the oracle's dd KKT, at
    the same objective to 1e-6 (its norms are summed in another order, so
    the iterates may differ in their last bits);
  - warm starts and new vectors are mapped into the engine's order.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

from nirnaya_b200 import lp as L  # noqa: E402
from nirnaya_b200 import pdhg  # noqa: E402
from oracle import ffi  # noqa: E402


def _lp():
    # power-law rows: the longest is far above 8x the mean, so the engine reorders
    return L.generate(L.ZIPF, 3, m=20000, n=50000, target_nnz=500000)


def _engine(lp, monkeypatch, mode):
    monkeypatch.setenv("NIR_PDHG_ROW_ORDER", mode)
    return pdhg.Engine(lp)


def test_the_power_law_lp_is_reordered():
    lp = _lp()
    rl = np.bincount(lp.row_index, minlength=lp.nrow)
    assert lp.nrow >= 1024 and rl.max() >= 8 * rl.mean()


def test_spmv_and_reference_loop_are_bit_identical_in_the_callers_order(monkeypatch):
    lp = _lp()
    rng = np.random.default_rng(5)
    x = rng.standard_normal(lp.ncol)
    y = rng.standard_normal(lp.nrow)
    out = {}
    for mode in ("0", "1"):
        with _engine(lp, monkeypatch, mode) as eng:
            ax = eng.spmv(x, transpose=False, kernel=0)
            aty = eng.spmv(y, transpose=True, kernel=0)
            ax1 = eng.spmv(x, transpose=False, kernel=1)
            p = pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, tol=0.0, max_iters=2000)
            xs, ys, info = eng.solve(p)
            rep = eng.verify(xs, claimed_obj=info.objective)
        out[mode] = (ax, aty, ax1, xs, ys, info.iterations, info.objective, rep)
    a, b = out["0"], out["1"]
    for k in (0, 1, 3, 4):
        assert np.array_equal(a[k], b[k]), k
    assert np.allclose(a[2], b[2], rtol=1e-12, atol=1e-12 * np.abs(a[2]).max())
    assert a[5] == b[5] and a[6] == b[6]
    assert a[7] == b[7]


def test_pdlp_reaches_the_same_optimum_in_either_order(monkeypatch):
    lp = _lp()
    res = {}
    for mode in ("0", "1"):
        with _engine(lp, monkeypatch, mode) as eng:
            x, y, info = eng.solve(pdhg.default_params(tol=1e-6))
            assert info.status == pdhg.OPTIMAL
            k = ffi.rel_kkt(lp, x, y)
            assert k.rel_kkt <= 1.05e-6
            assert info.objective == ffi.eval_objective(lp, x)
            res[mode] = (info.objective, info.iterations, y)
    o0, o1 = res["0"][0], res["1"][0]
    assert abs(o0 - o1) / (1.0 + abs(o0)) <= 1e-6
    # the duals come back in the caller's order: the two runs agree row by row
    assert np.corrcoef(res["0"][2], res["1"][2])[0, 1] > 0.999


def test_warm_start_and_new_vectors_are_mapped(monkeypatch):
    lp = _lp()
    first, kkt = {}, {}
    for mode in ("0", "1"):
        with _engine(lp, monkeypatch, mode) as eng:
            x, y, info = eng.solve(pdhg.default_params(tol=1e-6))
            first[mode] = (x, y, info.primal_weight)
    # the same warm start (the order-0 solution, in the caller's order) in
    # both orders: the same trajectory up to rounding, so y_init is mapped
    x, y, w = first["0"]
    for mode in ("0", "1"):
        with _engine(lp, monkeypatch, mode) as eng:
            _, _, info = eng.solve(pdhg.default_params(tol=0.0, max_iters=256), x_init=x, y_init=y, omega_init=w)
            kkt[mode] = eng.history(8)[:4, 1]
    assert np.allclose(kkt["0"], kkt["1"], rtol=1e-6), kkt
    with _engine(lp, monkeypatch, "1") as eng:
        # new row bounds, in the caller's order, give the LP the oracle sees
        rowlo = lp.rowlo.copy()
        rowup = lp.rowup.copy()
        fin = np.isfinite(rowlo)
        rowlo[fin] -= 0.1 * np.abs(rowlo[fin])  # looser lower bounds: still feasible
        eng.update_vectors(rowlo=rowlo, rowup=rowup)
        x2, y2, info2 = eng.solve(pdhg.default_params(tol=1e-6))
    lp2 = L.LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index, lp.value, lp.cost, lp.collo, lp.colup, rowlo, rowup)
    assert info2.status == pdhg.OPTIMAL
    assert ffi.rel_kkt(lp2, x2, y2).rel_kkt <= 1.05e-6
