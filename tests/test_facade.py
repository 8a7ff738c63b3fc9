"""Presolve and scaling before the PDHG path (libnir_facade.so) against the
reference's Presolver::presolve (src/presolve/presolve.hpp:32-345) and
scale_model (src/model/scaling.hpp:56-154), compiled here (oracle/_ref).

CPU only; bit-for-bit on every output.  The instances are built so that
every presolve rule fires: fixed columns (R4), empty and singleton rows
with either sign and integer rounding (R1, R3), activity infeasibility
(R6), redundant rows (R5), forcing rows at either activity bound (R14),
integer bound tightening from either side (R7), and empty columns with
positive, negative and zero cost (R2), including the early returns.
"""
import numpy as np
import pytest

from nirnaya_b200 import facade
from nirnaya_b200 import lp as L

KEYS = ("col_start", "row_index", "value", "cost", "collo", "colup", "rowlo", "rowup")
INF = float("inf")


def _ref():
    from oracle import ffi

    if not ffi.ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    return ffi


def _bits(a):
    return np.atleast_1d(np.asarray(a, np.float64)).view(np.uint64)


def _lp(m, n, rows, cols, vals, **kw):
    per_row = [([], []) for _ in range(m)]
    for i, j, v in zip(rows, cols, vals):
        per_row[i][0].append(j)
        per_row[i][1].append(v)
    return L.LP.from_rows(n, per_row, **kw)


def rich_instance(seed, m=400, n=900, int_frac=0.3, density=4):
    """A sparse model in which every presolve rule has something to do."""
    rng = np.random.default_rng([0x9E5, seed])
    rows, cols, vals = [], [], []
    for i in range(m):
        kind = rng.integers(0, 10)
        if kind == 0:
            k = 1  # singleton row
        elif kind == 1:
            k = 0  # empty row
        else:
            k = int(rng.integers(2, 2 * density))
        js = rng.choice(n, size=min(k, n), replace=False)
        for j in js:
            v = float(rng.choice([-3, -2, -1, -0.5, 0.5, 1, 2, 3, 1.5, -1.25]))
            rows.append(i)
            cols.append(int(j))
            vals.append(v)
    vt = (rng.random(n) < int_frac).astype(np.int8)
    collo = np.where(rng.random(n) < 0.85, np.round(rng.uniform(-2, 1, n)), -INF)
    width = np.round(rng.uniform(0, 4, n))
    colup = np.where(rng.random(n) < 0.85, np.where(np.isfinite(collo), collo + width, width - 1.0), INF)
    fixed = rng.random(n) < 0.08
    colup[fixed & np.isfinite(collo)] = collo[fixed & np.isfinite(collo)]
    colup = np.where(np.isfinite(collo), np.maximum(colup, collo), colup)
    cost = np.round(rng.normal(size=n), 2)
    cost[rng.random(n) < 0.1] = 0.0
    # mostly bounded below: no cost pushes a column toward an infinite bound
    # (a few keep it, so the unbounded stop of R2 is still reached)
    keep = rng.random(n) < 0.03
    cost = np.where(~keep & ~np.isfinite(collo) & (cost > 0), -cost, cost)
    cost = np.where(~keep & ~np.isfinite(colup) & (cost < 0), 0.0, cost)
    # row bounds around the activity of a point inside the column bounds
    x0 = np.clip(rng.uniform(-1, 2, n), np.where(np.isfinite(collo), collo, -5),
                 np.where(np.isfinite(colup), colup, 5))
    act = np.zeros(m)
    np.add.at(act, np.array(rows, int), np.array(vals) * x0[np.array(cols, int)])
    rowlo = np.where(rng.random(m) < 0.6, act - rng.uniform(0, 3, m), -INF)
    rowup = np.where(rng.random(m) < 0.6, act + rng.uniform(0, 3, m), INF)
    eq = rng.random(m) < 0.15
    rowlo[eq], rowup[eq] = act[eq], act[eq]
    lp = _lp(m, n, rows, cols, vals, cost=cost, collo=collo, colup=colup, rowlo=rowlo, rowup=rowup)
    return lp, vt


def forcing_instance(seed):
    """Rows whose activity bound equals a row bound (R14 at min and max),
    redundant rows, and integer rows that tighten bounds (R7).  Each row
    has columns of its own, so the model stays feasible and presolve runs
    to the reduced model; the columns no row uses are empty (R2)."""
    rng = np.random.default_rng([0xF0C, seed])
    n, m = 130, 30
    rows, cols, vals = [], [], []
    rowlo, rowup = np.full(m, -INF), np.full(m, INF)
    collo, colup = np.zeros(n), np.full(n, 4.0)
    vt = (rng.random(n) < 0.5).astype(np.int8)
    fresh = list(rng.permutation(n))  # each row gets columns of its own
    for i in range(m):
        r = i % 5
        k = int(rng.integers(2, 5))
        js = np.array([fresh.pop() for _ in range(k)])
        a = rng.choice([1.0, 2.0, -1.0, 0.5], size=js.size)
        rows += [i] * js.size
        cols += js.tolist()
        vals += a.tolist()
        mn = float(np.sum(np.where(a > 0, a * collo[js], a * colup[js])))
        mx = float(np.sum(np.where(a > 0, a * colup[js], a * collo[js])))
        if r == 0:
            rowup[i] = mn            # forcing at the minimum
        elif r == 1:
            rowlo[i] = mx            # forcing at the maximum
        elif r == 2:
            rowlo[i], rowup[i] = mn - 1, mx + 1  # redundant
        elif r == 3:
            rowup[i] = mn + 1.5      # tightening room for integers
        else:
            rowlo[i] = mx - 2.5
    cost = rng.normal(size=n)
    lp = _lp(m, n, rows, cols, vals, cost=cost, collo=collo, colup=colup, rowlo=rowlo, rowup=rowup)
    return lp, vt


def _check_presolve(lp, vt, threads=0, rounds=20):
    ffi = _ref()
    a = facade.presolve(lp, vt, rounds, threads)
    b = ffi.ref_presolve(lp, vt, 2, rounds)
    assert (a.status, a.solved_in_presolve, a.rows_removed, a.cols_removed, a.bound_tightenings) == (
        b["status"], b["solved_in_presolve"], b["rows_removed"], b["cols_removed"], b["bound_tightenings"])
    assert a.reduced.nrow == b["reduced"].nrow and a.reduced.ncol == b["reduced"].ncol
    for k in KEYS:
        x, y = getattr(a.reduced, k), getattr(b["reduced"], k)
        if k == "col_start" and a.reduced.ncol == 0:
            continue
        assert x.shape == y.shape and np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8)), k
    assert np.array_equal(_bits(a.reduced.obj_offset), _bits(b["reduced"].obj_offset))
    assert np.array_equal(a.vartype, b["vartype"])
    assert np.array_equal(a.orig_col_map, b["orig_col_map"]) and np.array_equal(a.orig_row_map, b["orig_row_map"])
    assert np.array_equal(_bits(a.fixed_x), _bits(b["fixed_x"])) and np.array_equal(a.is_col_fixed, b["is_col_fixed"])
    return a


@pytest.mark.parametrize("seed", range(12))
def test_presolve_rich_instances(seed):
    lp, vt = rich_instance(seed)
    a = _check_presolve(lp, vt, threads=1 + seed % 4)
    if seed == 0:
        assert a.rows_removed > 0 and a.cols_removed > 0


@pytest.mark.parametrize("seed", range(8))
def test_presolve_forcing_redundant_and_integer_rows(seed):
    lp, vt = forcing_instance(seed)
    a = _check_presolve(lp, vt, threads=3)
    assert a.rows_removed > 0


def test_presolve_rules_all_fire():
    """Across the instances above, every counter and every early return is
    reached at least once (so the parity above covers each rule)."""
    seen = {"infeasible": 0, "unbounded": 0, "tight": 0, "rows": 0, "cols": 0}
    for seed in range(40):
        for lp, vt in (rich_instance(seed, m=120, n=200), forcing_instance(seed)):
            a = facade.presolve(lp, vt)
            seen["infeasible"] += a.status == facade.INFEASIBLE
            seen["unbounded"] += a.status == facade.UNBOUNDED
            seen["tight"] += a.bound_tightenings > 0
            seen["rows"] += a.rows_removed > 0
            seen["cols"] += a.cols_removed > 0
    assert all(v > 0 for v in seen.values()), seen


def test_presolve_early_returns_match(tmp_path):
    for seed in range(40):
        lp, vt = rich_instance(seed, m=120, n=200)
        _check_presolve(lp, vt)


@pytest.mark.parametrize("kind,kw", [(1, dict(m=300, n=800)), (2, dict(m=3000, n=8000, target_nnz=60000)),
                                     (3, {}), (4, {}), (5, dict(m=60, n=150))])
def test_presolve_generated_families(kind, kw):
    lp = L.generate(kind, 3, **kw)
    for threads in (1, 8):
        _check_presolve(lp, None, threads=threads)


def test_presolve_round_limit_and_threads():
    lp, vt = rich_instance(5, m=800, n=1500)
    for rounds in (1, 2, 5):
        base = _check_presolve(lp, vt, threads=1, rounds=rounds)
        other = facade.presolve(lp, vt, rounds, 7)
        for k in KEYS:
            assert np.array_equal(getattr(base.reduced, k), getattr(other.reduced, k))


def test_postsolve_puts_values_back():
    lp, vt = forcing_instance(1)
    a = facade.presolve(lp, vt)
    x_red = np.arange(a.reduced.ncol, dtype=np.float64)
    x = a.postsolve(x_red)
    assert np.array_equal(x[a.orig_col_map], x_red)
    fixed = a.is_col_fixed
    assert np.array_equal(x[fixed], a.fixed_x[fixed])


# ---- scaling


def _check_scale(lp, vt=None, enable=True, q=None, threads=0):
    ffi = _ref()
    a = facade.scale(lp, vt, enable, q, threads)
    b = ffi.ref_scale(lp, vt, enable, q)
    assert a.active == b["active"]
    assert np.array_equal(_bits(a.R), _bits(b["R"])) and np.array_equal(_bits(a.C), _bits(b["C"]))
    for k in ("cost", "collo", "colup", "value", "rowlo", "rowup"):
        assert np.array_equal(_bits(getattr(a.lp, k)), _bits(b[k])), k
    if q is not None:
        assert np.array_equal(_bits(a.q_value), _bits(b["q_value"]))
    return a


@pytest.mark.parametrize("kind,kw", [(1, dict(m=300, n=800)), (2, dict(m=3000, n=8000, target_nnz=60000)),
                                     (5, dict(m=200, n=500)), (3, {})])
def test_scale_generated_families(kind, kw):
    lp = L.generate(kind, 4, **kw)
    for threads in (1, 5):
        _check_scale(lp, threads=threads)


@pytest.mark.parametrize("decades", [0.0, 1.0, 6.0])
def test_scale_two_and_six_passes_with_integers(decades):
    lp, vt = rich_instance(2, m=500, n=1200)
    rng = np.random.default_rng(9)
    lp = L.LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index, lp.value * 10.0 ** rng.uniform(-decades, decades, lp.nnz),
              lp.cost, lp.collo, lp.colup, lp.rowlo, lp.rowup)
    a = _check_scale(lp, vt, threads=4)
    # coefficients within a ratio of 10: no scaling; below 1e3: 2 passes; else 6
    assert a.active == (decades > 0.0)


def test_scale_off_and_quadratic():
    lp = L.generate(5, 1, m=40, n=90)
    _check_scale(lp, enable=False)
    n = lp.ncol
    qs = np.arange(n + 1, dtype=np.int64)
    qi = np.arange(n, dtype=np.int32)
    qv = np.linspace(0.5, 3.0, n)
    _check_scale(lp, q=(qs, qi, qv))


def test_c2_presolve_and_scale_match():
    """The 200k x 500k workload: what Solver::solve does before PDHG."""
    lp = L.generate(2, 1)
    a = _check_presolve(lp, None, threads=0)
    assert (a.reduced.nrow, a.reduced.ncol) == (87885, 398795)
    _check_scale(a.reduced, a.vartype)


def test_facade_exports_every_declared_symbol():
    import ctypes as C
    import os

    from conftest import ROOT
    from test_abi import declared

    lib = C.CDLL(os.path.join(ROOT, "nirnaya_b200", "libnir_facade.so"))
    names = declared("nir_facade.h")
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(facade.EXPORTED) == names


def test_facade_rejects_inconsistent_input():
    lp = L.generate(1, 0, m=20, n=50)
    bad = L.LP(lp.nrow, lp.ncol, lp.col_start, lp.row_index.copy(), lp.value, lp.cost, lp.collo, lp.colup,
               lp.rowlo, lp.rowup)
    bad.row_index[3] = lp.nrow + 5  # a row index out of range
    with pytest.raises(RuntimeError, match="status 12"):
        facade.presolve(bad)
    with pytest.raises(RuntimeError, match="status 12"):
        facade.scale(bad)


@pytest.mark.parametrize("case", ["empty", "cols_only", "rows_only", "rows_only_infeasible"])
def test_degenerate_models_match(case):
    """Models with no rows, no columns or neither, through presolve and
    scaling, as the reference treats them (solved in presolve, or the
    infeasible empty row)."""
    z64, z32, z = np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0)
    lp = {
        "empty": L.LP(0, 0, z64, z32, z, z, z, z, z, z),
        "cols_only": L.LP(0, 3, np.zeros(4, np.int64), z32, z, np.array([1.0, -1.0, 0.0]),
                          np.array([0.0, -INF, -1.0]), np.array([2.0, 5.0, 3.0]), z, z),
        "rows_only": L.LP(2, 0, z64, z32, z, z, z, z, np.array([-1.0, 0.0]), np.array([1.0, 0.0])),
        "rows_only_infeasible": L.LP(1, 0, z64, z32, z, z, z, z, np.array([1.0]), np.array([2.0])),
    }[case]
    a = _check_presolve(lp, None)
    assert a.solved_in_presolve
    _check_scale(lp)
