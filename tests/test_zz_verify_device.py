"""The solution check on the device (nir_pdhg_verify, nir_pdhg_batch_verify;
nirnaya_b200/csrc/k_verify.cuh) against the host check nir_verify_solution
(itself bit-identical to the reference's verify_solution,
src/io/sol_io.hpp:25-106): the same report, bit for bit.

CPU: the kernels' arithmetic, thread partitions and shuffle reductions,
compiled for the host from the same header
(tests/native/verify_device_emulation.cpp).  GPU: the C ABI on a B200.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from nirnaya_b200 import lp as L
from nirnaya_b200 import mps

INC = os.path.join(ROOT, "include")
CSRC = os.path.join(ROOT, "nirnaya_b200", "csrc")


def _same(a: dict, b: dict) -> bool:
    """Equal reports: every float field with the same bits."""
    if a.keys() != b.keys():
        return False
    for k in a:
        if isinstance(a[k], float):
            if np.float64(a[k]).view(np.uint64) != np.float64(b[k]).view(np.uint64):
                return False
        elif a[k] != b[k]:
            return False
    return True


def edge_lp(rng):
    """Duplicate entries within a column, bounds at and beyond 1e20 and
    infinite, an empty row and an empty column."""
    m, n = 7, 9
    cols = [[(0, 1.5), (0, -0.5), (2, 3.0)], [(1, 2.0)], [], [(3, 1.0), (4, -1.0), (3, 0.25)], [(5, 1e-3)],
            [(0, 2.0), (5, 4.0)], [(2, -7.0), (1, 1.0)], [(4, 0.5), (6, 1e3)], [(6, -2.0)]]
    start, idx, val = [0], [], []
    for c in cols:
        for r, v in c:
            idx.append(r)
            val.append(v)
        start.append(len(idx))
    big = [1e20, -1e20, 1e25, -1e30, np.inf, -np.inf, 5.0, -5.0, 0.0]
    collo = np.array([big[(j * 3) % 9] if j % 2 else -abs(rng.normal()) for j in range(n)])
    colup = np.array([big[(j * 5 + 1) % 9] if j % 3 else abs(rng.normal()) + 1 for j in range(n)])
    collo = np.where(collo > colup, -np.inf, collo)
    rowlo = np.array([-np.inf, 1.0, -1e21, 0.0, -2.0, -np.inf, 3.0])
    rowup = np.array([4.0, 1.0, 1e20, np.inf, 2.0, 9.99e19, np.inf])
    return L.LP(m, n, np.array(start, np.int64), np.array(idx, np.int32), np.array(val), rng.normal(size=n),
                collo, colup, rowlo, rowup, 2.5)


def empty_lp(m, n):
    return L.LP(m, n, np.zeros(n + 1, np.int64), np.zeros(0, np.int32), np.zeros(0), np.ones(n), np.zeros(n),
                np.ones(n), -np.ones(m), np.ones(m), 0.0)


def integer_lp(rng, m=5, n=50):
    """Free rows and boxed columns: with a point inside the box, the worst
    item can only be an integrality violation."""
    rows = rng.integers(0, m, size=2 * n)
    return L.LP(m, n, np.arange(0, 2 * n + 1, 2, dtype=np.int64), rows.astype(np.int32), rng.normal(size=2 * n),
                rng.normal(size=n), np.zeros(n), np.full(n, 10.0), np.full(m, -np.inf), np.full(m, np.inf), 0.0)


def tie_lp(m=600, n=1200):
    """With x = 2 everywhere, every column has the same upper-bound violation
    and every row (two entries of 1 each) the same lower-bound violation: the
    first maximum must win across threads and warps."""
    rng = np.random.default_rng(5)
    rows = rng.permutation(np.repeat(np.arange(m), n // m))
    lp = L.LP(m, n, np.arange(n + 1, dtype=np.int64), rows.astype(np.int32), np.ones(n), np.zeros(n),
              np.zeros(n), np.ones(n), np.full(m, 1e6), np.full(m, np.inf), 0.0)
    lp.extra["tie"] = True
    return lp


def a_point(lp, rng, mode):
    n = lp.ncol
    if mode == "tie":
        return np.full(n, 2.0)
    x = rng.normal(size=n) * 3
    lo = np.where(np.isfinite(lp.collo) & (np.abs(lp.collo) < 1e20), lp.collo, -50)
    up = np.where(np.isfinite(lp.colup) & (np.abs(lp.colup) < 1e20), lp.colup, 50)
    if mode == "feasible":
        x = np.clip(x, lo, up)
    elif mode == "integers":
        x = np.round(x) + np.where(rng.random(n) < 0.3, 0.5, 0.0)  # exact halves: round half away
    elif mode == "huge":
        x[rng.random(n) < 0.1] = 1e300 * np.sign(rng.normal())  # activities overflow to inf / nan
    x[rng.random(n) < 0.2] = 0.0
    if mode == "nan" and n:
        x[rng.integers(0, n)] = [np.nan, np.inf, -np.inf][rng.integers(0, 3)]
    return x


def batch_case(seed, with_empty=True):
    """Instances, points, integer marks, claimed objectives and a tolerance."""
    from test_facade import rich_instance

    rng = np.random.default_rng([0xDDC, seed])
    lps, vts = [], []
    lps.append(L.generate(L.RANDOM_EQ, seed, m=40, n=100))
    vts.append(None)
    r, vt = rich_instance(seed, m=60, n=100, int_frac=0.3)
    lps.append(r)
    vts.append(vt)
    lps.append(L.generate(L.MULTIPERIOD, seed + 1, m=600))
    vts.append(None)
    lps.append(edge_lp(rng))
    vts.append((rng.random(9) < 0.4).astype(np.int8) * 2)
    lps.append(L.generate(L.ZIPF, seed, m=300, n=700, target_nnz=4000))
    vts.append(None)
    lps.append(tie_lp())
    vts.append(None)
    lps.append(integer_lp(rng))
    vts.append(rng.integers(0, 3, size=50).astype(np.int8))
    if with_empty:
        lps.append(empty_lp(3, 0))
        vts.append(None)
        lps.append(empty_lp(0, 4))
        vts.append(None)
    modes = ["free", "feasible", "integers", "huge", "nan"]
    xs = []
    for k, lp in enumerate(lps):
        mode = "tie" if lp.extra.get("tie") else modes[(seed + k) % len(modes)]
        if lp.ncol == 50 and lp.nrow == 5:
            xs.append(rng.uniform(0.0, 10.0, size=50))  # inside the box, mostly fractional
            continue
        xs.append(a_point(lp, rng, mode))
    vts = [v if v is not None else np.zeros(lp.ncol, np.int8) for v, lp in zip(vts, lps)]
    claimed = np.array([[np.nan, np.inf, 0.0, rng.normal() * 10][(seed + k) % 4] for k in range(len(lps))])
    tol = [1e-9, 1e-6, 10.0, 0.3][seed % 4]
    return lps, xs, vts, claimed, tol


def host_reports(lps, xs, vts, claimed, tol):
    return [mps.verify_solution(lp, x, float(c), tol, vartype=vt) for lp, x, vt, c in zip(lps, xs, vts, claimed)]


# ---------------------------------------------------------------- CPU


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("vfy") / "libvfy_emu.so")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I" + INC, "-I" + CSRC,
                    os.path.join(ROOT, "tests", "native", "verify_device_emulation.cpp"), "-o", so], check=True)
    lib = C.CDLL(so)
    D = C.POINTER(C.c_double)
    lib.emu_batch_verify.argtypes = [C.POINTER(L.NirLpView), C.c_int, D, C.POINTER(C.c_int8), D, C.c_double,
                                     C.POINTER(mps.VerifyReport)]

    def run(lps, xs, vts, claimed, tol):
        views = (L.NirLpView * len(lps))(*[lp.view() for lp in lps])
        x = np.ascontiguousarray(np.concatenate(xs), np.float64)
        vt = np.ascontiguousarray(np.concatenate(vts), np.int8)
        cl = np.ascontiguousarray(claimed, np.float64)
        reps = (mps.VerifyReport * len(lps))()
        lib.emu_batch_verify(views, len(lps), x.ctypes.data_as(D), vt.ctypes.data_as(C.POINTER(C.c_int8)),
                             cl.ctypes.data_as(D), tol, reps)
        return [mps.report_dict(r) for r in reps]

    return run


@pytest.mark.parametrize("seed", range(8))
def test_device_check_arithmetic_matches_the_host_check(emu, seed):
    case = batch_case(seed)
    got, want = emu(*case), host_reports(*case)
    for k, (g, w) in enumerate(zip(got, want)):
        assert _same(g, w), (seed, k, g, w)


def test_the_cases_reach_every_outcome(emu):
    kinds, passed = set(), set()
    for seed in range(8):
        for rep in host_reports(*batch_case(seed)):
            kinds.add(rep["worst_item"].split(" on ")[0].split(" in ")[0])
            passed.add(rep["passed"])
    assert passed == {True, False}
    for item in ("Lower bound", "Upper bound", "Integrality", "Row lower bound", "Row upper bound", "NaN/Inf"):
        assert item in kinds, (item, kinds)


def test_ties_name_the_first_column_and_row(emu):
    lp = tie_lp()
    x = np.full(lp.ncol, 2.0)
    rep = emu([lp], [x], [np.zeros(lp.ncol, np.int8)], np.array([np.nan]), 1e-6)[0]
    assert rep == host_reports([lp], [x], [np.zeros(lp.ncol, np.int8)], [np.nan], 1e-6)[0]
    assert rep["worst_item"] == "Row lower bound on 0"
    # without the rows, the first column's upper bound is named
    cols_only = L.LP(0, lp.ncol, np.zeros(lp.ncol + 1, np.int64), np.zeros(0, np.int32), np.zeros(0), lp.cost,
                     lp.collo, lp.colup, np.zeros(0), np.zeros(0), 0.0)
    rep = emu([cols_only], [x], [np.zeros(lp.ncol, np.int8)], np.array([np.nan]), 1e-6)[0]
    assert rep["worst_item"] == "Upper bound on 0" and rep["max_bound_viol"] == 0.5


# ---------------------------------------------------------------- GPU


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_batch_verify_on_the_device_matches_the_host_check(seed):
    from nirnaya_b200 import batch as B

    lps, xs, vts, claimed, tol = batch_case(seed, with_empty=False)
    want = host_reports(lps, xs, vts, claimed, tol)
    with B.BatchEngine(lps) as eng:
        got = eng.verify(xs, claimed, tol, vts)
        again = eng.verify(xs, claimed, tol, vts)
    for k, (g, w) in enumerate(zip(got, want)):
        assert _same(g, w), (seed, k, g, w)
    assert all(_same(a, b) for a, b in zip(got, again))


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_batch_verify_checks_the_solved_points_in_place():
    from nirnaya_b200 import batch as B
    from nirnaya_b200 import pdhg

    lps = [L.generate(L.RANDOM_EQ, 21, m=200, n=500), L.generate(L.MULTIPERIOD, 22, m=600),
           L.generate(L.RANDOM_EQ, 23, m=80, n=200)]
    with B.BatchEngine(lps) as eng:
        with pytest.raises(RuntimeError, match="no batch solve"):
            eng.verify()
        res, _ = eng.solve(pdhg.default_params(tol=1e-6, max_iters=200000))
        claimed = np.array([info.objective for _, _, info in res])
        got = eng.verify(None, claimed, 1e-6)
    for lp, (x, _, _), c, g in zip(lps, res, claimed, got):
        assert _same(g, mps.verify_solution(lp, x, float(c), 1e-6))


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_single_handle_verify_matches_the_host_check():
    from nirnaya_b200 import pdhg

    rng = np.random.default_rng(7)
    lp = L.generate(L.ZIPF, 3, m=2000, n=5000, target_nnz=40000)
    with pdhg.Engine(lp) as eng:
        for mode in ("free", "feasible", "huge", "nan"):
            x = a_point(lp, rng, mode)
            vt = (rng.random(lp.ncol) < 0.2).astype(np.int8)
            for tol, claimed in ((1e-9, float(rng.normal())), (10.0, float("nan"))):
                got = eng.verify(x, claimed, tol, vartype=vt)
                want = mps.verify_solution(lp, x, claimed, tol, vartype=vt)
                assert _same(got, want), (mode, tol, got, want)


def test_device_check_random_sweep(emu):
    """30 random batches over all five generator kinds with bounds moved to
    the edge values (+-inf, +-1e20, beyond 1e20, 0), random non-finite
    entries, integer marks and tolerances: the emulated device check equals
    the host check bit for bit."""
    rng = np.random.default_rng(2024)
    kinds = [(L.RANDOM_EQ, dict(m=60, n=150)), (L.ZIPF, dict(m=200, n=500, target_nnz=3000)),
             (L.MULTIPERIOD, dict(m=500)), (L.BLEND_FAMILY, dict(m=100, n=250, target_nnz=1500)),
             (L.BADLY_SCALED, dict(m=80, n=200, target_nnz=1200))]
    edges = np.array([np.inf, -np.inf, 1e20, -1e20, 3e20, -5e25, 0.0])
    for trial in range(30):
        lps, xs, vts, claimed = [], [], [], []
        for _ in range(int(rng.integers(1, 5))):
            kind, kw = kinds[int(rng.integers(0, len(kinds)))]
            lp = L.generate(kind, int(rng.integers(0, 1000)), **kw)
            for arr in (lp.collo, lp.colup, lp.rowlo, lp.rowup):
                hit = rng.random(arr.size) < 0.05
                arr[hit] = edges[rng.integers(0, edges.size, int(hit.sum()))]
            x = rng.normal(size=lp.ncol) * 10 ** rng.uniform(-2, 2)
            x[rng.random(lp.ncol) < 0.3] = 0.0
            if rng.random() < 0.2:
                x[int(rng.integers(0, lp.ncol))] = [np.nan, np.inf][int(rng.integers(0, 2))]
            lps.append(lp)
            xs.append(x)
            vts.append((rng.random(lp.ncol) < 0.2).astype(np.int8) * int(rng.integers(1, 3)))
            claimed.append([np.nan, float(rng.normal() * 100)][int(rng.integers(0, 2))])
        tol = float(10 ** rng.uniform(-10, 1))
        got, want = emu(lps, xs, vts, np.array(claimed), tol), host_reports(lps, xs, vts, claimed, tol)
        for k, (g, w) in enumerate(zip(got, want)):
            assert _same(g, w), (trial, k, g, w)


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
@pytest.mark.parametrize("algorithm", ["pdlp", "reference"])
def test_single_handle_checks_its_solved_point_in_place(algorithm):
    """Engine.verify(None) after a solve (PDLP or the reference loop) checks
    the returned point on the device: the host check's report for it."""
    from nirnaya_b200 import pdhg

    lp = L.generate(L.RANDOM_EQ, 5, m=300, n=750)
    with pdhg.Engine(lp) as eng:
        with pytest.raises(RuntimeError, match="no solve"):
            eng.verify(None)
        algo = pdhg.ALGO_PDLP if algorithm == "pdlp" else pdhg.ALGO_REFERENCE
        x, _, info = eng.solve(pdhg.default_params(algorithm=algo, tol=1e-6, max_iters=20000))
        got = eng.verify(None, info.objective, 1e-6)
    assert _same(got, mps.verify_solution(lp, x, info.objective, 1e-6))


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_sharded_solve_checks_its_shard_on_the_device():
    """solve_sharded(verify_tol=...): the rank's solved points are checked in
    place and every result carries the verdict; solved instances pass."""
    from nirnaya_b200 import batch as B
    from nirnaya_b200 import pdhg

    lps = [L.generate(L.RANDOM_EQ, 31, m=200, n=500), L.generate(L.MULTIPERIOD, 32, m=600),
           L.generate(L.RANDOM_EQ, 33, m=80, n=200)]
    got = B.solve_sharded(lps, 0, 1, params=pdhg.default_params(tol=1e-6, max_iters=200000), verify_tol=1e-4)
    assert sorted(got) == [0, 1, 2]
    for obj, status, iterations, passed in got.values():
        assert status != pdhg.OPTIMAL or passed, (obj, status, iterations)
