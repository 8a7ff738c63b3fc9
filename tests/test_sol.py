"""SOL file I/O and the double-double solution check (libnir_mps.so,
include/nir_sol.h) against the reference's SolIo::write_sol / read_sol and
verify_solution (src/io/sol_io.hpp:25-170), compiled here.

CPU only.  write: identical bytes.  read: identical x and objective,
including how `istream >> double` treats odd tokens, and the same
exception where std::stod throws on the objective (read_sol runs as its
own process: oracle/_ref/ref_sol_tool).  verify: identical report fields
and worst item.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from nirnaya_b200 import lp as L
from nirnaya_b200 import mps


def _ffi():
    from oracle import ffi

    if not ffi.ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    return ffi


def _bits(a):
    return np.atleast_1d(np.asarray(a, np.float64)).view(np.uint64)


def test_sol_exports_every_declared_symbol():
    import ctypes as C

    from test_abi import declared

    lib = C.CDLL(os.path.join(ROOT, "nirnaya_b200", "libnir_mps.so"))
    names = declared("nir_sol.h")
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(mps.EXPORTED_SOL) == names


@pytest.mark.parametrize("case", ["plain", "few_names", "long_names", "special"])
def test_write_sol_bytes(tmp_path, case):
    ffi = _ffi()
    lp = L.generate(1, 2, m=40, n=120)
    rng = np.random.default_rng(3)
    x = rng.normal(size=lp.ncol) * 10.0 ** rng.integers(-8, 8, lp.ncol)
    names = [f"x_{j}" for j in range(lp.ncol)]
    nx = lp.ncol
    if case == "few_names":
        names = names[:50]     # the rest are written as C<j>
        nx = lp.ncol - 7       # fewer values than columns: lines stop there
    elif case == "long_names":
        names = ["n" * (200 + j) + str(j) for j in range(lp.ncol)]  # past the 256-byte line buffer
    elif case == "special":
        x[:6] = [np.inf, -np.inf, np.nan, -0.0, 5e-324, 1.7976931348623157e308]
    ours, ref = str(tmp_path / "o.sol"), str(tmp_path / "r.sol")
    mps.write_sol(ours, x[:nx], "optimal", 123.456, 1e-4, names, ncol=lp.ncol)
    # the reference writes the names of its model: pad to ncol with C<j>
    ref_names = names + [f"C{j}" for j in range(len(names), lp.ncol)]
    assert ffi.ref_write_sol(lp, ref_names, 0, 123.456, 1e-4, x[:nx], ref) == 0
    with open(ours, "rb") as a, open(ref, "rb") as b:
        assert a.read() == b.read()


SOL_LINES = [
    "C0 1.5", "C1 -2e-3", "C2 1.5e", "C3 1e400", "C4 1e-400", "C5 0x10", "C6 +.5", "C7 .", "C8 inf", "C9 nan",
    "C10 1.5abc", "  C11   7", "C12\t8", "C13", "", "nosuch 9", "C0 2.5", "C14 -0", "C15 00012.5e+1",
    "C16 1e", "C17 1e+", "C18 -.e5", "C19 4.", "C20 123456789012345678901234567890", "C21 1.0000000000000000000001",
    "#objective 5", "# gap 1", "# objective 42.5", "C22 3\r", "C23 9.9E9xyz", "C24 +-1", "C25 0.000e-2",
]


def _model_file(tmp_path, n=30):
    lp = L.generate(1, 0, m=5, n=n)
    lp.cost[lp.cost == 0.0] = 1.0  # every column appears in COLUMNS
    path = str(tmp_path / "model.mps")
    names = [f"C{j}" for j in range(n)]
    mps.write_mps(path, lp, name="solmodel", col_names=names)
    return lp, names, path


def _compare_read(tmp_path, text, names, model):
    ffi = _ffi()
    sol = str(tmp_path / "x.sol")
    with open(sol, "w", newline="") as f:
        f.write(text)
    ref = ffi.ref_read_sol(model, sol, len(names))
    try:
        x, obj, _ = mps.read_sol(sol, names)
        ours = ("ok", x, obj)
    except mps.MpsError:
        ours = ("exception",)
    assert ours[0] == ref[0], (ours, ref)
    if ref[0] == "ok":
        assert np.array_equal(_bits(ours[1]), _bits(ref[1])) and _bits(ours[2]) == _bits(ref[2])
    return ours


def test_read_sol_odd_tokens(tmp_path):
    lp, names, model = _model_file(tmp_path)
    ours = _compare_read(tmp_path, "\n".join(SOL_LINES) + "\n", names, model)
    assert ours[0] == "ok" and ours[2] == 42.5 and ours[1][0] == 2.5


@pytest.mark.parametrize("obj_line", ["# objective", "# objective abc", "# objective 1e400", "# objective 1e-400",
                                      "# objective 0x1p3", "# objective inf", "# objective 3d0"])
def test_read_sol_objective_like_stod(tmp_path, obj_line):
    lp, names, model = _model_file(tmp_path)
    _compare_read(tmp_path, f"# status optimal\n{obj_line}\nC0 1\n", names, model)


def test_read_sol_random_files(tmp_path):
    lp, names, model = _model_file(tmp_path, n=60)
    rng = np.random.default_rng(5)
    for _ in range(30):
        lines = list(rng.choice(SOL_LINES, size=40))
        lines += [f"C{rng.integers(0, 70)} {rng.normal() * 10.0 ** rng.integers(-300, 300):.17g}" for _ in range(40)]
        rng.shuffle(lines)
        _compare_read(tmp_path, rng.choice(["\n", "\r\n"]).join(lines), names, model)


def test_read_sol_of_written_file(tmp_path):
    lp = L.generate(2, 3, m=2000, n=5000, target_nnz=40000)
    lp.cost[lp.cost == 0.0] = 1.0
    names = [f"C{j}" for j in range(lp.ncol)]
    model = str(tmp_path / "m.mps")
    mps.write_mps(model, lp, col_names=names)
    x = np.random.default_rng(1).normal(size=lp.ncol)
    sol = str(tmp_path / "s.sol")
    mps.write_sol(sol, x, "optimal", 7.0, 0.0, names)
    xo, obj, _ = mps.read_sol(sol, names, threads=4)
    assert np.array_equal(xo, x) and obj == 7.0
    _compare_read(tmp_path, open(sol).read(), names, model)


def test_read_sol_missing_file(tmp_path):
    with pytest.raises(mps.MpsError) as e:
        mps.read_sol(str(tmp_path / "none.sol"), ["a"])
    assert e.value.status == 14


def _verify_pair(lp, x, claimed, tol, vt=None):
    ffi = _ffi()
    cn = [f"C{j}" for j in range(lp.ncol)]
    rn = [f"R{i}" for i in range(lp.nrow)]
    a = mps.verify_solution(lp, x, claimed, tol, vartype=vt, col_names=cn, row_names=rn, threads=3)
    b = ffi.ref_verify_full(lp, x, claimed, tol, vartype=vt)
    for k in ("max_bound_viol", "max_row_viol", "max_int_viol", "computed_obj", "obj_rel_err"):
        assert _bits(a[k]) == _bits(b[k]), k
    assert a["passed"] == b["passed"] and a["worst_item"] == b["worst_item"], (a, b)
    return a


@pytest.mark.parametrize("seed", range(10))
def test_verify_matches(seed):
    rng = np.random.default_rng(seed)
    lp = L.generate(int(rng.choice([1, 2, 5])), seed, m=300, n=700)
    vt = (rng.random(lp.ncol) < 0.3).astype(np.int8)
    x = rng.normal(size=lp.ncol) * 3
    if seed % 3 == 0:
        x = np.clip(x, lp.collo, lp.colup)
    if seed % 4 == 1:
        x[rng.integers(lp.ncol)] = np.nan
    x[rng.random(lp.ncol) < 0.2] = 0.0
    obj = mps.eval_objective(lp, x) if np.isfinite(x).all() else 1.0
    for tol in (1e-9, 1e-6, 10.0):
        _verify_pair(lp, x, obj * (1 + 1e-7 * seed), tol, vt)


def test_verify_size_mismatch_and_clean_solution():
    lp = L.generate(1, 1, m=50, n=100)
    a = _verify_pair(lp, np.zeros(lp.ncol - 1), 0.0, 1e-6)
    assert not a["passed"] and a["worst_item"] == "Solution size mismatch"


def test_eval_objective_matches():
    ffi = _ffi()
    for seed in range(5):
        lp = L.generate(2, seed, m=2000, n=5000, target_nnz=40000)
        lp.obj_offset = 0.1 * seed
        x = np.random.default_rng(seed).normal(size=lp.ncol)
        ref = ffi.ref_lib().ref_eval_objective(ffi.C.byref(lp.view()), ffi._dptr(x))
        assert _bits(mps.eval_objective(lp, x)) == _bits(ref)


def test_verify_splits_rows_into_ranges_on_larger_models():
    """Above 131,072 nonzeros the row activities are summed in row ranges,
    one per thread, each scanning the columns in order: the same report as
    the reference at every thread count, ties across ranges included."""
    ffi = _ffi()
    rng = np.random.default_rng(11)
    lp = L.generate(2, 4, m=20000, n=50000, target_nnz=600000)
    assert lp.nnz > 4 * 131072
    vt = (rng.random(lp.ncol) < 0.1).astype(np.int8)
    for trial in range(3):
        x = np.clip(rng.normal(size=lp.ncol) * 3, lp.collo, lp.colup) if trial else rng.normal(size=lp.ncol)
        x[rng.random(lp.ncol) < 0.3] = 0.0
        for tol in (1e-9, 10.0):
            b = ffi.ref_verify_full(lp, x, 1.0, tol, vartype=vt)
            for threads in (1, 3, 8):
                a = mps.verify_solution(lp, x, 1.0, tol, vartype=vt, col_names=[f"C{j}" for j in range(lp.ncol)],
                                        row_names=[f"R{i}" for i in range(lp.nrow)], threads=threads)
                for k in ("max_bound_viol", "max_row_viol", "max_int_viol", "computed_obj", "obj_rel_err"):
                    assert _bits(a[k]) == _bits(b[k]), (trial, tol, threads, k)
                assert a["passed"] == b["passed"] and a["worst_item"] == b["worst_item"], (trial, threads)
    # every row the same violation: the first row is named, whichever range reports it
    m, per = 60000, 5
    rows = rng.permutation(np.repeat(np.arange(m), per)).astype(np.int32)
    n = m * per
    tie = L.LP(m, n, np.arange(n + 1, dtype=np.int64), rows, np.ones(n), np.zeros(n), np.zeros(n), np.ones(n),
               np.full(m, 1e6), np.full(m, np.inf), 0.0)
    x = np.full(n, 0.5)
    b = ffi.ref_verify_full(tie, x, 0.0, 1e-6)
    for threads in (1, 2, 8):
        a = mps.verify_solution(tie, x, 0.0, 1e-6, row_names=[f"R{i}" for i in range(m)], threads=threads)
        assert a["worst_item"] == b["worst_item"] == "Row lower bound on R0"
        assert _bits(a["max_row_viol"]) == _bits(b["max_row_viol"])
