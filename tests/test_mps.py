"""The multi-threaded MPS reader (libnir_mps.so) against the reference's.

CPU only.  Parity is bit-for-bit on every array:
  * against tests/golden/mps_golden.json, recorded from the reference's own
    sov::MpsReader::read + Model::to_internal_min (src/io/mps_reader.hpp:
    15-304, src/model/model.hpp:101-178) by tests/golden/make_mps_golden.py;
  * against the reference compiled here (oracle/_ref), live, on the same
    cases, on seeded random layouts at several thread counts and on the
    reference's refinery models -- skipped where the reference is absent.
Where the reference lets std::stod's exception escape (status -1 in the
fixtures), this reader returns input error 12 with the line number.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from mps_cases import CASES, random_mps

GOLDEN = os.path.join(ROOT, "tests", "golden", "mps_golden.json")
# the reference checkout beside this repository, unless NIRNAYA_REF names another
REFINERY = os.path.join(os.environ.get("NIRNAYA_REF") or os.path.join(ROOT, os.pardir, "reference"), "data", "refinery")
KEYS = ("col_start", "row_index", "value", "cost", "collo", "colup", "rowlo", "rowup")


def _unhex(a):
    return np.array([float.fromhex(v) for v in a], dtype=np.float64)


def _write(tmp_path, name, text):
    p = tmp_path / (name + ".mps")
    with open(p, "w", newline="") as f:
        f.write(text)
    return str(p)


def _ours(path, threads=0):
    from nirnaya_b200 import mps

    try:
        m = mps.read_mps(path, threads=threads)
    except mps.MpsError as e:
        return {"status": e.status, "message": e.message}
    lp, qv = m.internal_min()
    return {"status": 0, "sense": m.sense, "lp": lp, "vartype": m.vartype, "q": (m.q_start, m.q_index, qv)}


def _same_bits(a, b):
    a, b = np.atleast_1d(np.asarray(a)), np.atleast_1d(np.asarray(b))
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def _check_against_golden(got, rec, name):
    if rec["status"] != 0:
        want = 12 if rec["status"] == -1 else rec["status"]
        assert got["status"] == want, (name, got, rec)
        if rec["status"] != -1:
            assert got["message"] == rec["message"], name
        return
    assert got["status"] == 0, (name, got)
    lp = got["lp"]
    assert got["sense"] == rec["sense"] and lp.nrow == rec["nrow"] and lp.ncol == rec["ncol"], name
    assert np.array_equal(lp.col_start, np.array(rec["col_start"], np.int64)), name
    assert np.array_equal(lp.row_index, np.array(rec["row_index"], np.int32)), name
    for k in ("value", "cost", "collo", "colup", "rowlo", "rowup"):
        assert _same_bits(getattr(lp, k), _unhex(rec[k])), (name, k)
    assert _same_bits(np.float64(lp.obj_offset), np.float64(float.fromhex(rec["obj_offset"]))), name
    assert np.array_equal(got["vartype"], np.array(rec["vartype"], np.int8)), name
    qs, qi, qv = got["q"]
    assert np.array_equal(qs, np.array(rec["q_start"], np.int64)), name
    assert np.array_equal(qi, np.array(rec["q_index"], np.int32)), name
    assert _same_bits(qv, _unhex(rec["q_value"])), name


def _check_against_reference(got, path, name):
    from oracle import ffi

    try:
        lp, sense, vt, (qs, qi, qv) = ffi.ref_read_mps_full(path)
    except ffi.RefMpsError as e:
        want = 12 if e.status == -1 else e.status
        assert got["status"] == want, (name, got, e)
        if e.status != -1:
            assert got["message"] == e.message, name
        return
    assert got["status"] == 0, (name, got)
    ours = got["lp"]
    assert got["sense"] == sense and ours.nrow == lp.nrow and ours.ncol == lp.ncol, name
    for k in KEYS:
        assert _same_bits(getattr(ours, k), getattr(lp, k)), (name, k)
    assert _same_bits(np.float64(ours.obj_offset), np.float64(lp.obj_offset)), name
    assert np.array_equal(got["vartype"], vt), name
    assert np.array_equal(got["q"][0], qs) and np.array_equal(got["q"][1], qi), name
    assert _same_bits(got["q"][2], qv), name


def _ref_available():
    from oracle import ffi

    return ffi.ref_available()


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def test_reader_exports_every_declared_symbol():
    import ctypes as C

    from test_abi import declared

    from nirnaya_b200 import mps

    lib = C.CDLL(os.path.join(ROOT, "nirnaya_b200", "libnir_mps.so"))
    names = declared("nir_mps.h")
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(mps.EXPORTED) == names


def test_golden_covers_every_case(golden):
    assert sorted(golden["cases"]) == sorted(CASES)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("threads", [1, 4])
def test_cases_match_the_reference_golden(tmp_path, golden, name, threads):
    path = _write(tmp_path, name, CASES[name])
    _check_against_golden(_ours(path, threads), golden["cases"][name], name)


def test_random_layouts_match_the_reference_golden(tmp_path, golden):
    from nirnaya_b200 import lp as L

    for rec in golden["random"]:
        lp = L.generate(rec["kind"], rec["seed"], **rec["kw"])
        path = _write(tmp_path, "random", random_mps(lp, rec["seed"], sense=rec["sense"]))
        for threads in (1, 3):
            _check_against_golden(_ours(path, threads), rec["result"], f"random kind {rec['kind']}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_cases_match_the_reference_live(tmp_path, name):
    if not _ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    path = _write(tmp_path, name, CASES[name])
    _check_against_reference(_ours(path, 2), path, name)


@pytest.mark.parametrize("kind,seed,kw,sense", [
    (1, 3, dict(m=300, n=800), 1),
    (2, 4, dict(m=3000, n=8000, target_nnz=60000), -1),
    (3, 5, dict(), 1),
    (4, 6, dict(), 1),
])
def test_random_layouts_match_the_reference_live(tmp_path, kind, seed, kw, sense):
    if not _ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    from nirnaya_b200 import lp as L

    lp = L.generate(kind, seed, **kw)
    path = _write(tmp_path, "random", random_mps(lp, seed, sense=sense))
    for threads in (1, 2, 8):
        _check_against_reference(_ours(path, threads), path, f"kind {kind} threads {threads}")


def test_files_written_by_the_reference_writer(tmp_path):
    """MpsReader::write's layout (src/io/mps_reader.hpp:306-412), read back."""
    if not _ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    from nirnaya_b200 import lp as L
    from oracle import ffi

    lp = L.generate(L.ZIPF, 7, m=5000, n=12000, target_nnz=100000)
    vt = (np.arange(lp.ncol) % 7 == 0).astype(np.int8)
    path = str(tmp_path / "written.mps")
    ffi.ref_write_mps(lp, path, vartype=vt, sense=-1)
    for threads in (1, 8):
        _check_against_reference(_ours(path, threads), path, f"written threads {threads}")


@pytest.mark.parametrize("name", sorted(f for f in os.listdir(REFINERY) if f.endswith(".mps"))
                         if os.path.isdir(REFINERY) else [])
def test_refinery_models(name):
    if not _ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    path = os.path.join(REFINERY, name)
    _check_against_reference(_ours(path, 3), path, name)


def test_thread_count_does_not_change_the_model(tmp_path):
    from nirnaya_b200 import lp as L

    lp = L.generate(L.ZIPF, 11, m=20000, n=50000, target_nnz=400000)
    path = _write(tmp_path, "big", random_mps(lp, 11))
    base = _ours(path, 1)
    assert base["status"] == 0
    for threads in (2, 5, 8, 16):
        got = _ours(path, threads)
        for k in KEYS:
            assert _same_bits(getattr(got["lp"], k), getattr(base["lp"], k)), (threads, k)
        assert np.array_equal(got["vartype"], base["vartype"])
    # and the LP itself came through: same nonzeros, same costs
    assert base["lp"].nnz == lp.nnz
    assert _same_bits(np.sort(base["lp"].value), np.sort(lp.value))


def test_missing_file_is_an_input_error(tmp_path):
    from nirnaya_b200 import mps

    with pytest.raises(mps.MpsError) as e:
        mps.read_mps(str(tmp_path / "nope.mps"))
    assert e.value.status == 12 and "Cannot open MPS file" in e.value.message


def test_errors_name_the_line(tmp_path):
    from nirnaya_b200 import mps

    text = "NAME X\nROWS\n N o\n L r\nCOLUMNS\n" + "".join(f" c{j} o 1 r 1\n" for j in range(5000)) + \
        " bad o 1 r 1x2e\n" + "".join(f" d{j} o 1 r 1\n" for j in range(5000)) + "ENDATA\n"
    path = _write(tmp_path, "bad", text.replace("1x2e", "x2e"))
    with pytest.raises(mps.MpsError) as e:
        mps.read_mps(path, threads=4)
    assert e.value.status == 12 and e.value.message == "invalid number 'x2e' at line 5006"


def test_decimal_conversion_matches_strtod(tmp_path):
    """The fast decimal conversion (nirnaya_b200/csrc/decimal.hpp) against
    strtod on random 17-digit renderings, digit strings with exponents
    across the whole range, exact ties and midpoints."""
    exe = tmp_path / "decimal_harness"
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "native", "decimal_harness.cpp"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), "1500000", "7"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    checked, accepted = int(out.stdout.split()[1]), int(out.stdout.split()[3])
    assert "mismatches 0" in out.stdout and accepted > 0.9 * checked, out.stdout


def test_directory_reads_as_an_empty_model(tmp_path):
    # std::ifstream opens a directory and getline yields nothing: an empty,
    # valid model (status 0), which the reference reader returns too
    from nirnaya_b200 import mps

    m = mps.read_mps(str(tmp_path))
    assert (m.lp.nrow, m.lp.ncol, m.lp.nnz, m.sense) == (0, 0, 0, 1)
    if _ref_available():
        _check_against_reference(_ours(str(tmp_path)), str(tmp_path), "directory")


def test_a_pipe_is_read_as_a_stream(tmp_path):
    import sys

    code = ("import sys; sys.path.insert(0, %r); from nirnaya_b200 import mps; m = mps.read_mps('/dev/stdin'); "
            "print(m.lp.nrow, m.lp.ncol, m.lp.nnz, repr(m.lp.cost.tolist()))" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], input=CASES["basic"], capture_output=True, text=True,
                         timeout=120)
    path = _write(tmp_path, "basic", CASES["basic"])
    from nirnaya_b200 import mps

    m = mps.read_mps(path)
    assert out.stdout.strip() == f"{m.lp.nrow} {m.lp.ncol} {m.lp.nnz} {m.lp.cost.tolist()!r}", out.stderr


def test_random_files_match_the_reference_live(tmp_path):
    """Differential fuzzing: 400 seeded random files (mps_cases.fuzz_mps),
    each read at 1-4 threads, against the reference reader.  Valid models,
    every error message and every status must agree."""
    if not _ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    from mps_cases import fuzz_mps

    outcomes = set()
    for seed in range(400):
        rng = np.random.default_rng([0xF22, seed])
        path = _write(tmp_path, "fuzz", fuzz_mps(rng))
        got = _ours(path, int(rng.integers(1, 5)))
        outcomes.add(got["status"] if got["status"] else ("ok", got["lp"].nnz > 0))
        _check_against_reference(got, path, f"fuzz seed {seed}")
    assert {("ok", True), 1, 12} <= outcomes


@pytest.mark.parametrize("seed", range(12))
def test_writer_bytes_match_the_reference_writer(tmp_path, seed):
    """nir_mps_write against MpsReader::write (src/io/mps_reader.hpp:306-412)
    on models with every bound shape (free, fixed, one-sided, boxed, binary,
    infinite and 1e20 bounds), integer runs, ranged and free rows, offsets
    and both senses."""
    if not _ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    from test_facade import rich_instance

    from nirnaya_b200 import mps
    from oracle import ffi

    rng = np.random.default_rng([0x3B1, seed])
    lp, vt = rich_instance(seed, m=int(rng.integers(5, 200)), n=int(rng.integers(5, 400)), int_frac=0.4)
    vt[(vt == 1) & (rng.random(lp.ncol) < 0.5)] = 2  # some binaries
    lp.collo[rng.random(lp.ncol) < 0.05] = 1e20
    lp.colup[rng.random(lp.ncol) < 0.05] = -1e30
    lp.rowlo[rng.random(lp.nrow) < 0.05] = -np.inf
    lp.obj_offset = float(rng.choice([0.0, 1.25, -3e-7]))
    sense = int(rng.choice([1, -1]))
    ours, ref = str(tmp_path / "o.mps"), str(tmp_path / "r.mps")
    mps.write_mps(ours, lp, vartype=vt, sense=sense, name="written", threads=int(rng.integers(1, 5)))
    ffi.ref_write_mps(lp, ref, vartype=vt, sense=sense)
    with open(ours, "rb") as a, open(ref, "rb") as b:
        assert a.read() == b.read()
