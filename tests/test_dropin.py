"""The drop-in: the reference's own programs built with
nirnaya_b200/sov/pdhg_solver.hpp in place of src/gpu/pdhg_solver.hpp
(nirnaya_b200/sov/Makefile), so that Solver::solve, the CLI's
`--method pdhg` / `--set method=pdhg`, the sov.h C API and the ctypes SDK
reach the B200 engine.

The binaries are built from the reference's sources where they are present
and travel prebuilt; the tests skip when they were not built.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import golden_io as G
from conftest import ROOT, has_gpu

DROPIN = os.path.join(ROOT, "nirnaya_b200", "sov", "_dropin")
GOLD = G.load()


def _need(name):
    path = os.path.join(DROPIN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (needs the reference sources: make -C nirnaya_b200/sov)")
    return path


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure mode")
def test_dropin_fails_loudly_without_gpu():
    exe = _need("unit_tests")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "no CUDA device" in (r.stdout + r.stderr)


def test_dropin_links_the_engine():
    exe = _need("unit_tests")
    out = subprocess.run(["readelf", "-d", exe], capture_output=True, text=True).stdout
    assert "libnir_pdhg.so" in out


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_reference_unit_tests_pass_on_the_gpu_engine():
    # tests/unit_tests.cpp: 12 tests, GPU/PDHG-01 asserts status Optimal and
    # objective 9 +- 1e-2 (:316-331); the other 11 must stay green
    r = subprocess.run([_need("unit_tests")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "12 / 12 tests passed" in r.stdout
    assert "[PASS] GPU/PDHG-01" in r.stdout


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_reference_bench_runner_pdhg_row():
    # tools/bench_runner.cpp:61-66,79-81: PDHG on Degenerate_Transport_LP
    r = subprocess.run([_need("bench_runner")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    row = [ln for ln in r.stdout.splitlines() if "PDHG (GPU)" in ln]
    assert row, r.stdout
    f = [t.strip() for t in row[0].split("|")]
    assert abs(float(f[2]) - 13.0) <= 1e-5 and f[5] == "PASS"


def _sov(lib_path):
    lib = C.CDLL(lib_path)
    lib.sov_env_create.restype = C.c_void_p
    lib.sov_model_create.restype = C.c_void_p
    lib.sov_model_create.argtypes = [C.c_void_p, C.c_char_p]
    lib.sov_add_col.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_char_p]
    lib.sov_add_row.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_int),
                                C.POINTER(C.c_double), C.c_char_p]
    lib.sov_set_sense.argtypes = [C.c_void_p, C.c_int]
    lib.sov_set_option_string.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
    lib.sov_optimize.argtypes = [C.c_void_p]
    lib.sov_get_status.argtypes = [C.c_void_p]
    lib.sov_get_obj.argtypes = [C.c_void_p]
    lib.sov_get_obj.restype = C.c_double
    lib.sov_get_x.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.sov_write_mps.argtypes = [C.c_void_p, C.c_char_p]
    lib.sov_error_message.argtypes = [C.c_void_p]
    lib.sov_error_message.restype = C.c_char_p
    lib.sov_model_free.argtypes = [C.c_void_p]
    lib.sov_env_free.argtypes = [C.c_void_p]
    return lib


def _build_model(lib, m, lp, sense):
    """Adds an internal-minimisation LP to a sov model in the user's sense."""
    sign = -1.0 if sense < 0 else 1.0
    for j in range(lp.ncol):
        lib.sov_add_col(m, sign * lp.cost[j], lp.collo[j], lp.colup[j], 0, f"x{j}".encode())
    rows = [[] for _ in range(lp.nrow)]
    for j in range(lp.ncol):
        for k in range(lp.col_start[j], lp.col_start[j + 1]):
            rows[lp.row_index[k]].append((j, lp.value[k]))
    for i, r in enumerate(rows):
        idx = (C.c_int * len(r))(*[a for a, _ in r])
        val = (C.c_double * len(r))(*[b for _, b in r])
        lib.sov_add_row(m, lp.rowlo[i], lp.rowup[i], len(r), idx, val, f"r{i}".encode())
    lib.sov_set_sense(m, sense)


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_c_api_and_ctypes_sdk_reach_the_engine():
    # the binding python/nirnaya.py makes (its :32-62), against the drop-in libsov.so
    lib = _sov(_need("libsov.so"))
    env = lib.sov_env_create()
    m = lib.sov_model_create(env, b"pdhg_lp")
    lib.sov_set_option_string(m, b"log_level", b"0")
    g = GOLD["unit_test_pdhg_lp"]
    _build_model(lib, m, G.lp_from(g["lp"]), 1)
    assert lib.sov_set_option_string(m, b"method", b"pdhg") == 0
    assert lib.sov_optimize(m) == 0, lib.sov_error_message(m)
    assert lib.sov_get_status(m) == 0
    assert abs(lib.sov_get_obj(m) - 9.0) <= 1e-4
    x = (C.c_double * 2)()
    lib.sov_get_x(m, x)
    assert abs(x[0] - 3.0) <= 1e-3 and abs(x[1] - 1.0) <= 1e-3
    lib.sov_model_free(m)
    lib.sov_env_free(env)


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
@pytest.mark.parametrize("args", [["--method", "pdhg"], ["--method=pdhg"], ["--method=gpu"], ["--set", "method=pdhg"],
                                  ["--set", "method=gpu"]])
def test_cli_method_pdhg_on_crude_blending(tmp_path, args):
    # data/refinery/MRPL_Crude_Blending_LP: optimum 22171.59777424483 (.sol:2)
    g = GOLD["crude_blending"]
    lib = _sov(_need("libsov.so"))
    env = lib.sov_env_create()
    m = lib.sov_model_create(env, b"MRPL_Crude_Blending_LP")
    _build_model(lib, m, G.lp_from(g["lp_internal_min"]), g["sense"])
    path = str(tmp_path / "crude.mps")
    assert lib.sov_write_mps(m, path.encode()) == 0
    lib.sov_model_free(m)
    lib.sov_env_free(env)
    sol = str(tmp_path / "crude.sol")
    r = subprocess.run([_need("sovsolve"), path, *args, "--sol", sol], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PDHG" in r.stdout
    obj = float(re.search(r"Objective:\s+([-0-9.eE+]+)", r.stdout).group(1))
    assert abs(obj - g["sol_objective"]) / g["sol_objective"] <= 1e-6
    assert "PASS=YES" in r.stdout


# ---- the MPS reader drop-in (nirnaya_b200/sov/mps_reader.hpp): CPU only

# the reference checkout beside this repository, unless NIRNAYA_REF names another
REF_DIR = os.environ.get("NIRNAYA_REF") or os.path.join(ROOT, os.pardir, "reference")
REFINERY = os.path.join(REF_DIR, "data", "refinery")
REF_CHECKER = os.path.join(ROOT, "oracle", "_ref", "checker")


def _refinery(ext):
    if not os.path.isdir(REFINERY):
        return []
    return sorted(f[:-len(ext)] for f in os.listdir(REFINERY) if f.endswith(ext))


def test_dropin_links_the_mps_reader():
    for exe in ("sovsolve", "libsov.so", "checker"):
        out = subprocess.run(["readelf", "-d", _need(exe)], capture_output=True, text=True).stdout
        assert "libnir_mps.so" in out, exe


@pytest.mark.parametrize("model", [m for m in _refinery(".sol") if m in _refinery(".mps")])
def test_dropin_checker_matches_the_reference_checker(model):
    """tools/checker.cpp built twice: on the drop-in reader and as it is."""
    if not os.path.exists(REF_CHECKER):
        pytest.skip("the reference checker (oracle/_ref/checker) is absent")
    args = [os.path.join(REFINERY, model + ".mps"), os.path.join(REFINERY, model + ".sol")]
    ours = subprocess.run([_need("checker"), *args], capture_output=True, text=True, timeout=120)
    ref = subprocess.run([REF_CHECKER, *args], capture_output=True, text=True, timeout=120)
    assert (ours.returncode, ours.stdout) == (ref.returncode, ref.stdout)


def _c_api_roundtrip(lib, src, dst):
    lib.sov_read_mps.argtypes = [C.c_void_p, C.c_char_p]
    env = lib.sov_env_create()
    m = lib.sov_model_create(env, b"rt")
    try:
        assert lib.sov_read_mps(m, src.encode()) == 0, lib.sov_error_message(m)
        assert lib.sov_write_mps(m, dst.encode()) == 0
    finally:
        lib.sov_model_free(m)
        lib.sov_env_free(env)


def _roundtrip_cases(tmp_path):
    from mps_cases import CASES, random_mps

    from nirnaya_b200 import lp as L

    paths = [os.path.join(REFINERY, f + ".mps") for f in _refinery(".mps")]
    for name in ("basic", "ranges", "integers", "objname", "bound_rules", "quadobj", "layout"):
        p = tmp_path / (name + ".mps")
        with open(p, "w", newline="") as f:
            f.write(CASES[name])
        paths.append(str(p))
    p = tmp_path / "random.mps"
    with open(p, "w", newline="") as f:
        f.write(random_mps(L.generate(L.ZIPF, 3, m=3000, n=8000, target_nnz=60000), 3, sense=-1))
    paths.append(str(p))
    return paths


def test_dropin_c_api_read_then_write_is_the_reference_bytes(tmp_path):
    """sov_read_mps + sov_write_mps (src/driver/c_api.cpp:101-120) on the
    drop-in against MpsReader::read + MpsReader::write of the reference:
    the files written must be identical, names and all."""
    from oracle import ffi

    if not ffi.ref_available():
        pytest.skip("the reference build (oracle/_ref) is absent")
    lib = _sov(_need("libsov.so"))
    for src in _roundtrip_cases(tmp_path):
        ours, ref = str(tmp_path / "ours.mps"), str(tmp_path / "ref.mps")
        _c_api_roundtrip(lib, src, ours)
        assert ffi.ref_mps_roundtrip(src, ref) == 0, src
        with open(ours, "rb") as a, open(ref, "rb") as b:
            assert a.read() == b.read(), src


def test_dropin_cli_reports_a_bad_number_as_an_input_error(tmp_path):
    # the reference's reader throws from std::stod here; the drop-in returns
    # InputError, which the CLI reports (src/driver/cli_main.cpp:89-93)
    p = tmp_path / "bad.mps"
    p.write_text("NAME B\nROWS\n N o\n L r\nCOLUMNS\n x o 1 r 1\n y o abc r 1\nENDATA\n")
    r = subprocess.run([_need("sovsolve"), str(p)], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "Input Error reading" in r.stderr and "invalid number 'abc' at line 7" in r.stderr


# ---- presolve and scaling drop-ins (presolve.hpp, scaling.hpp): the whole
# CLI path on the CPU methods, against the reference's own CLI

REF_SOVSOLVE = os.path.join(ROOT, "oracle", "_ref", "sovsolve")


def _cli_pair(tmp_path, model, args):
    if not os.path.exists(REF_SOVSOLVE):
        pytest.skip("the reference CLI (oracle/_ref/sovsolve) is absent")
    outs = []
    for tag, exe in (("ref", REF_SOVSOLVE), ("ours", _need("sovsolve"))):
        sol = str(tmp_path / f"{tag}.sol")
        r = subprocess.run([exe, model, *args, "--sol", sol], capture_output=True, text=True, timeout=300)
        text = "\n".join(ln for ln in r.stdout.splitlines() if "Time:" not in ln)
        body = open(sol).read() if os.path.exists(sol) else None
        outs.append((r.returncode, text, body))
    return outs


def test_dropin_links_presolve_and_scaling():
    out = subprocess.run(["readelf", "-d", _need("sovsolve")], capture_output=True, text=True).stdout
    assert "libnir_facade.so" in out


@pytest.mark.parametrize("model", _refinery(".mps"))
@pytest.mark.parametrize("method", ["dual", "ipm"])
def test_dropin_cli_cpu_methods_match_the_reference_cli(tmp_path, model, method):
    """sovsolve --method dual|ipm: read, presolve, scale, solve, verify and
    the .sol all equal the reference CLI's (only timings differ)."""
    ours, ref = _cli_pair(tmp_path, os.path.join(REFINERY, model + ".mps"), ["--method", method])[::-1]
    assert ours == ref


@pytest.mark.parametrize("method", ["dual", "ipm"])
def test_dropin_cli_accepts_the_method_equals_form(tmp_path, method):
    """`--method=<m>` (the reference's README.md:27) selects the method as `--method <m>`
    does; the reference's own loop drops that form (cli_main.cpp:77)."""
    model = os.path.join(REFINERY, "MRPL_Crude_Blending_LP.mps")
    if not os.path.exists(model):
        pytest.skip("the reference's refinery models are absent")
    ref = _cli_pair(tmp_path, model, ["--method", method])[0]
    exe = _need("sovsolve")
    sol = str(tmp_path / "eq.sol")
    r = subprocess.run([exe, model, f"--method={method}", f"--sol={sol}"], capture_output=True, text=True, timeout=300)
    text = "\n".join(ln for ln in r.stdout.splitlines() if "Time:" not in ln)
    assert (r.returncode, text, open(sol).read()) == ref


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure mode")
@pytest.mark.parametrize("form", [["--method=pdhg"], ["--method", "pdhg"], ["--method=gpu"]])
def test_dropin_cli_method_pdhg_form_reaches_the_engine(tmp_path, form):
    """Every spelling of the PDHG method reaches the GPU engine, which
    without a device fails loudly instead of falling back to the CPU."""
    model = os.path.join(REFINERY, "MRPL_Crude_Blending_LP.mps")
    if not os.path.exists(model):
        pytest.skip("the reference's refinery models are absent")
    r = subprocess.run([_need("sovsolve"), model, *form], capture_output=True, text=True, timeout=300)
    out = r.stdout + r.stderr
    assert "no CUDA device" in out, out
    assert "Simplex" not in out, out


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_dropin_cli_presolve_heavy_models_match(tmp_path, seed):
    from test_facade import rich_instance

    from nirnaya_b200 import mps

    lp, vt = rich_instance(seed, m=150, n=300, int_frac=0.0)
    # every column gets an objective entry: MpsReader::write leaves a column
    # with neither cost nor entries out of COLUMNS, and its bound line then
    # names an unknown column
    lp.cost[lp.cost == 0.0] = 0.5
    path = str(tmp_path / "rich.mps")
    mps.write_mps(path, lp, name=f"rich{seed}")
    ref, ours = _cli_pair(tmp_path, path, ["--method", "dual"])
    assert ours == ref
    assert "Presolve:" in ours[1] or "infeasible" in ours[1] or "unbounded" in ours[1]


def _harness(tmp_path, source, oracle=False, args=(), timeout=300):
    """Builds tests/native/<source> against a tree of the reference's headers
    with the five drop-in headers linked in; the engine entry point is the
    harness's own stand-in, so no GPU is needed."""
    if not os.path.isdir(os.path.join(REF_DIR, "include", "sov")):
        pytest.skip("the reference sources are absent")
    tree = tmp_path / "tree"
    for sub in ("include", "src"):
        for dirpath, _, files in os.walk(os.path.join(REF_DIR, sub)):
            rel = os.path.relpath(dirpath, REF_DIR)
            os.makedirs(tree / rel, exist_ok=True)
            for f in files:
                if f.endswith((".hpp", ".h")):
                    os.symlink(os.path.join(dirpath, f), tree / rel / f)
    sov = os.path.join(ROOT, "nirnaya_b200", "sov")
    for name, where in (("pdhg_solver.hpp", "src/gpu"), ("scaling.hpp", "src/model"), ("presolve.hpp", "src/presolve"),
                        ("mps_reader.hpp", "src/io"), ("sol_io.hpp", "src/io")):
        os.remove(tree / where / name)
        os.symlink(os.path.join(sov, name), tree / where / name)
    exe = tmp_path / "harness"
    orc = os.path.join(ROOT, "oracle")
    extra = [f"-I{orc}", f"-L{orc}", "-loracle", "-lnir_lpgen", f"-Wl,-rpath,{orc}"] if oracle else []
    subprocess.run(["g++", "-std=c++17", "-O2", "-fno-fast-math", f"-I{tree}", f"-I{os.path.join(ROOT, 'include')}",
                    os.path.join(ROOT, "tests", "native", source), "-o", str(exe),
                    f"-L{os.path.join(ROOT, 'nirnaya_b200')}", "-lnir_mps", "-lnir_facade",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'nirnaya_b200')}", *extra, "-lpthread"], check=True)
    return subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=timeout)


def test_dropin_pdhg_undoes_scale_model_exactly(tmp_path):
    """The drop-in PdhgSolver hands the engine the model before scale_model
    (bit for bit) and maps the returned point back exactly; checked with a
    stand-in for the engine entry point (tests/native/
    pdhg_dropin_scaling_harness.cpp), so no GPU is needed."""
    r = _harness(tmp_path, "pdhg_dropin_scaling_harness.cpp")
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_dropin_pdhg_retries_in_fp64_when_only_the_row_margin_is_missing(tmp_path):
    """A solve that meets the relative KKT but not the row margin at its cap
    goes on once in FP64 on the GPU from the point it reached (the retry
    Solver's presolve-less fallback would otherwise make from scratch,
    include/sov/solver.hpp:283-296); checked with a scripted stand-in for the
    engine entry point (tests/native/pdhg_dropin_retry_harness.cpp)."""
    r = _harness(tmp_path, "pdhg_dropin_retry_harness.cpp")
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_dropin_crossover_reaches_the_simplex_optimum(tmp_path):
    """NIR_PDHG_CROSSOVER: from an approximate optimum (the simplex's,
    perturbed by 1e-8, 1e-6 and 1e-3 relative), a real PDHG iterate (the
    reference loop in the oracle) or an interior point of an optimal face,
    the drop-in's crossover reaches the simplex's optimal
    objective with a passing dd check, in a small fraction of the simplex's
    own pivots.  Checked on the
    reference's worked example (x = (3, 1), duals (1.5, 0.5)), its PDHG and
    transport LPs and seeded random LPs.  It runs through Solver with
    presolve and scaling on and off, and `auto` runs only after an engine
    result short of Optimal (tests/native/pdhg_dropin_crossover_harness.cpp)."""
    r = _harness(tmp_path, "pdhg_dropin_crossover_harness.cpp", oracle=True)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith(("random_", "transport"))]
    assert len(lines) == 5
    for ln in lines:  # near an optimum the crash basis leaves (almost) nothing to pivot
        scratch = int(ln.split("simplex from slacks ")[1].split()[0])
        pivots = [int(ln.split("crossover ")[1].split()[0]), int(ln.split("), ")[1].split()[0])]
        assert max(pivots) <= scratch // 8, ln
    far = next(ln for ln in r.stdout.splitlines() if ln.startswith("far:"))
    assert int(far.split("off: ")[1].split()[0]) <= int(far.split("from slacks ")[1].rstrip(")")) // 8, far
    # from real PDHG iterates (the reference loop, restated in the oracle)
    its = [ln for ln in r.stdout.splitlines() if ln.startswith("pdhg_iterate_")]
    assert len(its) == 3
    for ln in its:
        pivots = int(ln.split("crossover ")[1].split()[0])
        assert pivots <= int(ln.split("from slacks ")[1].rstrip(")")) // 8, ln


def test_dropin_crossover_on_the_refinery_models(tmp_path):
    """The reference's data/refinery models as LPs (integrality dropped, the
    QPs skipped): crossover from each simplex optimum perturbed by 1e-6
    reaches that optimum with a passing dd check, in no more pivots than
    the simplex from slacks."""
    if not os.path.isdir(REFINERY):
        pytest.skip("the reference's refinery models are absent")
    files = sorted(os.path.join(REFINERY, f) for f in os.listdir(REFINERY) if f.endswith(".mps"))
    r = _harness(tmp_path, "pdhg_dropin_crossover_harness.cpp", oracle=True, args=["mps", *files])
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("MRPL_")]
    assert len(lines) >= 4
    for ln in lines:
        scratch = int(ln.split("simplex from slacks ")[1].split()[0])
        assert int(ln.rsplit("crossover ", 1)[1]) <= scratch, ln


@pytest.mark.skipif(os.environ.get("NIR_MEASURE_CROSSOVER") != "1",
                    reason="a measurement of several minutes: set NIR_MEASURE_CROSSOVER=1")
@pytest.mark.parametrize("model", [("measure", "3", "12", "600"), ("c1",)])
def test_crossover_measurement(tmp_path, model):
    """Crossover timings on CPU (printed; run with -s): the reference loop
    (oracle) for its own cap and six times that, then crossover from each
    point with the primal and the dual finish, against the simplex from its
    slack basis.  A multiperiod model (600 rows) and C1."""
    r = _harness(tmp_path, "pdhg_dropin_crossover_harness.cpp", oracle=True, args=model, timeout=3600)
    print(r.stdout)
    if model[0] == "measure":
        assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
@pytest.mark.parametrize("presolve,scale", [("0", "0"), ("2", "1")])
def test_c_api_pdhg_scaling_and_presolve_equivalence(presolve, scale):
    """tests/unit_tests.cpp:177-203's badly scaled LP (coefficients over three
    decades, a fixed column, a singleton row) with method=pdhg, with and
    without presolve and scaling: the same optimum, 29.5 (x = (6500, 4, 3)),
    and a passing double-double check.  With scaling on, the drop-in undoes
    scale_model's scales before the engine and maps the point back."""
    lib = _sov(_need("libsov.so"))
    lib.sov_get_status.restype = C.c_int
    env = lib.sov_env_create()
    m = lib.sov_model_create(env, b"Badly_Scaled_LP")
    for k, v in (("log_level", "0"), ("method", "pdhg"), ("presolve", presolve), ("scale", scale)):
        lib.sov_set_option_string(m, k.encode(), v.encode())
    for cost, lo, up in ((1e-3, 0.0, 1e4), (2.0, 0.0, 100.0), (5.0, 3.0, 3.0)):
        lib.sov_add_col(m, cost, lo, up, 0, None)
    for lo, cols, vals in ((10.0, [0, 1], [1e-3, 1.0]), (20.0, [0, 1, 2], [2e-3, 1.0, 1.0]), (4.0, [1], [1.0])):
        idx = (C.c_int * len(cols))(*cols)
        val = (C.c_double * len(vals))(*vals)
        lib.sov_add_row(m, lo, 1e20, len(cols), idx, val, None)
    try:
        assert lib.sov_optimize(m) == 0, lib.sov_error_message(m)
        assert lib.sov_get_status(m) == 0
        assert abs(lib.sov_get_obj(m) - 29.5) <= 1e-5 * 29.5
        x = (C.c_double * 3)()
        lib.sov_get_x(m, x)
        assert abs(x[0] - 6500.0) <= 1e-2 and abs(x[1] - 4.0) <= 1e-5 and x[2] == 3.0
    finally:
        lib.sov_model_free(m)
        lib.sov_env_free(env)


@pytest.mark.parametrize("objective_line", ["# objective 42.5", "# objective abc", "# objective 1e400"])
def test_dropin_checker_on_odd_sol_files_matches_the_reference(tmp_path, objective_line):
    """tools/checker.cpp on the drop-in SOL reader against the reference's:
    the same report on a file of odd value tokens, and the same failure
    when std::stod rejects the objective (the exception leaves main)."""
    if not os.path.exists(REF_CHECKER):
        pytest.skip("the reference checker (oracle/_ref/checker) is absent")
    from test_sol import SOL_LINES

    from nirnaya_b200 import lp as L
    from nirnaya_b200 import mps

    lp = L.generate(1, 0, m=5, n=30)
    lp.cost[lp.cost == 0.0] = 1.0
    model, sol = str(tmp_path / "m.mps"), str(tmp_path / "x.sol")
    mps.write_mps(model, lp, name="solmodel", col_names=[f"C{j}" for j in range(30)])
    lines = [ln for ln in SOL_LINES if "objective" not in ln] + [objective_line]
    with open(sol, "w", newline="") as f:
        f.write("\n".join(lines) + "\n")
    ours = subprocess.run([_need("checker"), model, sol], capture_output=True, text=True, timeout=120)
    ref = subprocess.run([REF_CHECKER, model, sol], capture_output=True, text=True, timeout=120)
    assert (ours.returncode, ours.stdout) == (ref.returncode, ref.stdout)
    if "abc" in objective_line or "1e400" in objective_line:
        assert ref.returncode != 0 and ("stod" in ref.stderr) == ("stod" in ours.stderr)
