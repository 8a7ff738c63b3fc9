"""The C-ABI libraries load and export every symbol their headers declare.

CPU only: no compute call is made here, except nir_pdhg_create on a
machine without a GPU, which must fail loudly (no CPU fallback).
"""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT, has_gpu

INCLUDE = os.path.join(ROOT, "include")


def declared(header):
    text = open(os.path.join(INCLUDE, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nir_[a-z0-9_]+)\s*\(", text)))


def test_engine_exports_every_declared_symbol():
    path = os.path.join(ROOT, "nirnaya_b200", "libnir_pdhg.so")
    if not os.path.exists(path):
        pytest.skip("libnir_pdhg.so not built (run __graft_entry__.build())")
    lib = C.CDLL(path)
    names = declared("nir_pdhg.h")
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
    from nirnaya_b200 import pdhg

    assert sorted(pdhg.EXPORTED) == sorted(n for n in names)


def test_lpgen_exports_every_declared_symbol():
    lib = C.CDLL(os.path.join(ROOT, "nirnaya_b200", "libnir_lpgen.so"))
    for name in declared("nir_lpgen.h"):
        assert hasattr(lib, name), name


def test_structs_match_header_sizes():
    from nirnaya_b200 import pdhg
    from nirnaya_b200.lp import NirLpView

    assert C.sizeof(NirLpView) == 4 + 4 + 8 + 8 * 8 + 8
    # nir_pdhg_params: 2 int32, 2 double, int64, double, 3 int32, 5 double,
    # double, 2 int32, double, 5 int32 (+pad), 2 pointers, 2 double
    assert C.sizeof(pdhg.Params) == 184
    assert C.sizeof(pdhg.Info) == 4 + 4 + 8 + 8 + 8 * 11 + 4 + 4 + 8


def test_ctypes_layouts_match_the_c_compiler(tmp_path):
    """sizeof and field offsets of every struct in include/*.h as gcc sees
    them, against the ctypes mirrors."""
    import subprocess

    from nirnaya_b200 import pdhg
    from nirnaya_b200.lp import NirLpView

    mirrors = {"nir_pdhg_params": pdhg.Params, "nir_pdhg_info": pdhg.Info, "nir_pdhg_kernel_time": pdhg.KernelTime,
               "nir_pdhg_layout": pdhg.Layout, "nir_lp_view": NirLpView}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "nir_pdhg.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in mirrors.items():
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure mode")
def test_create_without_gpu_fails_loudly():
    from nirnaya_b200 import lp as L
    from nirnaya_b200 import pdhg

    if not os.path.exists(pdhg.LIB_PATH):
        pytest.skip("libnir_pdhg.so not built")
    lp = L.generate(L.RANDOM_EQ, 1, m=20, n=50)
    with pytest.raises(RuntimeError, match="CUDA|device"):
        pdhg.Engine(lp)


def test_params_defaults_roundtrip():
    from nirnaya_b200 import pdhg

    if not os.path.exists(pdhg.LIB_PATH):
        pytest.skip("libnir_pdhg.so not built")
    p = pdhg.default_params()
    assert p.algorithm == pdhg.ALGO_PDLP and p.precision == pdhg.PREC_MIXED and p.tol == 1e-6
    assert p.check_every == 64 and p.reflection == 1.0 and p.use_graphs == 1


def test_python_solver_mirror_uses_the_dropin_iteration_cap():
    # as nirnaya_b200/sov/pdhg_solver.hpp: the reference's cap
    # max(5000, simplex_iter_limit / 10) for its own loop, ten times that
    # for the restarted methods, whose iterations replace many plain ones
    from nirnaya_b200 import pdhg

    p = pdhg.PdhgSolver.params_from(pdhg.Options(simplex_iter_limit=500000))
    assert p.max_iters == 500000 and p.algorithm == pdhg.ALGO_PDLP
    p = pdhg.PdhgSolver.params_from(pdhg.Options(simplex_iter_limit=1000, pdhg_algorithm=pdhg.ALGO_REFERENCE))
    assert p.max_iters == 5000
    p = pdhg.PdhgSolver.params_from(pdhg.Options(pdhg_max_iters=123, extra={"check_every": 32}))
    assert p.max_iters == 123 and p.check_every == 32


def test_verify_entry_points_reject_bad_arguments_before_any_device_call():
    """nir_pdhg_verify / nir_pdhg_batch_verify check their arguments on the
    host: a null handle or report is an input error with a message."""
    import ctypes as C

    from nirnaya_b200 import batch as B
    from nirnaya_b200 import mps
    from nirnaya_b200 import pdhg

    if not os.path.exists(pdhg.LIB_PATH):
        pytest.skip("libnir_pdhg.so not built")
    lib = B._lib()
    rep = mps.VerifyReport()
    assert lib.nir_pdhg_verify(None, None, None, 0.0, 1e-6, C.byref(rep)) == pdhg.INPUT_ERROR
    assert pdhg.last_error() == "null handle"
    assert lib.nir_pdhg_batch_verify(None, None, None, None, 1e-6, C.byref(rep)) == pdhg.INPUT_ERROR
    assert pdhg.last_error() == "null handle"
    assert lib.nir_pdhg_batch_verify(None, None, None, None, 1e-6, None) == pdhg.INPUT_ERROR
    assert pdhg.last_error() == "null report"


def test_a_start_is_a_device_address_as_is_or_a_kept_host_copy():
    # Engine.solve hands x_init / y_init to nir_pdhg_solve: an int is a device
    # address passed through unchanged; anything else becomes a contiguous
    # FP64 host copy that lives as long as the call's keep list
    import numpy as np

    from nirnaya_b200 import pdhg

    keep = []
    p = pdhg._start_ptr(0x7F0012345600, keep)
    assert C.cast(p, C.c_void_p).value == 0x7F0012345600 and keep == []
    p = pdhg._start_ptr(np.int64(4096), keep)
    assert C.cast(p, C.c_void_p).value == 4096 and keep == []
    p = pdhg._start_ptr([1, 2, 3], keep)
    assert len(keep) == 1 and keep[0].dtype == np.float64 and keep[0].flags.c_contiguous
    assert [p[i] for i in range(3)] == [1.0, 2.0, 3.0]
    strided = np.arange(10.0)[::2]
    p = pdhg._start_ptr(strided, keep)
    assert len(keep) == 2 and [p[i] for i in range(5)] == [0.0, 2.0, 4.0, 6.0, 8.0]
