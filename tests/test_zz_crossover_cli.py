"""The drop-in crossover (NIR_PDHG_CROSSOVER, nirnaya_b200/sov/pdhg_solver.hpp)
behind the real B200 engine, through the reference's CLI rebuilt on the
drop-ins.  The CPU checks of the crossover are in tests/test_dropin.py.
"""
import os
import subprocess

import pytest

import golden_io as G
from conftest import has_gpu
from test_dropin import _build_model, _need, _sov

GOLD = G.load()


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_cli_crossover_returns_the_vertex_on_crude_blending(tmp_path):
    """NIR_PDHG_CROSSOVER=1: after PDLP, the crash basis and the program's
    own simplex give the published optimum (.sol:2) to 1e-9 relative, where
    PDHG alone is within 1e-6."""
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
    r = subprocess.run([_need("sovsolve"), path, "--method", "pdhg", "--sol", sol], capture_output=True, text=True,
                       timeout=600, env=dict(os.environ, NIR_PDHG_CROSSOVER="1"))
    assert r.returncode == 0 and "PASS=YES" in r.stdout, r.stdout + r.stderr
    with open(sol) as f:
        obj = float(next(ln for ln in f if ln.startswith("# objective")).split()[2])
    assert abs(obj - g["sol_objective"]) <= 1e-9 * abs(g["sol_objective"]), (obj, g["sol_objective"])
