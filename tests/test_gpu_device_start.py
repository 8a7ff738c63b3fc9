"""Starting points in device memory (nir_pdhg_params.x_init / y_init given as
device addresses, include/nir_pdhg.h).

  - The engine copies a device-resident start on the device. The solve is
    the one from the same values in host memory, bit for bit. This holds on
    a plain LP, on one that the engine reorders by row length (the start's
    rows are remapped on the host) and on one with parallel columns (the
    start is re-expressed on the host).
  - The warm start's device-resident prediction (WarmStart.predict with
    device_out) holds the host prediction's values bit for bit. The warm
    solve from it is the one from the host prediction.

The SpMV layout is pinned (spmv_block_nnz) so that both solves of a pair
use the same one."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

import torch  # noqa: E402

from nirnaya_b200 import learned as LW  # noqa: E402
from nirnaya_b200 import lp as L  # noqa: E402
from nirnaya_b200 import pdhg  # noqa: E402


def _cudart():
    names = [os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64", "libcudart.so.12"),
             "libcudart.so.12", "libcudart.so"]
    for nm in names:
        try:
            return C.CDLL(nm)
        except OSError:
            continue
    pytest.skip("no CUDA runtime library to read device memory with")


def _download(addr, n):
    """n doubles at a device address, read into host memory."""
    rt = _cudart()
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    out = np.empty(n, np.float64)
    rc = rt.cudaMemcpy(out.ctypes.data, C.c_void_p(addr), n * 8, 2)  # device to host
    assert rc == 0, rc
    return out


def _same_solve(lp, p, x0, y0):
    xd = torch.tensor(x0, dtype=torch.float64, device="cuda")
    yd = torch.tensor(y0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    with pdhg.Engine(lp) as eng:
        xh, yh, ih = eng.solve(p, x_init=x0, y_init=y0)
        xg, yg, ig = eng.solve(p, x_init=xd.data_ptr(), y_init=yd.data_ptr())
    assert ih.iterations == ig.iterations and ih.status == ig.status
    assert np.array_equal(xh.view(np.int64), xg.view(np.int64))
    assert np.array_equal(yh.view(np.int64), yg.view(np.int64))
    return ih


@pytest.mark.parametrize("case", ["plain", "reordered", "parallel"])
def test_a_device_start_gives_the_host_start_solve(case):
    if case == "plain":
        lp = L.generate(L.RANDOM_EQ, 5, m=500, n=1250)
    elif case == "reordered":
        lp = L.generate(L.ZIPF, 3, m=4000, n=10000, target_nnz=100000)
        rl = np.bincount(lp.row_index, minlength=lp.nrow)
        assert lp.nrow >= 1024 and rl.max() >= 8 * rl.mean()  # the engine reorders its rows
    else:
        lp = L.generate(L.BADLY_SCALED, 1, m=500, n=1200, target_nnz=10000)
    p = pdhg.default_params(tol=1e-6, max_iters=4000, spmv_block_nnz=256)
    with pdhg.Engine(lp) as eng:
        x0, y0, _ = eng.solve(pdhg.default_params(tol=1e-6, max_iters=1000, spmv_block_nnz=256))
    info = _same_solve(lp, p, x0, y0)
    if case == "parallel":
        assert info.parallel_groups > 0


def test_the_warm_start_prediction_stays_on_the_device():
    fam = LW.BlendFamily(m=2000, n=5000, nnz=40000, family_seed=0)
    p = pdhg.default_params(tol=1e-6, max_iters=200000, spmv_block_nnz=256)
    with pdhg.Engine(fam.base) as eng:
        train = LW.solve_family(fam, range(1000, 1064), p, engine=eng)
    model = LW.WarmStart(fam, width=64, depth=2, seed=0, lr=1e-3)
    model.fit(train, epochs=2, batch=8192)
    try:
        with pdhg.Engine(fam.base) as eng:
            for seed in (5000, 5001):
                f, g = fam.factors(seed)
                xd, yd, wd = model.predict(f, g, device_out=True)
                xh, yh, wh = model.predict(f, g)
                assert isinstance(xd, int) and isinstance(yd, int) and wd == wh
                assert np.array_equal(_download(xd, fam.n).view(np.int64), xh.view(np.int64))
                assert np.array_equal(_download(yd, fam.m).view(np.int64), yh.view(np.int64))
                rowlo, cost = fam.vectors(f, g)
                eng.update_vectors(cost=cost, rowlo=rowlo)
                _, _, ih = eng.solve(p, x_init=xh, y_init=yh, omega_init=wh)
                _, _, ig = eng.solve(p, x_init=xd, y_init=yd, omega_init=wd)
                assert ig.status == pdhg.OPTIMAL and ih.iterations == ig.iterations
                assert ih.objective == ig.objective
    finally:
        model.close()
