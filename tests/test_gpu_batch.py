"""GPU parity of the batched solve (nir_pdhg_batch_*), through the C ABI.

Every instance of a mixed batch must reach the requested relative KKT as the
oracle measures it in that instance's own space, its objective must be the
double-double evaluation of c'x, and it must agree with the objective of the
same LP solved alone. The batch is deterministic (same inputs, same bits),
and a batch split into shards gives the same per-instance answers as the
whole batch solved at once up to the stopping tolerance.
"""
import numpy as np
import pytest

import golden_io as G
from conftest import has_gpu
from nirnaya_b200 import batch as B
from nirnaya_b200 import lp as L
from nirnaya_b200 import pdhg
from oracle import ffi

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

GOLD = G.load()


def mixed_batch():
    return [
        L.generate(L.RANDOM_EQ, 11, m=300, n=750),
        L.generate(L.MULTIPERIOD, 12, m=600),
        G.lp_from(GOLD["crude_blending"]["lp_internal_min"]),
        L.generate(L.BLEND_FAMILY, 13, m=500, n=1250, target_nnz=10000),
        G.lp_from(GOLD["unit_test_pdhg_lp"]["lp"]),
        L.generate(L.MULTIPERIOD, 14, m=1500),
        L.generate(L.RANDOM_EQ, 15, m=120, n=300),
    ]


@pytest.mark.parametrize("prec", [pdhg.PREC_FP64, pdhg.PREC_MIXED])
def test_batch_each_instance_reaches_tolerance(prec):
    lps = mixed_batch()
    tol = 1e-6
    with B.BatchEngine(lps) as eng:
        res, total = eng.solve(pdhg.default_params(precision=prec, tol=tol, max_iters=300000))
    assert total.status == pdhg.OPTIMAL
    for lp, (x, y, info) in zip(lps, res):
        assert info.status == pdhg.OPTIMAL, (pdhg.STATUS_NAMES.get(info.status), info.rel_kkt)
        k = ffi.rel_kkt(lp, x, y)
        assert k.rel_kkt <= 1.05 * tol, k.rel_kkt
        assert info.objective == ffi.eval_objective(lp, x)
        # an independent optimum (HiGHS), to the relative objective error of
        # src/io/sol_io.hpp:96-102 at 1e-6
        opt = G.highs_optimum(lp)
        assert abs(info.objective - opt) / (1 + abs(opt)) <= 1e-6, (info.objective, opt)
    assert total.iterations == max(r[2].iterations for r in res)


def test_batch_is_deterministic():
    lps = mixed_batch()[:4]
    p = pdhg.default_params(precision=pdhg.PREC_MIXED, tol=1e-6, max_iters=100000)
    with B.BatchEngine(lps) as eng:
        a, _ = eng.solve(p)
        b, _ = eng.solve(p)
    for (xa, ya, ia), (xb, yb, ib) in zip(a, b):
        assert np.array_equal(G.bits(xa), G.bits(xb)) and np.array_equal(G.bits(ya), G.bits(yb))
        assert ia.iterations == ib.iterations


def test_sharded_batch_matches_whole_batch():
    lps = mixed_batch()
    # a fixed row-block capacity: the autotuner could pick another one for
    # a smaller batch, and the block boundaries set the summation order
    p = pdhg.default_params(precision=pdhg.PREC_FP64, tol=1e-7, max_iters=300000, spmv_block_nnz=256)
    with B.BatchEngine(lps) as eng:
        whole, _ = eng.solve(p)
    got = {}
    shards = B.shard_instances([lp.nnz for lp in lps], 3)
    for idx in shards:
        if not idx:
            continue
        with B.BatchEngine([lps[i] for i in idx]) as eng:
            part, _ = eng.solve(p)
        for i, (x, y, inf) in zip(idx, part):
            got[i] = inf
    for i, (_, _, inf) in enumerate(whole):
        assert got[i].status == pdhg.OPTIMAL
        # an instance's iteration does not depend on the batch around it:
        # same layout, same per-instance reductions, same bits
        assert got[i].iterations == inf.iterations
        assert got[i].objective == inf.objective


@pytest.mark.parametrize("prec", [pdhg.PREC_FP64, pdhg.PREC_MIXED])
def test_persistent_batch_chunks_are_bit_identical(prec):
    # the non-check iterations of a chunk in one cooperative launch with grid
    # barriers: the same blocks, the same per-row order, the same bits
    lps = mixed_batch()[:5]
    base = dict(precision=prec, tol=1e-6, max_iters=20000, spmv_block_nnz=256)
    with B.BatchEngine(lps) as eng:
        a, ta = eng.solve(pdhg.default_params(persistent=0, **base))
        b, tb = eng.solve(pdhg.default_params(persistent=1, **base))
    assert ta.status == tb.status
    for (xa, ya, ia), (xb, yb, ib) in zip(a, b):
        assert ia.iterations == ib.iterations and ia.status == ib.status
        assert np.array_equal(G.bits(xa), G.bits(xb)) and np.array_equal(G.bits(ya), G.bits(yb))


def test_persistent_batch_barrier_wait_is_bounded():
    # persistent=2 makes the barrier wait for one CTA more than the launch
    # has: the wait gives up after ~0.1 s, every instance ends with
    # INTERNAL_ERROR, and the same handle then solves normally
    import time

    lps = mixed_batch()[:3]
    with B.BatchEngine(lps) as eng:
        t = time.time()
        with pytest.raises(RuntimeError, match="internal_error"):
            eng.solve(pdhg.default_params(persistent=2, max_iters=5000))
        assert time.time() - t < 30
        res, total = eng.solve(pdhg.default_params(persistent=1))
        assert total.status == pdhg.OPTIMAL


def test_batch_rejects_bad_input():
    with pytest.raises(RuntimeError):
        with B.BatchEngine([L.generate(L.RANDOM_EQ, 1, m=50, n=100)]) as eng:
            eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE))
