"""Batched PDLP: many independent LPs in one solve, and instance sharding
across ranks.

The reference solves one model per call (src/gpu/pdhg_solver.hpp:25-27,
PdhgSolver::solve); its batch tooling runs models one after another
(bench/bench_runner.cpp, one solve per .mps file). Here a batch of LPs is
laid out block-diagonally on one GPU and every chunk of iterations advances
all of them with one launch per operator (nir_pdhg_batch_solve in
include/nir_pdhg.h): each instance keeps its own step size, primal weight,
restart state and stopping test, and an instance that has converged stops
moving while the others carry on.

Across GPUs the instances are independent, so a job shards them over ranks
with no data-path collective (`shard_instances`, longest-processing-time
first on nonzero counts); the results are gathered on rank 0 once at the end
(`gather_results`).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import pdhg as P
from .lp import LP, NirLpView
from .mps import VerifyReport, report_dict

_bound = False


def _lib():
    global _bound
    L = P.lib()
    if not _bound:
        D = C.POINTER(C.c_double)
        L.nir_pdhg_batch_create.argtypes = [C.POINTER(NirLpView), C.c_int32, C.c_int, C.POINTER(C.c_void_p)]
        L.nir_pdhg_batch_solve.argtypes = [C.c_void_p, C.POINTER(P.Params), P.POLL_FN, C.c_void_p, D, D,
                                           C.POINTER(P.Info), C.POINTER(P.Info)]
        L.nir_pdhg_batch_free.argtypes = [C.c_void_p]
        L.nir_pdhg_batch_verify.argtypes = [C.c_void_p, D, C.POINTER(C.c_int8), D, C.c_double,
                                            C.POINTER(VerifyReport)]
        _bound = True
    return L


class BatchEngine:
    """A batch of LPs resident on one GPU (nir_pdhg_batch_create ... _free)."""

    def __init__(self, lps: list[LP], device: int = 0):
        if not lps:
            raise ValueError("empty batch")
        self.lps = list(lps)
        views = (NirLpView * len(lps))(*[lp.view() for lp in lps])
        self._h = C.c_void_p()
        rc = _lib().nir_pdhg_batch_create(views, len(lps), device, C.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"nir_pdhg_batch_create failed ({P.STATUS_NAMES.get(rc, rc)}): {P.last_error()}")
        self.n = sum(lp.ncol for lp in lps)
        self.m = sum(lp.nrow for lp in lps)

    def close(self):
        if self._h:
            _lib().nir_pdhg_batch_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def solve(self, params: P.Params | None = None, poll=None):
        """Returns ([(x_i, y_i, info_i)], total): per-instance primal and
        dual solutions in each LP's own space and per-instance Info, plus
        the batch total (status = the first non-optimal instance status)."""
        p = params if params is not None else P.default_params()
        x = np.zeros(self.n)
        y = np.zeros(self.m)
        infos = (P.Info * len(self.lps))()
        total = P.Info()
        cb = P.POLL_FN(0) if poll is None else P.POLL_FN(lambda _ctx: 1 if poll() else 0)
        rc = _lib().nir_pdhg_batch_solve(self._h, C.byref(p), cb, None, P._dptr(x), P._dptr(y), infos,
                                         C.byref(total))
        if rc in (P.INPUT_ERROR, P.INTERNAL_ERROR):
            raise RuntimeError(f"nir_pdhg_batch_solve failed ({P.STATUS_NAMES[rc]}): {P.last_error()}")
        out = []
        c0 = r0 = 0
        for lp, inf in zip(self.lps, infos):
            out.append((x[c0:c0 + lp.ncol].copy(), y[r0:r0 + lp.nrow].copy(), inf))
            c0 += lp.ncol
            r0 += lp.nrow
        return out, total

    def verify(self, xs=None, claimed=None, tol: float = 1e-6, vartypes=None) -> list[dict]:
        """verify_solution (src/io/sol_io.hpp:25-106) for every instance on
        the GPU (nir_pdhg_batch_verify): per instance, the report
        mps.verify_solution gives on the host, bit for bit.  xs: one point
        per instance, or None for the points the last solve returned (still
        on the device).  claimed: one objective per instance or None.
        vartypes: one int8 array per instance or None."""
        x = None
        if xs is not None:
            if len(xs) != len(self.lps):
                raise ValueError(f"{len(xs)} points for {len(self.lps)} instances")
            for xi, lp in zip(xs, self.lps):
                if np.shape(xi) != (lp.ncol,):
                    raise ValueError("a point's length differs from its instance's column count")
            x = np.ascontiguousarray(np.concatenate([np.asarray(xi, np.float64) for xi in xs]))
        vt = None
        if vartypes is not None:
            vt = np.ascontiguousarray(np.concatenate([np.asarray(v, np.int8) for v in vartypes]), np.int8)
            if vt.size != self.n:
                raise ValueError("vartypes do not match the instances' column counts")
        cl = None if claimed is None else np.ascontiguousarray(claimed, np.float64)
        if cl is not None and cl.size != len(self.lps):
            raise ValueError(f"{cl.size} claimed objectives for {len(self.lps)} instances")
        reps = (VerifyReport * len(self.lps))()
        rc = _lib().nir_pdhg_batch_verify(self._h, None if x is None else P._dptr(x),
                                          None if vt is None else vt.ctypes.data_as(C.POINTER(C.c_int8)),
                                          None if cl is None else P._dptr(cl), float(tol), reps)
        if rc != 0:
            raise RuntimeError(f"nir_pdhg_batch_verify failed ({P.STATUS_NAMES.get(rc, rc)}): {P.last_error()}")
        return [report_dict(r) for r in reps]


def shard_instances(work, world: int) -> list[list[int]]:
    """Deterministic longest-processing-time assignment of instances to
    `world` ranks by their work (e.g. nonzeros); every rank gets a list of
    instance indices in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-float(work[i]), i))
    load = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += float(work[i])
    return [sorted(s) for s in shards]


def gather_results(local: dict, rank: int, world: int):
    """Collects every rank's {instance index: result} on rank 0 (one
    gather at the end of the job; None on the other ranks)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist

    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0)
    if rank != 0:
        return None
    merged: dict = {}
    for p in parts:
        merged.update(p)
    return merged


def solve_sharded(lps: list[LP], rank: int, world: int, device: int = 0, params: P.Params | None = None,
                  solve_fn=None, verify_tol: float | None = None):
    """Solves this rank's shard of `lps` as one batch and gathers
    {index: (objective, status, iterations)} on rank 0.

    With verify_tol, each rank also checks its solved points where they lie,
    on the device (BatchEngine.verify: verify_solution bit for bit).  Each
    result then ends with the check's verdict: (objective, status,
    iterations, passed).

    `solve_fn(lps)` replaces the device solve, which lets the sharding run
    on hosts without a GPU.  It returns one such tuple per LP.  The check
    runs on the device solve only, so solve_fn and verify_tol together are
    an error."""
    if solve_fn is not None and verify_tol is not None:
        raise ValueError("verify_tol checks the device solve's points; it cannot be combined with solve_fn")
    mine = shard_instances([lp.nnz for lp in lps], world)[rank]
    local = {}
    if mine:
        sub = [lps[i] for i in mine]
        if solve_fn is None:
            with BatchEngine(sub, device) as eng:
                res, _ = eng.solve(params)
                vals = [(inf.objective, inf.status, inf.iterations) for _, _, inf in res]
                if verify_tol is not None:
                    reps = eng.verify(None, [v[0] for v in vals], verify_tol)
                    vals = [v + (r["passed"],) for v, r in zip(vals, reps)]
        else:
            vals = solve_fn(sub)
        local = {i: v for i, v in zip(mine, vals)}
    return gather_results(local, rank, world)
