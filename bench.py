"""Benchmark of the PDHG path on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2] [--impl ours|reference]

A step is one solve of the workload to 1e-6 relative KKT (the metric of the
reference's PDHG path is time to tolerance).  Workloads (seeded synthetic
instances of include/nir_lpgen.h; the reference publishes no dataset):

  c2  ZIPF 200,000 x 500,000, ~5M nonzeros, mixed precision (default)
  c1  RANDOM_EQ 2,000 x 5,000, 40,000 nonzeros
  c5  BADLY_SCALED 50,000 x 120,000, ~1M nonzeros
  c4  learned warm start on the fixed-matrix blending family (m 20,000,
      n 50,000, 400k nonzeros): PDLP solves --c4-train instances, the
      network (3 x 512, hand-written BF16 tensor-core kernels) trains on
      them, and --c4-test held-out instances are solved cold and warm to
      1e-6; also plain FP64 PDHG on --c4-pdhg of them.  Time per held-out
      instance (mean).
  c3  256 MULTIPERIOD instances, m log-uniform in [500, 20,000], n = 2.5 m
      (~1.3M rows, ~3.3M columns, ~33M nonzeros in total), solved as one
      batch (nir_pdhg_batch_solve); with --gpus N the instances are sharded
      over the ranks (strong scaling, no data-path collective)

`value` is the time to tolerance with the LP already resident in HBM
(handle created before the timed region); `e2e` is the same metric through
the one-shot C ABI (nir_pdhg_solve_lp) from host arrays, host->device copy,
transpose and device->host copy of x and y included.  `roofline` covers the
dominant kernel (the fused A'y SpMV + primal update) timed with CUDA events
on the engine's stream during a solve.  `cpu_baseline` times the
reference's own PdhgSolver::solve (compiled from source into oracle/_ref) on
a bounded sample of the same workload.

With --gpus N > 1 (torchrun), every rank solves its own replica (the path
does not shard a single LP) and the time is the max over
ranks.  --impl reference runs the reference's CPU PDHG on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to 1e-6 rel KKT: learned-warm/mixed vs plain PDHG on B200; SpMV GB/s"
L2_BYTES = 126 * 2 ** 20

WORKLOADS = {
    "c2": dict(kind=2, seed=1, kw={}, label="zipf_200000x500000_nnz5M", precision=1),
    "c1": dict(kind=1, seed=1, kw={}, label="random_eq_2000x5000_nnz40000", precision=1),
    "c5": dict(kind=5, seed=1, kw={}, label="badly_scaled_50000x120000_nnz1M", precision=1),
    "c3": dict(kind=3, seed=1000, kw={}, label="multiperiod_batch256_m500-20000", precision=1, batch=256),
    "c4": dict(kind=4, seed=0, kw={}, label="blend_family_20000x50000_nnz400k_learned_warm", precision=1,
               learned=True),
}


def batch_instances(wl):
    """The c3 batch: instance i is MULTIPERIOD seed (seed + i) with m drawn
    log-uniformly from [500, 20000] by a seeded generator."""
    import numpy as np

    from nirnaya_b200 import lp as L

    rng = np.random.default_rng(wl["seed"])
    ms = np.exp(rng.uniform(np.log(500), np.log(20000), wl["batch"])).astype(int)
    return [L.generate(wl["kind"], wl["seed"] + i, m=int(m)) for i, m in enumerate(ms)]


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(kernel_tag: str):
    """Per-launch DRAM bytes of the fused kernel from the committed ncu
    summary (profiles/*.md line `traffic_bytes_per_launch[<tag>]: N`)."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    pat = re.compile(r"traffic_bytes_per_launch\[" + re.escape(kernel_tag) + r"\]:\s*([0-9.eE+]+)")
    for fn in sorted(os.listdir(pdir)):
        if fn.endswith((".md", ".txt")):
            with open(os.path.join(pdir, fn)) as f:
                m = pat.search(f.read())
            if m:
                return float(m.group(1))
    return None


def committed_ref_iterations(label: str):
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None, None
    pat = re.compile(r"reference_iterations_to_tol\[" + re.escape(label) + r"\]:\s*([0-9]+)(\s*lower_bound)?")
    for fn in sorted(os.listdir(pdir)):
        if fn.endswith((".md", ".txt")):
            with open(os.path.join(pdir, fn)) as f:
                m = pat.search(f.read())
            if m:
                return int(m.group(1)), bool(m.group(2))
    return None, None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def primal_bytes(lp, w, vw=None):
    """Algorithmic bytes of one fused A'y + primal-update launch, counted
    unfused: the CSR SpMV of A' (n rows; vw-byte values, 4-byte indices and
    row pointers, y read once, A'y written once) plus the primal update
    (x, c, l, u, A'y read, x and x-bar written), w = 4 (FP32) or 8 (FP64)
    the vector width, vw the value width (w unless the values are FP32 with
    FP64 vectors)."""
    n, m, nnz = lp.ncol, lp.nrow, lp.nnz
    vw = w if vw is None else vw
    return (4 + vw) * nnz + 4 * (n + 1) + w * m + w * n + 7 * w * n


def dual_bytes(lp, w, vw=None):
    """Same for the fused A x-bar + dual-update launch: SpMV of A (m rows)
    plus the dual update (y, A x-bar, row bounds read, y written)."""
    n, m, nnz = lp.ncol, lp.nrow, lp.nnz
    vw = w if vw is None else vw
    return (4 + vw) * nnz + 4 * (m + 1) + w * n + w * m + 5 * w * m


def spmv_bytes_w(lp, transpose, vword, xword):
    """spmv_bytes with separate value and vector widths (FP32 values with
    FP64 vectors stream 8 bytes per nonzero but read and write FP64)."""
    R, Cc = (lp.ncol, lp.nrow) if transpose else (lp.nrow, lp.ncol)
    return (4 + vword) * lp.nnz + 4 * (R + 1) + xword * Cc + xword * R


def spmv_bytes(lp, transpose, word):
    """Algorithmic bytes of a plain CSR SpMV: index and value per nonzero, row
    pointers, the input vector read once, the output vector written once."""
    R, Cc = (lp.ncol, lp.nrow) if transpose else (lp.nrow, lp.ncol)
    iw = 4
    return (iw + word) * lp.nnz + 4 * (R + 1) + word * Cc + word * R


def dist_setup(gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def allmax(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch

    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()


def run_ours(args, rank, world, local):
    import numpy as np
    import torch

    from nirnaya_b200 import lp as L
    from nirnaya_b200 import pdhg

    wl = WORKLOADS[args.workload]
    lp = L.generate(wl["kind"], wl["seed"], **wl["kw"])
    params = pdhg.default_params(precision=wl["precision"], tol=1e-6, max_iters=args.max_iters)
    eng = pdhg.Engine(lp, local)
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    launches = 0
    infos = []
    for _ in range(args.warmup):
        flush.fill_(1)
        eng.solve(params)
    barrier(world)
    with ClockSampler(local) as clk:
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for _ in range(args.steps):
            flush.fill_(1)  # every solve starts with a cold L2
            x, y, info = eng.solve(params)
            launches += info.kernel_launches
            infos.append(info.as_dict())
        b.record()
        torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    ms = allmax(ms, world)
    # end-to-end through the one-shot C ABI with host arrays
    e2e_s = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x = np.zeros(lp.ncol)
        y = np.zeros(lp.nrow)
        info = pdhg.Info()
        import ctypes as C

        pdhg.lib().nir_pdhg_solve_lp(C.byref(lp.view()), local, C.byref(params), pdhg.POLL_FN(0), None,
                                     x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)),
                                     C.byref(info))
        e2e_s.append(time.perf_counter() - t0)
    e2e = allmax(statistics.median(e2e_s), world)
    # steady-state event timing of the fused kernels on the solved state,
    # in the precision of each phase of the timed solves
    kt = {}
    flush.fill_(1)
    eng.solve(params)
    lay_first = eng.layout()
    kt[wl["precision"]] = eng.time_iteration(wl["precision"], reps=100)
    # the same workload in FP64 throughout: one solve, for the mixed-precision gain
    fp64 = None
    if wl["precision"] != pdhg.PREC_FP64:
        p64 = pdhg.default_params(precision=pdhg.PREC_FP64, tol=1e-6, max_iters=args.max_iters)
        eng.solve(p64)  # the FP64 layout is tuned here (untimed)
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, _, i64 = eng.solve(p64)
        torch.cuda.synchronize()
        fp64 = dict(seconds=time.perf_counter() - t0, iterations=i64.iterations, status=i64.status,
                    rel_kkt=i64.rel_kkt, objective=i64.objective)
    kt[pdhg.PREC_FP64] = eng.time_iteration(pdhg.PREC_FP64, reps=100)
    lay64 = eng.layout()
    # plain SpMV with a cold L2 (the SpMV GB/s of the metric): both layout
    # families in each precision and the row-less gather ceilings
    spmv = spmv_figures(eng, lp, lay_first, reps=20)
    eng.close()
    return dict(lp=lp, ms=ms, infos=infos, launches=launches, e2e=e2e, kt=kt, lay=lay_first, lay64=lay64,
                clocks=clk.summary(), spmv=spmv, fp64=fp64)


def spmv_figures(eng, lp, lay=None, reps=20):
    """Cold-L2 CUDA-event times of the plain SpMV kernels of both layout
    families (warp row blocks at the capacity the solve chose for that
    orientation, else 256 and 128; CTA blocks of 256 x 4 nonzeros) in each
    precision, and of the row-less ceilings over the same stream, with the
    algorithmic GB/s of each.  `best_f32` / `best_f64` per orientation is the
    faster family."""
    from nirnaya_b200 import pdhg

    out = {}
    for tr, side in ((False, "A"), (True, "At")):
        chosen = None if lay is None else (lay.block_nnz_at if tr else lay.block_nnz)
        warp_caps = [chosen] if chosen is not None and chosen <= 256 else [256, 128]
        rows = []
        for cap in warp_caps:
            rows += [("warp_f32", pdhg.K_WARP32, 4, 4, cap), ("warp_f64", pdhg.K_WARP64, 8, 8, cap)]
        for cap in ((1024,) if lay is not None else (1024, 2048)):
            rows += [("cta_f32", pdhg.K_CTA32, 4, 4, cap), ("cta_f32val_f64x", pdhg.K_CTA_MIXED, 4, 8, cap),
                     ("cta_f64", pdhg.K_CTA64, 8, 8, cap)]
        rows += [("ceiling_gather_f32", pdhg.K_CEIL_GATHER32, 4, 4, 0),
                 ("ceiling_gather_f64", pdhg.K_CEIL_GATHER64, 8, 8, 0),
                 ("ceiling_stream_f64", pdhg.K_CEIL_STREAM64, 8, 8, 0)]
        for kname, kind, vw, xw, cap in rows:
            us = eng.time_kernel(tr, kind, cap, reps=reps, flush_l2=True)
            by = spmv_bytes_w(lp, tr, vw, xw)
            key = f"{side}_{kname}"
            fig = {"us": us, "GBs": by / (us * 1e-6) / 1e9, "bytes": by, "block_nnz": cap}
            if key not in out or us < out[key]["us"]:
                out[key] = fig
        for prec in ("f32", "f64"):
            fam = min(("warp", "cta"), key=lambda f: out[f"{side}_{f}_{prec}"]["us"])
            out[f"{side}_best_{prec}"] = {**out[f"{side}_{fam}_{prec}"], "family": fam,
                                         "chosen_by_solve": None if chosen is None else
                                         ("cta" if chosen > 256 else "warp")}
    return out


def cpu_baseline(lp, label, seconds=15.0, threads=None):
    """The reference's PdhgSolver::solve (oracle/_ref) on this host for a
    bounded wall time, at 1 thread and at all host threads (its ThreadPool
    size, Options.threads): iterations per second of the faster, then time
    to tolerance from the reference algorithm's iteration count on this
    instance when known."""
    from oracle import ffi

    if not ffi.ref_available():
        return None
    nproc = threads or os.cpu_count() or 1
    rates = {}
    for th in sorted({1, nproc}):
        t0 = time.perf_counter()
        x, y, st, obj, it = ffi.ref_pdhg(lp, threads=th, simplex_iter_limit=10 ** 9, time_limit=seconds / 2)
        rates[th] = it / (time.perf_counter() - t0)
    best = max(rates, key=rates.get)
    it_s = rates[best]
    n_ref, lower = committed_ref_iterations(label)
    value = (n_ref / it_s) if n_ref else None
    return dict(value=value, unit="s", cores=best, kind="reference",
                sample=f"PdhgSolver::solve for {seconds / 2:.0f} s wall at each of threads="
                       f"{sorted(rates)} ({', '.join(f'{k}: {v:.1f} it/s' for k, v in sorted(rates.items()))}); "
                       f"time = iterations the reference algorithm needs to 1e-6 relative KKT on this instance "
                       f"({n_ref if n_ref else 'unknown'}{' lower bound' if lower else ''}) / the faster rate",
                iterations_per_s=it_s, iterations_per_s_by_threads={str(k): v for k, v in rates.items()},
                lower_bound=bool(lower))


def run_batch_ours(args, rank, world, local):
    """c3: this rank's shard of the 256 instances as one batch."""
    import ctypes as C

    import numpy as np
    import torch

    from nirnaya_b200 import batch as B
    from nirnaya_b200 import pdhg
    from nirnaya_b200.lp import NirLpView

    wl = WORKLOADS[args.workload]
    lps = batch_instances(wl)
    mine = B.shard_instances([lp.nnz for lp in lps], world)[rank]
    sub = [lps[i] for i in mine]
    params = pdhg.default_params(precision=wl["precision"], tol=1e-6, max_iters=args.max_iters)
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    eng = B.BatchEngine(sub, local)
    for _ in range(args.warmup):
        flush.fill_(1)
        eng.solve(params)
    barrier(world)
    launches = 0
    with ClockSampler(local) as clk:
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for _ in range(args.steps):
            flush.fill_(1)
            res, total = eng.solve(params)
            launches += total.kernel_launches
        b.record()
        torch.cuda.synchronize()
    ms = allmax(a.elapsed_time(b) / args.steps, world)
    eng.close()
    # end to end: create (host->device copy, transpose), solve, copy out, free
    views = (NirLpView * len(sub))(*[lp.view() for lp in sub])
    n = sum(lp.ncol for lp in sub)
    m = sum(lp.nrow for lp in sub)
    e2e_s = []
    L = B._lib()
    for _ in range(max(1, min(args.steps, 2))):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = C.c_void_p()
        if L.nir_pdhg_batch_create(views, len(sub), local, C.byref(h)) != 0:
            raise RuntimeError(pdhg.last_error())
        x = np.zeros(n)
        y = np.zeros(m)
        infos = (pdhg.Info * len(sub))()
        tot = pdhg.Info()
        L.nir_pdhg_batch_solve(h, C.byref(params), pdhg.POLL_FN(0), None, pdhg._dptr(x), pdhg._dptr(y), infos,
                               C.byref(tot))
        L.nir_pdhg_batch_free(h)
        e2e_s.append(time.perf_counter() - t0)
    e2e = allmax(statistics.median(e2e_s), world)
    per = [dict(status=r[2].status, iterations=r[2].iterations, rel_kkt=r[2].rel_kkt) for r in res]
    # algorithmic bytes of the iterations actually run: per instance and
    # iteration, one FP32 pass over A' and one over A (index + value per
    # nonzero, row pointers, the gathered vector and the epilogue vectors)
    alg = 0.0
    for lp, r in zip(sub, per):
        alg += r["iterations"] * (16.0 * lp.nnz + 4 * 9 * lp.ncol + 4 * 8 * lp.nrow)
    return dict(ms=ms, per=per, launches=launches, e2e=e2e, clocks=clk.summary(), alg=alg,
                h2d=sum(lp.host_bytes() for lp in sub), d2h=8 * (n + m), rows=m, cols=n,
                nnz=sum(lp.nnz for lp in sub), count=len(sub))


def batch_line(args, r, world):
    peak, peak_kind = peaks()
    alg_total = allmax(r["alg"], 1)
    achieved = alg_total / (r["ms"] * 1e-3) / 1e9
    per = r["per"]
    return {
        "metric": METRIC,
        "value": r["ms"] / 1000.0,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": r["ms"],
        "higher_is_better": False,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic (seeded generator, include/nir_lpgen.h)",
        "config": {"workload": WORKLOADS["c3"]["label"], "instances": 256, "instances_rank0": r["count"],
                   "rows_rank0": r["rows"], "cols_rank0": r["cols"], "nnz_rank0": r["nnz"], "tol": 1e-6,
                   "algorithm": "pdlp batch (per-instance restarts, primal weight and stop)",
                   "precision": "mixed (fp32 + fp64 polish)",
                   "parallelism": f"instance shards x{world}" if world > 1 else "single gpu",
                   "l2": "flushed (2x L2 write) before every solve; the batch (~0.5 GB of matrix) exceeds L2"},
        "instances_per_s": 256 / (r["ms"] / 1000.0) if world == 1 else None,
        "status_counts": {str(k): sum(1 for p in per if p["status"] == k) for k in sorted({p["status"] for p in per})},
        "iterations_max": max(p["iterations"] for p in per),
        "iterations_median": statistics.median(p["iterations"] for p in per),
        "rel_kkt_max": max(p["rel_kkt"] for p in per),
        "e2e": {"value": r["e2e"], "unit": "s", "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]},
        "gpu_launches": r["launches"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None,
                     "kernel": "whole batch loop (k_bprimal + k_bdual + checks), algorithmic bytes of the "
                               "iterations each instance ran / solve time (rank 0)",
                     "peak_kind": peak_kind},
        "cpu_baseline": None,
        "clocks": r["clocks"],
    }


def learned_figures(n_train, n_test, n_pdhg, pdhg_iters, epochs):
    """The learned warm start on the blending family (c4): PDLP solves
    n_train training instances, the network trains on them, n_test held-out
    instances are solved cold and warm (prediction included) to 1e-6, and
    n_pdhg of them also by cold FP64 PDLP and by plain unrestarted FP64 PDHG.
    Returns (figures, clocks)."""
    import numpy as np

    from nirnaya_b200 import learned as LW
    from nirnaya_b200 import pdhg

    fam = LW.BlendFamily(m=20000, n=50000, nnz=400000, family_seed=0)
    p = pdhg.default_params(tol=1e-6, max_iters=1000000)
    eng = pdhg.Engine(fam.base, 0)
    t0 = time.perf_counter()
    train = LW.solve_family(fam, range(100000, 100000 + n_train), p, engine=eng)
    t_gen = time.perf_counter() - t0
    model = LW.WarmStart(fam, width=512, depth=3, seed=0, lr=1e-3)
    t0 = time.perf_counter()
    fit = model.fit(train, epochs=epochs, batch=8192, cols_per_instance=1024, rows_per_instance=512)
    t_fit = time.perf_counter() - t0
    losses = fit["col_loss"]
    us_step, flops_step = model.col_net.step_stats()
    held = list(range(900000, 900000 + n_test))
    with ClockSampler(0) as clk:
        ev = LW.evaluate(fam, model, held, p, engine=eng)
    summ = ev.summary()
    # baselines on a subset: cold FP64 PDLP and plain (unrestarted) FP64 PDHG
    sub_ = held[:n_pdhg]
    p64 = pdhg.default_params(tol=1e-6, max_iters=1000000, precision=pdhg.PREC_FP64)
    pp = pdhg.default_params(tol=1e-6, max_iters=pdhg_iters, precision=pdhg.PREC_FP64, algorithm=pdhg.ALGO_PDHG)
    t64, tpl, itpl, stpl = [], [], [], []
    for sd in sub_:
        rowlo, cost = fam.vectors(*fam.factors(sd))
        eng.update_vectors(cost=cost, rowlo=rowlo)
        t1 = time.perf_counter()
        eng.solve(p64)
        t64.append(time.perf_counter() - t1)
        t1 = time.perf_counter()
        _, _, ip = eng.solve(pp)
        tpl.append(time.perf_counter() - t1)
        itpl.append(ip.iterations)
        stpl.append(ip.status)
    # what a warm start must achieve: PDLP iterations from the instance's own
    # accurate solution (tol 1e-9) perturbed per entry by a relative Gaussian
    # error, from the training mean, and from the network's prediction, with
    # the relative distance of each start from that solution
    ok = train.status == pdhg.OPTIMAL
    xbar = train.x[ok].astype(np.float64).mean(0)
    ybar = train.y[ok].astype(np.float64).mean(0)
    sens = {"instances": len(sub_), "iterations": {}, "rel_dist_x": {}, "rel_dist_y": {}}
    rows_ = []
    for sd in sub_:
        f_, g_ = fam.factors(sd)
        rowlo, cost = fam.vectors(f_, g_)
        eng.update_vectors(cost=cost, rowlo=rowlo)
        _, _, ci = eng.solve(p)
        xs, ys, si = eng.solve(pdhg.default_params(tol=1e-9, max_iters=1000000))
        xp, yp, wp = model.predict(f_, g_)
        rng = np.random.default_rng(sd)
        starts = {"cold": None, "network": (xp, yp, wp), "training_mean": (xbar, ybar, wp)}
        for eps in (1e-3, 1e-2, 1e-1):
            starts[f"own_solution_rel_err_{eps:g}"] = (xs * (1 + eps * rng.standard_normal(xs.size)),
                                                        ys * (1 + eps * rng.standard_normal(ys.size)), si.primal_weight)
        rec = {}
        for k, st_ in starts.items():
            if st_ is None:
                rec[k] = (ci.iterations, 0.0, 0.0)
                continue
            x0 = np.clip(st_[0], fam.base.collo, fam.base.colup)
            _, _, wi = eng.solve(p, x_init=x0, y_init=st_[1], omega_init=st_[2])
            rec[k] = (wi.iterations, float(np.linalg.norm(x0 - xs) / max(np.linalg.norm(xs), 1e-300)),
                      float(np.linalg.norm(st_[1] - ys) / max(np.linalg.norm(ys), 1e-300)))
        rows_.append(rec)
    for k in rows_[0] if rows_ else []:
        sens["iterations"][k] = float(np.mean([r[k][0] for r in rows_]))
        sens["rel_dist_x"][k] = float(np.mean([r[k][1] for r in rows_]))
        sens["rel_dist_y"][k] = float(np.mean([r[k][2] for r in rows_]))
    eng.close()
    model.close()
    warm_s = summ["warm_seconds_mean"]
    pdhg_reached = all(s_ == pdhg.OPTIMAL for s_ in stpl)
    fig = {
        "workload": WORKLOADS["c4"]["label"], "m": fam.m, "n": fam.n, "nnz": int(fam.base.nnz),
        "train_instances": n_train, "test_instances": n_test,
        "network": "per-column and per-row 3 x 512 ReLU MLPs (shared weights)",
        "learned_warm_mixed_s": warm_s,
        "cold_mixed_pdlp_s": summ["cold_seconds_mean"],
        "cold_fp64_pdlp_s": float(np.mean(t64)) if t64 else None,
        "plain_fp64_pdhg_s": float(np.mean(tpl)) if tpl else None,
        "plain_fp64_pdhg_iterations": float(np.mean(itpl)) if itpl else None,
        "plain_fp64_pdhg_reached_tol": pdhg_reached, "baseline_subset": len(sub_),
        "ratio_plain_fp64_pdhg_over_learned_warm": (float(np.mean(tpl)) / warm_s) if tpl else None,
        "network_gain_cold_over_warm": summ["cold_seconds_mean"] / warm_s,
        "learned": {**summ, "train_generation_s": t_gen, "train_fit_s": t_fit,
                    "train_loss_first_last": [float(losses[0]), float(losses[-1])],
                    "row_loss_first_last": [float(fit["row_loss"][0]), float(fit["row_loss"][-1])],
                    "col_samples": fit["col_samples"], "row_samples": fit["row_samples"],
                    "train_solutions_optimal": int((train.status == pdhg.OPTIMAL).sum())},
        "warm_start_sensitivity": sens,
        "note": None if pdhg_reached else "plain PDHG hit its iteration cap on some instances: its time is a lower bound",
        "train_step_us": us_step, "train_step_flops": flops_step,
    }
    return fig, clk.summary()


def run_learned(args, world):
    """c4: the learned warm start pipeline on one GPU (replicas only)."""
    fig, clocks = learned_figures(args.c4_train, args.c4_test, args.c4_pdhg, args.c4_pdhg_iters, args.c4_epochs)
    peak_tf = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak_tf = float(json.load(f)["bf16_tflops"])
    except Exception:
        peak_tf = 1590.0
    us_step, flops_step = fig["train_step_us"], fig["train_step_flops"]
    tf = flops_step / (us_step * 1e-6) / 1e12 if us_step > 0 else None
    warm_s = fig["learned_warm_mixed_s"]
    line = {
        "metric": METRIC, "value": warm_s, "unit": "s", "n_gpus": world, "steps": args.c4_test, "warmup": 0,
        "ms_per_step": 1000 * warm_s, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 values + f64 iterates (PDLP), bf16 x fp32 (network)", "data": "synthetic (seeded blending family)",
        "config": {"workload": WORKLOADS["c4"]["label"], "m": fig["m"], "n": fig["n"], "nnz": fig["nnz"],
                   "train_instances": args.c4_train, "test_instances": args.c4_test, "network": fig["network"],
                   "tol": 1e-6, "parallelism": "single gpu"},
        "learned": fig["learned"],
        "warm_start_sensitivity": fig["warm_start_sensitivity"],
        "baselines": {k: fig[k] for k in ("cold_mixed_pdlp_s", "cold_fp64_pdlp_s", "plain_fp64_pdhg_s",
                                          "plain_fp64_pdhg_iterations", "plain_fp64_pdhg_reached_tol",
                                          "baseline_subset", "ratio_plain_fp64_pdhg_over_learned_warm", "note")},
        "roofline": {"bound": "tensor", "achieved": tf, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": (tf / peak_tf) if tf else None, "traffic": None,
                     "kernel": "column network training step (k_gemm BF16, FP32 accumulate), 8192-sample batch",
                     "us_per_step": us_step, "flops_per_step": flops_step},
        "cpu_baseline": None,
        "clocks": clocks,
    }
    print(json.dumps(line))


def run_blocks(args, local):
    """The headline figures of the other configurations, measured in the
    same run as the c2 line (one GPU), within the bench's time budget:
      batch    c3: the 256 instances as one batch, time to 1e-6 for all of
               them (mean of 2 solves after 1 warm-up), and the cold plain
               SpMV of the block-diagonal batch matrix;
      learned  c4: learned warm start vs cold mixed PDLP vs plain FP64 PDHG
               (fewer training and held-out instances than --workload c4;
               the counts are in the block);
      c5       the badly scaled LP: one mixed and one FP64 solve;
      c1       the 2,000 x 5,000 random LP: mean of 5 solves."""
    import numpy as np
    import scipy.sparse as sp
    import torch

    from nirnaya_b200 import batch as B
    from nirnaya_b200 import lp as L
    from nirnaya_b200 import pdhg

    out = {}
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    # c3
    lps = batch_instances(WORKLOADS["c3"])
    p = pdhg.default_params(tol=1e-6, max_iters=args.max_iters)
    t0 = time.perf_counter()
    with B.BatchEngine(lps, local) as eng:
        t_create = time.perf_counter() - t0
        eng.solve(p)
        times = []
        for _ in range(2):
            flush.fill_(1)
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            res, total = eng.solve(p)
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b) / 1000.0)
        # the same batch with each chunk's non-check iterations in one
        # cooperative persistent launch (grid barriers between half-iterations)
        pp_ = pdhg.default_params(tol=1e-6, max_iters=args.max_iters, persistent=1)
        eng.solve(pp_)
        ptimes = []
        for _ in range(2):
            flush.fill_(1)
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            pres, _ = eng.solve(pp_)
            b.record()
            torch.cuda.synchronize()
            ptimes.append(a.elapsed_time(b) / 1000.0)
    st = [r[2].status for r in res]
    its = [r[2].iterations for r in res]
    alg = sum(r[2].iterations * (12.0 * lp.nnz + 8 * 9 * lp.ncol + 8 * 8 * lp.nrow) for lp, r in zip(lps, res))
    tts = float(np.mean(times))
    out["batch"] = {"workload": WORKLOADS["c3"]["label"], "instances": len(lps),
                    "nnz": int(sum(lp.nnz for lp in lps)), "time_to_tol_s": tts, "instances_per_s": len(lps) / tts,
                    "create_s": t_create, "status_counts": {str(k): st.count(k) for k in sorted(set(st))},
                    "iterations_max": int(max(its)), "iterations_median": float(np.median(its)),
                    "rel_kkt_max": float(max(r[2].rel_kkt for r in res)),
                    "loop_algorithmic_GBs": alg / tts / 1e9,
                    "persistent_time_to_tol_s": float(np.mean(ptimes)),
                    "persistent_same_iterations": [r[2].iterations for r in pres] == its,
                    "launch_mode": "graph-launched kernels per half-iteration (the default); "
                                   "persistent_time_to_tol_s: the cooperative persistent chunk kernel",
                    "note": "algorithmic bytes of the iterations each instance ran, counted at FP32 values with "
                            "FP64 vectors, over the device time of the whole solve"}
    # the batch matrix as one block-diagonal LP: cold plain SpMV GB/s
    Ab = sp.block_diag([sp.csc_matrix((lp.value, lp.row_index, lp.col_start), shape=(lp.nrow, lp.ncol))
                        for lp in lps], format="csc")
    big = L.LP(Ab.shape[0], Ab.shape[1], Ab.indptr.astype(np.int64), Ab.indices.astype(np.int32), Ab.data,
               np.concatenate([lp.cost for lp in lps]), np.concatenate([lp.collo for lp in lps]),
               np.concatenate([lp.colup for lp in lps]), np.concatenate([lp.rowlo for lp in lps]),
               np.concatenate([lp.rowup for lp in lps]))
    del Ab
    with pdhg.Engine(big, local) as eng:
        sp_fig = spmv_figures(eng, big, None, reps=10)
        out["batch"]["spmv_cold"] = sp_fig
    del big
    # c4
    fig, _ = learned_figures(args.block_c4_train, args.block_c4_test, args.block_c4_pdhg, args.c4_pdhg_iters,
                             args.c4_epochs)
    out["learned"] = {k: v for k, v in fig.items() if k not in ("train_step_us", "train_step_flops")}
    # c5 and c1
    for key in ("c5", "c1"):
        wl = WORKLOADS[key]
        lp = L.generate(wl["kind"], wl["seed"], **wl["kw"])
        rec = {"workload": wl["label"]}
        with pdhg.Engine(lp, local) as eng:
            for tag, prec in (("mixed", pdhg.PREC_MIXED), ("fp64", pdhg.PREC_FP64)):
                pp = pdhg.default_params(precision=prec, tol=1e-6, max_iters=args.max_iters)
                eng.solve(pp)  # warm-up (layout tuning, graph capture)
                ts = []
                for _ in range(5 if key == "c1" else 1):
                    flush.fill_(1)
                    torch.cuda.synchronize()
                    t1 = time.perf_counter()
                    _, _, inf = eng.solve(pp)
                    ts.append(time.perf_counter() - t1)
                rec[tag] = {"seconds": float(np.mean(ts)), "status": inf.status, "iterations": inf.iterations,
                            "iterations_fp64": inf.iterations_fp64, "rel_kkt": inf.rel_kkt,
                            "objective": inf.objective, "parallel_groups": inf.parallel_groups}
        out[key] = rec
    return out


def mlp_perf(args):
    """Throughput of the warm-start network's hand-written GEMM on a few
    shapes and of one per-variable training step (16 -> 3 x 512 -> 8,
    8192-sample batches); one JSON line."""
    import numpy as np

    from nirnaya_b200 import mlp

    peak = 1590.0
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except Exception:
        pass
    out = {"peak_bf16_tflops": peak, "gemm": {}}
    with mlp.Mlp(16, 8, width=512, depth=3, seed=0) as net:
        for shape in ((8192, 8192, 8192), (4096, 4096, 4096), (8192, 512, 512), (256, 512, 52000)):
            tf = net.gemm_tflops(*shape, reps=10)
            out["gemm"]["x".join(map(str, shape))] = {"tflops": tf, "frac": tf / peak}
        rng = np.random.default_rng(0)
        net.set_data(rng.normal(size=(262144, 16)).astype(np.float32), rng.normal(size=(262144, 8)).astype(np.float32))
        net.train(2, 8192)
        us, fl = net.step_stats()
    out["train_step"] = {"us": us, "gflop": fl / 1e9, "tflops": fl / (us * 1e-6) / 1e12}
    print(json.dumps(out))


def mps_read_bench(args):
    """Reads the workload's LP from an MPS file: libnir_mps.so with all host
    threads (W warm-up reads, K timed reads) and with one thread, against
    the reference's MpsReader::read (oracle/_ref, one read) on the same
    file, with a bit-for-bit comparison of the models.  The file is written
    once by nir_mps_write (the reference writer's bytes) under --mps-dir.
    One JSON line; wall-clock timing (host-only work)."""
    import numpy as np

    from nirnaya_b200 import lp as L
    from nirnaya_b200 import mps
    from oracle import ffi

    wl = WORKLOADS[args.workload]
    os.makedirs(args.mps_dir, exist_ok=True)
    path = os.path.join(args.mps_dir, wl["label"] + ".mps")
    lp = L.generate(wl["kind"], wl["seed"], **wl["kw"])
    t0 = time.perf_counter()
    mps.write_mps(path, lp, name=wl["label"])
    t_write = time.perf_counter() - t0
    size = os.path.getsize(path)
    nproc = os.cpu_count() or 1
    for _ in range(args.warmup):
        mps.read_mps(path)
    times, phases = [], None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        m = mps.read_mps(path)
        times.append(time.perf_counter() - t0)
        phases = m.timings
    t = float(np.median(times))
    by_threads = {}
    for th in sorted({1, 2, 4, nproc}):
        if th > nproc:
            continue
        best = None
        for _ in range(2):
            t0 = time.perf_counter()
            mps.read_mps(path, threads=th)
            d = time.perf_counter() - t0
            best = d if best is None else min(best, d)
        by_threads[str(th)] = best
    t1 = by_threads["1"]
    ref = None
    if ffi.ref_available():
        t0 = time.perf_counter()
        rl, rs, rvt, _ = ffi.ref_read_mps_full(path)
        tr = time.perf_counter() - t0
        ours, _ = m.internal_min()
        same = rs == m.sense and np.array_equal(rvt, m.vartype) and all(
            np.array_equal(getattr(ours, k).view(np.uint8), getattr(rl, k).view(np.uint8))
            for k in ("col_start", "row_index", "value", "cost", "collo", "colup", "rowlo", "rowup"))
        ref = {"seconds": tr, "MB_per_s": size / tr / 1e6, "cores": 1, "kind": "reference",
               "sample": "sov::MpsReader::read + Model::validate (+ to_internal_min) of the whole file, once",
               "models_bit_identical": bool(same)}
    line = {"metric": "mps_read_throughput", "value": size / t / 1e6, "unit": "MB/s", "higher_is_better": True,
            "steps": args.steps, "warmup": args.warmup, "seconds": t,
            "data": "synthetic (seeded generator, include/nir_lpgen.h), written as MPS",
            "config": {"workload": wl["label"] + ".mps", "bytes": size, "rows": lp.nrow, "cols": lp.ncol,
                       "nnz": lp.nnz, "threads": nproc},
            "phases_s": phases, "single_thread": {"seconds": t1, "MB_per_s": size / t1 / 1e6},
            "seconds_by_threads": by_threads,
            "writer_seconds": t_write, "reference": ref,
            "speedup_vs_reference": (ref["seconds"] / t) if ref else None}
    os.remove(path)  # a few hundred MB: not left in the tree
    print(json.dumps(line))


def host_path_bench(args):
    """The host steps of the CLI path around PdhgSolver::solve
    (include/sov/solver.hpp:135-313): read the MPS file, presolve, scale;
    then, on a solution (the reduced model's bound-clipped midpoint, put
    back by postsolve), verify it in double-double and write the SOL file.
    This package's libraries (all host threads; each step's best of three
    runs after one warm-up) against the reference's own code (oracle/_ref,
    one thread, as it runs; each step once), with a bit-for-bit comparison of the scaled model handed to
    PDHG and of the verification report.  One JSON line; wall-clock timing
    (host-only work)."""
    import numpy as np

    from nirnaya_b200 import facade
    from nirnaya_b200 import lp as L
    from nirnaya_b200 import mps
    from oracle import ffi

    wl = WORKLOADS[args.workload]
    os.makedirs(args.mps_dir, exist_ok=True)
    path = os.path.join(args.mps_dir, wl["label"] + ".mps")
    lp = L.generate(wl["kind"], wl["seed"], **wl["kw"])
    mps.write_mps(path, lp, name=wl["label"])

    def solution(lpm, pre):
        lo = np.where(np.isfinite(pre.reduced.collo), pre.reduced.collo, -1.0)
        up = np.where(np.isfinite(pre.reduced.colup), pre.reduced.colup, 1.0)
        return pre.postsolve(0.5 * (lo + up))

    def ours():
        t = {}
        t0 = time.perf_counter()
        m = mps.read_mps(path)
        t["read"] = time.perf_counter() - t0
        lpm, _ = m.internal_min()
        t0 = time.perf_counter()
        pre = facade.presolve(lpm, m.vartype)
        t["presolve"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        sc = facade.scale(pre.reduced, pre.vartype)
        t["scale"] = time.perf_counter() - t0
        x = solution(lpm, pre)
        t0 = time.perf_counter()
        obj = mps.eval_objective(lpm, x)
        rep = mps.verify_solution(lpm, x, obj, 1e-6, m.vartype)
        t["verify"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        mps.write_sol(path + ".ours.sol", x, "optimal", obj, 0.0)  # the file's names are C<j>
        t["write_sol"] = time.perf_counter() - t0
        return t, sc, x, obj, rep

    ours()
    runs = [ours() for _ in range(3)]
    t_ours = {k: min(r[0][k] for r in runs) for k in runs[0][0]}  # each step's best of three
    _, sc, x, obj, rep = runs[-1]
    ref = None
    if ffi.ref_available():
        t = {}
        t0 = time.perf_counter()
        rl, _, rvt, _ = ffi.ref_read_mps_full(path)
        t["read"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        rp = ffi.ref_presolve(rl, rvt)
        t["presolve"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        rs = ffi.ref_scale(rp["reduced"], rp["vartype"])
        t["scale"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        rrep = ffi.ref_verify_full(rl, x, obj, 1e-6, vartype=rvt)
        t["verify"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        ffi.ref_write_sol(rl, None, 0, obj, 0.0, x, path + ".ref.sol")
        t["write_sol"] = time.perf_counter() - t0
        same = (sc.active == rs["active"] and np.array_equal(sc.R, rs["R"]) and np.array_equal(sc.C, rs["C"]) and
                all(np.array_equal(getattr(sc.lp, k).view(np.uint8), rs[k].view(np.uint8))
                    for k in ("cost", "collo", "colup", "value", "rowlo", "rowup")))
        same_rep = all(np.float64(rep[k]).tobytes() == np.float64(rrep[k]).tobytes()
                       for k in ("max_bound_viol", "max_row_viol", "max_int_viol", "computed_obj", "obj_rel_err"))
        with open(path + ".ours.sol", "rb") as a, open(path + ".ref.sol", "rb") as b:
            same_sol = a.read() == b.read()
        ref = {"seconds": t, "total": sum(t.values()), "cores": 1, "kind": "reference",
               "sample": "MpsReader::read, Presolver::presolve (level 2), scale_model, verify_solution, "
                         "SolIo::write_sol, once each",
               "scaled_model_bit_identical": bool(same), "verification_bit_identical": bool(same_rep),
               "sol_bytes_identical": bool(same_sol)}
    size = os.path.getsize(path)
    for suffix in (".ours.sol", ".ref.sol", ""):  # a few hundred MB: not left in the tree
        if os.path.exists(path + suffix):
            os.remove(path + suffix)
    total = sum(t_ours.values())
    print(json.dumps({"metric": "host_path_seconds", "value": total, "unit": "s", "higher_is_better": False,
                      "data": "synthetic (seeded generator, include/nir_lpgen.h), written as MPS",
                      "config": {"workload": wl["label"] + ".mps", "bytes": size,
                                 "threads": os.cpu_count(), "reduced": [sc.lp.nrow, sc.lp.ncol, sc.lp.nnz]},
                      "seconds": t_ours, "reference": ref,
                      "speedup_vs_reference": (ref["total"] / total) if ref else None}))


def verify_batch_bench(args):
    """C3's 256 solution checks (verify_solution, src/io/sol_io.hpp:25-106)
    on the device (nir_pdhg_batch_verify), against this package's host check
    and the reference's.  Two device figures:
      - in place: the points a short batch solve left on the device, so the
        call is the three kernels plus 2 KB of claimed objectives in and the
        reports out;
      - from the host: seeded points near each instance's construction point,
        copied in by the call (the end-to-end figure).
    Every device report is compared with the host check's, bit for bit."""
    import numpy as np

    from nirnaya_b200 import batch as B
    from nirnaya_b200 import mps, pdhg

    wl = WORKLOADS["c3"]
    lps = batch_instances(wl)
    rng = np.random.default_rng(7)
    xs = [lp.x0 + 1e-7 * rng.normal(size=lp.ncol) for lp in lps]
    claimed = np.array([float(np.dot(lp.cost, x)) + lp.obj_offset for lp, x in zip(lps, xs)])
    tol = 1e-6
    t0 = time.perf_counter()
    host = [mps.verify_solution(lp, x, float(c), tol) for lp, x, c in zip(lps, xs, claimed)]
    t_host = time.perf_counter() - t0
    # the same checks spread over all host threads, one instance per task
    # (the library call releases the interpreter lock)
    from concurrent.futures import ThreadPoolExecutor

    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as pool:
        pooled = list(pool.map(lambda a: mps.verify_solution(a[0], a[1], float(a[2]), tol, threads=1),
                               zip(lps, xs, claimed)))
    t_host_pool = time.perf_counter() - t0
    if any(p != h for p, h in zip(pooled, host)):
        raise RuntimeError("the host check differs between thread layouts")
    t_ref = None  # the cpu_baseline leg: the reference's own check, built from its sources
    try:
        from oracle import ffi

        t0 = time.perf_counter()
        for lp, x, c in zip(lps, xs, claimed):
            ffi.ref_verify_full(lp, x, float(c), tol)
        t_ref = time.perf_counter() - t0
    except Exception as e:  # the reference library is built only where its sources are
        print(f"reference check not timed: {e}", file=sys.stderr)

    def same(a, b):
        return all(np.float64(a[k]).view(np.uint64) == np.float64(b[k]).view(np.uint64)
                   if isinstance(a[k], float) else a[k] == b[k] for k in a)

    with B.BatchEngine(lps, 0) as eng:
        for _ in range(args.warmup):
            dev = eng.verify(xs, claimed, tol)
        e2e = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            dev = eng.verify(xs, claimed, tol)
            e2e.append(time.perf_counter() - t0)
        from_host_ok = all(same(d, h) for d, h in zip(dev, host))
        res, _ = eng.solve(pdhg.default_params(max_iters=64, tol=0.0))
        solved_claimed = np.array([r[2].objective for r in res])
        for _ in range(args.warmup):
            eng.verify(None, solved_claimed, tol)
        with ClockSampler(0) as clk:
            resident = []
            for _ in range(args.steps):
                t0 = time.perf_counter()
                inplace = eng.verify(None, solved_claimed, tol)
                resident.append(time.perf_counter() - t0)
        in_place_ok = all(same(d, mps.verify_solution(lp, r[0], float(c), tol))
                          for d, lp, r, c in zip(inplace, lps, res, solved_claimed))
    nnz = sum(lp.nnz for lp in lps)
    m = sum(lp.nrow for lp in lps)
    n = sum(lp.ncol for lp in lps)
    alg = 12.0 * nnz + 38.0 * m + 40.0 * n
    t_dev = statistics.median(resident)
    peak, peak_kind = peaks()
    achieved = alg / t_dev / 1e9
    print(json.dumps({
        "metric": "C3 solution check: verify_solution for 256 instances",
        "value": t_dev, "unit": "s", "higher_is_better": False, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "dtype": "f64 (double-double sums)", "data": "synthetic (seeded generator)",
        "config": {"workload": wl["label"], "instances": len(lps), "nnz": nnz, "rows": m, "cols": n, "tol": tol,
                   "points": "in place: a 64-iteration batch solve's; from the host: x0 + 1e-7 N(0,1)",
                   "timing": "host clock around the synchronous call (median)"},
        "e2e": {"value": statistics.median(e2e), "unit": "s", "h2d_bytes_per_step": 8 * n + 8 * len(lps),
                "d2h_bytes_per_step": 48 * len(lps)},
        "host_check_s": t_host, "host_check_all_threads_s": t_host_pool, "host_threads": cores,
        "cpu_baseline": None if t_ref is None else {
            "value": t_ref, "unit": "s", "cores": 1, "kind": "reference",
            "sample": "the reference's verify_solution on all 256 instances, once, one after another"},
        "reports_bit_identical": {"from_host": from_host_ok, "in_place": in_place_ok},
        "gpu_launches": 3 * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "k_vfy_cols + k_vfy_rows + k_vfy_report, 12 B/nnz + 38 B/row "
                                                "+ 40 B/column over the call time",
                     "peak_kind": peak_kind},
        "clocks": clk.summary(),
    }), flush=True)


def reference_iterations(args):
    """Counts the reference PDHG's iterations to 1e-6 relative KKT on the
    workload: the bit-identical GPU restatement of its loop
    (NIR_ALGO_REFERENCE) with the KKT probe every 32 iterations, bounded by
    --ref-iterations and --ref-seconds; also reports where the reference's
    own stopping rule (max row violation <= 1e-6) fired.  One JSON line."""
    from nirnaya_b200 import lp as L
    from nirnaya_b200 import pdhg

    wl = WORKLOADS[args.workload]
    lp = L.generate(wl["kind"], wl["seed"], **wl["kw"])
    p = pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, max_iters=args.ref_iterations, tol=1e-6,
                            time_limit=args.ref_seconds)
    with pdhg.Engine(lp, 0) as eng:
        t0 = time.perf_counter()
        _, _, info = eng.solve(p)
        dt = time.perf_counter() - t0
    print(json.dumps({"workload": wl["label"], "iterations_to_1e-6_rel_kkt": info.iterations_to_tol,
                      "iterations_run": info.iterations, "status": pdhg.STATUS_NAMES.get(info.status),
                      "stopped_by_reference_rule": info.status == pdhg.OPTIMAL and info.iterations < args.ref_iterations,
                      "last_probe_rel_kkt": info.rel_kkt, "rel_primal": info.rel_primal, "rel_dual": info.rel_dual,
                      "rel_gap": info.rel_gap, "seconds": dt, "objective": info.objective}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--max-iters", type=int, default=1000000)
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="reference CPU sample: half of it at 1 thread, half at all host threads")
    ap.add_argument("--no-blocks", action="store_true",
                    help="c2: leave out the batch (c3), learned (c4), badly scaled (c5) and c1 figures")
    ap.add_argument("--c4-train", type=int, default=4096)
    ap.add_argument("--c4-test", type=int, default=512)
    ap.add_argument("--c4-pdhg", type=int, default=16)
    ap.add_argument("--c4-pdhg-iters", type=int, default=400000)
    ap.add_argument("--c4-epochs", type=int, default=4)
    ap.add_argument("--block-c4-train", type=int, default=512, help="c2 run's learned block: training instances")
    ap.add_argument("--block-c4-test", type=int, default=64, help="c2 run's learned block: held-out instances")
    ap.add_argument("--block-c4-pdhg", type=int, default=4, help="c2 run's learned block: plain-PDHG subset")
    ap.add_argument("--ref-iterations", type=int, default=0,
                    help="count the reference loop's iterations to its stopping rule (cap), then exit")
    ap.add_argument("--ref-seconds", type=float, default=600.0)
    ap.add_argument("--mlp-perf", action="store_true",
                    help="throughput of the warm-start network's GEMM and training step, then exit")
    ap.add_argument("--ncu-case", action="store_true",
                    help="one short solve (--ncu-iters iterations) of the workload for an ncu capture, then exit")
    ap.add_argument("--ncu-iters", type=int, default=1024)
    ap.add_argument("--ncu-precision", choices=["fp64", "mixed", "fp32"], default=None,
                    help="iterate precision of the ncu case (default: the workload's)")
    ap.add_argument("--ncu-cap", type=int, default=0,
                    help="warp row-block capacity of the ncu case (0: autotuned; the tuner times launches, "
                         "which a profiler that serialises every launch perturbs)")
    ap.add_argument("--mps-read", action="store_true",
                    help="MPS reader throughput on the workload written as an MPS file, then exit")
    ap.add_argument("--mps-dir", default=os.path.join(ROOT, "_bench_tmp"),
                    help="where --mps-read writes its input file")
    ap.add_argument("--verify-batch", action="store_true",
                    help="C3's 256 solution checks on the device against the host check and the reference's")
    ap.add_argument("--host-path", action="store_true",
                    help="the CLI's host steps around PDHG (read, presolve, scale, verify, write_sol) "
                         "against the reference's")
    ap.add_argument("--spmv-case", action="store_true",
                    help="cold-L2 times of the plain SpMV kernels of both layout families and of the row-less "
                         "gather ceilings on the workload's matrix (one JSON line), then exit")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.spmv_case:
        from nirnaya_b200 import lp as L
        from nirnaya_b200 import pdhg

        lp = L.generate(wl["kind"], wl["seed"], **wl["kw"])
        with pdhg.Engine(lp, 0) as eng:
            fig = spmv_figures(eng, lp, None, reps=10)
        peak, peak_kind = peaks()
        print(json.dumps({"workload": wl["label"], "nnz": lp.nnz, "hbm_peak_GBs": peak, "peak_kind": peak_kind,
                          "timing": "CUDA events on the engine's stream, L2 flushed (512 MB write) before each "
                                    "of 10 launches after one warm-up", "kernels": fig}))
        return
    if args.host_path:
        host_path_bench(args)
        return
    if args.verify_batch:
        verify_batch_bench(args)
        return
    if args.mps_read:
        mps_read_bench(args)
        return
    if args.ref_iterations > 0:
        reference_iterations(args)
        return
    if args.mlp_perf:
        mlp_perf(args)
        return
    if args.ncu_case:
        from nirnaya_b200 import lp as L
        from nirnaya_b200 import pdhg

        if args.ncu_precision:
            wl = dict(wl, precision={"fp64": 0, "mixed": 1, "fp32": 2}[args.ncu_precision])

        if wl.get("batch"):
            from nirnaya_b200 import batch as B

            with B.BatchEngine(batch_instances(wl)[:32], 0) as eng:
                eng.solve(pdhg.default_params(precision=wl["precision"], max_iters=args.ncu_iters, tol=0.0))
            return
        lp = L.generate(wl["kind"], wl["seed"], **wl["kw"])
        with pdhg.Engine(lp, 0) as eng:
            eng.solve(pdhg.default_params(precision=wl["precision"], max_iters=args.ncu_iters, tol=0.0,
                                          spmv_block_nnz=args.ncu_cap))
        return
    if args.impl == "reference":
        # the reference runs on the host cores of rank 0; the other ranks of a
        # torchrun launch have nothing to do and open no process group
        if int(os.environ.get("RANK", "0")) != 0:
            return
        from nirnaya_b200 import lp as L

        if wl.get("batch"):
            # the reference solves one model per call; its rate on the
            # median-size instance of the batch is reported, without a time
            # to tolerance (its iteration counts on these are not recorded)
            lps = batch_instances(wl)
            lp = sorted(lps, key=lambda q: q.nnz)[len(lps) // 2]
            res = cpu_baseline(lp, wl["label"] + ":median", seconds=args.cpu_seconds)
            if res is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_nirnaya.so was not built "
                                  "from the reference sources"}))
                return
            print(json.dumps({"impl": "reference", "metric": METRIC, "value": None, "unit": "s",
                              "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": None,
                              "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic (seeded generator, include/nir_lpgen.h)",
                              "config": {"workload": wl["label"], "tol": 1e-6, "threads": res["cores"]},
                              "cpu_baseline": res,
                              "e2e": {"value": None, "unit": "s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
            return
        lp = L.generate(wl["kind"], wl["seed"], **wl["kw"])
        # one sample of at least 5 s per thread count, whatever --steps says:
        # the reference runs for hours to this tolerance, so its time is the
        # iteration count it needs over its measured rate
        res = cpu_baseline(lp, wl["label"], seconds=max(10.0, args.cpu_seconds))
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_nirnaya.so was not built "
                              "from the reference sources"}))
            return
        v = res["value"]
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None if v is None else 1000 * v,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator, include/nir_lpgen.h)",
                "config": {"workload": wl["label"], "tol": 1e-6, "threads": res["cores"]},
                "lower_bound": bool(res.get("lower_bound")),
                "per_iteration_s": 1.0 / res["iterations_per_s"],
                "how": "value = iterations the reference algorithm needs to 1e-6 relative KKT on this instance "
                       "(counted with its bit-identical GPU restatement; a lower bound when that count did not "
                       "reach the tolerance) / the reference's own measured iterations per second here",
                "cpu_baseline": res,
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    rank, world, local = dist_setup(args.gpus)
    try:
        run_arm(args, wl, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            if dist.is_initialized():
                dist.destroy_process_group()


def run_arm(args, wl, rank, world, local):
    """Our arm: one JSON line from rank 0."""
    if wl.get("learned"):
        if rank == 0:
            run_learned(args, world)
        return
    if wl.get("batch"):
        r = run_batch_ours(args, rank, world, local)
        if rank == 0:
            print(json.dumps(batch_line(args, r, world)))
        return
    r = run_ours(args, rank, world, local)
    blocks = {}
    if args.workload == "c2" and world == 1 and not args.no_blocks:
        # the other configurations' headline figures, in the same run
        blocks = run_blocks(args, local)
    if rank != 0:
        return
    from nirnaya_b200 import pdhg

    lp, infos = r["lp"], r["infos"]
    last = infos[-1]
    peak, peak_kind = peaks()
    kt = r["kt"]
    # dominant kernel of the solve: steady-state launch time x launches, per
    # kernel and precision (the first phase, then the FP64 polish)
    it64 = last["iterations_fp64"]
    it_first = last["iterations"] - it64
    first = WORKLOADS[args.workload]["precision"]
    kernels = {}
    phases = [(first, it_first)] if first != pdhg.PREC_FP64 else []
    phases.append((pdhg.PREC_FP64, it64 if first != pdhg.PREC_FP64 else last["iterations"]))
    for prec, its in phases:
        if its <= 0 or prec not in kt:
            continue
        vw, xw = {pdhg.PREC_FP64: (8, 8), pdhg.PREC_MIXED: (4, 8), pdhg.PREC_FP32: (4, 4)}[prec]
        tv = "double" if vw == 8 else "float"
        tx = "double" if xw == 8 else "float"
        p_us, d_us, pair_us = kt[prec]
        for kname, us, alg in (("k_primal", p_us, primal_bytes(lp, xw, vw)), ("k_dual", d_us, dual_bytes(lp, xw, vw))):
            kernels[f"{kname}<{tv},{tx}>"] = {
                "launch_us": us, "launches": its, "share_s": us * its * 1e-6,
                "algorithmic_bytes_per_launch": alg, "achieved_GBs": alg / (us * 1e-6) / 1e9,
                "pair_us": pair_us}
    if kernels:
        dom_name, dom = max(kernels.items(), key=lambda kv: kv[1]["share_s"])
    else:
        dom_name, dom = "none", {"achieved_GBs": None, "algorithmic_bytes_per_launch": None, "launch_us": None}
    achieved = dom["achieved_GBs"]
    wl = WORKLOADS[args.workload]
    dom_family = "cta" if (r["lay"].block_nnz_at if "primal" in dom_name else r["lay"].block_nnz) > 256 else "warp"
    traffic = committed_traffic(f"{dom_name}[{dom_family}]:{wl['label']}")
    # the reference on the host cores: rank 0 at N=1 only
    cpu = cpu_baseline(lp, wl["label"], seconds=args.cpu_seconds) if world == 1 else None
    fp64 = r["fp64"]
    if cpu and fp64 and fp64["iterations"]:
        # seconds per iteration: the reference on the host cores vs the FP64 GPU solve
        gpu_it_s = fp64["seconds"] / fp64["iterations"]
        cpu["per_iteration_s"] = 1.0 / cpu["iterations_per_s"]
        cpu["gpu_fp64_per_iteration_s"] = gpu_it_s
        cpu["per_iteration_ratio_fp64"] = cpu["per_iteration_s"] / gpu_it_s
    line = {
        "metric": METRIC,
        "value": r["ms"] / 1000.0,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": r["ms"],
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 values + f64 iterates, f64 polish" if first == pdhg.PREC_MIXED else
                 ("f64" if first == pdhg.PREC_FP64 else "f32"),
        "data": "synthetic (seeded generator, include/nir_lpgen.h)",
        "config": {"workload": wl["label"], "m": lp.nrow, "n": lp.ncol, "nnz": lp.nnz, "tol": 1e-6,
                   "algorithm": "pdlp (restarted reflected Halpern PDHG)",
                   "precision": "mixed: fp32 matrix values with fp64 iterates, then fp64 values (polish)",
                   "block_nnz": r["lay"].block_nnz,
                   "parallelism": f"replicas x{world}" if world > 1 else "single gpu",
                   "l2": "flushed (2x L2 write) before every solve; inside a solve the working set stays resident"},
        "status": last["status"],
        "iterations": last["iterations"],
        "iterations_fp64": last["iterations_fp64"],
        "fp64_iteration_share": (last["iterations_fp64"] / last["iterations"]) if last["iterations"] else None,
        "rel_kkt": last["rel_kkt"],
        "objective": last["objective"],
        "setup_s": last["setup_seconds"],
        "fp64_solve": None if fp64 is None else {
            **fp64, "mixed_speedup": (fp64["seconds"] / (r["ms"] / 1000.0)) if fp64["seconds"] else None,
            "note": "the same workload with FP64 values and iterates throughout, one solve with a cold L2, "
                    "host clock around the synchronous call"},
        "e2e": {"value": r["e2e"], "unit": "s", "h2d_bytes_per_step": lp.host_bytes(),
                "d2h_bytes_per_step": 8 * (lp.ncol + lp.nrow)},
        "gpu_launches": r["launches"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": f"{dom_name} (fused SpMV + update over "
                               f"{'CTA blocks' if dom_family == 'cta' else 'warp row blocks'}), "
                               "dominant by time in the solve",
                     "algorithmic_bytes_per_launch": dom["algorithmic_bytes_per_launch"],
                     "launch_us": dom["launch_us"],
                     "timing": "steady state: 100 back-to-back launches on the solved state, CUDA events on "
                               "the engine's stream (nir_pdhg_time_iteration)",
                     "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "kernels": kernels,
                     "kernel_share_sum_s": sum(k["share_s"] for k in kernels.values()),
                     "spmv_cold": r["spmv"]},
        "cpu_baseline": cpu,
        "clocks": r["clocks"],
    }
    line.update(blocks)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
