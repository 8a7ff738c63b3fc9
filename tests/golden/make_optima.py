"""Generates the optimal objectives that pin PDLP parity at the workload sizes.

The reference's simplex does not finish these LPs in reasonable time (it
did not finish the 2,000 x 5,000 random LP in 600 s), so their optima come
from an independent LP solver: HiGHS through scipy.optimize.linprog, its
interior-point method followed by crossover (method "highs-ipm", presolve on).
The instances are the seeded generator's (include/nir_lpgen.h), so the
fixture stores only how to rebuild each one and its optimal objective:

  c1_random_eq_2000x5000       the full 2,000 x 5,000 random LP, seed 1
  c4_blend_member_900000       one held-out instance of the 20,000 x 50,000
                               blending family (family seed 0, instance seed
                               900000)
  c3_multiperiod_<i>           8 instances of the 256-instance multiperiod
                               batch (seed 1000 + i, m drawn as the batch draws
                               it; the first eight with m <= 4,000)
  c5_badly_scaled_5000x12000   the badly scaled construction (scales 10^U[-4,4],
                               half the columns duplicated with a 1e-9
                               perturbation) at 5,000 x 12,000, 100,000 nonzeros

Run once where scipy is present (it is slow: the badly scaled LP takes
about 12 minutes):

    python tests/golden/make_optima.py [name ...]

With --confirm, each named entry is solved again by HiGHS's dual simplex
(method "highs-ds"), a second algorithm, and the entry records that
objective beside the first; the two must agree to 1e-9 relative:

    python tests/golden/make_optima.py --confirm c5_badly_scaled_5000x12000

Objectives are stored as hex strings (exact) and as decimals (readable).
Several runs may fill the file at once: each merges its entry into it.
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

OUT = os.path.join(HERE, "optima.json")


def c3_members():
    """(index, m) of the first eight batch instances with m <= 4000, drawn as
    the c3 batch draws its sizes (log-uniform in [500, 20000], seed 1000)."""
    rng = np.random.default_rng(1000)
    ms = np.exp(rng.uniform(np.log(500), np.log(20000), 256)).astype(int)
    return [(i, int(m)) for i, m in enumerate(ms) if m <= 4000][:8]


def instances():
    """name -> (kind, seed, generator keyword arguments)."""
    from nirnaya_b200 import lp as L

    d = {
        "c1_random_eq_2000x5000": (L.RANDOM_EQ, 1, {}),
        "c4_blend_member_900000": (L.BLEND_FAMILY, 900000, {}),
        "c5_badly_scaled_5000x12000": (L.BADLY_SCALED, 1, {"m": 5000, "n": 12000, "target_nnz": 100000}),
    }
    for i, m in c3_members():
        d[f"c3_multiperiod_{i}"] = (L.MULTIPERIOD, 1000 + i, {"m": m})
    return d


def highs_optimum(lp, method="highs-ipm"):
    """Optimal objective (with the LP's offset) by HiGHS: IPM + crossover,
    or the dual simplex with method "highs-ds"."""
    import scipy
    import scipy.sparse as sp
    from scipy.optimize import linprog

    A = sp.csc_matrix((lp.value, lp.row_index, lp.col_start), shape=(lp.nrow, lp.ncol)).tocsr()
    fin = lambda v: np.isfinite(v) & (np.abs(v) < 1e20)  # noqa: E731  (src/core/types.hpp:49-51)
    rl, ru = lp.rowlo, lp.rowup
    eq = fin(rl) & fin(ru) & (rl == ru)
    ub, lb = ~eq & fin(ru), ~eq & fin(rl)
    A_ub = sp.vstack([A[ub], -A[lb]]).tocsr()
    b_ub = np.concatenate([ru[ub], -rl[lb]])
    bounds = np.stack([np.where(fin(lp.collo), lp.collo, -np.inf), np.where(fin(lp.colup), lp.colup, np.inf)], axis=1)
    t0 = time.time()
    r = linprog(lp.cost, A_ub=A_ub if A_ub.shape[0] else None, b_ub=b_ub if A_ub.shape[0] else None,
                A_eq=A[eq] if eq.any() else None, b_eq=rl[eq] if eq.any() else None, bounds=bounds,
                method=method, options={"presolve": True})
    if r.status != 0:
        raise RuntimeError(f"HiGHS did not solve the LP: {r.message}")
    return float(r.fun) + float(lp.obj_offset), time.time() - t0, f"scipy {scipy.__version__} linprog {method}"


def main():
    from nirnaya_b200 import build
    from nirnaya_b200 import lp as L

    build.build_lpgen()
    args = sys.argv[1:]
    confirm = "--confirm" in args
    want = set(a for a in args if a != "--confirm")
    for name, (kind, seed, kw) in instances().items():
        if want and name not in want:
            continue
        lp = L.generate(kind, seed, **kw)
        if confirm:
            out = json.load(open(OUT))
            e = out[name]
            obj, secs, how = highs_optimum(lp, "highs-ds")
            ref = float.fromhex(e["objective_hex"])
            rel = abs(obj - ref) / (1.0 + abs(ref))
            if rel > 1e-9:
                raise RuntimeError(f"{name}: the dual simplex gives {obj!r}, the fixture {ref!r} (rel {rel:.2e})")
            out = json.load(open(OUT))  # merged: several runs may fill it
            out[name]["confirmed"] = {"solver": how, "objective_hex": obj.hex(), "rel_diff": rel,
                                      "solver_seconds": round(secs, 1)}
            print(name, "confirmed", obj, f"rel {rel:.1e}", f"{secs:.1f}s", flush=True)
            with open(OUT, "w") as f:
                json.dump(out, f, indent=1, sort_keys=True)
            continue
        obj, secs, how = highs_optimum(lp)
        out = json.load(open(OUT)) if os.path.exists(OUT) else {}  # merged: several runs may fill it
        out[name] = {"kind": kind, "seed": seed, "kw": kw, "nrow": lp.nrow, "ncol": lp.ncol, "nnz": int(lp.nnz),
                     "objective": obj, "objective_hex": obj.hex(), "solver": how, "solver_seconds": round(secs, 1)}
        print(name, obj, f"{secs:.1f}s", flush=True)
        with open(OUT, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
