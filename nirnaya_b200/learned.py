"""Learned warm start for a fixed-structure LP family.

The family (the blending family of include/nir_lpgen.h, kind
NIR_GEN_BLEND_FAMILY): one constraint matrix A fixed by `family_seed`;
instance k multiplies the demand rows' lower bounds by factors
f ~ clip(1 + 0.2 N(0,1), 0.1, 1.9) and the costs by g ~ clip(1 + 0.1 N(0,1),
0.5, 1.5), drawn from a generator seeded with k (x0 of the base construction
stays feasible, every cost keeps its sign).

`WarmStart` holds two multilayer perceptrons (libnir_mlp.so: hand-written
BF16 tensor-core training and inference kernels) applied per column and per
row with shared weights, trained only on solutions the PDLP engine
generates for training instances.  Its prediction seeds the engine
(x_init, y_init, omega_init); `evaluate` solves each held-out instance cold
and warm to the same relative-KKT tolerance: a warm result is accepted only
when its solve reaches that tolerance, otherwise the cold result stands
(the cold-start PDLP is both the fallback and the arbiter).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import lp as L
from . import mlp as MLP
from . import pdhg as P


class BlendFamily:
    """Instances of the fixed-matrix blending family, as vectors over one
    base LP (so a solver handle can keep A resident and swap vectors)."""

    def __init__(self, m=20000, n=50000, nnz=400000, family_seed=0):
        base = L.generate(L.BLEND_FAMILY, 0, m=m, n=n, target_nnz=nnz, family_seed=family_seed)
        f0 = base.extra["demand_factors"]
        g0 = base.extra["cost_factors"]
        self.nd = len(f0)
        self.base = base
        self.m, self.n = base.nrow, base.ncol
        self.rowlo0 = base.rowlo.copy()
        self.rowlo0[: self.nd] /= f0
        self.cost0 = base.cost / g0

    def factors(self, seed: int):
        rng = np.random.default_rng([0xC4, int(seed)])
        f = np.clip(1.0 + 0.2 * rng.standard_normal(self.nd), 0.1, 1.9)
        g = np.clip(1.0 + 0.1 * rng.standard_normal(self.n), 0.5, 1.5)
        return f, g

    def vectors(self, f, g):
        rowlo = self.rowlo0.copy()
        rowlo[: self.nd] *= f
        return rowlo, self.cost0 * g

    def instance(self, seed: int) -> L.LP:
        """The instance as a standalone LP (for checks against the oracle)."""
        f, g = self.factors(seed)
        rowlo, cost = self.vectors(f, g)
        b = self.base
        return L.LP(b.nrow, b.ncol, b.col_start, b.row_index, b.value, cost, b.collo, b.colup, rowlo, b.rowup,
                    b.obj_offset)


@dataclass
class Solutions:
    seeds: np.ndarray             # N instance seeds
    x: np.ndarray                 # N x n
    y: np.ndarray                 # N x m
    omega: np.ndarray             # N
    iterations: np.ndarray        # N
    seconds: np.ndarray           # N
    status: np.ndarray            # N


def solve_family(fam: BlendFamily, seeds, params: P.Params | None = None, device=0, engine: P.Engine | None = None):
    """PDLP solutions of the family's instances (A stays resident)."""
    own = engine is None
    eng = engine or P.Engine(fam.base, device)
    p = params or P.default_params()
    N = len(seeds)
    out = Solutions(np.asarray(list(seeds), np.int64), np.zeros((N, fam.n), np.float32),
                    np.zeros((N, fam.m), np.float32), np.zeros(N), np.zeros(N, np.int64), np.zeros(N),
                    np.zeros(N, np.int32))
    try:
        for i, s in enumerate(seeds):
            f, g = fam.factors(s)
            rowlo, cost = fam.vectors(f, g)
            eng.update_vectors(cost=cost, rowlo=rowlo)
            t0 = time.perf_counter()
            x, y, info = eng.solve(p)
            out.seconds[i] = time.perf_counter() - t0
            out.x[i], out.y[i] = x, y
            out.omega[i] = info.primal_weight
            out.iterations[i] = info.iterations
            out.status[i] = info.status
    finally:
        if own:
            eng.close()
    return out


def _atx(lp: L.LP, x: np.ndarray) -> np.ndarray:
    """A x for the LP's CSC matrix."""
    cols = np.repeat(np.arange(lp.ncol), np.diff(lp.col_start))
    return np.bincount(lp.row_index, weights=lp.value * x[cols], minlength=lp.nrow)


def _aty(lp: L.LP, y: np.ndarray) -> np.ndarray:
    """A' y for the LP's CSC matrix."""
    cols = np.repeat(np.arange(lp.ncol), np.diff(lp.col_start))
    return np.bincount(cols, weights=lp.value * y[lp.row_index], minlength=lp.ncol)


COL_FEATURES = 16
ROW_FEATURES = 16


class WarmStart:
    """Per-variable networks with shared weights.

    One MLP maps each column's local features to x_j / u_j, another maps
    each row's to its dual value (standardised per row); every instance
    therefore contributes n column samples and m row samples, which is what
    lets 3 x 512 networks generalise from a few thousand instances.  Column
    features: the cost factor and the perturbed cost, the reduced cost at
    the training-mean duals, the training-mean value and how often the
    column sat at each bound, the demand perturbation of the rows it serves
    (weighted by its coefficients), its bound.  Row features: whether it is
    a demand row and its factor, the training-mean dual, how often the row
    was tight, its slack at the training-mean primal under the perturbed
    bound, and the cost perturbation of its columns.  The primal weight is
    the training geometric mean (the exact final weight measured no faster
    than the engine's own initial estimate).
    """

    def __init__(self, fam: BlendFamily, width=512, depth=3, seed=0, lr=1e-3, device=0):
        self.fam = fam
        self.col_net = MLP.Mlp(COL_FEATURES, 8, width=width, depth=depth, seed=seed, lr=lr, device=device)
        self.row_net = MLP.Mlp(ROW_FEATURES, 8, width=width, depth=depth, seed=seed + 1, lr=lr, device=device)
        w = np.zeros(8, np.float32)
        w[0] = 1.0
        self.col_net.set_output_weights(w)
        self.row_net.set_output_weights(w)
        b = fam.base
        self.u = b.colup.copy()
        self.cols = np.repeat(np.arange(fam.n), np.diff(b.col_start))
        dem = b.row_index < fam.nd
        self.dem_w = np.bincount(self.cols[dem], weights=b.value[dem], minlength=fam.n)  # sum of demand coefficients
        self.row_abs = np.bincount(b.row_index, weights=np.abs(b.value), minlength=fam.m)
        # the two per-instance aggregations of the features as fixed sparse
        # operators (built once): demand perturbation per column and cost
        # perturbation per row
        import scipy.sparse as sp

        self._dem_t = sp.csr_matrix((b.value[dem], (self.cols[dem], b.row_index[dem])), shape=(fam.n, fam.nd))
        self._abs_a = sp.csr_matrix((np.abs(b.value), (b.row_index, self.cols)), shape=(fam.m, fam.n))
        self.device = device
        self._dev = None  # the features on the device (MLP.BlendFeatures), built after a fit
        self._affine = False  # the networks' output maps for device_out are set
        self.fitted = False

    # ---- statistics of the training solutions
    def _stats(self, sol: Solutions):
        fam = self.fam
        self._colF = self._rowF = None
        self._affine = False
        if self._dev is not None:
            self._dev.close()
            self._dev = None
        ok = sol.status == P.OPTIMAL
        X = sol.x[ok].astype(np.float64)
        Y = sol.y[ok].astype(np.float64)
        u = self.u
        self.xbar = X.mean(axis=0)
        self.p_up = (X >= u - 1e-6 * (1 + u)).mean(axis=0)
        self.p_zero = (X <= 1e-6).mean(axis=0)
        self.ybar = Y.mean(axis=0)
        self.ysd = np.maximum(Y.std(axis=0), 1e-6 + 1e-3 * np.abs(self.ybar))
        self.p_tight = (np.abs(Y) > 1e-9 * (1 + np.abs(Y).max())).mean(axis=0)
        self.atybar = _aty(fam.base, self.ybar)
        self.axbar = _atx(fam.base, self.xbar)
        self.cscale = np.abs(fam.cost0).mean() + 1e-30
        b = fam.base
        self.bscale = np.where(np.isfinite(fam.rowlo0), np.abs(fam.rowlo0), np.abs(b.rowup))
        self.bscale = np.where(np.isfinite(self.bscale), self.bscale, 1.0) + 1e-9
        self.log_omega = float(np.mean(np.log(np.maximum(sol.omega[ok], 1e-30))))

    # ---- features of one instance
    def _col_base(self) -> np.ndarray:
        """The instance-independent column features (built once per fit)."""
        if getattr(self, "_colF", None) is None:
            fam = self.fam
            F = np.zeros((fam.n, COL_FEATURES), np.float32)
            F[:, 3] = self.xbar / self.u
            F[:, 4] = self.p_up
            F[:, 5] = self.p_zero
            F[:, 7] = self.u / 10.0
            F[:, 8] = fam.cost0 / self.cscale
            F[:, 9] = 1.0
            self._colF = F
        return self._colF

    def _row_base(self) -> np.ndarray:
        """The instance-independent row features (built once per fit)."""
        if getattr(self, "_rowF", None) is None:
            fam = self.fam
            F = np.zeros((fam.m, ROW_FEATURES), np.float32)
            F[: fam.nd, 0] = 1.0
            F[:, 2] = self.ybar / self.ysd
            F[:, 3] = self.p_tight
            F[:, 7] = 1.0
            self._rowF = F
        return self._rowF

    def col_features(self, f, g) -> np.ndarray:
        fam = self.fam
        c = fam.cost0 * g
        F = self._col_base().copy()
        dpert = self._dem_t @ (f - 1.0)
        F[:, 0] = (g - 1.0) / 0.1
        F[:, 1] = c / self.cscale
        F[:, 2] = (c - self.atybar) / self.cscale
        F[:, 6] = dpert / np.maximum(self.dem_w, 1e-12) / 0.2
        return F

    def row_features(self, f, g) -> np.ndarray:
        fam, b = self.fam, self.fam.base
        F = self._row_base().copy()
        nd = fam.nd
        rowlo = fam.rowlo0.copy()
        rowlo[:nd] *= f
        gpert = self._abs_a @ (g - 1.0)
        F[:nd, 1] = (f - 1.0) / 0.2
        slack_lo = np.where(np.isfinite(rowlo), self.axbar - rowlo, 0.0)
        slack_up = np.where(np.isfinite(b.rowup), b.rowup - self.axbar, 0.0)
        F[:, 4] = slack_lo / self.bscale
        F[:, 5] = slack_up / self.bscale
        F[:, 6] = gpert / np.maximum(self.row_abs, 1e-12) / 0.1
        return F

    def fit(self, sol: Solutions, epochs=20, batch=1024, cols_per_instance=4096, rows_per_instance=2048,
            seed=0) -> dict:
        fam = self.fam
        self._stats(sol)
        rng = np.random.default_rng(seed)
        ok = np.flatnonzero(sol.status == P.OPTIMAL)
        nc = min(cols_per_instance, fam.n)
        nr = min(rows_per_instance, fam.m)
        XC = np.zeros((len(ok) * nc, COL_FEATURES), np.float32)
        TC = np.zeros((len(ok) * nc, 8), np.float32)
        XR = np.zeros((len(ok) * nr, ROW_FEATURES), np.float32)
        TR = np.zeros((len(ok) * nr, 8), np.float32)
        for t, i in enumerate(ok):
            f, g = fam.factors(sol.seeds[i])
            jc = rng.choice(fam.n, size=nc, replace=False) if nc < fam.n else np.arange(fam.n)
            ir = rng.choice(fam.m, size=nr, replace=False) if nr < fam.m else np.arange(fam.m)
            XC[t * nc:(t + 1) * nc] = self.col_features(f, g)[jc]
            TC[t * nc:(t + 1) * nc, 0] = sol.x[i, jc] / self.u[jc]
            XR[t * nr:(t + 1) * nr] = self.row_features(f, g)[ir]
            TR[t * nr:(t + 1) * nr, 0] = (sol.y[i, ir] - self.ybar[ir]) / self.ysd[ir]
        self.col_net.set_data(XC[: len(XC) // 8 * 8], TC[: len(TC) // 8 * 8])
        self.row_net.set_data(XR[: len(XR) // 8 * 8], TR[: len(TR) // 8 * 8])
        lc = self.col_net.train(epochs, batch)
        lr = self.row_net.train(epochs, batch)
        self.fitted = True
        return {"col_loss": lc, "row_loss": lr, "col_samples": len(XC), "row_samples": len(XR)}

    def device_features(self):
        """The feature builder on the device (the same features as
        col_features / row_features, include/nir_mlp.h), created on first
        use after a fit; None when the sizes are not multiples of 8 (the
        networks take whole groups of 8 samples from the device)."""
        fam = self.fam
        if fam.n % 8 or fam.m % 8:
            return None
        if self._dev is None:
            b = fam.base
            dt, aa = self._dem_t, self._abs_a
            self._dev = MLP.BlendFeatures(dict(
                n=fam.n, m=fam.m, nd=fam.nd, nf=COL_FEATURES, col_template=self._col_base(),
                row_template=self._row_base(), cost0=fam.cost0, atybar=self.atybar, dem_w=self.dem_w,
                cscale=self.cscale, dem_rp=dt.indptr.astype(np.int64), dem_ci=dt.indices, dem_val=dt.data,
                rowlo0=fam.rowlo0, rowup=b.rowup, axbar=self.axbar, bscale=self.bscale, row_abs=self.row_abs,
                abs_rp=aa.indptr.astype(np.int64), abs_ci=aa.indices, abs_val=aa.data), self.device)
        return self._dev

    def predict(self, f, g, on_device: bool = True, device_out: bool = False):
        """x0, y0, omega for one instance: the features built on the device
        (or, with on_device False or sizes the device path does not take,
        on the host), then one pass of each network.

        With device_out, x0 and y0 are the device addresses (int) of FP64
        vectors owned by the networks, valid until their next prediction,
        which Engine.solve takes as its start with no trip through the host;
        their values are those of the host form bit for bit."""
        dev = self.device_features() if (on_device or device_out) else None
        if device_out:
            if dev is None:
                raise ValueError("device_out needs the device features (n and m multiples of 8)")
            if not self._affine:
                # x0 = u * clip(p, 0, 1); y0 = ybar + ysd * p
                self.col_net.set_affine(self.fam.n, 0, 0.0, 1.0, scale=self.u)
                self.row_net.set_affine(self.fam.m, 0, scale=self.ysd, shift=self.ybar)
                self._affine = True
            col, row = dev.build(f, g)
            x0 = self.col_net.predict_device_affine(col, self.fam.n)
            y0 = self.row_net.predict_device_affine(row, self.fam.m)
            return x0, y0, float(np.exp(self.log_omega))
        if dev is not None:
            col, row = dev.build(f, g)
            xc = self.col_net.predict_device(col, self.fam.n)[:, 0].astype(np.float64)
            yr = self.row_net.predict_device(row, self.fam.m)[:, 0].astype(np.float64)
        else:
            xc = self.col_net.predict(self.col_features(f, g))[:, 0].astype(np.float64)
            yr = self.row_net.predict(self.row_features(f, g))[:, 0].astype(np.float64)
        x = np.clip(xc, 0.0, 1.0) * self.u
        y = self.ybar + self.ysd * yr
        return x, y, float(np.exp(self.log_omega))

    def close(self):
        if self._dev is not None:
            self._dev.close()
            self._dev = None
        self.col_net.close()
        self.row_net.close()


@dataclass
class Evaluation:
    cold_iterations: np.ndarray
    warm_iterations: np.ndarray
    cold_seconds: np.ndarray
    warm_seconds: np.ndarray       # the warm solve, prediction excluded
    predict_seconds: float         # all held-out predictions
    accepted: np.ndarray           # warm solve reached the tolerance
    cold_objective: np.ndarray
    warm_objective: np.ndarray
    extra: dict = field(default_factory=dict)

    def summary(self) -> dict:
        acc = self.accepted
        # the result a user gets: warm when accepted, else cold after warm
        used_s = np.where(acc, self.warm_seconds, self.warm_seconds + self.cold_seconds)
        return {
            "instances": int(len(acc)),
            "accepted": int(acc.sum()),
            "cold_iterations_mean": float(self.cold_iterations.mean()),
            "warm_iterations_mean": float(self.warm_iterations.mean()),
            "cold_seconds_mean": float(self.cold_seconds.mean()),
            "warm_seconds_mean": float(used_s.mean() + self.predict_seconds / len(acc)),
            "warm_solve_seconds_mean": float(self.warm_seconds.mean()),
            "predict_seconds_mean": float(self.predict_seconds / len(acc)),
            "iteration_ratio": float(self.cold_iterations.mean() / max(self.warm_iterations.mean(), 1.0)),
            "time_ratio": float(self.cold_seconds.mean() / (used_s.mean() + self.predict_seconds / len(acc))),
            "max_rel_objective_gap": float(np.max(np.abs(self.warm_objective - self.cold_objective)
                                                  / (1.0 + np.abs(self.cold_objective)))),
            **self.extra,
        }


def evaluate(fam: BlendFamily, model: WarmStart, seeds, params: P.Params | None = None, device=0,
             engine: P.Engine | None = None) -> Evaluation:
    """Cold and warm PDLP solves of held-out instances to the same tolerance."""
    own = engine is None
    eng = engine or P.Engine(fam.base, device)
    p = params or P.default_params()
    N = len(seeds)
    ev = Evaluation(np.zeros(N, np.int64), np.zeros(N, np.int64), np.zeros(N), np.zeros(N), 0.0,
                    np.zeros(N, bool), np.zeros(N), np.zeros(N))
    # the start stays on the device from features to solve where it can
    dev_out = model.device_features() is not None
    if N:
        # one untimed prediction: the networks' first call sizes their
        # device buffers, a one-off cost of the handle, not of an instance
        model.predict(*fam.factors(seeds[0]), device_out=dev_out)
    try:
        for i, s in enumerate(seeds):
            f, g = fam.factors(s)
            rowlo, cost = fam.vectors(f, g)
            t0 = time.perf_counter()
            x0, y0, w0 = model.predict(f, g, device_out=dev_out)
            ev.predict_seconds += time.perf_counter() - t0
            eng.update_vectors(cost=cost, rowlo=rowlo)
            t0 = time.perf_counter()
            _, _, ci = eng.solve(p)
            ev.cold_seconds[i] = time.perf_counter() - t0
            t0 = time.perf_counter()
            _, _, wi = eng.solve(p, x_init=x0, y_init=y0, omega_init=w0)
            ev.warm_seconds[i] = time.perf_counter() - t0
            ev.cold_iterations[i], ev.warm_iterations[i] = ci.iterations, wi.iterations
            ev.cold_objective[i], ev.warm_objective[i] = ci.objective, wi.objective
            ev.accepted[i] = wi.status == P.OPTIMAL and wi.rel_kkt <= p.tol * 1.0000001
    finally:
        if own:
            eng.close()
    return ev
