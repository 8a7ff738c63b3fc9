"""LP container in the reference's layout and the seeded instance generator.

`LP` holds exactly the arrays of the reference's internal-minimisation
`sov::Model` for a continuous LP (src/model/model.hpp:21-40): CSC matrix with
int64 column starts, int32 row indices and float64 values
(src/core/csc_matrix.hpp:18-23), cost, collo/colup, rowlo/rowup (+-inf or
|b| >= 1e20 meaning "no bound", src/core/types.hpp:49-51) and obj_offset.
`LP.view()` packs it into the `nir_lp_view` struct of include/nir_lp.h that
every C-ABI entry point takes.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


class NirLpView(C.Structure):
    _fields_ = [
        ("nrow", C.c_int32),
        ("ncol", C.c_int32),
        ("nnz", C.c_int64),
        ("col_start", C.POINTER(C.c_int64)),
        ("row_index", C.POINTER(C.c_int32)),
        ("value", C.POINTER(C.c_double)),
        ("cost", C.POINTER(C.c_double)),
        ("collo", C.POINTER(C.c_double)),
        ("colup", C.POINTER(C.c_double)),
        ("rowlo", C.POINTER(C.c_double)),
        ("rowup", C.POINTER(C.c_double)),
        ("obj_offset", C.c_double),
    ]


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class LP:
    nrow: int
    ncol: int
    col_start: np.ndarray          # int64[ncol+1]
    row_index: np.ndarray          # int32[nnz]
    value: np.ndarray              # float64[nnz]
    cost: np.ndarray               # float64[ncol]
    collo: np.ndarray
    colup: np.ndarray
    rowlo: np.ndarray              # float64[nrow]
    rowup: np.ndarray
    obj_offset: float = 0.0
    x0: np.ndarray | None = None   # generator's interior point, if any
    extra: dict = field(default_factory=dict)

    def __post_init__(self):
        self.col_start = np.ascontiguousarray(self.col_start, dtype=np.int64)
        self.row_index = np.ascontiguousarray(self.row_index, dtype=np.int32)
        for k in ("value", "cost", "collo", "colup", "rowlo", "rowup"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.float64))
        self._view = None

    @property
    def nnz(self) -> int:
        return int(self.col_start[-1]) if len(self.col_start) else 0

    def view(self) -> NirLpView:
        if self._view is None:
            v = NirLpView()
            v.nrow, v.ncol, v.nnz = self.nrow, self.ncol, self.nnz
            v.col_start = _ptr(self.col_start, C.c_int64)
            v.row_index = _ptr(self.row_index, C.c_int32)
            v.value = _ptr(self.value, C.c_double)
            v.cost = _ptr(self.cost, C.c_double)
            v.collo = _ptr(self.collo, C.c_double)
            v.colup = _ptr(self.colup, C.c_double)
            v.rowlo = _ptr(self.rowlo, C.c_double)
            v.rowup = _ptr(self.rowup, C.c_double)
            v.obj_offset = float(self.obj_offset)
            self._view = v
        return self._view

    def host_bytes(self) -> int:
        """Bytes of the arrays a solve copies to the device."""
        return (self.col_start.nbytes + self.row_index.nbytes + self.value.nbytes + self.cost.nbytes
                + self.collo.nbytes + self.colup.nbytes + self.rowlo.nbytes + self.rowup.nbytes)

    @staticmethod
    def from_rows(ncol: int, rows, cost, collo, colup, rowlo, rowup, obj_offset=0.0) -> "LP":
        """Build from row lists [(cols, vals), ...] (a ModelBuilder::add_row
        sequence, src/model/model.hpp:198-210); duplicates are summed and
        zeros dropped as CscMatrix::from_triplets does."""
        tr, tc, tv = [], [], []
        for i, (cols, vals) in enumerate(rows):
            for j, v in zip(cols, vals):
                if v != 0.0:
                    tr.append(i)
                    tc.append(j)
                    tv.append(float(v))
        m = len(rows)
        order = sorted(range(len(tr)), key=lambda k: (tc[k], tr[k], k))
        start = np.zeros(ncol + 1, np.int64)
        idx, val = [], []
        k = 0
        while k < len(order):
            j, i = tc[order[k]], tr[order[k]]
            s = tv[order[k]]
            k2 = k + 1
            while k2 < len(order) and tc[order[k2]] == j and tr[order[k2]] == i:
                s += tv[order[k2]]
                k2 += 1
            if s != 0.0:
                idx.append(i)
                val.append(s)
                start[j + 1] += 1
            k = k2
        start = np.cumsum(start)
        return LP(m, ncol, start, np.array(idx, np.int32), np.array(val, np.float64),
                  np.array(cost, float), np.array(collo, float), np.array(colup, float),
                  np.array(rowlo, float), np.array(rowup, float), obj_offset)


# ---------------------------------------------------------------- generator

RANDOM_EQ, ZIPF, MULTIPERIOD, BLEND_FAMILY, BADLY_SCALED = 1, 2, 3, 4, 5


class _GenOpts(C.Structure):
    _fields_ = [
        ("m", C.c_int32),
        ("n", C.c_int32),
        ("target_nnz", C.c_int64),
        ("per_col", C.c_int32),
        ("zipf_cap", C.c_int32),
        ("family_seed", C.c_uint64),
        ("scale_decades", C.c_double),
    ]


_gen_lib = None


def _lpgen():
    global _gen_lib
    if _gen_lib is None:
        path = os.path.join(_HERE, "libnir_lpgen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build() first")
        lib = C.CDLL(path)
        lib.nir_lpgen_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(_GenOpts), C.POINTER(C.c_void_p)]
        lib.nir_lpgen_view.argtypes = [C.c_void_p, C.POINTER(NirLpView)]
        lib.nir_lpgen_x0.argtypes = [C.c_void_p]
        lib.nir_lpgen_x0.restype = C.POINTER(C.c_double)
        lib.nir_lpgen_demand_factors.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        lib.nir_lpgen_demand_factors.restype = C.POINTER(C.c_double)
        lib.nir_lpgen_cost_factors.argtypes = [C.c_void_p]
        lib.nir_lpgen_cost_factors.restype = C.POINTER(C.c_double)
        lib.nir_lpgen_free.argtypes = [C.c_void_p]
        lib.nir_lpgen_last_error.restype = C.c_char_p
        _gen_lib = lib
    return _gen_lib


def _copy(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def generate(kind: int, seed: int, m: int = 0, n: int = 0, target_nnz: int = 0, per_col: int = 0,
             zipf_cap: int = 0, family_seed: int = 0, scale_decades: float = 0.0) -> LP:
    """One seeded instance (kinds and defaults: include/nir_lpgen.h)."""
    lib = _lpgen()
    o = _GenOpts(m, n, target_nnz, per_col, zipf_cap, family_seed, scale_decades)
    h = C.c_void_p()
    if lib.nir_lpgen_create(kind, seed, C.byref(o), C.byref(h)) != 0:
        raise ValueError(lib.nir_lpgen_last_error().decode())
    try:
        v = NirLpView()
        lib.nir_lpgen_view(h, C.byref(v))
        lp = LP(v.nrow, v.ncol, _copy(v.col_start, v.ncol + 1, np.int64), _copy(v.row_index, v.nnz, np.int32),
                _copy(v.value, v.nnz, np.float64), _copy(v.cost, v.ncol, np.float64),
                _copy(v.collo, v.ncol, np.float64), _copy(v.colup, v.ncol, np.float64),
                _copy(v.rowlo, v.nrow, np.float64), _copy(v.rowup, v.nrow, np.float64), v.obj_offset)
        lp.x0 = _copy(lib.nir_lpgen_x0(h), v.ncol, np.float64)
        nd = C.c_int32(0)
        dptr = lib.nir_lpgen_demand_factors(h, C.byref(nd))
        if dptr:
            lp.extra["demand_factors"] = _copy(dptr, nd.value, np.float64)
            lp.extra["cost_factors"] = _copy(lib.nir_lpgen_cost_factors(h), v.ncol, np.float64)
        lp.extra["kind"], lp.extra["seed"] = kind, seed
        return lp
    finally:
        lib.nir_lpgen_free(h)
