"""ctypes binding of libnir_mlp.so (include/nir_mlp.h): the warm-start
network's hand-written tensor-core training and inference."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnir_mlp.so")

EXPORTED = [
    "nir_mlp_create", "nir_mlp_free", "nir_mlp_last_error", "nir_mlp_param_count", "nir_mlp_get_params",
    "nir_mlp_set_params", "nir_mlp_set_output_weights", "nir_mlp_set_data", "nir_mlp_train", "nir_mlp_predict",
    "nir_mlp_gradients", "nir_mlp_gemm_check", "nir_mlp_gemm_time", "nir_mlp_step_stats", "nir_mlp_predict_device",
    "nir_mlp_set_affine", "nir_mlp_predict_device_affine",
]
BLEND_EXPORTED = ["nir_blend_features_create", "nir_blend_features_build", "nir_blend_features_free"]


class Config(C.Structure):
    _fields_ = [("d_in", C.c_int32), ("width", C.c_int32), ("depth", C.c_int32), ("d_out", C.c_int32),
                ("seed", C.c_uint64), ("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("eps", C.c_float)]


class BlendFeatureData(C.Structure):
    """nir_blend_feature_data (include/nir_mlp.h)."""
    _fields_ = [("n", C.c_int32), ("m", C.c_int32), ("nd", C.c_int32), ("nf", C.c_int32),
                ("col_template", C.POINTER(C.c_float)), ("row_template", C.POINTER(C.c_float)),
                ("cost0", C.POINTER(C.c_double)), ("atybar", C.POINTER(C.c_double)),
                ("dem_w", C.POINTER(C.c_double)), ("cscale", C.c_double),
                ("dem_rp", C.POINTER(C.c_int64)), ("dem_ci", C.POINTER(C.c_int32)), ("dem_val", C.POINTER(C.c_double)),
                ("rowlo0", C.POINTER(C.c_double)), ("rowup", C.POINTER(C.c_double)), ("axbar", C.POINTER(C.c_double)),
                ("bscale", C.POINTER(C.c_double)), ("row_abs", C.POINTER(C.c_double)),
                ("abs_rp", C.POINTER(C.c_int64)), ("abs_ci", C.POINTER(C.c_int32)), ("abs_val", C.POINTER(C.c_double))]


_lib = None
F = C.POINTER(C.c_float)


def lib():
    """Loads libnir_mlp.so (raises if it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m nirnaya_b200.build`")
        L = C.CDLL(LIB_PATH)
        VP = C.c_void_p
        L.nir_mlp_create.argtypes = [C.POINTER(Config), C.c_int, C.POINTER(VP)]
        L.nir_mlp_free.argtypes = [VP]
        L.nir_mlp_last_error.restype = C.c_char_p
        L.nir_mlp_param_count.argtypes = [VP]
        L.nir_mlp_param_count.restype = C.c_int64
        L.nir_mlp_get_params.argtypes = [VP, F]
        L.nir_mlp_set_params.argtypes = [VP, F]
        L.nir_mlp_set_output_weights.argtypes = [VP, F]
        L.nir_mlp_set_data.argtypes = [VP, F, F, C.c_int32]
        L.nir_mlp_train.argtypes = [VP, C.c_int32, C.c_int32, F]
        L.nir_mlp_predict.argtypes = [VP, F, C.c_int32, F]
        L.nir_mlp_gradients.argtypes = [VP, F, F, C.c_int32, F, F]
        L.nir_mlp_gemm_check.argtypes = [VP, C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int32, F, C.c_int32, F,
                                         C.c_int32, F]
        L.nir_mlp_step_stats.argtypes = [VP, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.nir_mlp_gemm_time.argtypes = [VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
        L.nir_mlp_predict_device.argtypes = [VP, VP, C.c_int32, F]
        D = C.POINTER(C.c_double)
        L.nir_mlp_set_affine.argtypes = [VP, C.c_int32, C.c_int32, C.c_double, C.c_double, D, D]
        L.nir_mlp_predict_device_affine.argtypes = [VP, VP, C.c_int32, C.POINTER(VP)]
        L.nir_blend_features_create.argtypes = [C.POINTER(BlendFeatureData), C.c_int32, C.POINTER(VP)]
        L.nir_blend_features_build.argtypes = [VP, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(VP),
                                               C.POINTER(VP)]
        L.nir_blend_features_free.argtypes = [VP]
        _lib = L
    return _lib


def _f(a):
    return a.ctypes.data_as(F)


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Mlp:
    """d_in -> width x depth (ReLU) -> d_out on one GPU."""

    def __init__(self, d_in, d_out, width=512, depth=3, seed=0, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8,
                 device=0):
        self.cfg = Config(d_in, width, depth, d_out, seed, lr, beta1, beta2, eps)
        self.dims = [d_in] + [width] * depth + [d_out]
        self._h = C.c_void_p()
        rc = lib().nir_mlp_create(C.byref(self.cfg), device, C.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"nir_mlp_create failed: {lib().nir_mlp_last_error().decode()}")

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed: {lib().nir_mlp_last_error().decode()}")

    def close(self):
        if self._h:
            lib().nir_mlp_free(self._h)
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

    def param_count(self) -> int:
        return int(lib().nir_mlp_param_count(self._h))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.param_count(), np.float32)
        self._check(lib().nir_mlp_get_params(self._h, _f(out)), "get_params")
        return out

    def set_params(self, p):
        p = _c32(p)
        assert p.size == self.param_count()
        self._check(lib().nir_mlp_set_params(self._h, _f(p)), "set_params")

    def set_output_weights(self, w):
        w = _c32(w)
        self._check(lib().nir_mlp_set_output_weights(self._h, _f(w)), "set_output_weights")

    def set_data(self, X, T):
        X, T = _c32(X), _c32(T)
        self._check(lib().nir_mlp_set_data(self._h, _f(X), _f(T), X.shape[0]), "set_data")

    def train(self, epochs, batch) -> np.ndarray:
        losses = np.zeros(max(epochs, 1), np.float32)
        self._check(lib().nir_mlp_train(self._h, epochs, batch, _f(losses)), "train")
        return losses[:epochs]

    def predict(self, X) -> np.ndarray:
        X = _c32(X)
        n = X.shape[0]
        pad = (-n) % 8
        if pad:
            X = np.vstack([X, np.zeros((pad, X.shape[1]), np.float32)])
        Y = np.zeros((X.shape[0], self.dims[-1]), np.float32)
        self._check(lib().nir_mlp_predict(self._h, _f(X), X.shape[0], _f(Y)), "predict")
        return Y[:n]

    def predict_device(self, x_dev: int, n: int) -> np.ndarray:
        """Forward pass of n FP32 samples already on the device (the address
        x_dev, n x d_in row-major; n a multiple of 8)."""
        Y = np.zeros((n, self.dims[-1]), np.float32)
        self._check(lib().nir_mlp_predict_device(self._h, C.c_void_p(x_dev), n, _f(Y)), "predict_device")
        return Y

    def set_affine(self, n: int, col: int = 0, lo: float = -np.inf, hi: float = np.inf, scale=None, shift=None):
        """The map of predict_device_affine: shift + scale * clamp(pred[:, col], lo, hi)."""
        keep = [None if v is None else np.ascontiguousarray(v, np.float64) for v in (scale, shift)]
        for v in keep:
            assert v is None or v.shape == (n,)
        ptr = [None if v is None else v.ctypes.data_as(C.POINTER(C.c_double)) for v in keep]
        self._check(lib().nir_mlp_set_affine(self._h, int(n), int(col), float(lo), float(hi), ptr[0], ptr[1]),
                    "set_affine")

    def predict_device_affine(self, x_dev: int, n: int) -> int:
        """Forward pass of n FP32 samples on the device and the set_affine map:
        the device address of n FP64 results, valid until the next call."""
        out = C.c_void_p()
        self._check(lib().nir_mlp_predict_device_affine(self._h, C.c_void_p(x_dev), int(n), C.byref(out)),
                    "predict_device_affine")
        return int(out.value)

    def gradients(self, X, T):
        X, T = _c32(X), _c32(T)
        g = np.zeros(self.param_count(), np.float32)
        loss = C.c_float()
        self._check(lib().nir_mlp_gradients(self._h, _f(X), _f(T), X.shape[0], C.byref(loss), _f(g)), "gradients")
        return float(loss.value), g

    def gemm(self, a_kmaj, b_kmaj, M, N, K, A, lda, B, ldb) -> np.ndarray:
        A, B = _c32(A), _c32(B)
        Cm = np.zeros((M, N), np.float32)
        self._check(lib().nir_mlp_gemm_check(self._h, int(a_kmaj), int(b_kmaj), M, N, K, _f(A), lda, _f(B), ldb,
                                             _f(Cm)), "gemm_check")
        return Cm

    def gemm_tflops(self, M, N, K, reps=20) -> float:
        """Throughput of the forward GEMM on an M x N x K problem."""
        us = C.c_double()
        self._check(lib().nir_mlp_gemm_time(self._h, M, N, K, reps, C.byref(us)), "gemm_time")
        return 2.0 * M * N * K / (us.value * 1e-6) / 1e12

    def step_stats(self):
        us, fl = C.c_double(), C.c_double()
        lib().nir_mlp_step_stats(self._h, C.byref(us), C.byref(fl))
        return us.value, fl.value


class BlendFeatures:
    """The blending family's per-variable features built on the device
    (nir_blend_features_*): the family's data is copied once, and each
    instance uploads only its factors (f, g)."""

    def __init__(self, data: dict, device: int = 0):
        self._keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dt)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(np.ctypeslib.as_ctypes_type(dt)))

        d = BlendFeatureData()
        d.n, d.m, d.nd, d.nf = data["n"], data["m"], data["nd"], data["nf"]
        d.col_template = arr(data["col_template"], np.float32)
        d.row_template = arr(data["row_template"], np.float32)
        for k in ("cost0", "atybar", "dem_w", "dem_val", "rowlo0", "rowup", "axbar", "bscale", "row_abs", "abs_val"):
            setattr(d, k, arr(data[k], np.float64))
        d.cscale = float(data["cscale"])
        d.dem_rp = arr(data["dem_rp"], np.int64)
        d.abs_rp = arr(data["abs_rp"], np.int64)
        d.dem_ci = arr(data["dem_ci"], np.int32)
        d.abs_ci = arr(data["abs_ci"], np.int32)
        h = C.c_void_p()
        rc = lib().nir_blend_features_create(C.byref(d), device, C.byref(h))
        self._keep = []  # the library has copied everything
        if rc != 0:
            raise RuntimeError(f"nir_blend_features_create failed ({rc}): {lib().nir_mlp_last_error().decode()}")
        self._h = h
        self.n, self.m, self.nf = d.n, d.m, d.nf

    def build(self, f, g):
        """Device addresses (col, row) of instance (f, g)'s features, valid
        until the next build."""
        f = np.ascontiguousarray(f, np.float64)
        g = np.ascontiguousarray(g, np.float64)
        col, row = C.c_void_p(), C.c_void_p()
        rc = lib().nir_blend_features_build(self._h, f.ctypes.data_as(C.POINTER(C.c_double)),
                                            g.ctypes.data_as(C.POINTER(C.c_double)), C.byref(col), C.byref(row))
        if rc != 0:
            raise RuntimeError(f"nir_blend_features_build failed ({rc}): {lib().nir_mlp_last_error().decode()}")
        return col.value, row.value

    def close(self):
        if getattr(self, "_h", None):
            lib().nir_blend_features_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
