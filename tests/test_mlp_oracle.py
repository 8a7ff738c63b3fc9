"""CPU checks of the warm-start network's oracle and C ABI (no GPU).

The oracle's exact float64 backward pass agrees with central differences
(this pins the formulas the GPU gradients are checked against), its BF16
rounding is round-to-nearest-even as torch's, and libnir_mlp.so exports
every function include/nir_mlp.h declares and fails loudly without a GPU.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest
import torch

from conftest import ROOT, has_gpu
from oracle import mlp_oracle as M


def _net(rng, dims):
    n = sum(dims[i] * dims[i + 1] + dims[i + 1] for i in range(len(dims) - 1))
    return rng.normal(size=n) * 0.5


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    dims = [6, 5, 4, 3]
    p = _net(rng, dims)
    X = rng.normal(size=(7, 6))
    T = rng.normal(size=(7, 3))
    w = np.array([1.0, 0.0, 2.0])
    _, g = M.loss_and_grads(p, dims, X, T, w, emulate=False)
    idx = rng.choice(p.size, size=40, replace=False)
    fd = M.finite_difference(p, dims, X, T, w, idx)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-7)


def test_oracle_bf16_rounding_matches_torch():
    rng = np.random.default_rng(1)
    a = np.concatenate([rng.normal(size=10000) * 10.0 ** rng.uniform(-8, 8, 10000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.005859375, 65504.0]])
    want = torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16(a), want)


def test_mlp_library_exports_every_declared_symbol():
    from nirnaya_b200 import mlp

    header = open(os.path.join(ROOT, "include", "nir_mlp.h")).read()
    declared = set(re.findall(r"\b(nir_mlp_\w+)\s*\(", header))
    assert declared == set(mlp.EXPORTED)
    blend = set(re.findall(r"\b(nir_blend_features_\w+)\s*\(", header))
    assert blend == set(mlp.BLEND_EXPORTED)
    lib = C.CDLL(mlp.LIB_PATH)
    for name in declared | blend:
        assert hasattr(lib, name), name


def test_blend_feature_data_layout_matches_the_c_compiler(tmp_path):
    import subprocess

    from nirnaya_b200 import mlp

    src = tmp_path / "b.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "nir_mlp.h"', 'int main(void){',
             'printf("%zu\\n", sizeof(nir_blend_feature_data));']
    lines += [f'printf("%zu\\n", offsetof(nir_blend_feature_data, {f}));' for f, _ in mlp.BlendFeatureData._fields_]
    lines += ["return 0;}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "b"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals[0] == C.sizeof(mlp.BlendFeatureData)
    assert vals[1:] == [getattr(mlp.BlendFeatureData, f).offset for f, _ in mlp.BlendFeatureData._fields_]


def test_mlp_config_layout_matches_the_c_compiler(tmp_path):
    import subprocess

    from nirnaya_b200 import mlp

    src = tmp_path / "l.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "nir_mlp.h"', 'int main(void){',
             'printf("%zu\\n", sizeof(nir_mlp_config));']
    lines += [f'printf("%zu\\n", offsetof(nir_mlp_config, {f}));' for f, _ in mlp.Config._fields_]
    lines += ["return 0;}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "l"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals[0] == C.sizeof(mlp.Config)
    assert vals[1:] == [getattr(mlp.Config, f).offset for f, _ in mlp.Config._fields_]


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure mode")
def test_mlp_create_without_gpu_fails_loudly():
    from nirnaya_b200 import mlp

    with pytest.raises(RuntimeError):
        mlp.Mlp(16, 8, width=16, depth=1)


def test_blend_family_instances_keep_the_base_point_feasible():
    from nirnaya_b200 import learned as LW
    from oracle import ffi

    fam = LW.BlendFamily(m=400, n=1000, nnz=8000, family_seed=0)
    x0 = fam.base.x0
    for seed in (1, 2, 3):
        lp = fam.instance(seed)
        ax = ffi.spmv(lp, x0)
        assert np.all(ax >= lp.rowlo - 1e-9 * (1 + np.abs(lp.rowlo)))
        assert np.all(ax <= lp.rowup + 1e-9 * (1 + np.abs(lp.rowup)))
        f, g = fam.factors(seed)
        assert f.min() >= 0.1 and f.max() <= 1.9 and g.min() >= 0.5 and g.max() <= 1.5
        assert np.all(np.sign(lp.cost) == np.sign(fam.base.cost))
    a, b = fam.factors(7), fam.factors(7)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
