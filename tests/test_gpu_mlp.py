"""GPU checks of the warm-start network's hand-written tensor-core kernels
(libnir_mlp.so) against the numpy oracle (oracle/mlp_oracle.py).

  * the GEMM in all four operand layouts, with ragged tiles and split K,
    equals the float64 product of the BF16-rounded operands up to FP32
    accumulation error;
  * forward outputs, the loss and every gradient equal the oracle's
    BF16-emulating float64 network (tolerances in each test);
  * training reduces the loss, parameters round-trip, bad shapes fail.
"""
import numpy as np
import pytest

from conftest import has_gpu
from nirnaya_b200 import mlp
from oracle import mlp_oracle as M

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]


def _operand(rng, rows, K, kmaj, ld_pad=0):
    """Random (rows x K) operand stored K-major or MN-major, as FP32 plus
    the BF16-rounded logical matrix."""
    logical = rng.normal(size=(rows, K))
    if kmaj:
        ld = K + ld_pad
        store = np.zeros((rows, ld))
        store[:, :K] = logical
    else:
        ld = rows + ld_pad
        store = np.zeros((K, ld))
        store[:, :rows] = logical.T
    return store.astype(np.float32), ld, M.bf16(logical)


@pytest.mark.parametrize("a_kmaj,b_kmaj", [(True, True), (True, False), (False, False), (False, True)])
@pytest.mark.parametrize("Mr,N,K", [(24, 40, 48), (136, 264, 1000), (64, 128, 8192), (8, 520, 72)])
def test_gemm_layouts_match_numpy(a_kmaj, b_kmaj, Mr, N, K):
    rng = np.random.default_rng(Mr * 7 + N + K)
    A, lda, Al = _operand(rng, Mr, K, a_kmaj, ld_pad=8)
    B, ldb, Bl = _operand(rng, N, K, b_kmaj, ld_pad=16)
    with mlp.Mlp(8, 8, width=8, depth=1) as net:
        C = net.gemm(a_kmaj, b_kmaj, Mr, N, K, A, lda, B, ldb)
    ref = Al @ Bl.T
    mag = np.abs(Al) @ np.abs(Bl).T
    # FP32 accumulation of K exact BF16 products
    assert np.all(np.abs(C - ref) <= 4e-6 * mag + 1e-6), np.max(np.abs(C - ref) / (mag + 1e-6))


def _rand_net(net, rng, scale=0.3):
    p = (rng.normal(size=net.param_count()) * scale).astype(np.float32)
    net.set_params(p)
    return p


@pytest.mark.parametrize("d_in,width,depth,d_out,rows", [(64, 32, 2, 24, 16), (2048, 64, 3, 136, 64)])
def test_forward_loss_and_gradients_match_oracle(d_in, width, depth, d_out, rows):
    rng = np.random.default_rng(d_in + rows)
    with mlp.Mlp(d_in, d_out, width=width, depth=depth, seed=3) as net:
        p = _rand_net(net, rng, scale=1.0 / np.sqrt(d_in / 8))
        assert np.array_equal(net.get_params(), p)
        w = np.ones(d_out, np.float32)
        w[-5:] = 0.0  # padding outputs
        net.set_output_weights(w)
        X = rng.normal(size=(rows, d_in)).astype(np.float32)
        T = rng.normal(size=(rows, d_out)).astype(np.float32)
        Y = net.predict(X)
        loss, g = net.gradients(X, T)
    dims = net.dims
    Yo, _ = M.forward(p, dims, X)
    assert np.allclose(Y, Yo, rtol=2e-2, atol=2e-2 * np.abs(Yo).max())
    # relative error of the whole output, dominated by rare BF16 rounding flips
    assert np.linalg.norm(Y - Yo) <= 5e-3 * np.linalg.norm(Yo)
    lo, go = M.loss_and_grads(p, dims, X, T, w)
    assert abs(loss - lo) <= 5e-3 * lo
    o = 0
    for i in range(len(dims) - 1):
        n_in, n_out = dims[i], dims[i + 1]
        for part, n in (("W", n_in * n_out), ("b", n_out)):
            a, b = g[o:o + n], go[o:o + n]
            o += n
            assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b) + 1e-7, (i, part)
    assert o == g.size
    # gradient of the padding outputs' bias is exactly zero
    assert np.all(g[-5:] == 0.0)


def test_training_reduces_loss_on_a_teacher_network():
    rng = np.random.default_rng(5)
    d_in, d_out, n = 128, 64, 1024
    X = rng.normal(size=(n, d_in)).astype(np.float32)
    Wt = rng.normal(size=(d_in, d_out)) / np.sqrt(d_in)
    T = (np.tanh(X @ Wt) + 0.1 * X[:, :d_out]).astype(np.float32)
    with mlp.Mlp(d_in, d_out, width=128, depth=3, seed=1, lr=2e-3) as net:
        net.set_data(X, T)
        losses = net.train(40, 64)
        us, flops = net.step_stats()
        Y = net.predict(X[:256])
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.2 * losses[0], losses[[0, -1]]
    assert np.mean((Y - T[:256]) ** 2) < 0.3 * np.mean(T[:256] ** 2)
    assert us > 0 and flops > 0


def test_bad_shapes_fail_loudly():
    with pytest.raises(RuntimeError):
        mlp.Mlp(12, 8, width=8, depth=1)  # d_in not a multiple of 8
    with mlp.Mlp(16, 8, width=8, depth=1) as net:
        with pytest.raises(RuntimeError):
            net.gradients(np.zeros((12, 16)), np.zeros((12, 8)))  # rows not a multiple of 8
        with pytest.raises(RuntimeError):
            net.train(1, 12)
