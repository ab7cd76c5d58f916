"""Warm-start MLP on the tensor cores (fs_gemm.cuh, fs_mlp.cu).

GEMM: BF16 operands, FP32 accumulation, against float64 products of the same
BF16 values (relative error 1e-5 of the largest entry). Forward pass and
gradients against oracle/mlp_oracle.py, which rounds to BF16 where the kernels
hold BF16 values and sums in float64: relative Frobenius error 2e-2 per tensor
(the remaining differences are FP32 accumulation order and expf, which can move
single BF16 roundings by one unit).
"""
import ctypes

import numpy as np
import pytest
import torch

from filsim_b200 import abi
from filsim_b200.configs import params_for
from filsim_b200.fcm import Context
from filsim_b200.learn import WarmStartModel

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def ctx(gpu_lib):
    c = Context(params_for(32), max_beads=64, max_filaments=8)
    yield c
    c.close()


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (128, 128, 128), (256, 384, 192), (512, 256, 512),
                                   (1024, 512, 1024), (4096, 4864, 256), (8192, 2560, 576)])
def test_gemm_bf16_matches_fp64(ctx, M, N, K):
    g = torch.Generator(device="cuda")
    g.manual_seed(M + N + K)
    A = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    D = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    ctx.call("fs_gemm_bf16", _ptr(A), _ptr(B), _ptr(D), M, N, K)
    ref = A.double() @ B.double().T
    assert torch.isfinite(D).all()
    assert float((D.double() - ref).abs().max() / ref.abs().max()) < 1e-5


def test_gemm_rejects_unaligned_shapes(ctx):
    A = torch.zeros((100, 64), dtype=torch.bfloat16, device="cuda")
    D = torch.zeros((100, 128), dtype=torch.float32, device="cuda")
    st = abi.lib().fs_gemm_bf16(ctx.h, _ptr(A), _ptr(A), _ptr(D), 100, 128, 64)
    assert st == abi.FS_ERR_INVALID_ARG


def _model_case(ctx, n=200, seed=0):
    m = WarmStartModel(ctx, nw=8, hidden=128, batch_capacity=256, seed=seed + 3)
    rng = np.random.default_rng(seed)
    feats = rng.standard_normal((n, m.n_features)).astype(np.float32) * 3 + 1
    tgts = rng.standard_normal((n, m.n_targets)).astype(np.float32)
    norm = (rng.normal(size=m.n_features).astype(np.float32), rng.uniform(0.5, 4, m.n_features).astype(np.float32),
            rng.normal(size=m.n_targets).astype(np.float32), rng.uniform(0.5, 2, m.n_targets).astype(np.float32))
    m.set_normalization(*norm)
    # the kernels clip normalised values to +-10 standard deviations
    x = np.zeros((m.capacity, m.k_in), np.float32)
    x[:n, :m.n_features] = np.clip((feats - norm[0]) / norm[1], -10, 10)
    t = np.zeros((m.capacity, m.k_out), np.float32)
    t[:n, :m.n_targets] = np.clip((tgts - norm[2]) / norm[3], -10, 10)
    return m, feats, tgts, norm, x, t


def test_mlp_forward_matches_oracle(ctx):
    from oracle import mlp_oracle
    m, feats, tgts, norm, x, t = _model_case(ctx)
    y = m.forward(torch.as_tensor(feats)).cpu().numpy()
    layers = mlp_oracle.unflatten(m.params(), m.dims)
    yr, _ = mlp_oracle.forward(layers, x)
    yr = yr[:feats.shape[0], :m.n_targets] * norm[3] + norm[2]
    assert np.linalg.norm(y - yr) / np.linalg.norm(yr) < 2e-2


def test_mlp_gradients_match_oracle(ctx):
    from oracle import mlp_oracle
    m, feats, tgts, norm, x, t = _model_case(ctx, seed=1)
    g, loss = m.gradients(torch.as_tensor(feats), torch.as_tensor(tgts))
    layers = mlp_oracle.unflatten(m.params(), m.dims)
    loss_ref, grads = mlp_oracle.loss_and_gradients(layers, x, t, feats.shape[0], m.n_targets)
    assert abs(loss - loss_ref) / loss_ref < 1e-3
    got = mlp_oracle.unflatten(g, m.dims)
    for l in range(4):
        for a, b in zip(got[l], grads[l]):
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 2e-2, l


def test_mlp_training_reduces_loss(ctx):
    """A smooth synthetic map learned by the library's Adam steps: 240 steps take the
    normalised loss from about 1 to about 0.22 (an FP32 PyTorch model with the same
    widths, optimiser and schedule reaches 0.21)."""
    m = WarmStartModel(ctx, nw=8, hidden=128, batch_capacity=256, seed=7)
    rng = np.random.default_rng(5)
    n = 2048
    feats = rng.standard_normal((n, m.n_features)).astype(np.float32)
    P = rng.standard_normal((m.n_features, m.n_targets)).astype(np.float32) / np.sqrt(m.n_features)
    tgts = np.tanh(feats @ P).astype(np.float32)
    ft, tt = torch.as_tensor(feats, device="cuda"), torch.as_tensor(tgts, device="cuda")
    m.fit_normalization(ft, tt)
    losses = m.fit(ft, tt, epochs=30, batch=256, lr=2e-3, lr_final=2e-4, seed=0)
    assert losses[-1] < 0.3 * losses[0]


def test_mlp_params_roundtrip(ctx, tmp_path):
    m, feats, *_ = _model_case(ctx, seed=2)
    y0 = m.forward(torch.as_tensor(feats)).cpu().numpy()
    path = tmp_path / "w.npz"
    m.save(path)
    m2 = WarmStartModel(ctx, nw=8, hidden=128, batch_capacity=256, seed=99)
    m2.load(path)
    y1 = m2.forward(torch.as_tensor(feats)).cpu().numpy()
    assert np.array_equal(y0, y1)
