"""The MLP of the learned PCG start on the GPU (csaige_b200.learn, through the C ABI)
against a CPU reference of the same network in PyTorch FP32 autograd, with the same
BF16-rounded weights in the forward pass (the library takes the gradient through that
rounding as the identity, which is what differentiating with respect to the rounded
weights gives)."""
import numpy as np
import pytest
import torch

import csaige_b200 as cs
import csaige_b200.learn as L

pytestmark = pytest.mark.gpu


def _torch_mlp(params, feats):
    pb = torch.tensor(params, dtype=torch.float32).to(torch.bfloat16).to(torch.float32)
    pb.requires_grad_(True)
    w1 = pb[0:512].view(64, 8)
    b1 = pb[512:576]
    w2 = pb[576:4672].view(64, 64)
    b2 = pb[4672:4736]
    w3 = pb[4736:8832].view(64, 64)
    b3 = pb[8832:8896]
    w4 = pb[8896:8960]
    b4 = pb[8960]
    x = torch.tensor(feats, dtype=torch.float32)
    h1 = torch.tanh(x @ w1.T + b1)
    h2 = torch.tanh(h1 @ w2.T + b2)
    h3 = torch.tanh(h2 @ w3.T + b3)
    return h3 @ w4 + b4, pb


@pytest.mark.parametrize("n_ex", [1, 129, 1000])
def test_forward_and_gradient_match_torch(n_ex):
    rng = np.random.default_rng(n_ex)
    p = L.initial_params(7)
    p += rng.normal(0, 0.05, p.size).astype(np.float32)
    f = rng.standard_normal((n_ex, 8)).astype(np.float32)
    t = rng.standard_normal(n_ex).astype(np.float32)
    out, grad, sse = L.mlp_eval(p, f, t, want_grad=True)
    y, pb = _torch_mlp(p, f)
    loss = ((y - torch.tensor(t)) ** 2).mean()
    loss.backward()
    assert np.allclose(out, y.detach().numpy(), rtol=1e-5, atol=2e-6)
    assert abs(sse - float(((y.detach() - torch.tensor(t)) ** 2).sum())) <= 1e-4 * max(sse, 1e-6)
    g = pb.grad.numpy()
    assert np.allclose(grad, g, rtol=1e-3, atol=1e-6 * np.abs(g).max())


def test_initial_weights_are_the_documented_uniform():
    p = L.initial_params(12345)
    assert p.size == L.param_count() == 8961
    assert np.abs(p[0:512]).max() <= 1 / np.sqrt(8) and np.abs(p[576:4672]).max() <= 1 / 8
    assert not np.array_equal(p, L.initial_params(1))


def test_training_reduces_held_out_error():
    rng = np.random.default_rng(0)
    n, q = 4000, 6
    f = rng.standard_normal((n * q, 8)).astype(np.float32)
    t = (np.tanh(f[:, 0]) + 0.5 * f[:, 1] * f[:, 2] - 0.3 * f[:, 3]).astype(np.float32)
    p0 = L.initial_params(3)
    p1, before, after, tms = L.mlp_train(p0, f, t, n, q, steps=300, batch=8192, lr=3e-3)
    assert after < 0.1 * before and after < 0.1 * tms
    # the trained weights reproduce the reported held-out error
    out, _, _ = L.mlp_eval(p1, f)
    held = (np.arange(n * q) % n) % 8 == 0
    assert abs(np.mean((out[held] - t[held]) ** 2) - after) <= 1e-3 * max(after, 1e-9) + 1e-9


def test_training_is_deterministic():
    rng = np.random.default_rng(1)
    n, q = 1500, 4
    f = rng.standard_normal((n * q, 8)).astype(np.float32)
    t = np.sin(f[:, 0]).astype(np.float32)
    a = L.mlp_train(L.initial_params(5), f, t, n, q, steps=50, batch=4096)[0]
    b = L.mlp_train(L.initial_params(5), f, t, n, q, steps=50, batch=4096)[0]
    assert np.array_equal(a, b)
