"""The MLP of the learned PCG start on the GPU (csaige_b200.learn, through the C ABI)
against a CPU reference of the same network in PyTorch FP32 autograd, with the same
BF16-rounded weights and BF16-rounded activations in the forward pass (the library
takes the gradient through those roundings as the identity, which is what
differentiating through the rounded values gives).  The two 256 x 256 layers run on the
tensor cores with FP32 accumulation in another order than PyTorch's, so an activation
may round to the neighbouring BF16 value: the tolerances are written per test."""
import numpy as np
import pytest
import torch

import csaige_b200 as cs
import csaige_b200.learn as L

pytestmark = pytest.mark.gpu

IN, H = 16, 256
# offsets of W1, b1, W2, b2, W3, b3, w4, b4
OFF = np.cumsum([0, H * IN, H, H * H, H, H * H, H, H, 1])


def _torch_mlp(params, feats):
    pb = torch.tensor(params, dtype=torch.float32).to(torch.bfloat16).to(torch.float32)
    pb.requires_grad_(True)
    w1 = pb[OFF[0]:OFF[1]].view(H, IN)
    b1 = pb[OFF[1]:OFF[2]]
    w2 = pb[OFF[2]:OFF[3]].view(H, H)
    b2 = pb[OFF[3]:OFF[4]]
    w3 = pb[OFF[4]:OFF[5]].view(H, H)
    b3 = pb[OFF[5]:OFF[6]]
    w4 = pb[OFF[6]:OFF[7]]
    b4 = pb[OFF[7]]
    bf = lambda a: a + (a.detach().to(torch.bfloat16).to(torch.float32) - a.detach())
    x = torch.tensor(feats, dtype=torch.float32)
    h1 = bf(torch.tanh(x @ w1.T + b1))
    h2 = bf(torch.tanh(h1 @ w2.T + b2))
    h3 = bf(torch.tanh(h2 @ w3.T + b3))
    return h3 @ w4 + b4, pb


@pytest.mark.parametrize("n_ex", [1, 129, 1000, 3000])
def test_forward_and_gradient_match_torch(n_ex):
    rng = np.random.default_rng(n_ex)
    p = L.initial_params(7)
    p += rng.normal(0, 0.02, p.size).astype(np.float32)
    f = rng.standard_normal((n_ex, IN)).astype(np.float32)
    t = rng.standard_normal(n_ex).astype(np.float32)
    out, grad, sse = L.mlp_eval(p, f, t, want_grad=True)
    y, pb = _torch_mlp(p, f)
    loss = ((y - torch.tensor(t)) ** 2).mean()
    loss.backward()
    yt = y.detach().numpy()
    # an activation that lands on the other side of a BF16 rounding boundary moves y by
    # up to one BF16 step (2^-8 relative) of one of 256 terms of size ~ |w4| / 16
    assert np.abs(out - yt).max() <= 2e-3 * max(1.0, np.abs(yt).max())
    assert abs(sse - float(((y.detach() - torch.tensor(t)) ** 2).sum())) <= 5e-3 * max(sse, 1e-6)
    g = pb.grad.numpy()
    for a, b, name in [(OFF[0], OFF[2], "layer 1"), (OFF[2], OFF[4], "layer 2"),
                       (OFF[4], OFF[6], "layer 3"), (OFF[6], OFF[8], "output")]:
        rel = np.linalg.norm(grad[a:b] - g[a:b]) / max(np.linalg.norm(g[a:b]), 1e-30)
        assert rel <= 2e-2, (name, rel)


def test_initial_weights_are_the_documented_uniform():
    p = L.initial_params(12345)
    assert p.size == L.param_count() == OFF[-1]
    assert np.abs(p[OFF[0]:OFF[1]]).max() <= 1 / np.sqrt(IN)
    assert np.abs(p[OFF[2]:OFF[3]]).max() <= 1 / np.sqrt(H)
    assert not np.array_equal(p, L.initial_params(1))


def test_training_reduces_held_out_error():
    rng = np.random.default_rng(0)
    n, q = 6000, 6
    f = rng.standard_normal((n * q, IN)).astype(np.float32)
    t = (np.tanh(f[:, 0]) + 0.5 * f[:, 1] * f[:, 2] - 0.3 * f[:, 3]).astype(np.float32)
    p0 = L.initial_params(3)
    p1, before, after, tms = L.mlp_train(p0, f, t, n, q, steps=300, lr=1e-3)
    assert after < 0.1 * before and after < 0.1 * tms
    # the trained weights reproduce the reported held-out error
    out, _, _ = L.mlp_eval(p1, f)
    held = (np.arange(n * q) % n) % 8 == 0
    assert abs(np.mean((out[held] - t[held]) ** 2) - after) <= 1e-3 * max(after, 1e-9) + 1e-9


def test_training_is_deterministic():
    rng = np.random.default_rng(1)
    n, q = 3000, 4
    f = rng.standard_normal((n * q, IN)).astype(np.float32)
    t = np.sin(f[:, 0]).astype(np.float32)
    a = L.mlp_train(L.initial_params(5), f, t, n, q, steps=50)[0]
    b = L.mlp_train(L.initial_params(5), f, t, n, q, steps=50)[0]
    assert np.array_equal(a, b)
