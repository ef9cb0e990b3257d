"""The MLP of the learned PCG start (SAIGE_WARM_LEARNED), exposed for checking:
16 inputs, three tanh layers of 256 units, one linear output; BF16 weights and
activations in the forward pass (the 256 x 256 layers on the tensor cores), FP32
master weights and arithmetic.  Parameter layout W1[256][16], b1[256], W2[256][256],
b2[256], W3[256][256], b3[256], w4[256], b4."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._lib import LIB, check

N_IN, N_HIDDEN = 16, 256


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def param_count() -> int:
    return int(LIB.saige_mlp_param_count())


def initial_params(seed: int = 12345) -> np.ndarray:
    p = np.empty(param_count(), np.float32)
    check(LIB.saige_mlp_initial_params(seed, _fp(p)))
    return p


def mlp_eval(params, features, targets=None, want_grad: bool = False, device: int = -1):
    """(out, grad or None, sum of squared errors or None) from the library's kernels."""
    p = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(features, np.float32).reshape(-1, N_IN)
    n = f.shape[0]
    t = None if targets is None else np.ascontiguousarray(targets, np.float32).reshape(n)
    out = np.empty(n, np.float32)
    grad = np.empty(param_count(), np.float32) if want_grad else None
    sse = C.c_double(0.0)
    check(LIB.saige_mlp_eval(_fp(p), _fp(f), None if t is None else _fp(t), n, _fp(out),
                             None if grad is None else _fp(grad),
                             C.byref(sse) if t is not None else None, device))
    return out, grad, (sse.value if t is not None else None)


def mlp_train(params, features, targets, n: int, q: int, steps: int = 200, lr: float = 1e-3,
              holdout: int = 8, device: int = -1):
    """Trains a copy of params; returns (params, held-out MSE before, after, mean square target)."""
    p = np.ascontiguousarray(params, np.float32).copy()
    f = np.ascontiguousarray(features, np.float32).reshape(-1, N_IN)
    t = np.ascontiguousarray(targets, np.float32).reshape(-1)
    b, a, m = C.c_double(), C.c_double(), C.c_double()
    check(LIB.saige_mlp_train(_fp(p), _fp(f), _fp(t), n, q, steps, lr, holdout,
                              C.byref(b), C.byref(a), C.byref(m), device))
    return p, b.value, a.value, m.value
