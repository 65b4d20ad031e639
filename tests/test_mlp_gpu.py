"""The learned (alpha, PC count) proposal's perceptron on the GPU, through the C ABI.

No reference counterpart: the float64 restatement in oracle/ha_oracle.py (itself checked against
finite differences in test_oracle.py) is the checker.  Tolerances:
  * gradient of the mean cross-entropy (float32 kernels vs float64): relative 2-norm <= 1e-4,
    loss relative <= 1e-5
  * bfloat16 inference vs the float64 forward: the same class for >= 97 % of samples where the
    float64 top two probabilities differ by more than 0.05; probability of the chosen class within
    0.1 (mean within 0.01): bfloat16 weights carry ~2^-9 relative error into logits of size ~10
"""

import ctypes

import numpy as np
import pytest

from hyperalignment_b200 import _lib as L
from oracle import ha_oracle as O

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _params(gpu, C, seed):
    import torch
    P = gpu.ha_b200_mlp_param_count(C)
    d = torch.zeros(P, dtype=torch.float32, device="cuda")
    assert gpu.ha_b200_mlp_init(ctypes.c_void_p(d.data_ptr()), C, seed) == 0
    return d


def _toy(seed, n, C):
    # labels from a fixed rule of the features (a linear score over a few inputs, binned)
    rng = np.random.default_rng(seed)
    X = rng.uniform(0.0, 1.0, (n, O.MLP_IN)).astype(np.float32)
    X[:, 64] = np.log(rng.integers(50, 500, n))
    score = X[:, 0] * 2.0 - X[:, 3] + 0.5 * X[:, 10] + 0.1 * X[:, 64]
    edges = np.quantile(score, np.linspace(0, 1, C + 1)[1:-1])
    y = np.searchsorted(edges, score).astype(np.int32)
    return X, y


@pytest.mark.parametrize("C,n", [(40, 100), (7, 33), (64, 257)])
def test_mlp_gradient_matches_oracle(gpu, C, n):
    import torch
    rng = np.random.default_rng(C)
    d = _params(gpu, C, 3)
    X = rng.standard_normal((n, O.MLP_IN)).astype(np.float32)
    y = rng.integers(0, C, n).astype(np.int32)
    dX, dy = _dev(X, np.float32), _dev(y, np.int32)
    g = torch.zeros_like(d)
    loss = ctypes.c_float()
    assert gpu.ha_b200_mlp_grad(ctypes.c_void_p(d.data_ptr()), C, ctypes.c_void_p(dX.data_ptr()),
                                ctypes.c_void_p(dy.data_ptr()), n, ctypes.c_void_p(g.data_ptr()),
                                ctypes.byref(loss)) == 0
    rl, rg = O.mlp_loss_grad(d.cpu().numpy().astype(np.float64), C, X.astype(np.float64), y)
    got = g.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(got - rg) <= 1e-4 * np.linalg.norm(rg)
    assert abs(loss.value - rl) <= 1e-5 * abs(rl)


def test_mlp_rejects_bad_labels(gpu):
    import torch
    d = _params(gpu, 5, 1)
    dX = _dev(np.zeros((4, O.MLP_IN)), np.float32)
    dy = _dev(np.array([0, 1, 5, 2]), np.int32)
    g = torch.zeros_like(d)
    assert gpu.ha_b200_mlp_grad(ctypes.c_void_p(d.data_ptr()), 5, ctypes.c_void_p(dX.data_ptr()),
                                ctypes.c_void_p(dy.data_ptr()), 4, ctypes.c_void_p(g.data_ptr()), None) == L.ERROR_ARG


def test_mlp_training_learns_and_bf16_inference_agrees(gpu):
    import torch
    C = 8
    X, y = _toy(1, 4000, C)
    Xt, yt = _toy(2, 1000, C)
    d = _params(gpu, C, 7)
    dX, dy = _dev(X, np.float32), _dev(y, np.int32)
    loss0 = ctypes.c_float()
    g = torch.zeros_like(d)
    assert gpu.ha_b200_mlp_grad(ctypes.c_void_p(d.data_ptr()), C, ctypes.c_void_p(dX.data_ptr()),
                                ctypes.c_void_p(dy.data_ptr()), 4000, ctypes.c_void_p(g.data_ptr()),
                                ctypes.byref(loss0)) == 0
    loss1 = ctypes.c_float()
    assert gpu.ha_b200_mlp_train(ctypes.c_void_p(d.data_ptr()), C, ctypes.c_void_p(dX.data_ptr()),
                                 ctypes.c_void_p(dy.data_ptr()), 4000, 60, 128, 3e-3, 11, ctypes.byref(loss1)) == 0
    assert loss1.value < 0.5 * loss0.value
    dXt = _dev(Xt, np.float32)
    cls = torch.zeros(1000, dtype=torch.int32, device="cuda")
    prob = torch.zeros(1000, dtype=torch.float32, device="cuda")
    assert gpu.ha_b200_mlp_infer(ctypes.c_void_p(d.data_ptr()), C, ctypes.c_void_p(dXt.data_ptr()), 1000,
                                 ctypes.c_void_p(cls.data_ptr()), ctypes.c_void_p(prob.data_ptr()), None) == 0
    torch.cuda.synchronize()
    c, p = cls.cpu().numpy(), prob.cpu().numpy()
    assert (c == yt).mean() > 0.8  # held-out accuracy on the toy rule
    z = O.mlp_forward(d.cpu().numpy().astype(np.float64), C, Xt.astype(np.float64))
    pr = np.exp(z - z.max(1, keepdims=True))
    pr /= pr.sum(1, keepdims=True)
    top = np.sort(pr, axis=1)
    clear = (top[:, -1] - top[:, -2]) > 0.05
    assert (c[clear] == pr.argmax(1)[clear]).mean() >= 0.97
    dp = np.abs(p - pr[np.arange(1000), c])
    assert dp.max() <= 0.1 and dp.mean() <= 0.01
