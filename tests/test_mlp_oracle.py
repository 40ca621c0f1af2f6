"""The learned-h MLP's CPU oracle (FP64) and the parameter layout, checked without a GPU."""
import numpy as np

import oracle
from botheadstudios_b200 import _lib, learned_h


def _params(seed=0):
    rng = np.random.default_rng(seed)
    p = learned_h.zero_params()
    p[:_lib.MLP_TRAINABLE] = rng.normal(0.0, 0.2, _lib.MLP_TRAINABLE)
    p[learned_h.XM:learned_h.XM + 8] = rng.normal(0.0, 0.5, 8)
    p[learned_h.XS:learned_h.XS + 8] = rng.uniform(0.5, 2.0, 8)
    p[learned_h.YM], p[learned_h.YS] = 0.01, 0.02
    return p


def test_layout_constants_agree():
    assert oracle.mlp_param_count() == _lib.MLP_PARAMS == 4819
    assert oracle.mlp_param_count(True) == _lib.MLP_TRAINABLE == 4801
    assert learned_h.B3 + 1 == _lib.MLP_TRAINABLE and learned_h.YS + 1 == _lib.MLP_PARAMS


def test_oracle_gradient_matches_finite_differences():
    p = _params(1)
    rng = np.random.default_rng(2)
    x = rng.normal(size=(48, 8)).astype(np.float32)
    t = rng.normal(0.01, 0.02, 48).astype(np.float32)
    _, g = oracle.mlp_grad(p, x, t, bf16=False)
    for k in [0, 77, learned_h.B1 + 3, learned_h.W2 + 1000, learned_h.B2 + 5, learned_h.W3 + 9, learned_h.B3]:
        e = 1e-2 * max(abs(float(p[k])), 0.1)
        q1, q2 = p.copy(), p.copy()
        q1[k] += e
        q2[k] -= e
        l1, _ = oracle.mlp_grad(q1, x, t, bf16=False)
        l2, _ = oracle.mlp_grad(q2, x, t, bf16=False)
        fd = (l1 - l2) / (float(q1[k]) - float(q2[k]))
        assert abs(fd - g[k]) <= 1e-4 * max(abs(g[k]), 1e-2), (k, fd, g[k])


def test_bf16_emulation_is_a_small_perturbation():
    p = _params(3)
    x = np.random.default_rng(4).normal(size=(256, 8)).astype(np.float32)
    y64 = oracle.mlp_forward(p, x, bf16=False)
    y16 = oracle.mlp_forward(p, x, bf16=True)
    scale = np.abs(y64 - p[learned_h.YM]).max()
    assert 0 < np.abs(y16 - y64).max() < 0.05 * scale
