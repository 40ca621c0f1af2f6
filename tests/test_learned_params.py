"""The learned smoothing length's parameter block on the host (no GPU): its layout matches the C ABI's
SPH_MLP_PARAMS / SPH_MLP_TRAINABLE, the shipped trained network loads with that layout and sane
normalisation, the normalisation rule, and the zero network's proposal (none) through the oracle."""
import os
import re

import numpy as np

import oracle
from botheadstudios_b200 import learned_h
from botheadstudios_b200._lib import MLP_PARAMS, MLP_TRAINABLE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _define(name):
    text = open(os.path.join(ROOT, "include", "sph_b200.h")).read()
    return int(re.search(rf"#define {name} (\d+)", text).group(1))


def test_layout_matches_the_c_abi():
    assert MLP_PARAMS == _define("SPH_MLP_PARAMS") and MLP_TRAINABLE == _define("SPH_MLP_TRAINABLE")
    n_in, n_h = learned_h.N_IN, learned_h.N_H
    assert MLP_TRAINABLE == n_in * n_h + n_h + n_h * n_h + n_h + n_h + 1  # W1 b1 W2 b2 W3 b3
    assert MLP_PARAMS == MLP_TRAINABLE + 2 * n_in + 2                  # x_mean x_scale y_mean y_scale
    assert (learned_h.W1, learned_h.B1, learned_h.W2) == (0, 512, 576)
    assert (learned_h.B2, learned_h.W3, learned_h.B3) == (4672, 4736, 4800)
    assert (learned_h.XM, learned_h.XS, learned_h.YM, learned_h.YS) == (4801, 4809, 4817, 4818)


def test_shipped_network_loads():
    p = learned_h.load()
    assert p.dtype == np.float32 and p.shape == (MLP_PARAMS,)
    assert np.isfinite(p).all()
    assert (p[learned_h.XS:learned_h.XS + learned_h.N_IN] > 0).all() and p[learned_h.YS] > 0
    assert np.abs(p[:MLP_TRAINABLE]).max() > 0  # trained, not the zero network


def test_normalisation_rule():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(1000, 8)) * np.arange(1, 9) + np.arange(8)
    X[:, 5] = 1.0  # a constant feature (one material)
    T = rng.normal(0.01, 0.002, 1000)
    xm, xs, ym, ys = learned_h.normalisation(X, T)
    assert np.allclose(xm, X.mean(0), atol=1e-5)
    assert xs[5] == 1.0
    others = [k for k in range(8) if k != 5]
    assert np.allclose(xs[others], 1.0 / X.std(0)[others], rtol=1e-5)
    assert ym == T.mean() and ys == T.std()


def test_zero_network_proposes_nothing():
    x = np.random.default_rng(1).normal(size=(64, 8)).astype(np.float32)
    for bf16 in (True, False):
        assert np.array_equal(oracle.mlp_forward(learned_h.zero_params(), x, bf16=bf16), np.zeros(64))
