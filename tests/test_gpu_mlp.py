"""The learned-h MLP on the GPU: tensor-core forward and backward against the FP64 CPU oracle (with the same
BF16 operand rounding), training, and the solver's learned smoothing-length mode."""
import numpy as np
import pytest

import oracle
from botheadstudios_b200 import _lib, ic, learned_h
from botheadstudios_b200.gpusph import GpuSph

pytestmark = pytest.mark.gpu

BLOCKS = dict(W1=(learned_h.W1, learned_h.B1), b1=(learned_h.B1, learned_h.W2), W2=(learned_h.W2, learned_h.B2),
              b2=(learned_h.B2, learned_h.W3), W3=(learned_h.W3, learned_h.B3), b3=(learned_h.B3, learned_h.B3 + 1))


def _params(seed):
    rng = np.random.default_rng(seed)
    p = learned_h.init_params(rng.normal(0, 0.3, 8), rng.uniform(0.5, 2.0, 8), 0.004, 0.01, seed=seed)
    p[learned_h.W3:learned_h.B3] *= 10.0  # a network whose output moves with its inputs
    p[learned_h.B1:learned_h.W2] = rng.normal(0, 0.1, 64)
    return p


def test_forward_matches_oracle():
    p = _params(5)
    x = np.random.default_rng(6).normal(size=(1000, 8)).astype(np.float32)
    got = learned_h.forward(p, x)
    want = oracle.mlp_forward(p, x, bf16=True)
    scale = np.abs(want - p[learned_h.YM]).max()
    # FP32 sums in another order than the FP64 oracle: ≤ 2e-3 of the output range
    assert np.abs(got - want).max() <= 2e-3 * scale


def test_gradient_matches_oracle():
    p = _params(7)
    rng = np.random.default_rng(8)
    x = rng.normal(size=(1000, 8)).astype(np.float32)  # 7 full tiles of 128 and a partial one
    t = (0.004 + 0.01 * np.tanh(x[:, 2]) + 0.003 * x[:, 0] * x[:, 1]).astype(np.float32)
    lg, gg = learned_h.grad(p, x, t)
    lc, gc = oracle.mlp_grad(p, x, t, bf16=True)
    _, g64 = oracle.mlp_grad(p, x, t, bf16=False)
    assert abs(lg - lc) <= 1e-3 * lc
    for name, (a, b) in BLOCKS.items():
        ref = np.linalg.norm(gc[a:b])
        # same BF16 operands, FP32 vs FP64 sums: 1 %; against the unrounded FP64 gradient: 5 %
        assert np.linalg.norm(gg[a:b] - gc[a:b]) <= 1e-2 * ref, name
        assert np.linalg.norm(gg[a:b] - g64[a:b]) <= 5e-2 * np.linalg.norm(g64[a:b]), name


def test_training_fits_a_smooth_target():
    rng = np.random.default_rng(9)
    x = rng.normal(size=(40_000, 8)).astype(np.float32)
    t = (0.004 + 0.01 * np.tanh(x[:, 2]) + 0.003 * x[:, 0] * x[:, 1]).astype(np.float32)
    p, losses = learned_h.fit(x[:32_000], t[:32_000], schedule=((25, 3e-3),), batch=2048)
    assert losses[-1] < 0.05 * losses[0]
    pred = learned_h.forward(p, x[32_000:])
    err = np.sqrt(np.mean((pred - t[32_000:]) ** 2))
    assert err < 0.2 * t[32_000:].std()


def _impact():
    return ic.impact(8192, 2048, n_ngb=64.0, seed=12)


def test_learned_mode_with_zero_network_matches_the_iterative_solve():
    I = _impact()
    out = {}
    for mode in ("solve", "learned"):
        with GpuSph(len(I.particles), **learned_h.solver_config(I.units, h_mode=mode, h_iters=4)) as s:
            s.upload(I.particles, I.eos, I.softening)
            s.encode_kdk(2)
            out[mode] = (s.inspect("RHO"), s.diag())
    rho_s, d_s = out["solve"]
    rho_l, d_l = out["learned"]
    assert d_l["h_residual"] <= 2e-3 and d_s["h_residual"] <= 2e-3
    assert 0 < d_l["h_accepted"] <= len(I.particles)
    # two solves within their tolerance of the same equation after one learned step
    assert np.abs(rho_l / rho_s - 1.0).max() < 5e-3


def test_recorded_features():
    I = _impact()
    with GpuSph(len(I.particles), **learned_h.solver_config(I.units, h_mode="solve")) as s:
        s.upload(I.particles, I.eos, I.softening)
        s.mlp_record(True)
        s.set_progress(0.25)
        s.encode_kdk(2)
        f, d = s.mlp_features()
        mat = I.particles["mat"]
    assert np.isfinite(f).all() and np.array_equal(d, -f[:, 0])  # the zero network proposes h(rho)
    assert np.array_equal(f[:, 5], mat.astype(np.float32))
    assert np.all(f[:, 7] == np.float32(0.25))
    assert 0.5 < np.median(f[:, 3]) < 1.5            # neighbours / target
    assert np.abs(np.median(f[:, 0])) < 0.05          # h sits at h(rho) after the solve
    assert np.abs(f[:, 2]).max() < 0.5               # div v dt: a fraction of the volume per step


def _run(I, params, mode="learned", steps=6):
    with GpuSph(len(I.particles), **learned_h.solver_config(I.units, h_mode=mode, h_iters=2)) as s:
        if params is not None:
            s.mlp_set(params)
        s.upload(I.particles, I.eos, I.softening)
        s.encode_kdk(2)  # the fresh solve and the first learned step
        acc, res = [], []
        for k in range(steps):
            s.set_progress(k / steps)
            s.encode_kdk(1)
            d = s.diag()
            acc.append(d["h_accepted"] / len(I.particles))
            res.append(d["h_residual"])
        return np.array(acc), np.array(res), s.readback()


def _density_error(I, state):
    """Relative density error of a final state against a converged solve (8 Newton iterations) on the same
    positions: (rms, max)."""
    with GpuSph(len(I.particles), **learned_h.solver_config(I.units, h_mode="solve", h_iters=8)) as s:
        s.upload(state, I.eos, I.softening)
        s.eval_forces()
        rho_conv = s.inspect("RHO")
    e = np.abs(state["rho"] / rho_conv - 1.0)
    return float(np.sqrt(np.mean(e * e))), float(e.max())


def test_trained_network_gains_over_the_method_without_it():
    # held out: a 33,000-particle impact (the network saw the 10,240-particle impact and a planet)
    I = ic.impact(30_000, 3_000, n_ngb=64.0, seed=77)
    acc_t, res_t, out_t = _run(I, learned_h.load())
    acc_0, res_0, out_0 = _run(I, None)  # without the network: the proposal is h(rho) of the last step
    # what the network gains: several times more particles pass the first check ...
    assert acc_t.mean() > 2.5 * acc_0.mean() and acc_t.mean() > 0.3
    # ... with every final residual within the tolerance (1e-3) ...
    assert res_t.max() <= 1.0001e-3 and res_0.max() <= 1.3e-3
    # ... and densities closer to a converged solve than without it (rms well inside 1e-3)
    rms_t, max_t = _density_error(I, out_t)
    rms_0, max_0 = _density_error(I, out_0)
    assert rms_t <= rms_0 and max_t <= max_0
    assert rms_t <= 3e-4 and max_t <= 3e-3
