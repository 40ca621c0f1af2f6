"""Learned smoothing lengths: the network's parameter block, training data from the solver's own trajectories,
training on the GPU through the library's kernels, and the parameter file the solver loads.

The network (8 → 64 → 64 → 1, GELU) proposes each particle's Δlog h for the coming step; see sph_b200.h for the
features. Training targets are log(h_next/h(ρ)): the smoothing lengths a converged iterative solve reaches at
the next step, relative to the equilibrium h(ρ) = η(m/ρ)^(1/3) of the current density,
recorded while the plain solver runs (SPH_H_SOLVE with many iterations), so the network learns to land where
the iteration would. In SPH_H_LEARNED the solver checks every proposal's density residual and iterates only
the rejected particles, so a poor proposal costs iterations, never accuracy.

    python -m botheadstudios_b200.learned_h train [--out FILE]    # collect, train, save (needs a GPU)
    python -m botheadstudios_b200.learned_h eval                  # held-out comparison with plain Newton
"""
from __future__ import annotations

import argparse
import ctypes as C
import os

import numpy as np

from . import _lib, ic
from ._lib import MLP_PARAMS, MLP_TRAINABLE

N_IN, N_H = 8, 64
W1, B1 = 0, N_IN * N_H
W2 = B1 + N_H
B2 = W2 + N_H * N_H
W3 = B2 + N_H
B3 = W3 + N_H
XM, XS = MLP_TRAINABLE, MLP_TRAINABLE + N_IN
YM, YS = XS + N_IN, XS + N_IN + 1
assert YS + 1 == MLP_PARAMS

FEATURES = ("log h/h(rho)", "log rho/rho0", "div v dt", "neighbours/target", "log(1+|a|h/c^2)", "material",
            "log(1+u/E_iv)", "progress")
DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "learned_h.npz")


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(st, what):
    if st < 0:
        raise RuntimeError(f"{what} failed: {_lib.load().sph_status_string(st).decode()}")


def zero_params() -> np.ndarray:
    """The zero network (Δlog h = 0): what the solver holds before sph_mlp_set."""
    p = np.zeros(MLP_PARAMS, np.float32)
    p[XS:XS + N_IN] = 1.0
    p[YS] = 1.0
    return p


def init_params(x_mean, x_scale, y_mean, y_scale, seed: int = 0) -> np.ndarray:
    """He-normal hidden weights, small output weights, the given normalisation."""
    rng = np.random.default_rng(seed)
    p = zero_params()
    p[W1:B1] = rng.normal(0.0, np.sqrt(2.0 / N_IN), N_IN * N_H)
    p[W2:B2] = rng.normal(0.0, np.sqrt(2.0 / N_H), N_H * N_H)
    p[W3:B3] = rng.normal(0.0, 0.1 / np.sqrt(N_H), N_H)
    p[XM:XM + N_IN] = x_mean
    p[XS:XS + N_IN] = x_scale
    p[YM], p[YS] = y_mean, y_scale
    return p


def normalisation(X: np.ndarray, T: np.ndarray):
    """Per-feature mean and inverse spread (constant features get scale 1), target mean and spread."""
    xm = X.mean(0)
    sd = X.std(0)
    xs = np.where(sd > 1e-12, 1.0 / np.maximum(sd, 1e-12), 1.0)
    return xm.astype(np.float32), xs.astype(np.float32), float(T.mean()), float(max(T.std(), 1e-12))


# ---- the library's kernels ---------------------------------------------------------------------------------
def forward(params: np.ndarray, X: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(X, np.float32).reshape(-1, N_IN)
    out = np.zeros(len(x), np.float32)
    _check(_lib.load().sph_mlp_forward(_ptr(p), _ptr(x), len(x), _ptr(out)), "sph_mlp_forward")
    return out


def grad(params: np.ndarray, X: np.ndarray, T: np.ndarray):
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(X, np.float32).reshape(-1, N_IN)
    t = np.ascontiguousarray(T, np.float32)
    g = np.zeros(MLP_TRAINABLE, np.float32)
    loss = C.c_float()
    _check(_lib.load().sph_mlp_grad(_ptr(p), _ptr(x), _ptr(t), len(x), _ptr(g), C.byref(loss)), "sph_mlp_grad")
    return float(loss.value), g


def train(params: np.ndarray, X: np.ndarray, T: np.ndarray, epochs: int = 20, batch: int = 4096,
          lr: float = 2e-3, seed: int = 0, weight_decay: float = 0.0):
    """Adam on the GPU; returns (trained parameters, per-epoch mean training loss)."""
    p = np.ascontiguousarray(params, np.float32).copy()
    x = np.ascontiguousarray(X, np.float32).reshape(-1, N_IN)
    t = np.ascontiguousarray(T, np.float32)
    cfg = _lib.MlpTrainCfg(epochs=epochs, batch=batch, lr=lr, beta1=0.9, beta2=0.999, eps=1e-8,
                           weight_decay=weight_decay, seed=seed)
    losses = np.zeros(max(epochs, 1), np.float32)
    _check(_lib.load().sph_mlp_train(_ptr(p), _ptr(x), _ptr(t), len(x), C.byref(cfg), _ptr(losses)),
           "sph_mlp_train")
    return p, losses[:epochs]


# ---- training data -------------------------------------------------------------------------------------------
def solver_config(units, h_mode: int = 1, h_iters: int = 2, **over) -> dict:
    """The learned-h method's solver (the 1M/4M impact method: Wendland C2, 64 neighbours, θ = 0.6 with
    quadrupoles, 16-particle leaves, CFL 0.3)."""
    kw = dict(theta=0.6, leaf_size=16, kernel="wendland", multipole=1, h_mode=h_mode, h_neighbours=64.0,
              h_iters=h_iters, max_neighbours=192, cfl=0.3, **ic.config_kwargs(units))
    kw.update(over)
    return kw


def collect(I, steps: int, every: int = 1, h_iters: int = 6, device: int = -1, max_rows: int | None = None,
            seed: int = 0, skip: int = 0):
    """Run the plain solver (a converged iterative solve) on initial conditions I for `steps` KDK steps and
    record (features at the start of each step's drift, Δlog h the solve reached), leaving out the first
    `skip` steps (the settling of the initial lattice). Returns (X, T)."""
    from .gpusph import GpuSph
    rng = np.random.default_rng(seed)
    Xs, Ts = [], []
    with GpuSph(len(I.particles), device=device, **solver_config(I.units, h_mode=1, h_iters=h_iters)) as s:
        s.upload(I.particles, I.eos, I.softening)
        s.mlp_record(True)
        s.encode_kdk(1)  # the first force evaluation: h solved from the initial guess
        for k in range(steps):
            s.set_progress(k / max(steps - 1, 1))
            h0 = s.inspect("H").astype(np.float64)
            s.encode_kdk(1)
            if k < skip or k % every:
                continue
            f, _ = s.mlp_features()
            h1 = s.inspect("H").astype(np.float64)
            # the network's target: log(h_next / h(rho)) = log(h_next / h) + log(h / h(rho))
            t = (np.log(h1 / h0) + f[:, 0]).astype(np.float32)
            if max_rows and len(t) > max_rows:
                sel = rng.choice(len(t), max_rows, replace=False)
                f, t = f[sel], t[sel]
            Xs.append(f)
            Ts.append(t)
    return np.concatenate(Xs), np.concatenate(Ts)


def training_set(device: int = -1, quick: bool = False):
    """Trajectories of the two training shapes: the 10,240-particle two-body impact (8,192 + 2,048) and an
    equilibrium planet (131,072 particles; 16,384 for a quick set), both with the learned-h method's solver."""
    steps_i, steps_p = (30, 10) if quick else (300, 80)
    Ii = ic.impact(8192, 2048, n_ngb=64.0, seed=5)
    Ip = ic.planet(16_384 if quick else 131_072, n_ngb=64.0, seed=6)
    Xa, Ta = collect(Ii, steps_i, device=device, skip=3 if quick else 10)
    Xb, Tb = collect(Ip, steps_p, device=device, max_rows=None if quick else 32_768, skip=2 if quick else 5)
    return np.concatenate([Xa, Xb]), np.concatenate([Ta, Tb])


# (epochs, learning rate) stages; Adam restarts at each stage
SCHEDULE = ((80, 2e-3), (40, 5e-4), (20, 1.25e-4))


def fit(X, T, schedule=SCHEDULE, batch: int = 4096, seed: int = 0):
    """Train from a fresh initialisation through the stages of `schedule`; returns (params, losses)."""
    xm, xs, ym, ys = normalisation(X, T)
    p = init_params(xm, xs, ym, ys, seed=seed)
    losses = []
    for k, (epochs, lr) in enumerate(schedule):
        p, l = train(p, X, T, epochs=epochs, batch=batch, lr=lr, seed=seed + k)
        losses.append(l)
    return p, np.concatenate(losses)


def save(params: np.ndarray, path: str = DEFAULT_PATH, **meta):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=np.asarray(params, np.float32), **{k: np.asarray(v) for k, v in meta.items()})


def load(path: str = DEFAULT_PATH) -> np.ndarray:
    p = np.load(path)["params"].astype(np.float32)
    if p.shape != (MLP_PARAMS,):
        raise ValueError(f"{path}: expected {MLP_PARAMS} parameters, found {p.shape}")
    return p


def evaluate(I, params=None, mode: str = "learned", steps: int = 6, h_iters: int = 2, device: int = -1) -> dict:
    """One held-out run: 2 steps to settle, then `steps` timed KDK steps; first-pass acceptance, residual,
    smoothing-length phase time per rebuild, and the final densities' error against an 8-iteration solve on the
    same positions."""
    from .gpusph import GpuSph
    with GpuSph(len(I.particles), device=device, **solver_config(I.units, h_mode=mode, h_iters=h_iters)) as s:
        if params is not None:
            s.mlp_set(params)
        s.upload(I.particles, I.eos, I.softening)
        s.encode_kdk(2)
        s.sync()
        acc, res = [], []
        s.profile_enable(True)
        for k in range(steps):
            s.set_progress(k / steps)
            s.encode_kdk(1)
            d = s.diag()
            acc.append(d["h_accepted"] / len(I.particles))
            res.append(d["h_residual"])
        pr = s.profile_read()
        out = s.readback()
    with GpuSph(len(I.particles), device=device, **solver_config(I.units, h_mode="solve", h_iters=8)) as s:
        s.upload(out, I.eos, I.softening)
        s.eval_forces()
        rho_conv = s.inspect("RHO")
    e = np.abs(out["rho"] / rho_conv - 1.0)
    return dict(accepted=float(np.mean(acc)), residual=float(max(res)), hsolve_ms_per_step=pr["ms"]["hsolve"] / steps,
                step_ms=sum(pr["ms"].values()) / steps, density_rms=float(np.sqrt(np.mean(e * e))),
                density_max=float(e.max()))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--quick", action="store_true")
    a = ap.parse_args(argv)
    if a.cmd == "eval":
        # held-out impacts (the network saw the 10,240-particle impact and the planet)
        import json
        p = load()
        for nt, ni, seed in ((30_000, 3_000, 77), (953_250, 95_326, 79)):
            I = ic.impact(nt, ni, n_ngb=64.0, seed=seed)
            rows = dict(trained=evaluate(I, p), zero_network=evaluate(I, None),
                        newton2=evaluate(I, None, mode="solve"), newton1=evaluate(I, None, mode="solve", h_iters=1))
            print(json.dumps(dict(particles=nt + ni, **rows)), flush=True)
        return
    X, T = training_set(quick=a.quick)
    p, losses = fit(X, T, schedule=((5, 2e-3),) if a.quick else SCHEDULE)
    save(p, a.out, losses=losses, rows=len(X))
    print(f"trained on {len(X)} rows: loss {losses[0]:.4g} -> {losses[-1]:.4g}; saved {a.out}")


if __name__ == "__main__":
    main()
