"""CPU pins of the oracle's smoothing-length solve, relaxation step and Courant signal (no GPU).

The reference keeps h fixed (crates/engine/src/hydrostatic.rs:59-61), so the solve has no reference test to
reproduce; it is pinned by what the method promises: the f64 Newton iteration of Price (2012) settles on
ρ_i h_i³ = m_i η³ wherever no limit holds h, contracts by a large factor per step, and the f32 restatement (the
device's sequence) reaches the same solution. cs_relax (sph_step.wgsl:245-257) and cs_signal (:263-269) are
checked against closed forms and against the f64 HydroBody::courant_dt (hydrostatic.rs:366-374).
"""
import numpy as np
import pytest

import oracle
from botheadstudios_b200 import ic
from botheadstudios_b200 import materials as M

SKIN = 0.15


def _body(n=4000, seed=3):
    I = ic.planet(n, n_ngb=64.0, seed=seed)
    p = I.particles
    return I, p, np.float32(ic.eta_for(64.0))


def _clamped(h, h0, skin=SKIN):
    """Particles held at a skin bound of the limited iteration (the surface, where ρ(h) cannot reach the
    target inside one rebuild's box)."""
    hi = h0 * (1.0 + skin) * 0.999
    lo = h0 / ((1.0 + skin) * 1.001)
    return (np.abs(h / hi - 1.0) < 1e-9) | (np.abs(h / lo - 1.0) < 1e-9)


def test_f64_solve_settles_on_the_target_density():
    I, p, eta = _body()
    h0 = p["h"].astype(np.float64)
    h, rho, res, steps = oracle.h_solve64(p["pos"].astype(np.float64), h0, p["mass"].astype(np.float64),
                                          float(eta), SKIN)
    assert steps <= 60
    free = ~_clamped(h, h0)
    assert free.mean() > 0.5
    # ρ_i h_i³ = m_i η³ where no limit holds the particle (Price 2012, eq. 10)
    lhs = rho[free] * h[free] ** 3
    rhs = p["mass"][free].astype(np.float64) * float(eta) ** 3
    assert np.max(np.abs(lhs / rhs - 1.0)) < 1e-10
    assert np.max(res[free]) < 1e-10


def test_f64_iteration_contracts_in_the_interior():
    """Each Jacobi-Newton step cuts the interior residual by at least 5×: the per-particle Newton step is
    exact in h_i, and what is left comes from the neighbours' h_j moving in the same step (the symmetric h_ij
    couples them), so the coupled iteration converges linearly with a small ratio."""
    I, p, eta = _body(3000, seed=5)
    args = (p["pos"].astype(np.float64), p["h"].astype(np.float64), p["mass"].astype(np.float64), float(eta), SKIN)
    h_final, *_ = oracle.h_solve64(*args)
    free = ~_clamped(h_final, p["h"].astype(np.float64))
    r = []
    for k in (1, 2, 3, 4, 5):
        _, _, res, _ = oracle.h_solve64(*args, step_tol=0.0, max_iter=k)
        r.append(float(np.percentile(res[free], 90)))
    for a, b in zip(r, r[1:]):
        assert b < 0.2 * a, r


def test_f32_solve_reaches_the_f64_solution():
    I, p, eta = _body()
    pos4 = np.ascontiguousarray(np.concatenate([p["pos"], p["h"][:, None]], 1), dtype=np.float32)
    h64, _, _, _ = oracle.h_solve64(p["pos"].astype(np.float64), p["h"].astype(np.float64),
                                    p["mass"].astype(np.float64), float(eta), SKIN)
    h32, rho32, res32 = oracle.h_solve32(pos4, p["mass"], eta, SKIN, 30)
    assert np.max(np.abs(h32 / h64 - 1.0)) < 2e-6
    # the final density pass is the density sum at the final h
    pf = pos4.copy()
    pf[:, 3] = h32
    assert np.max(np.abs(oracle.density32(pf, p["mass"], kernel=1) / rho32 - 1.0)) < 1e-6
    # two iterations (the benchmark's) already bring the interior within 1 %
    h2, _, _ = oracle.h_solve32(pos4, p["mass"], eta, SKIN, 2)
    free = ~_clamped(h64, p["h"].astype(np.float64))
    assert np.percentile(np.abs(h2[free] / h64[free] - 1.0), 90) < 1e-2


def test_relax32_closed_form():
    """cs_relax on a particle at rest with no force: only the centrifugal term ω²(x, y, 0) acts."""
    pos4 = np.array([[3.0, -2.0, 5.0, 1.0], [0.0, 0.0, 1.0, 1.0]], np.float32)
    vel4 = np.zeros((2, 4), np.float32)
    acc4 = np.zeros((2, 4), np.float32)
    dt, damp, w = 0.5, 0.9, 0.2
    p, v = oracle.relax32(pos4, vel4, acc4, dt, damp, w)
    want_v = np.float32(w * w) * pos4[0, :3] * np.float32(dt) * np.float32(damp)
    want_v[2] = 0.0
    assert np.allclose(v[0, :3], want_v, rtol=1e-6)
    assert np.allclose(p[0, :3], pos4[0, :3] + want_v * np.float32(dt), rtol=1e-6)
    assert np.array_equal(v[1, :3], np.zeros(3, np.float32)) and np.array_equal(p[1], pos4[1])
    assert p[0, 3] == pos4[0, 3]  # h untouched


def test_signal32_matches_hydrobody_courant_dt():
    """cfl·min of the shader's signal (f32, sound speed with 1e-3 steps) against the CPU path's courant_dt
    (f64, 1e-4 steps) on the sph-verify cluster, in SI units as the reference runs it."""
    from refcases import verify_config
    pos4, vel4, mass, mat, rho = verify_config(300)
    eos10 = M.eos_table64()
    hb = oracle.HydroBody(pos4[:, :3], vel4[:, :3], mass, vel4[:, 3], pos4[:, 3], mat, eos10, 1.0e4)
    hb.compute_density()
    dt64 = hb.courant_dt(0.3)
    rho_o = oracle.density32(pos4, mass)
    _, c = oracle.eos32(M.eos_table(), mat, rho_o, vel4[:, 3])
    dt32 = 0.3 * float(oracle.signal32(pos4, vel4, c).min())
    assert dt32 == pytest.approx(dt64, rel=2e-3)
    # a particle at rest in a vacuum of sound: the floor of 1 m/s applies
    s = oracle.signal32(np.array([[0, 0, 0, 2.0]], np.float32), np.zeros((1, 4), np.float32),
                        np.zeros(1, np.float32))
    assert s[0] == np.float32(2.0)
