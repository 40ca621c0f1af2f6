"""Seeded synthetic initial conditions for the giant-impact workloads.

Bodies are differentiated: 30 % iron core / 70 % basalt mantle by mass, equal-mass particles, each region
seeded on its own cubic lattice at the material's reference density (the reference's construction,
``crates/engine/src/hydrostatic.rs:97-144`` ``new_differentiated``, uses equal-mass particles at the same
densities on Fibonacci shells; a lattice is used here), with a uniform ±jitter·h displacement per axis.
Smoothing lengths target a neighbour count inside the support radius h: (4π/3)(h/Δ)³ = N_ngb.
Impacts: impactor mass ratio q, speed v_imp = f·v_esc at contact, impact angle from the contact normal,
initial centre separation d0 (in target radii); the pair is placed on the straight-line approach that has
that contact speed and impact parameter (energy and angular momentum of the two-body orbit), in the
centre-of-mass frame. All values are in the unit system passed in (code units by default: G = M_t = R_t = 1).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from ._lib import PARTICLE_DTYPE
from .materials import G_SI, MAT_BASALT, MAT_IRON, TILLOTSON_SI, Units, code_units, eos_table


def eta_for(n_ngb: float) -> float:
    """h = eta·Δ such that (4π/3)(h/Δ)³ = n_ngb."""
    return (3.0 * n_ngb / (4.0 * math.pi)) ** (1.0 / 3.0)


def _lattice_ball(n: int, spacing: float, r_in: float, offset: float) -> np.ndarray:
    """The n lattice points (spacing Δ, shifted by offset·Δ) closest to the origin outside radius r_in."""
    r_out = (r_in ** 3 + n * spacing ** 3 * 3.0 / (4.0 * math.pi)) ** (1.0 / 3.0)
    m = int(math.ceil(r_out * 1.08 / spacing)) + 2
    while True:
        ax = (np.arange(-m, m + 1, dtype=np.float64) + offset) * spacing
        g = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), axis=-1).reshape(-1, 3)
        r = np.sqrt((g * g).sum(1))
        keep = r >= r_in
        g, r = g[keep], r[keep]
        if len(r) >= n:
            break
        m = int(m * 1.3) + 2
    # deterministic: by radius, ties by lattice order (stable sort)
    idx = np.argsort(r, kind="stable")[:n]
    return g[idx]


@dataclass
class Body:
    pos: np.ndarray
    mass: np.ndarray
    mat: np.ndarray
    h: np.ndarray
    radius: float
    total_mass: float
    spacing_min: float


def differentiated_body(n: int, total_mass: float, units: Units, n_ngb: float, iron_frac: float = 0.3,
                        jitter: float = 0.1, rng: np.random.Generator | None = None) -> Body:
    rfe = TILLOTSON_SI["iron"][0] / units.density
    rba = TILLOTSON_SI["basalt"][0] / units.density
    m = total_mass / n
    n_core = int(round(iron_frac * n))
    n_mant = n - n_core
    d_core = (m / rfe) ** (1.0 / 3.0)
    d_mant = (m / rba) ** (1.0 / 3.0)
    core = _lattice_ball(n_core, d_core, 0.0, 0.5) if n_core else np.zeros((0, 3))
    r_core = float(np.sqrt((core * core).sum(1)).max()) + 0.5 * d_core if n_core else 0.0
    mant = _lattice_ball(n_mant, d_mant, r_core, 0.25)
    pos = np.concatenate([core, mant])
    eta = eta_for(n_ngb)
    h = np.concatenate([np.full(n_core, eta * d_core), np.full(n_mant, eta * d_mant)])
    mat = np.concatenate([np.full(n_core, MAT_IRON, np.uint32), np.full(n_mant, MAT_BASALT, np.uint32)])
    if jitter > 0.0:
        rng = rng or np.random.default_rng(1)
        pos = pos + rng.uniform(-jitter, jitter, size=pos.shape) * h[:, None]
    radius = float(np.sqrt((pos * pos).sum(1)).max())
    return Body(pos=pos, mass=np.full(n, m), mat=mat, h=h, radius=radius, total_mass=total_mass,
                spacing_min=min(d_core, d_mant))


@dataclass
class Impact:
    particles: np.ndarray  # PARTICLE_DTYPE
    eos: np.ndarray        # [2, 12] float32
    softening: float
    units: Units
    pos64: np.ndarray      # f64 positions (the exchange format holds f32)
    n_target: int
    n_impactor: int


def impact(n_target: int, n_impactor: int, n_ngb: float = 48.0, mass_ratio: float = 0.1, v_factor: float = 1.1,
           angle_deg: float = 45.0, separation: float = 3.0, seed: int = 1, jitter: float = 0.1,
           u0_si: float = 1.0e6, units: Units | None = None) -> Impact:
    """Two differentiated bodies on an oblique collision course (configs of the giant-impact benchmark)."""
    units = units or code_units()
    rng = np.random.default_rng(seed)
    M_t = 1.0  # the target mass is the mass unit
    if units.G != 1.0:
        raise ValueError("impact() builds code-unit bodies (G = 1); pass code_units()")
    tgt = differentiated_body(n_target, 1.0, units, n_ngb, jitter=jitter, rng=rng)
    imp = differentiated_body(n_impactor, mass_ratio, units, n_ngb, jitter=jitter, rng=rng)
    M_i = mass_ratio
    R_sum = tgt.radius + imp.radius
    mu = M_t + M_i
    v_esc = math.sqrt(2.0 * mu / R_sum)
    v_c = v_factor * v_esc
    b_c = math.sin(math.radians(angle_deg)) * R_sum
    d0 = separation * tgt.radius
    v0 = math.sqrt(max(v_c * v_c - 2.0 * mu * (1.0 / R_sum - 1.0 / d0), 1e-12))
    b0 = min(b_c * v_c / v0, 0.999 * d0)
    rel_pos = np.array([math.sqrt(d0 * d0 - b0 * b0), b0, 0.0])
    rel_vel = np.array([-v0, 0.0, 0.0])
    # centre-of-mass frame
    ft, fi = M_i / mu, M_t / mu
    pos = np.concatenate([tgt.pos - ft * rel_pos, imp.pos + fi * rel_pos])
    vel = np.concatenate([np.tile(-ft * rel_vel, (n_target, 1)), np.tile(fi * rel_vel, (n_impactor, 1))])
    n = n_target + n_impactor
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["pos"] = pos.astype(np.float32)
    p["h"] = np.concatenate([tgt.h, imp.h]).astype(np.float32)
    p["vel"] = vel.astype(np.float32)
    p["u"] = np.float32(u0_si / units.energy)
    p["mass"] = np.concatenate([tgt.mass, imp.mass]).astype(np.float32)
    p["mat"] = np.concatenate([tgt.mat, imp.mat])
    rho0 = np.array([TILLOTSON_SI["basalt"][0], TILLOTSON_SI["iron"][0]]) / units.density
    p["rho"] = rho0[p["mat"]].astype(np.float32)
    p["prov"] = np.concatenate([np.zeros(n_target, np.uint32), np.ones(n_impactor, np.uint32)])
    soft = 0.5 * min(tgt.spacing_min, imp.spacing_min)
    return Impact(particles=p, eos=eos_table(units), softening=soft, units=units, pos64=pos, n_target=n_target,
                  n_impactor=n_impactor)


def planet(n: int, n_ngb: float = 64.0, seed: int = 3, jitter: float = 0.1, u0_si: float = 1.0e6,
           units: Units | None = None) -> Impact:
    """A single differentiated planet at rest (the equilibrium-planet precision workload)."""
    units = units or code_units()
    rng = np.random.default_rng(seed)
    b = differentiated_body(n, 1.0, units, n_ngb, jitter=jitter, rng=rng)
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["pos"] = b.pos.astype(np.float32)
    p["h"] = b.h.astype(np.float32)
    p["u"] = np.float32(u0_si / units.energy)
    p["mass"] = b.mass.astype(np.float32)
    p["mat"] = b.mat
    rho0 = np.array([TILLOTSON_SI["basalt"][0], TILLOTSON_SI["iron"][0]]) / units.density
    p["rho"] = rho0[p["mat"]].astype(np.float32)
    return Impact(particles=p, eos=eos_table(units), softening=0.5 * b.spacing_min, units=units, pos64=b.pos,
                  n_target=n, n_impactor=0)


def config_kwargs(units: Units) -> dict:
    """The unit-dependent fields of sph_config for these initial conditions."""
    return dict(G=units.G, rho_floor=units.rho_floor, du_floor=units.du_floor, r_min=units.r_min,
                sig_floor=units.sig_floor)


@dataclass
class Batch:
    particles: np.ndarray  # PARTICLE_DTYPE, impacts concatenated
    offsets: np.ndarray    # uint32 [n_impacts + 1]
    softening: np.ndarray  # float32 [n_impacts]
    eos: np.ndarray
    units: Units
    params: list           # per impact: dict(n, mass_ratio, angle_deg, v_factor, seed)

    @property
    def n_impacts(self) -> int:
        return len(self.offsets) - 1

    def impact(self, k: int) -> np.ndarray:
        return self.particles[self.offsets[k]:self.offsets[k + 1]]


def batch_draws(n_impacts: int, n_min: int, n_max: int, seed: int, mass_ratio=(0.05, 0.15), angle_deg=(0.0, 75.0),
                v_factor=(1.0, 1.5)) -> list:
    """The seeded per-impact draws of batch() (sizes and collision parameters) without building bodies."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_impacts):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        q = float(rng.uniform(*mass_ratio))
        ang = float(rng.uniform(*angle_deg))
        vf = float(rng.uniform(*v_factor))
        s = int(rng.integers(1, 2 ** 31 - 1))
        out.append(dict(n=n, mass_ratio=q, angle_deg=ang, v_factor=vf, seed=s))
    return out


def batch(n_impacts: int, n_min: int = 20_000, n_max: int = 200_000, n_ngb: float = 64.0, seed: int = 11,
          mass_ratio=(0.05, 0.15), angle_deg=(0.0, 75.0), v_factor=(1.0, 1.5)) -> Batch:
    """Independent two-body impacts of uneven size (the batched workload): total particle counts log-uniform
    in [n_min, n_max], impactor mass ratio, impact angle and v_imp/v_esc uniform in the given ranges, every
    draw from one seeded generator. Particles have equal mass within an impact, so the impactor holds the
    fraction q/(1+q) of them."""
    parts, offs, soft, params = [], [0], [], []
    I = None
    for d in batch_draws(n_impacts, n_min, n_max, seed, mass_ratio, angle_deg, v_factor):
        n, q, ang, vf, s = d["n"], d["mass_ratio"], d["angle_deg"], d["v_factor"], d["seed"]
        n_i = max(1, int(round(n * q / (1.0 + q))))
        I = impact(n - n_i, n_i, n_ngb=n_ngb, mass_ratio=q, v_factor=vf, angle_deg=ang, seed=s)
        parts.append(I.particles)
        offs.append(offs[-1] + len(I.particles))
        soft.append(I.softening)
        params.append(dict(n=n, mass_ratio=q, angle_deg=ang, v_factor=vf, seed=s))
    return Batch(particles=np.concatenate(parts), offsets=np.asarray(offs, np.uint32),
                 softening=np.asarray(soft, np.float32), eos=I.eos, units=I.units, params=params)


# ---- post-impact fields for the disk measurement -------------------------------------------------------
SCENE_R = 6.4e6  # m
# (members, orbit radius / SCENE_R, internal velocity dispersion m/s, azimuth rad): bound outside the Roche
# limit (the candidate), bound outside it and lighter, bound inside it, hot and unbound
SCENE_CLUMPS = ((40, 4.5, 5.0, 0.0), (25, 5.2, 5.0, math.pi), (30, 2.2, 5.0, 0.5 * math.pi),
                (30, 4.0, 1000.0, 1.5 * math.pi))


def _ball_si(rng, n, radius):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v * (radius * rng.random(n) ** (1.0 / 3.0))[:, None]


def post_impact_scene(seed=0, n_rem=6000, n_ring=300, n_esc=100, clumps=SCENE_CLUMPS, m_rem=1.0e21,
                      m_debris=1.0e18, h_rem=7.0e5, h_debris=2.0e5, clump_radius=3.0e5, rho_clump=3000.0):
    """A seeded post-impact particle field in SI (the input of the disk measurement): a remnant ball of n_rem
    particles of radius R = SCENE_R, a thin ring of n_ring near-circular orbits between 1.6 R and 6 R, n_esc
    particles leaving at twice the local escape speed, and clumps (members, orbit radius / R, velocity dispersion
    m/s, azimuth) on circular orbits. Provenance 0 is the target. The particles come out in a random order."""
    G = G_SI
    rng = np.random.default_rng(seed)
    M = n_rem * m_rem
    pos, vel, mass, h, rho, prov = [], [], [], [], [], []

    def add(p, v, m, hh, r, pv):
        pos.append(p)
        vel.append(v)
        mass.append(np.full(len(p), m))
        h.append(np.full(len(p), hh) * (1.0 + 0.1 * rng.random(len(p))))
        rho.append(np.full(len(p), r))
        prov.append(pv)

    # remnant: a nearly static ball, mostly target material
    add(_ball_si(rng, n_rem, SCENE_R), rng.normal(scale=10.0, size=(n_rem, 3)), m_rem, h_rem, 5000.0,
        (rng.random(n_rem) < 0.1).astype(np.uint32))
    # ring: near-circular orbits in a thin sheet, kept away from the clumps' azimuths
    r = SCENE_R * (1.6 + 4.4 * rng.random(n_ring))
    phi = rng.random(n_ring) * 2.0 * math.pi
    for c in clumps:
        d = np.angle(np.exp(1j * (phi - c[3])))
        phi = np.where(np.abs(d) < 0.35, phi + 0.7, phi)
    p = np.stack([r * np.cos(phi), r * np.sin(phi), rng.normal(scale=0.02 * SCENE_R, size=n_ring)], 1)
    vc = np.sqrt(G * M / r) * (0.97 + 0.03 * rng.random(n_ring))
    v = np.stack([-vc * np.sin(phi), vc * np.cos(phi), np.zeros(n_ring)], 1)
    add(p, v, m_debris, h_debris, 2000.0, (rng.random(n_ring) < 0.6).astype(np.uint32))
    # escaping: outward at twice the local escape speed
    r = SCENE_R * (2.0 + 2.0 * rng.random(n_esc))
    d = rng.normal(size=(n_esc, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    add(d * r[:, None], d * (2.0 * np.sqrt(2.0 * G * M / r))[:, None], m_debris, h_debris, 2000.0,
        (rng.random(n_esc) < 0.5).astype(np.uint32))
    # clumps on circular orbits
    for n, rr, sigma, ang in clumps:
        c = np.array([rr * SCENE_R * math.cos(ang), rr * SCENE_R * math.sin(ang), 0.0])
        vc = math.sqrt(G * M / (rr * SCENE_R))
        cv = np.array([-vc * math.sin(ang), vc * math.cos(ang), 0.0])
        add(c + _ball_si(rng, n, clump_radius), cv + rng.normal(scale=sigma, size=(n, 3)), m_debris, h_debris,
            rho_clump, (rng.random(n) < 0.7).astype(np.uint32))
    out = np.zeros(sum(len(x) for x in pos), PARTICLE_DTYPE)
    out["pos"] = np.concatenate(pos)
    out["vel"] = np.concatenate(vel)
    out["mass"] = np.concatenate(mass)
    out["h"] = np.concatenate(h)
    out["rho"] = np.concatenate(rho)
    out["prov"] = np.concatenate(prov)
    out["u"] = 1.0e5
    out["mat"] = 0
    perm = rng.permutation(len(out))  # no ordering for the measurement to lean on
    return out[perm]
