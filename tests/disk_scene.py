"""Seeded synthetic post-impact scenes (SI) for the disk measurement: a remnant ball, a thin ring of orbiting
debris, escaping particles and a few clumps placed to exercise each gate of the Moon-candidate test (bound and
outside the Roche limit, bound but inside it, unbound and hot). Provenance 0 is the target, 1 the impactor."""
import math

import numpy as np

from botheadstudios_b200._lib import PARTICLE_DTYPE
from botheadstudios_b200.materials import eos_table

G = 6.674e-11
R = 6.4e6  # m

# (members, orbit radius / R, internal velocity dispersion m/s, angle rad)
CLUMPS = ((40, 4.5, 5.0, 0.0), (25, 5.2, 5.0, math.pi), (30, 2.2, 5.0, 0.5 * math.pi), (30, 4.0, 1000.0, 1.5 * math.pi))


def _ball(rng, n, radius):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v * (radius * rng.random(n) ** (1.0 / 3.0))[:, None]


def scene(seed=0, n_rem=6000, n_ring=300, n_esc=100, clumps=CLUMPS, m_rem=1.0e21, m_debris=1.0e18,
          h_rem=7.0e5, h_debris=2.0e5, clump_radius=3.0e5, rho_clump=3000.0):
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
    add(_ball(rng, n_rem, R), rng.normal(scale=10.0, size=(n_rem, 3)), m_rem, h_rem, 5000.0,
        (rng.random(n_rem) < 0.1).astype(np.uint32))
    # ring: near-circular orbits in a thin sheet, kept away from the clumps' azimuths
    r = R * (1.6 + 4.4 * rng.random(n_ring))
    phi = rng.random(n_ring) * 2.0 * math.pi
    for c in clumps:
        d = np.angle(np.exp(1j * (phi - c[3])))
        phi = np.where(np.abs(d) < 0.35, phi + 0.7, phi)
    p = np.stack([r * np.cos(phi), r * np.sin(phi), rng.normal(scale=0.02 * R, size=n_ring)], 1)
    vc = np.sqrt(G * M / r) * (0.97 + 0.03 * rng.random(n_ring))
    v = np.stack([-vc * np.sin(phi), vc * np.cos(phi), np.zeros(n_ring)], 1)
    add(p, v, m_debris, h_debris, 2000.0, (rng.random(n_ring) < 0.6).astype(np.uint32))
    # escaping: outward at twice the local escape speed
    r = R * (2.0 + 2.0 * rng.random(n_esc))
    d = rng.normal(size=(n_esc, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    add(d * r[:, None], d * (2.0 * np.sqrt(2.0 * G * M / r))[:, None], m_debris, h_debris, 2000.0,
        (rng.random(n_esc) < 0.5).astype(np.uint32))
    # clumps on circular orbits
    for n, rr, sigma, ang in clumps:
        c = np.array([rr * R * math.cos(ang), rr * R * math.sin(ang), 0.0])
        vc = math.sqrt(G * M / (rr * R))
        cv = np.array([-vc * math.sin(ang), vc * math.cos(ang), 0.0])
        add(c + _ball(rng, n, clump_radius), cv + rng.normal(scale=sigma, size=(n, 3)), m_debris, h_debris,
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


def eos():
    return eos_table()
