"""Inputs of the reference's own tests, regenerated from their seeded generators.

* ``splitmix`` / ``cloud``: the splitmix64 stream and the 1e6 m random cloud of
  ``crates/engine/src/bhtree.rs:197-215`` and ``tools/gpu-bh-verify/src/main.rs:115-138`` (masses 1e18·(0.5+U)).
* ``neighbour_cloud``: the 800-point cloud of ``crates/engine/src/neighbors.rs:94-117``.
* ``verify_config``: the 300-particle Fibonacci cluster of ``tools/sph-verify/src/main.rs:253-289``.
"""
from __future__ import annotations

import math

import numpy as np

from botheadstudios_b200.materials import MAT_BASALT, MAT_IRON

M64 = (1 << 64) - 1


def splitmix(state: int):
    """One splitmix64 step as in bhtree.rs:197-203: returns (new_state, value in [0,1))."""
    state = (state + 0x9E3779B97F4A7C15) & M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return state, ((z ^ (z >> 31)) >> 11) / float(1 << 53)


def cloud(n: int, seed: int):
    """gpu-bh-verify build_cloud: returns (bodies f32 [n,4], pos f64 [n,3], mass f64 [n])."""
    s = seed
    pos = np.empty((n, 3))
    mass = np.empty(n)
    for i in range(n):
        s, a = splitmix(s)
        s, b = splitmix(s)
        s, c = splitmix(s)
        pos[i] = (a * 1.0e6, b * 1.0e6, c * 1.0e6)
        s, m = splitmix(s)
        mass[i] = 1.0e18 * (0.5 + m)
    bodies = np.concatenate([pos, mass[:, None]], axis=1).astype(np.float32)
    return bodies, pos, mass


def neighbour_cloud(n: int = 800, seed: int = 0x12345678):
    s = seed
    pos = np.empty((n, 3))
    for i in range(n):
        for k in range(3):
            s, v = splitmix(s)
            pos[i, k] = v * 100.0
    return pos


def _rnd(i: int, salt: int) -> float:
    """sph-verify rnd(): deterministic in [-1, 1)."""
    x = ((i + salt) * 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    return ((x >> 40) & 0xFFFF) / 32768.0 - 1.0


def verify_config(n: int = 300):
    """sph-verify build_config(n): AoS fields as f32 arrays (pos4 with h in w, vel4 with u in w, mass, mat, rho)."""
    r0 = 1.0e5
    vol_per = 4.0 / 3.0 * math.pi * r0 * r0 * r0 / n
    spacing = vol_per ** (1.0 / 3.0)
    h = np.float32(2.6 * spacing)
    golden = math.pi * (3.0 - math.sqrt(5.0))
    pos4 = np.zeros((n, 4), np.float32)
    vel4 = np.zeros((n, 4), np.float32)
    mass = np.zeros(n, np.float32)
    mat = np.zeros(n, np.uint32)
    rho = np.zeros(n, np.float32)
    for i in range(n):
        rr = r0 * ((i + 0.5) / n) ** (1.0 / 3.0)
        y = 1.0 - 2.0 * (i + 0.5) / n
        rad = math.sqrt(max(1.0 - y * y, 0.0))
        th = golden * i
        pos4[i, :3] = (math.cos(th) * rad * rr, y * rr, math.sin(th) * rad * rr)
        pos4[i, 3] = h
        m = MAT_IRON if rr < 0.5 * r0 else MAT_BASALT
        rho0 = 7850.0 if m == MAT_IRON else 2700.0
        vel4[i, :3] = (200.0 * _rnd(i, 1), 200.0 * _rnd(i, 2), 200.0 * _rnd(i, 3))
        vel4[i, 3] = 1.0e6
        mass[i] = rho0 * vol_per
        mat[i] = m
        rho[i] = rho0
    return pos4, vel4, mass, mat, rho


def splitmix_subsample(n_total: int, n: int, seed: int = 2) -> np.ndarray:
    """n distinct indices of range(n_total), ascending, drawn by a partial Fisher-Yates shuffle whose random
    numbers are the splitmix64 stream (bhtree.rs:197-203) started at `seed`."""
    idx = np.arange(n_total, dtype=np.int64)
    s = seed
    for k in range(n):
        s, u = splitmix(s)
        j = k + min(int(u * (n_total - k)), n_total - k - 1)
        idx[k], idx[j] = idx[j], idx[k]
    return np.sort(idx[:n])


def subsample_impact(I, n: int, seed: int = 2):
    """A seeded n-particle subsample of a built impact as a self-consistent body: the chosen particles keep
    their positions, velocities, u and materials; mass and smoothing length scale by N/n and (N/n)^(1/3) so the
    density and the neighbour count stay those of the full impact (the softening scales with h).
    Returns (particles, softening)."""
    N = len(I.particles)
    sel = splitmix_subsample(N, n, seed)
    p = I.particles[sel].copy()
    f = N / n
    p["mass"] = (p["mass"].astype(np.float64) * f).astype(np.float32)
    p["h"] = (p["h"].astype(np.float64) * f ** (1.0 / 3.0)).astype(np.float32)
    return p, float(I.softening * f ** (1.0 / 3.0))
