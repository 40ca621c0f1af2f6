"""The reference's own deterministic body builders, restated (SI units, as the reference builds them).

The engine seeds its impacts on Fibonacci spheres with equal-volume radii, no random numbers:
``fib_dir`` (crates/engine/src/hydrostatic.rs:32-38), ``HydroBody::new_sphere`` (:66-90),
``HydroBody::new_differentiated`` (:97-139), ``HydroBody::new_lod`` (:146-184), ``HydroBody::particalize``
(:199-238) with ``LayeredBody::temperature_at`` (crates/engine/src/planet.rs:87-97), and the offline impact
tool's 48-byte builders ``build_differentiated`` / ``build_lod`` (tools/impact-run/src/main.rs:103-176) with its
ensemble jitter ``hash_jitter`` (:179-190). Each builder returns 48-byte particles (`PARTICLE_DTYPE`, positions
rounded to f32 as the tool does) plus its softening, so a reference-built body goes through the CUDA path as
the reference would upload it. Material indices follow the engine's table (basalt 0, iron 1).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from ._lib import PARTICLE_DTYPE
from .materials import MAT_BASALT, MAT_IRON, TILLOTSON_SI

FOUR_THIRDS_PI = 4.0 / 3.0 * math.pi
M64 = (1 << 64) - 1


def fib_dir(i: np.ndarray, n: int, offset: float) -> np.ndarray:
    """Near-uniform directions on the unit sphere (hydrostatic.rs:32-38): y = 1 − 2(i + ½)/n, azimuth
    golden·i + offset with golden = π(3 − √5). Vectorised over i."""
    golden = math.pi * (3.0 - math.sqrt(5.0))
    i = np.asarray(i, dtype=np.float64)
    y = 1.0 - 2.0 * (i + 0.5) / n
    r = np.sqrt(np.maximum(1.0 - y * y, 0.0))
    th = golden * i + offset
    return np.stack([np.cos(th) * r, y, np.sin(th) * r], axis=-1)


def smoothing_for(m: float, rho0: float) -> float:
    """h ≈ two mean spacings of material at ρ0 (hydrostatic.rs:59-61)."""
    return 2.0 * (m / rho0) ** (1.0 / 3.0)


@dataclass
class RefBody:
    particles: np.ndarray  # PARTICLE_DTYPE
    softening: float
    pos64: np.ndarray      # the f64 positions before the f32 rounding of the exchange format


def _pack(pos, h, mass, u, mat, rho, prov=0) -> np.ndarray:
    n = len(pos)
    p = np.zeros(n, PARTICLE_DTYPE)
    p["pos"] = np.asarray(pos, np.float64).astype(np.float32)
    p["h"] = np.asarray(h, np.float64).astype(np.float32)
    p["u"] = np.asarray(u, np.float64).astype(np.float32)
    p["mass"] = np.asarray(mass, np.float64).astype(np.float32)
    p["mat"] = np.asarray(mat, np.uint32)
    p["rho"] = np.asarray(rho, np.float64).astype(np.float32)
    p["prov"] = prov
    return p


def _ball(n: int, radius: float, offset: float) -> np.ndarray:
    """n points at equal-volume radii r = R((i + ½)/n)^⅓ on the Fibonacci spiral."""
    i = np.arange(n)
    rr = radius * ((i + 0.5) / n) ** (1.0 / 3.0)
    return fib_dir(i, n, offset) * rr[:, None]


def _shell(n: int, r_in: float, r_out: float, offset: float) -> np.ndarray:
    """n points at equal-volume radii through the shell [r_in, r_out]."""
    i = np.arange(n)
    rc3, rt3 = r_in ** 3, r_out ** 3
    rr = (rc3 + (rt3 - rc3) * (i + 0.5) / n) ** (1.0 / 3.0)
    return fib_dir(i, n, offset) * rr[:, None]


def new_sphere(material: str, total_mass: float, temp_k: float, specific_heat: float, n: int) -> RefBody:
    """HydroBody::new_sphere (hydrostatic.rs:66-90): one material at ρ0, u = c·T."""
    rho0 = TILLOTSON_SI[material][0]
    r0 = (total_mass / (FOUR_THIRDS_PI * rho0)) ** (1.0 / 3.0)
    m_i = total_mass / n
    pos = _ball(n, r0, 0.0)
    mat = MAT_IRON if material == "iron" else MAT_BASALT
    p = _pack(pos, np.full(n, smoothing_for(m_i, rho0)), np.full(n, m_i), np.full(n, specific_heat * temp_k),
              np.full(n, mat), np.full(n, rho0))
    return RefBody(p, 0.5 * (m_i / rho0) ** (1.0 / 3.0), pos)


def _round(x: float) -> int:
    """Rust's f64::round: halves away from zero (Python's round() rounds halves to even)."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def _counts(m_core: float, m_mantle: float, m_i_core: float, m_i_mantle: float):
    n_core = max(_round(m_core / m_i_core), 1)
    n_mantle = max(_round(m_mantle / m_i_mantle), 1)
    return n_core, n_mantle


def new_differentiated(core_radius: float, total_radius: float, u_specific: float, target_n: int,
                       prov: int = 0) -> RefBody:
    """HydroBody::new_differentiated (hydrostatic.rs:97-139) = impact-run build_differentiated (main.rs:103-141):
    an iron core inside core_radius and a basalt mantle out to total_radius at their ρ0, equal-mass particles
    (mass chosen so the count is ≈ target_n), each with its material's h; softening half the core spacing."""
    rfe, rba = TILLOTSON_SI["iron"][0], TILLOTSON_SI["basalt"][0]
    m_core = rfe * FOUR_THIRDS_PI * core_radius ** 3
    m_mantle = rba * FOUR_THIRDS_PI * (total_radius ** 3 - core_radius ** 3)
    m_i = (m_core + m_mantle) / target_n
    n_core, n_mantle = _counts(m_core, m_mantle, m_i, m_i)
    pos = np.concatenate([_ball(n_core, core_radius, 0.0), _shell(n_mantle, core_radius, total_radius, 1.7)])
    n = n_core + n_mantle
    core = np.arange(n) < n_core
    h = np.where(core, smoothing_for(m_i, rfe), smoothing_for(m_i, rba))
    p = _pack(pos, h, np.full(n, m_i), np.full(n, u_specific), np.where(core, MAT_IRON, MAT_BASALT),
              np.where(core, rfe, rba), prov)
    return RefBody(p, 0.5 * (m_i / rfe) ** (1.0 / 3.0), pos)


def new_lod(core_radius: float, total_radius: float, u_specific: float, m_fine: float, coarse_factor: float,
            prov: int = 0) -> RefBody:
    """HydroBody::new_lod (hydrostatic.rs:146-184) = impact-run build_lod (main.rs:143-176): a coarse iron core
    (particle mass m_fine·coarse_factor) and a fine basalt mantle (m_fine); softening half the fine spacing."""
    rfe, rba = TILLOTSON_SI["iron"][0], TILLOTSON_SI["basalt"][0]
    m_coarse = m_fine * coarse_factor
    m_core = rfe * FOUR_THIRDS_PI * core_radius ** 3
    m_mantle = rba * FOUR_THIRDS_PI * (total_radius ** 3 - core_radius ** 3)
    n_core, n_mantle = _counts(m_core, m_mantle, m_coarse, m_fine)
    pos = np.concatenate([_ball(n_core, core_radius, 0.0), _shell(n_mantle, core_radius, total_radius, 1.7)])
    n = n_core + n_mantle
    core = np.arange(n) < n_core
    mass = np.where(core, m_coarse, m_fine)
    h = np.where(core, smoothing_for(m_coarse, rfe), smoothing_for(m_fine, rba))
    p = _pack(pos, h, mass, np.full(n, u_specific), np.where(core, MAT_IRON, MAT_BASALT), np.where(core, rfe, rba),
              prov)
    return RefBody(p, 0.5 * (m_fine / rba) ** (1.0 / 3.0), pos)


@dataclass
class Layer:
    """One layer of a LayeredBody (crates/engine/src/planet.rs): material index, outer radius (m), declared
    in-situ density (kg/m³), specific heat (J/kg/K) and the geotherm's inner and outer temperatures (K)."""
    mat: int
    outer_r: float
    density: float
    specific_heat: float
    t_inner: float
    t_outer: float


def temperature_at(layers, r: np.ndarray) -> np.ndarray:
    """LayeredBody::temperature_at (planet.rs:87-97): linear in radius through the layer that holds r."""
    r = np.asarray(r, np.float64)
    out = np.full(r.shape, layers[-1].t_outer if layers else 0.0)
    inner = 0.0
    done = np.zeros(r.shape, bool)
    for l in layers:
        sel = (~done) & (r <= l.outer_r)
        f = np.clip((r[sel] - inner) / max(l.outer_r - inner, 1.0), 0.0, 1.0)
        out[sel] = l.t_inner + (l.t_outer - l.t_inner) * f
        done |= sel
        inner = l.outer_r
    return out


def particalize(layers, resolution: int) -> RefBody:
    """HydroBody::particalize (hydrostatic.rs:199-238): equal-mass particles across the body's real layers, each
    layer's count from its declared density, equal-volume radii on a per-layer offset spiral (0.7 per layer),
    u = c·T(r) from the geotherm, h from the declared density; softening a quarter of the smallest h."""
    vols = []
    inner = 0.0
    for l in layers:
        vols.append(FOUR_THIRDS_PI * (l.outer_r ** 3 - inner ** 3))
        inner = l.outer_r
    total = sum(l.density * v for l, v in zip(layers, vols))
    m_i = max(total / max(resolution, 1), 1.0)
    parts = []
    inner = 0.0
    for li, (l, v) in enumerate(zip(layers, vols)):
        n = max(_round(l.density * v / m_i), 1)
        pos = _shell(n, inner, l.outer_r, li * 0.7)
        r = np.linalg.norm(pos, axis=1)
        parts.append((pos, np.full(n, smoothing_for(m_i, l.density)), np.full(n, m_i),
                      l.specific_heat * temperature_at(layers, r), np.full(n, l.mat), np.full(n, l.density)))
        inner = l.outer_r
    cols = [np.concatenate([p[k] for p in parts]) for k in range(6)]
    p = _pack(*cols)
    return RefBody(p, 0.25 * float(cols[1].min()), cols[0])


def hash_jitter(run: int, i: np.ndarray, axis: int) -> np.ndarray:
    """tools/impact-run/src/main.rs:179-190: a splitmix64-style hash of (run, particle, axis) in [-1, 1)."""
    i = np.asarray(i, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = (np.uint64(run) * np.uint64(0x9E3779B97F4A7C15)) ^ (i * np.uint64(0xD1B54A32D192ED03)) ^ \
            (np.uint64(axis) * np.uint64(0xCA5A826395121157)) ^ np.uint64(0x2545F4914F6CDD1D)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x ^= x >> np.uint64(31)
    return x.astype(np.float64) / float(M64) * 2.0 - 1.0
