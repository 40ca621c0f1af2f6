"""The reference's deterministic body builders restated (botheadstudios_b200/refbodies.py), on the CPU: the
Fibonacci directions, the equal-volume radii, the particle counts and masses, and the reference's own
assertions about them (crates/engine/src/hydrostatic.rs:1333-1346 Earth-mass differentiated body,
:1411-1437 particalize of Earth's real layers and of a pure-ice body)."""
import math

import numpy as np
import pytest

from botheadstudios_b200 import refbodies as RB
from botheadstudios_b200.materials import MAT_BASALT, MAT_ICE, MAT_IRON, MAT_PERIDOTITE, SPECIFIC_HEAT, TILLOTSON_SI


def _fib_scalar(i, n, offset):
    golden = math.pi * (3.0 - math.sqrt(5.0))
    y = 1.0 - 2.0 * (i + 0.5) / n
    r = math.sqrt(max(1.0 - y * y, 0.0))
    th = golden * i + offset
    return (math.cos(th) * r, y, math.sin(th) * r)


def test_fib_dir_unit_vectors_and_scalar_form():
    d = RB.fib_dir(np.arange(1000), 1000, 1.7)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-12)
    for i in (0, 1, 499, 999):
        assert np.array_equal(d[i], np.array(_fib_scalar(i, 1000, 1.7)))
    # y is uniform in (−1, 1): the hemispheres hold equal counts
    assert (d[:, 1] > 0).sum() == 500


def test_differentiated_earth_mass_body():
    """hydrostatic.rs:1343-1346: radii 0.55·7.37e6 / 7.37e6 m at the materials' ρ0 give about an Earth mass."""
    total_r, core_r = 7.37e6, 0.55 * 7.37e6
    b = RB.new_differentiated(core_r, total_r, 1.0e6, 3000, prov=1)
    p = b.particles
    m = p["mass"].astype(np.float64).sum()
    assert m == pytest.approx(5.97e24, rel=0.01)
    iron = p["mat"] == MAT_IRON
    v_core, v_all = core_r ** 3, total_r ** 3
    m_core = TILLOTSON_SI["iron"][0] * 4 / 3 * math.pi * v_core
    m_mantle = TILLOTSON_SI["basalt"][0] * 4 / 3 * math.pi * (v_all - v_core)
    m_i = (m_core + m_mantle) / 3000
    assert iron.sum() == math.floor(m_core / m_i + 0.5) and (~iron).sum() == math.floor(m_mantle / m_i + 0.5)
    r = np.linalg.norm(b.pos64, axis=1)
    assert r[iron].max() <= core_r and r[~iron].min() >= core_r and r.max() <= total_r
    assert np.all(p["prov"] == 1) and np.all(p["u"] == np.float32(1.0e6))
    assert p["h"][iron][0] == np.float32(2.0 * (m_i / 7850.0) ** (1 / 3))
    assert p["h"][~iron][0] == np.float32(2.0 * (m_i / 2700.0) ** (1 / 3))
    assert b.softening == pytest.approx(0.5 * (m_i / 7850.0) ** (1 / 3))
    # equal-volume radii: the core's mean r³ is half its radius cubed
    assert np.mean(r[iron] ** 3) == pytest.approx(0.5 * v_core, rel=1e-3)


def test_lod_body_masses():
    b = RB.new_lod(2.5e6, 5.0e6, 1.0e6, 1.0e21, 8.0)
    p = b.particles
    core = p["mat"] == MAT_IRON
    assert np.all(p["mass"][core] == np.float32(8.0e21)) and np.all(p["mass"][~core] == np.float32(1.0e21))
    assert b.softening == pytest.approx(0.5 * (1.0e21 / 2700.0) ** (1 / 3))


EARTH = [  # assets/bodies/earth.json: material, outer radius (m), density (kg/m3), T inner, T outer (K)
    ("iron", 1221500.0, 12900.0, 5900.0, 5800.0),
    ("iron", 2350000.0, 11900.0, 5800.0, 5150.0),
    ("iron", 3480000.0, 10600.0, 5150.0, 4150.0),
    ("peridotite", 6346000.0, 4500.0, 2900.0, 1600.0),
    ("basalt", 6371000.0, 2900.0, 900.0, 288.0),
]
MAT = dict(iron=MAT_IRON, basalt=MAT_BASALT, peridotite=MAT_PERIDOTITE, ice=MAT_ICE)


def _layers(rows):
    return [RB.Layer(MAT[m], r, d, SPECIFIC_HEAT[m], ti, to) for m, r, d, ti, to in rows]


def test_particalize_earth_and_ice_reference_assertions():
    """hydrostatic.rs:1411-1437: Earth's real mass within 2 %, >= 3 materials, iron innermost, u following the
    geotherm (core hotter than crust); a pure-ice body is ice and keeps its mass within 3 %."""
    layers = _layers(EARTH)
    real = sum(l.density * 4 / 3 * math.pi * (l.outer_r ** 3 - (layers[k - 1].outer_r if k else 0.0) ** 3)
               for k, l in enumerate(layers))
    b = RB.particalize(layers, 2000)
    p = b.particles
    assert p["mass"].astype(np.float64).sum() == pytest.approx(real, rel=0.02)
    assert len(set(p["mat"].tolist())) >= 3
    assert p["mat"][0] == MAT_IRON and p["u"][0] > p["u"][-1]
    assert b.softening == pytest.approx(0.25 * float(p["h"].astype(np.float64).min()), rel=1e-6)
    ice = RB.particalize(_layers([("ice", 1.0e6, 917.0, 120.0, 120.0)]), 400)
    mi = ice.particles["mass"].astype(np.float64).sum()
    assert np.all(ice.particles["mat"] == MAT_ICE)
    assert mi == pytest.approx(917.0 * 4 / 3 * math.pi * 1.0e18, rel=0.03)


def test_temperature_at_is_linear_in_each_layer():
    layers = _layers(EARTH)
    t = RB.temperature_at(layers, np.array([0.0, 1221500.0, 0.5 * (3480000.0 + 6346000.0), 7.0e6]))
    assert t[0] == 5900.0 and t[1] == 5800.0 and t[2] == pytest.approx(0.5 * (2900.0 + 1600.0)) and t[3] == 288.0


def test_hash_jitter_matches_integer_arithmetic():
    M = (1 << 64) - 1

    def ref(run, i, axis):
        x = ((run * 0x9E3779B97F4A7C15) & M) ^ ((i * 0xD1B54A32D192ED03) & M) ^ ((axis * 0xCA5A826395121157) & M) \
            ^ 0x2545F4914F6CDD1D
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M
        x ^= x >> 31
        return float(x) / float(M) * 2.0 - 1.0
    i = np.arange(0, 5000, 7, dtype=np.uint64)
    got = RB.hash_jitter(3, i, 2)
    assert np.array_equal(got, np.array([ref(3, int(k), 2) for k in i]))
    assert got.min() >= -1.0 and got.max() < 1.0
