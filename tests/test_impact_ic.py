"""The seeded impact generator reproduces the benchmark configurations' shapes (host side, no GPU): particle
counts, mass ratio, 30 % iron / 70 % basalt by mass, the initial separation, and the collision the bodies are
on — speed 1.1 v_esc and a 45° angle at contact, checked through the two-body orbit's energy and angular
momentum — in the centre-of-mass frame."""
import math

import numpy as np
import pytest

from botheadstudios_b200 import ic, workloads
from botheadstudios_b200.materials import MAT_BASALT, MAT_IRON


@pytest.mark.parametrize("name, n_t, n_i", [("impact_1m", 953_250, 95_326), ("impact_4m", 3_813_004, 381_300),
                                            ("impact_10k", 8_192, 2_048)])
def test_workload_shapes(name, n_t, n_i):
    wl = workloads.WORKLOADS[name]
    assert (wl["n_target"], wl["n_impactor"]) == (n_t, n_i)
    assert workloads.n_particles(wl) == n_t + n_i
    if name != "impact_10k":  # the large shapes have equal particle masses at mass ratio 0.1
        assert n_i / n_t == pytest.approx(0.1, rel=1e-4)


def _bodies(I):
    p = I.particles
    return p[p["prov"] == 0], p[p["prov"] == 1], I.pos64[p["prov"] == 0], I.pos64[p["prov"] == 1]


def test_small_impact_configuration():
    I = ic.impact(8_192, 2_048, n_ngb=48.0, seed=1)
    tgt, imp, xt, xi = _bodies(I)
    assert (len(tgt), len(imp)) == (8_192, 2_048)
    mt, mi = tgt["mass"].astype(np.float64), imp["mass"].astype(np.float64)
    assert mt.sum() == pytest.approx(1.0, rel=1e-6) and mi.sum() == pytest.approx(0.1, rel=1e-6)
    for b, m in ((tgt, mt), (imp, mi)):
        iron = m[b["mat"] == MAT_IRON].sum() / m.sum()
        assert iron == pytest.approx(0.3, abs=1.0 / len(b))
        assert set(np.unique(b["mat"])) == {MAT_IRON, MAT_BASALT}
    # centre-of-mass frame: no net momentum; the bodies are placed by their lattice origins, which the jittered
    # lattices' centres of mass miss by ~1e-3 of a radius, so the system's centre of mass is that close to 0
    m = np.concatenate([mt, mi])
    v = np.concatenate([tgt["vel"], imp["vel"]]).astype(np.float64)
    x = np.concatenate([xt, xi])
    assert np.abs((m[:, None] * v).sum(0)).max() < 1e-6
    assert np.linalg.norm((m[:, None] * x).sum(0) / m.sum()) < 2e-3
    # the relative orbit of the two centres of mass (within the same ~0.2 % of the lattice placement)
    ct, ci = (mt[:, None] * xt).sum(0) / mt.sum(), (mi[:, None] * xi).sum(0) / mi.sum()
    rt = np.sqrt(((xt - ct) ** 2).sum(1)).max()
    ri = np.sqrt(((xi - ci) ** 2).sum(1)).max()
    r = ci - ct
    d0 = np.linalg.norm(r)
    assert d0 == pytest.approx(3.0 * rt, rel=5e-3)
    vrel = imp["vel"][0].astype(np.float64) - tgt["vel"][0].astype(np.float64)
    mu = mt.sum() + mi.sum()
    R = rt + ri
    v_esc = math.sqrt(2.0 * mu / R)
    # energy: the speed at contact separation R
    v_c = math.sqrt(vrel @ vrel + 2.0 * mu * (1.0 / R - 1.0 / d0))
    assert v_c == pytest.approx(1.1 * v_esc, rel=2e-3)
    # angular momentum: the impact parameter at contact, sin(angle) = b_c / R
    b_c = np.linalg.norm(np.cross(r, vrel)) / v_c
    assert math.degrees(math.asin(b_c / R)) == pytest.approx(45.0, abs=0.2)
    # closing, not separating
    assert r @ vrel < 0.0


def test_impact_is_seeded():
    a = ic.impact(2_000, 400, seed=9)
    b = ic.impact(2_000, 400, seed=9)
    c = ic.impact(2_000, 400, seed=10)
    assert np.array_equal(a.particles, b.particles)
    assert not np.array_equal(a.particles["pos"], c.particles["pos"])
