"""The reference's own seeded bodies through the CUDA path: two differentiated bodies built exactly as
HydroBody::new_differentiated / impact-run build_differentiated build them (crates/engine/src/hydrostatic.rs:97-139,
tools/impact-run/src/main.rs:103-141; the Earth/Theia pair of hydrostatic.rs:1172-1173), in SI units, set on a
collision course, and evaluated with the reference's method (cubic spline, the bodies' own h, monopole
Barnes-Hut θ = 0.5 with one particle per leaf). Against the oracle: the per-particle walk's tree and
accelerations bit for bit (PARTICLE mode), the neighbour sets bit for bit, density, EOS and SPH forces within
the tolerances of the other parity tests, and the group walk's gravity (quadrupoles, 8-particle leaves) against the FP64 direct sum."""
import math

import numpy as np
import pytest

import oracle
from botheadstudios_b200 import materials as M
from botheadstudios_b200 import refbodies as RB
from botheadstudios_b200.gpusph import GpuSph

pytestmark = pytest.mark.gpu
G = M.G_SI


@pytest.fixture(scope="module")
def impact():
    earth = RB.new_differentiated(0.5 * 5.0e6, 5.0e6, 1.0e6, 1800, prov=0)
    theia = RB.new_differentiated(0.5 * 2.7e6, 2.7e6, 1.0e6, 300, prov=1)
    p = np.concatenate([earth.particles, theia.particles])
    nt = len(theia.particles)
    p["pos"][-nt:] += np.array([1.1e7, 3.0e6, 0.0], np.float32)
    p["vel"][-nt:] = np.array([-9.0e3, 0.0, 0.0], np.float32)
    return p, min(earth.softening, theia.softening)


def _ctx(p, soft, **kw):
    cfg = dict(G=G, kernel="cubic", h_mode="fixed", theta=0.5, leaf_size=1, multipole=0, max_neighbours=256)
    cfg.update(kw)
    s = GpuSph(len(p), **cfg)
    s.upload(p, M.eos_table(), soft)
    s.eval_forces()
    return s


def test_reference_bodies_particle_walk_and_sph_match_oracle(impact):
    p, soft = impact
    n = len(p)
    pos4 = np.ascontiguousarray(np.concatenate([p["pos"], p["h"][:, None]], 1), dtype=np.float32)
    vel4 = np.ascontiguousarray(np.concatenate([p["vel"], p["u"][:, None]], 1), dtype=np.float32)
    bodies = np.ascontiguousarray(np.concatenate([p["pos"], p["mass"][:, None]], 1), dtype=np.float32)
    with _ctx(p, soft, mac=1) as s:
        t = oracle.tree_pipeline32(bodies, K=1, theta=0.5, soft=soft, G=G)
        assert np.array_equal(s.inspect("ORDER"), t["order"])
        assert np.array_equal(s.inspect("LEFT"), t["left"]) and np.array_equal(s.inspect("RIGHT"), t["right"])
        assert np.array_equal(s.inspect("ACC_GRAV")[:, :3], t["acc"][:, :3])
        nb = s.neighbour_sets()
        want = oracle.neighbours32(pos4, cap=256)
        assert all(np.array_equal(nb[i], want[i]) for i in range(n))
        rho, c, acc = s.inspect("RHO"), s.inspect("SOUND"), s.inspect("ACC_SPH")
    rho_o = oracle.density32(pos4, p["mass"])
    assert np.max(np.abs(rho - rho_o) / rho_o) < 2e-6
    P_o, c_o = oracle.eos32(M.eos_table(), p["mat"], rho_o, p["u"])
    assert np.max(np.abs(c - c_o) / np.maximum(c_o, 1.0)) < 2e-3
    f_o = oracle.sph_forces32(pos4, vel4, p["mass"], rho_o, P_o, c)
    da = acc[:, :3].astype(np.float64) - f_o[:, :3]
    assert math.sqrt((da ** 2).sum() / (f_o[:, :3].astype(np.float64) ** 2).sum()) < 1e-4


def test_reference_bodies_group_walk_gravity_against_fp64_direct(impact):
    p, soft = impact
    with _ctx(p, soft, mac=0, multipole=1, leaf_size=8) as s:
        g = s.inspect("ACC_GRAV")[:, :3].astype(np.float64)
    ref = oracle.gravity_direct64(p["pos"].astype(np.float64), p["mass"].astype(np.float64), soft, G)
    rms = math.sqrt(((g - ref) ** 2).sum() / (ref ** 2).sum())
    assert rms < 1e-2, rms
