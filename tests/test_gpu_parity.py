"""GPU parity: the sm_100a path (through the C ABI) against the CPU oracle on the reference's own inputs.

Bit-exact: bounding box, Morton codes, sort permutation, Karras topology, node moments, neighbour sets and
the reference-MAC monopole Barnes-Hut accelerations. Tolerances (stated per test) for density, EOS, SPH
forces and multi-step integration, whose f32 summation order differs from the oracle's.
"""
import math

import numpy as np
import pytest

import oracle
from botheadstudios_b200 import ic
from botheadstudios_b200 import materials as M
from botheadstudios_b200.gpusph import GpuSph, particles_from_arrays
from refcases import cloud, verify_config

pytestmark = pytest.mark.gpu
G = M.G_SI


def _ctx_from_bodies(bodies4, K=1, theta=0.5, h=1.0, quad=False, mac=1, **kw):
    n = len(bodies4)
    parts = particles_from_arrays(bodies4[:, :3], np.full(n, h, np.float32), np.zeros((n, 3), np.float32),
                                  np.zeros(n, np.float32), bodies4[:, 3], np.zeros(n, np.uint32))
    s = GpuSph(n, G=G, theta=theta, leaf_size=K, multipole=int(quad), max_neighbours=64, mac=mac, **kw)
    s.upload(parts, M.eos_table(), softening=5.0e3)
    s.eval_forces()
    s.sync()
    return s


@pytest.mark.parametrize("K", [1, 8, 16, 32])
def test_tree_stages_bit_exact(K):
    bodies, _, _ = cloud(2000, 0x51A17EED ^ 2000)
    t = oracle.tree_pipeline32(bodies, K=K, theta=0.5, soft=5.0e3, G=G)
    with _ctx_from_bodies(bodies, K=K) as s:
        bb = s.inspect("BBOX")
        assert np.array_equal(bb[:3], t["lo"]) and np.array_equal(bb[3:], t["hi"])
        assert np.array_equal(s.inspect("CODES"), t["sorted_codes"])
        assert np.array_equal(s.inspect("ORDER"), t["order"])
        assert s.n_leaves() == t["L"]
        assert np.array_equal(s.inspect("LEFT"), t["left"])
        assert np.array_equal(s.inspect("RIGHT"), t["right"])
        assert np.array_equal(s.inspect("PARENT"), t["parent"])
        com, bmin, bmax = s.inspect("NODE_COM"), s.inspect("NODE_BMIN"), s.inspect("NODE_BMAX")
        assert np.array_equal(com, t["com"])
        assert np.array_equal(bmin[:, :3], t["bmin"][:, :3]) and np.array_equal(bmax[:, :3], t["bmax"][:, :3])
        assert oracle.verify_tree(s.inspect("LEFT"), s.inspect("RIGHT"), s.inspect("PARENT"), s.n_leaves())


@pytest.mark.parametrize("theta", [0.5, 0.25, 0.1, 1.0e-4])
def test_bh_monopole_matches_reference_walk_bitwise(theta):
    """Warp-cooperative traversal == the reference's per-particle cs_gravity_bh walk, bit for bit."""
    bodies, pos, mass = cloud(1500, 0xABCD1234)
    t = oracle.tree_pipeline32(bodies, K=1, theta=theta, soft=5.0e3, G=G)
    with _ctx_from_bodies(bodies, K=1, theta=theta) as s:
        a = s.inspect("ACC_GRAV")[:, :3]
    assert np.array_equal(a, t["acc"][:, :3])


@pytest.mark.parametrize("K", [1, 16])
def test_theta_sweep_against_f64_direct(K):
    """gpu-bh-verify main.rs:546-568: RMS < 1e-2 for θ ∈ {0.5, 0.25, 0.1}, < 1e-4 for θ → 0."""
    bodies, pos, mass = cloud(1500, 0xABCD1234)
    ref = oracle.gravity_direct64(pos, mass, 5.0e3, G)
    for theta, bound in ((0.5, 1e-2), (0.25, 1e-2), (0.1, 1e-2), (1e-4, 1e-4)):
        with _ctx_from_bodies(bodies, K=K, theta=theta) as s:
            a = s.inspect("ACC_GRAV")[:, :3].astype(np.float64)
        rms = math.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum())
        assert rms < bound, (theta, rms)


def test_quadrupole_beats_monopole():
    bodies, pos, mass = cloud(4000, 7)
    ref = oracle.gravity_direct64(pos, mass, 5.0e3, G)
    errs = {}
    for quad in (False, True):
        with _ctx_from_bodies(bodies, K=16, theta=0.6, quad=quad) as s:
            a = s.inspect("ACC_GRAV")[:, :3].astype(np.float64)
        errs[quad] = math.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum())
    assert errs[True] < 0.5 * errs[False], errs


def _verify_ctx(gravity="direct", **kw):
    pos4, vel4, mass, mat, rho = verify_config(300)
    parts = particles_from_arrays(pos4[:, :3], pos4[:, 3], vel4[:, :3], vel4[:, 3], mass, mat, rho)
    s = GpuSph(300, G=G, gravity=gravity, max_neighbours=256, **kw)
    s.upload(parts, M.eos_table(), softening=1.0e4)
    return s, (pos4, vel4, mass, mat)


def test_neighbour_sets_exact_verify_config():
    s, (pos4, _, _, _) = _verify_ctx()
    with s:
        s.eval_forces()
        got = s.neighbour_sets()
    want = oracle.neighbours32(pos4, cap=300)
    for i in range(300):
        assert np.array_equal(got[i], want[i]), i


def test_sph_eval_matches_f32_oracle():
    """cs_density / EOS / SPH forces: GPU vs the f32 restatement on the sph-verify cluster (SI units)."""
    s, (pos4, vel4, mass, mat) = _verify_ctx(gravity="none")
    with s:
        s.eval_forces()
        rho, P, c, acc = s.inspect("RHO"), s.inspect("PRESSURE"), s.inspect("SOUND"), s.inspect("ACC_SPH")
    rho_o = oracle.density32(pos4, mass)
    P_o, c_o = oracle.eos32(M.eos_table(), mat, rho_o, vel4[:, 3])
    f_o = oracle.sph_forces32(pos4, vel4, mass, rho_o, P_o, c_o)
    assert np.max(np.abs(rho - rho_o) / rho_o) < 2e-6
    pscale = np.abs(P_o).max()
    assert np.max(np.abs(P - P_o)) / pscale < 2e-5
    assert np.max(np.abs(c - c_o) / np.maximum(c_o, 1.0)) < 2e-3
    da = acc[:, :3] - f_o[:, :3]
    assert math.sqrt((da ** 2).sum() / (f_o[:, :3] ** 2).sum()) < 1e-4
    du = acc[:, 3] - f_o[:, 3]
    assert math.sqrt((du ** 2).sum() / (f_o[:, 3] ** 2).sum()) < 1e-3


def test_sph_eval_matches_f64_verifier():
    """tools/sph-verify main.rs:304-343: force RMS < 3e-2, du/dt < 5e-2 vs the f64 CPU physics."""
    s, (pos4, vel4, mass, mat) = _verify_ctx(gravity="direct")
    with s:
        s.eval_forces()
        rho, acc, grav = s.inspect("RHO"), s.inspect("ACC_SPH"), s.inspect("ACC_GRAV")
    rho64, acc64, dudt64 = oracle.cpu_forces64(pos4[:, :3], vel4[:, :3], pos4[:, 3], mass, vel4[:, 3],
                                               mat.astype(np.int32), M.eos_table64(), 1.0e4, G)
    total = acc[:, :3].astype(np.float64) + grav[:, :3]
    rms = math.sqrt(((total - acc64) ** 2).sum() / (acc64 ** 2).sum())
    du = math.sqrt(((acc[:, 3] - dudt64) ** 2).sum() / (dudt64 ** 2).sum())
    assert np.max(np.abs(rho - rho64) / rho64) < 1e-5
    assert rms < 3e-2 and du < 5e-2
    assert rms < 1e-4 and du < 1e-3


def test_kdk_integration_tracks_f64_cpu():
    """tools/sph-verify main.rs:356-395: 50 KDK steps at dt = 0.5 s, pos/vel/u RMS < 5e-3 vs f64."""
    s, (pos4, vel4, mass, mat) = _verify_ctx(gravity="direct")
    with s:
        s.set_dt(0.5, 1.0)
        s.encode_kdk(50)
        out = s.readback()
    p64, v64, u64 = oracle.cpu_kdk64(pos4[:, :3], vel4[:, :3], pos4[:, 3], mass, vel4[:, 3], mat.astype(np.int32),
                                     M.eos_table64(), 1.0e4, 0.5, 50, G=G)
    disp = p64 - pos4[:, :3]
    pe = math.sqrt(((out["pos"] - p64) ** 2).sum() / (disp ** 2).sum())
    ve = math.sqrt(((out["vel"] - v64) ** 2).sum() / (v64 ** 2).sum())
    ue = math.sqrt(((out["u"] - u64) ** 2).sum() / (u64 ** 2).sum())
    assert pe < 5e-3 and ve < 5e-3 and ue < 5e-3, (pe, ve, ue)


def test_readback_roundtrip_clamp_and_invalid():
    I = ic.impact(2000, 500)
    p = I.particles
    with GpuSph(2000, **ic.config_kwargs(I.units)) as s:
        with pytest.warns(UserWarning):
            assert s.upload(p, I.eos, I.softening) == 1  # SPH_CLAMPED: 2500 > 2000
        assert s.count() == 2000
        back = s.readback()
        assert np.array_equal(back, p[:2000])
        s.eval_forces()
        back2 = s.readback()
        assert np.array_equal(back2["pos"], p[:2000]["pos"]) and np.array_equal(back2["prov"], p[:2000]["prov"])
        bad = p[:100].copy()
        bad["mat"][5] = 7
        from botheadstudios_b200.gpusph import SphError
        with pytest.raises(SphError):
            s.upload(bad, I.eos, I.softening)


def test_impact_config1_one_eval_parity():
    """10,240-particle impact (code units): neighbour sets exact, density/forces vs f32 oracle, gravity vs f64."""
    I = ic.impact(8192, 2048, n_ngb=48)
    p = I.particles
    n = len(p)
    kw = ic.config_kwargs(I.units)
    with GpuSph(n, theta=0.5, leaf_size=1, **kw) as s:
        s.upload(p, I.eos, I.softening)
        s.eval_forces()
        nb = s.neighbour_sets()
        rho, acc, grav = s.inspect("RHO"), s.inspect("ACC_SPH"), s.inspect("ACC_GRAV")
        d = s.diag()
    pos4 = np.concatenate([p["pos"], p["h"][:, None]], axis=1)
    want = oracle.neighbours32(pos4, cap=256)
    assert all(np.array_equal(nb[i], want[i]) for i in range(n))
    rho_o = oracle.density32(pos4, p["mass"])
    assert np.max(np.abs(rho - rho_o) / rho_o) < 2e-6
    vel4 = np.concatenate([p["vel"], p["u"][:, None]], axis=1)
    P_o, c_o = oracle.eos32(I.eos, p["mat"], rho_o, p["u"], du_floor=I.units.du_floor, rho_floor=I.units.rho_floor)
    f_o = oracle.sph_forces32(pos4, vel4, p["mass"], rho_o, P_o, c_o, r_min=I.units.r_min)
    da = acc[:, :3] - f_o[:, :3]
    assert math.sqrt((da ** 2).sum() / (f_o[:, :3] ** 2).sum()) < 1e-4
    ref = oracle.gravity_direct64(I.pos64, p["mass"].astype(np.float64), I.softening, 1.0)
    g = grav[:, :3].astype(np.float64)
    assert math.sqrt(((g - ref) ** 2).sum() / (ref ** 2).sum()) < 1e-2
    assert d["overflow_flags"] == 0 and 20 < d["max_neighbours_seen"] <= 256
