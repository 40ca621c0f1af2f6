"""The ground scene of the granular pipeline (particle_step.wgsl cs_integrate :477-576 with terrain_* :338-452 and
the headroom of cs_forces :282-336): Newton cooling, aerodynamic drag, terrain contact as a non-injecting
constraint, the settle counter and the incandescent glow.

CPU: the oracle against the closed forms the shader's comments state (terminal speed of a grain in air, the
exponential relaxation of u toward c·300 K, the glow of a hot grain) and the terrain constraint's promises (it
never adds kinetic energy, it supports a resting grain on a slope, a buried grain under a stack is not rammed up).
GPU: the device step against the oracle on the same grains."""
import math

import numpy as np
import pytest

import oracle
from botheadstudios_b200._lib import GRAIN_DTYPE

G = 9.81
PRM = dict(dt=2.0e-3, stiffness=4000.0, normal_damp=30.0, friction=0.6, tangent_damp=40.0, cohesion=5.0)
W = D = 32
CENTER = (16.0, 0.0, 16.0)


def _prm(gravity=(0.0, -G, 0.0)):
    return oracle.dem_params(PRM["stiffness"], PRM["normal_damp"], PRM["friction"], PRM["tangent_damp"],
                             PRM["cohesion"], PRM["dt"], gravity)


def ramp():
    """A 32 × 32 heightfield rising one voxel every four columns along x (a bilinear 1:4 slope)."""
    return np.tile((np.arange(W) // 4).astype(np.int32), (D, 1))


def terrain_h(heights, x, z):
    """terrain_h (particle_step.wgsl:352) in f64, for placing grains."""
    vx, vz = x + CENTER[0], z + CENTER[2]
    cx, cz = math.floor(vx), math.floor(vz)

    def top(a, b):
        return heights[min(max(b, 0), D - 1), min(max(a, 0), W - 1)] - CENTER[1] - 0.5

    fx, fz = vx - cx, vz - cz
    return ((top(cx, cz) * (1 - fx) + top(cx + 1, cz) * fx) * (1 - fz)
            + (top(cx, cz + 1) * (1 - fx) + top(cx + 1, cz + 1) * fx) * fz)


def grains(n, seed=0, spacing=3.0, y0=5.0, vel=20.0, u0=800.0 * 1500.0):
    rng = np.random.default_rng(seed)
    m = int(math.ceil(math.sqrt(n)))
    g = np.zeros(n, GRAIN_DTYPE)
    ij = np.stack(np.meshgrid(np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 2)[:n]
    g["offset"][:, 0] = (ij[:, 0] - m / 2) * spacing
    g["offset"][:, 2] = (ij[:, 1] - m / 2) * spacing
    g["offset"][:, 1] = y0 + rng.uniform(0.0, 1.0, n)
    g["vel"] = rng.uniform(-vel, vel, (n, 3))
    g["radius"] = 0.5
    g["rho"] = rng.uniform(1500.0, 3000.0, n)
    g["u"] = u0 * rng.uniform(0.5, 1.5, n)
    return g


def on_ramp(n, seed=0, sink=0.002):
    """One layer of grains on the ramp, each pressed `sink` metres into the surface, apart from each other."""
    rng = np.random.default_rng(seed)
    h = ramp()
    m = int(math.ceil(math.sqrt(n)))
    g = np.zeros(n, GRAIN_DTYPE)
    for k in range(n):
        x = (k // m - m / 2) * 1.3 + rng.uniform(-0.05, 0.05)
        z = (k % m - m / 2) * 1.3 + rng.uniform(-0.05, 0.05)
        g["offset"][k] = (x, terrain_h(h, x, z) + 0.5 - sink, z)
    g["vel"] = rng.uniform(-0.5, 0.5, (n, 3))
    g["radius"] = 0.5
    g["rho"] = 2700.0
    g["u"] = 800.0 * 300.0
    return g, h


GROUND = (*CENTER, 1.2, 0.5, 800.0, 0.05)  # center, air_rho, drag_cd, specific_heat, cool_rate


def test_oracle_terminal_speed_in_air():
    """a = ½ ρ_air v² C_d / (ρ_grain s), s = 2r: a grain falling from rest approaches v_t = √(2 g ρ s / (ρ_air C_d))."""
    g = grains(1, vel=0.0, y0=1.0e5)
    g["rho"] = 2000.0
    prm = _prm()
    prm[5] = 0.05  # dt: one free grain, 200 s ≈ 7.7 drag time constants
    out = oracle.dem_ground_step32(g, prm, GROUND, None, substeps=4000)
    v_t = math.sqrt(2 * G * 2000.0 * 1.0 / (1.2 * 0.5))
    assert abs(-out["vel"][0, 1] - v_t) / v_t < 2e-3


def test_oracle_cooling_and_glow():
    g = grains(4, vel=0.0, y0=1.0e4)
    u0 = g["u"].astype(np.float64).copy()
    out = oracle.dem_ground_step32(g, _prm(), GROUND, None, substeps=500)
    u_amb = 800.0 * 300.0
    want = u_amb + (u0 - u_amb) * math.exp(-0.05 * 500 * PRM["dt"])
    assert np.allclose(out["u"], want, rtol=2e-5)
    t = out["u"].astype(np.float64) / 800.0
    x = t - 800.0
    inten = np.clip(x / 2200.0, 0.0, 4.0)
    glow = np.stack([inten, np.clip(x / 2200.0, 0, 1) * inten, np.clip((t - 2600.0) / 2400.0, 0, 1) * inten], 1)
    glow[t <= 800.0] = 0.0
    assert np.allclose(out["emission"], glow, rtol=1e-5, atol=1e-6)


def test_oracle_terrain_never_adds_kinetic_energy_and_supports():
    """Isolated grains thrown at the ramp: the constraint only removes energy; afterwards they rest on it."""
    g = grains(36, spacing=8.0, y0=3.0, vel=5.0)  # far apart: no grain-grain contact in 0.4 s
    h = ramp()
    prm = _prm(gravity=(0.0, 0.0, 0.0))  # no gravity: any KE gain would be the terrain's
    ground = (*CENTER, 0.0, 0.0, 0.0, 0.0)
    ke = lambda a: float((a["vel"].astype(np.float64) ** 2).sum())  # noqa: E731
    cur = g
    for _ in range(200):
        nxt = oracle.dem_ground_step32(cur, prm, ground, h)
        assert ke(nxt) <= ke(cur) * (1 + 1e-6) + 1e-9
        cur = nxt
    rest, _ = on_ramp(49)
    out = oracle.dem_ground_step32(rest, _prm(), ground, h, substeps=500)
    surf = np.array([terrain_h(h, x, z) for x, _, z in out["offset"].astype(np.float64)])
    assert (out["offset"][:, 1] - 0.5 - surf > -0.01).all()  # supported on the slope
    assert (out["resting"] == 500).all()


def test_oracle_headroom_keeps_a_stack_in_place():
    """A grain buried by a surface that rose under it, with a grain resting right above: the projection is capped by
    the headroom (0 here), so the buried grain is not rammed into the one above it."""
    h = np.zeros((D, W), np.int32)
    h[:, :] = 2  # the surface is at y = 1.5 in centred coordinates
    g = np.zeros(2, GRAIN_DTYPE)
    g["offset"] = [(0.3, 1.5, 0.3), (0.3, 2.5, 0.3)]  # the lower grain's centre on the surface, touching the upper
    g["radius"] = 0.5
    g["rho"] = 2700.0
    prm = _prm(gravity=(0.0, 0.0, 0.0))
    out = oracle.dem_ground_step32(g, prm, (*CENTER, 0, 0, 0, 0), h)
    assert abs(out["offset"][0, 1] - 1.5) < 1e-3  # not projected up by the 1 cm cap
    h1 = np.zeros((D, W), np.int32)  # same surface, no grain above: the projection runs at its 1 cm cap
    out1 = oracle.dem_ground_step32(g[:1], prm, (*CENTER, 0, 0, 0, 0), h1 + 2)
    assert abs(out1["offset"][0, 1] - 1.51) < 1e-4


# ---- device parity ------------------------------------------------------------------------------------------
def _device(g, heights, substeps, ground=GROUND, gravity=(0.0, -G, 0.0)):
    from botheadstudios_b200.grains import GpuGrains
    with GpuGrains(len(g)) as s:
        s.set_params(gravity=gravity, **PRM)
        s.set_ground(center=ground[:3], air_rho=ground[3], drag_cd=ground[4], specific_heat=ground[5],
                     cool_rate=ground[6])
        s.set_terrain(heights)
        s.replace(g)
        s.dispatch(substeps)
        return s.readback()


@pytest.mark.gpu
def test_gpu_drag_and_cooling_match_oracle():
    g = grains(400, spacing=3.0, y0=50.0)
    got = _device(g, None, 40)
    want = oracle.dem_ground_step32(g, _prm(), GROUND, None, substeps=40)
    assert np.abs(got["offset"] - want["offset"]).max() < 1e-4
    assert np.abs(got["vel"] - want["vel"]).max() < 1e-4 * np.abs(want["vel"]).max()
    assert np.allclose(got["u"], want["u"], rtol=1e-5)  # 40 substeps of one f32 relaxation each
    assert np.allclose(got["emission"], want["emission"], rtol=1e-4, atol=1e-6)
    assert (got["resting"] == 0).all()
    for f in ("radius", "rho", "color", "material"):
        assert np.array_equal(got[f], g[f]), f


@pytest.mark.gpu
def test_gpu_grains_resting_on_slope_match_oracle():
    g, h = on_ramp(400, seed=1)
    got = _device(g, h, 60)
    want = oracle.dem_ground_step32(g, _prm(), GROUND, h, substeps=60)
    # the device keeps f64 positions; the shader's f32 positions round each ~4e-5 m settle-and-project cycle
    # (a grain at the stick/slip edge of the Coulomb clamp can take the other branch from such a difference)
    assert np.abs(got["offset"] - want["offset"]).max() < 1e-3
    dv = np.abs(got["vel"] - want["vel"]).max(1)
    assert (dv < 1e-3).mean() > 0.97 and dv.max() < 0.05
    assert np.array_equal(got["resting"], want["resting"]) and (got["resting"] == 60).all()


@pytest.mark.gpu
def test_gpu_pile_falls_onto_terrain():
    """A dense pack lands on the ramp (grain-grain contacts, touchdown thresholds): the device tracks the oracle
    grain by grain except where a touchdown threshold falls within rounding of a grain, and no grain ends up
    below the surface."""
    from botheadstudios_b200.grains import grain_pack
    h = ramp()
    g = grain_pack(500, seed=4, vel_scale=0.5)
    g["offset"] -= g["offset"].mean(0)
    g["offset"][:, 1] += 5.2 - g["offset"][:, 1].min()  # above the ramp (its surface is 2.5-4.5 m below the pack)
    g["vel"][:, 1] -= 8.0  # the high side of the ramp is reached within the 40 substeps
    g["u"] = 800.0 * 900.0
    got = _device(g, h, 40)
    want = oracle.dem_ground_step32(g, _prm(), GROUND, h, substeps=40)
    close = np.abs(got["offset"] - want["offset"]).max(1) < 1e-3
    assert close.mean() > 0.97
    surf = np.array([terrain_h(h, x, z) for x, _, z in got["offset"].astype(np.float64)])
    assert (got["offset"][:, 1] - 0.5 - surf > -0.05).all()
    assert (got["resting"] > 0).mean() == pytest.approx((want["resting"] > 0).mean(), abs=0.03)


@pytest.mark.gpu
def test_gpu_headroom_keeps_a_stack_in_place():
    h = np.full((D, W), 2, np.int32)
    g = np.zeros(2, GRAIN_DTYPE)
    g["offset"] = [(0.3, 1.5, 0.3), (0.3, 2.5, 0.3)]
    g["radius"] = 0.5
    g["rho"] = 2700.0
    got = _device(g, h, 1, ground=(*CENTER, 0, 0, 0, 0), gravity=(0.0, 0.0, 0.0))
    want = oracle.dem_ground_step32(g, _prm(gravity=(0.0, 0.0, 0.0)), (*CENTER, 0, 0, 0, 0), h)
    assert np.abs(got["offset"] - want["offset"]).max() < 1e-5
    assert abs(got["offset"][0, 1] - 1.5) < 1e-3
