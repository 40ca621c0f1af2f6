"""GPU tests of the step's control paths against the oracle, through the C ABI:

* the damped relaxation in a rotating frame (cs_relax, sph_step.wgsl:245-257) against the oracle's f32 step,
  one step in isolation and ten steps with the whole force evaluation restated;
* the device's per-impact adaptive dt (cs_signal, sph_step.wgsl:263-269, reduced on the device instead of the
  host min of tools/impact-run/src/main.rs:345-356) against cfl · min h/max(c + |v|, floor);
* the hi/lo precision mode against the FP64 direct sum;
* the overflow flags: a neighbour list and a traversal stack that are too small raise SPH_ERR_OVERFLOW
  through sph_diag (the reference drops silently, bh_gravity.wgsl:388-391), without a fault.
"""
import math

import numpy as np
import pytest

import oracle
from botheadstudios_b200 import _lib, ic
from botheadstudios_b200 import materials as M
from botheadstudios_b200.gpusph import GpuSph, SphError, particles_from_arrays
from refcases import cloud

pytestmark = pytest.mark.gpu
G_SI = M.G_SI


def _pos4(p, h=None):
    h = p["h"] if h is None else h
    return np.ascontiguousarray(np.concatenate([p["pos"], np.asarray(h, np.float32)[:, None]], 1), dtype=np.float32)


def _vel4(p):
    return np.ascontiguousarray(np.concatenate([p["vel"], p["u"][:, None]], 1), dtype=np.float32)


# ---- relaxation ------------------------------------------------------------------------------------------
def _relax_ctx(I, gravity):
    kw = dict(kernel="cubic", h_mode="fixed", gravity=gravity, theta=0.5, leaf_size=1, max_neighbours=256,
              **ic.config_kwargs(I.units))
    return GpuSph(len(I.particles), **kw)


def test_relax_step_with_spin_matches_oracle_step():
    """One cs_relax step with ω != 0 from the device's own accelerations: v = (v + (a + ω²(x, y, 0))·dt)·damp,
    x += v·dt. The device keeps f64 master positions; the oracle steps in f32 (at most an ulp apart)."""
    I = ic.planet(3000, n_ngb=48.0, seed=9)
    p = I.particles
    dt, damp, w = 5.0e-3, 0.95, 0.3
    with _relax_ctx(I, "tree") as s:
        s.upload(p, I.eos, I.softening)
        s.set_omega(w)
        s.set_dt(dt, damp)
        s.eval_forces()
        a = s.inspect("ACC_SPH")[:, :3].astype(np.float32) + s.inspect("ACC_GRAV")[:, :3]
        pre = s.readback()
        s.encode_relax(1)
        post = s.readback()
    acc4 = np.zeros((len(p), 4), np.float32)
    acc4[:, :3] = a
    p_o, v_o = oracle.relax32(_pos4(pre), _vel4(pre), acc4, dt, damp, w)
    vscale = np.abs(v_o[:, :3]).max()
    assert vscale > 0.0
    assert np.abs(post["vel"] - v_o[:, :3]).max() < 1e-5 * vscale
    assert np.abs(post["pos"] - p_o[:, :3]).max() < 1e-6 * np.abs(p_o[:, :3]).max() + 2.0 * dt * 1e-5 * vscale
    assert np.array_equal(post["u"], pre["u"]) and np.array_equal(post["h"], pre["h"])
    # the centrifugal term acts in x and y only: with ω the x/y velocities differ from a run without it
    p0, v0 = oracle.relax32(_pos4(pre), _vel4(pre), acc4, dt, damp, 0.0)
    assert np.abs(v0[:, 2] - v_o[:, 2]).max() == 0.0 and np.abs(v0[:, 0] - v_o[:, 0]).max() > 0.0


def test_relax_ten_steps_track_the_oracle():
    """Ten relaxation steps with ω != 0 against the oracle running the reference's own evaluation
    (cs_density, the EOS, the SPH forces and the direct gravity sum in f32, sph_step.wgsl:120-211) then
    cs_relax, on the same particles."""
    I = ic.planet(1500, n_ngb=48.0, seed=10)
    p = I.particles
    u = I.units
    dt, damp, w, steps = 5.0e-3, 0.9, 0.3, 10
    with _relax_ctx(I, "direct") as s:
        s.upload(p, I.eos, I.softening)
        s.set_omega(w)
        s.set_dt(dt, damp)
        s.encode_relax(steps)
        got = s.readback()
    pos4, vel4 = _pos4(p), _vel4(p)
    soft2 = np.float32(I.softening) * np.float32(I.softening)
    for _ in range(steps):
        rho = oracle.density32(pos4, p["mass"], kernel=0)
        P, c = oracle.eos32(I.eos, p["mat"], rho, vel4[:, 3], du_floor=u.du_floor, rho_floor=u.rho_floor)
        f = oracle.sph_forces32(pos4, vel4, p["mass"], rho, P, c, r_min=u.r_min, kernel=0)
        bodies = np.ascontiguousarray(np.concatenate([pos4[:, :3], p["mass"][:, None]], 1), dtype=np.float32)
        g = oracle.gravity_direct32(bodies, soft2, u.G)
        acc4 = np.zeros_like(f)
        acc4[:, :3] = f[:, :3] + g[:, :3]
        pos4, vel4 = oracle.relax32(pos4, vel4, acc4, dt, damp, w)
    assert np.abs(got["pos"] - pos4[:, :3]).max() < 1e-5
    assert np.abs(got["vel"] - vel4[:, :3]).max() < 1e-3 * np.abs(vel4[:, :3]).max()


# ---- adaptive dt --------------------------------------------------------------------------------------------
def _dt_oracle(p, h, c, cfl, floor):
    sig = oracle.signal32(_pos4(p, h), _vel4(p), c, floor=floor)
    return float(np.float32(cfl)) * float(sig.min())


def test_device_dt_reference_method_matches_cs_signal():
    """The small plain-method impact (cubic spline, 48 neighbours, fixed h, θ = 0.5 monopole, CFL 0.3): the
    first step's dt is cfl · min signal of the uploaded state, with the oracle's density and sound speed (c
    differs by the EOS's finite-difference noise) and, exactly, with the device's own sound speed."""
    I = ic.impact(8192, 2048, n_ngb=48.0, seed=1)
    p = I.particles
    u = I.units
    kw = dict(kernel="cubic", h_mode="fixed", theta=0.5, leaf_size=1, multipole=0, cfl=0.3, max_neighbours=256,
              **ic.config_kwargs(u))
    with GpuSph(len(p), **kw) as s:
        s.upload(p, I.eos, I.softening)
        s.eval_forces()
        c_dev = s.inspect("SOUND")
        s.encode_kdk(1)
        dt_dev = float(s.impact_dt()[0])
        assert s.diag()["dt"] == dt_dev
    rho_o = oracle.density32(_pos4(p), p["mass"], kernel=0)
    _, c_o = oracle.eos32(I.eos, p["mat"], rho_o, p["u"], du_floor=u.du_floor, rho_floor=u.rho_floor)
    assert dt_dev == pytest.approx(_dt_oracle(p, p["h"], c_o, 0.3, u.sig_floor), rel=2e-3)
    assert dt_dev == pytest.approx(_dt_oracle(p, p["h"], c_dev, 0.3, u.sig_floor), rel=1e-6)


def test_device_dt_benchmark_method_and_batch():
    """The benchmark's method (Wendland, the h-solve, quadrupoles θ = 0.6, 16-particle leaves) in a batch of
    three impacts: each impact's dt is cfl · min over its own particles of h/max(c + |v|, floor), at the solved
    h and the device's sound speed."""
    B = ic.batch(3, 3000, 9000, n_ngb=64.0, seed=4)
    u = B.units
    kw = dict(kernel="wendland", h_mode="solve", h_neighbours=64.0, h_iters=2, theta=0.6, leaf_size=16,
              multipole=1, cfl=0.3, max_neighbours=192, **ic.config_kwargs(u))
    with GpuSph(len(B.particles), **kw) as s:
        s.upload_batch(B.particles, B.offsets, B.eos, B.softening)
        s.eval_forces()
        h, c = s.inspect("H"), s.inspect("SOUND")
        st = s.readback()
        s.encode_kdk(1)
        dts = s.impact_dt()
    for k in range(3):
        a, b = int(B.offsets[k]), int(B.offsets[k + 1])
        want = _dt_oracle(st[a:b], h[a:b], c[a:b], 0.3, u.sig_floor)
        assert float(dts[k]) == pytest.approx(want, rel=1e-6), k
    assert len(set(map(float, dts))) == 3


# ---- hi/lo precision mode -----------------------------------------------------------------------------------
@pytest.mark.parametrize("mac,K,quad,theta,bound", [(0, 16, 1, 0.6, 2e-3), (1, 1, 0, 0.5, 1e-2)])
def test_hilo_precision_against_fp64_direct(mac, K, quad, theta, bound):
    """precision = HILO (f64 master split into f32 hi + lo inside the walks, compensated sums) on 24,000
    points: within the bound against the FP64 direct sum, no worse than plain f32 (the tree truncation, not
    the coordinates, sets the error), and the direct-sum limit θ → 0 to 1e-5."""
    bodies, pos, mass = cloud(24000, 0x5EED)
    n = len(bodies)
    parts = particles_from_arrays(bodies[:, :3], np.full(n, 1.0, np.float32), np.zeros((n, 3), np.float32),
                                  np.zeros(n, np.float32), bodies[:, 3], np.zeros(n, np.uint32))
    tg = np.random.default_rng(1).choice(n, 4096, replace=False)
    ref = oracle.gravity_direct64(pos, mass, 5.0e3, G_SI, targets=tg)
    rms = {}
    for prec in (0, 1):
        for th in (theta, 1.0e-4):
            with GpuSph(n, G=G_SI, theta=th, leaf_size=K, multipole=quad, mac=mac, precision=prec,
                        max_neighbours=64) as s:
                s.upload(parts, M.eos_table(), softening=5.0e3)
                s.eval_forces()
                a = s.inspect("ACC_GRAV")[:, :3].astype(np.float64)[tg]
            rms[prec, th] = math.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum())
    assert rms[1, theta] < bound, rms
    assert rms[1, theta] <= 1.1 * rms[0, theta], rms
    assert rms[1, 1.0e-4] < 1e-5 and rms[0, 1.0e-4] < 1e-5, rms


# ---- overflow flags -----------------------------------------------------------------------------------------
def _overflow_ctx(n, h, **kw):
    bodies, pos, mass = cloud(n, 77)
    parts = particles_from_arrays(bodies[:, :3], np.full(n, h, np.float32), np.zeros((n, 3), np.float32),
                                  np.full(n, 1.0e5, np.float32), bodies[:, 3], np.zeros(n, np.uint32))
    s = GpuSph(n, G=G_SI, **kw)
    s.upload(parts, M.eos_table(), softening=5.0e3)
    return s


def _assert_overflow(s, bit):
    with pytest.raises(SphError) as e:
        s.diag()
    assert e.value.status == _lib.SPH_ERR_OVERFLOW
    d = s.diag(check=False)
    assert d["overflow_flags"] & bit
    return d


def test_neighbour_list_overflow_is_reported():
    """Lists of 8 entries for ~40 neighbours: the walk keeps counting past the capacity, writes nothing beyond
    it, and sph_diag reports SPH_ERR_OVERFLOW; the gather passes stay within the list."""
    with _overflow_ctx(3000, 1.5e5, theta=0.5, leaf_size=8, multipole=1, max_neighbours=8) as s:
        s.eval_forces()
        d = _assert_overflow(s, 1)
        assert d["max_neighbours_seen"] > 8
        assert np.isfinite(s.inspect("RHO")).all()
    with _overflow_ctx(3000, 1.5e5, theta=0.5, leaf_size=8, multipole=1, max_neighbours=128) as s:
        s.eval_forces()
        assert s.diag()["overflow_flags"] == 0


@pytest.mark.parametrize("mac,K,limit", [(0, 8, 24), (1, 1, 6)])
def test_traversal_stack_overflow_is_reported(mac, K, limit):
    """A traversal stack limited to a few entries (sph_config.walk_stack) drops the children that do not fit
    and raises the stack flag through sph_diag, in both walks; the full stack raises nothing."""
    with _overflow_ctx(20000, 1.0e3, theta=0.3, leaf_size=K, multipole=1 - mac, mac=mac, max_neighbours=64,
                       walk_stack=limit) as s:
        s.eval_forces()
        _assert_overflow(s, 2)
    with _overflow_ctx(20000, 1.0e3, theta=0.3, leaf_size=K, multipole=1 - mac, mac=mac, max_neighbours=64) as s:
        s.eval_forces()
        assert s.diag()["overflow_flags"] == 0
