"""Relaxed-body assembly: `body_bulk` (gpu_sph.rs:260-293) and `assemble_from_relaxed_n` (gpu_sph.rs:309-339).

CPU: the oracle restatement reproduces the reference's own assembly test (gpu_sph.rs:1262-1300: three bodies
each land at their placement with their own velocity, and a spin about x gives the target a vz) and the reason
body_bulk exists (gpu_sph.rs:250-259: a stray far out must not drag the centre). GPU: sph_body_bulk and
sph_assemble against the oracle on the same particles, directly after an upload and after relaxation steps
(the state sorted on the device), then a KDK step on the assembled state."""
import numpy as np
import pytest

import oracle
from botheadstudios_b200._lib import PARTICLE_DTYPE
from botheadstudios_b200.materials import eos_table

R_E, R_M = 6.4e6, 1.7e6
PLACEMENTS = [((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), (3.0e-4, 0.0, 0.0)),
              ((1.5e7, 2.0e6, 0.0), (-8000.0, 0.0, 0.0), (0.0, 0.0, 0.0)),
              ((0.0, 1.6e7, 0.0), (0.0, -7000.0, 0.0), (0.0, 0.0, 0.0))]


def _ball(rng, n, radius, centre):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return np.asarray(centre) + v * (radius * rng.random(n) ** (1.0 / 3.0))[:, None]


def bodies(seed=0, n=(1200, 250, 250), strays=True):
    """Three relaxed-looking bodies (prov 0, 1, 2) far apart, a few strays flung out of each, and particles of a
    provenance without a placement (prov 7)."""
    rng = np.random.default_rng(seed)
    parts = []
    for prov, (k, rad, c, m) in enumerate([(n[0], R_E, (0.0, 0.0, 0.0), 5.0e21),
                                           (n[1], R_M, (4.0e7, 0.0, 0.0), 3.0e20),
                                           (n[2], R_M, (-4.0e7, 0.0, 0.0), 3.0e20)]):
        p = np.zeros(k, PARTICLE_DTYPE)
        p["pos"] = _ball(rng, k, rad, c)
        if strays:
            p["pos"][:3] = np.asarray(c) + rng.normal(size=(3, 3)) * 20 * rad  # strays a relax leaves
        p["vel"] = rng.normal(scale=30.0, size=(k, 3))
        p["mass"] = m * (1.0 + 0.01 * rng.random(k))
        p["h"] = 1.4 * rad * (4.0 / 3.0 * np.pi / k) ** (1 / 3) * (1 + 0.05 * rng.random(k))
        p["u"] = 1.0e5
        p["rho"] = 4000.0
        p["mat"] = rng.integers(0, 2, k)
        p["prov"] = prov
        parts.append(p)
    extra = np.zeros(5, PARTICLE_DTYPE)
    extra["pos"] = rng.normal(size=(5, 3)) * 1e8
    extra["h"] = 1e6
    extra["mass"] = 1e20
    extra["prov"] = 7
    out = np.concatenate(parts + [extra])
    return out[rng.permutation(len(out))]


def _com(p, prov, field="pos"):
    s = p[p["prov"] == prov]
    m = s["mass"].astype(np.float64)
    return (s[field].astype(np.float64) * m[:, None]).sum(0) / m.sum()


def test_oracle_assembly_places_every_body_and_spins_about_any_axis():
    """gpu_sph.rs:1262-1300, on these bodies (without strays, as there)."""
    p = bodies(strays=False)
    out, soft, dt = oracle.assemble(p, PLACEMENTS)
    assert len(out) == len(p) - 5 and not (out["prov"] == 7).any()
    c0, c1, c2 = (_com(out, k) for k in range(3))
    v0, v1, v2 = (_com(out, k, "vel") for k in range(3))
    assert np.linalg.norm(c0) < 0.02 * R_E
    assert np.linalg.norm(c1 - c0 - PLACEMENTS[1][0]) < 0.02 * R_E
    assert np.linalg.norm(c2 - c0 - PLACEMENTS[2][0]) < 0.02 * R_E
    assert np.linalg.norm(v1 - v0 - PLACEMENTS[1][1]) < 1.0
    assert np.linalg.norm(v2 - v0 - PLACEMENTS[2][1]) < 1.0
    assert np.abs(out["vel"][out["prov"] == 0][:, 2]).max() > 1.0  # an x spin gives vz
    keep = p[p["prov"] != 7]
    for f in ("h", "u", "mass", "mat", "rho", "prov"):
        assert np.array_equal(out[f], keep[f]), f  # only positions and velocities change, order kept
    assert soft == np.float32(0.25) * keep["h"].min()
    assert dt == np.float32(0.01 * float(keep["h"].min()) / (20000.0 + 8000.0))


def test_oracle_body_bulk_resists_strays():
    """gpu_sph.rs:250-259: one stray far out drags a plain mass-weighted centre; the clipped bulk does not."""
    p = bodies(strays=False)
    ball = p[p["prov"] == 1].copy()
    ball["pos"][0] = (4.0e7 + 20 * R_M, 0.0, 0.0)
    ball["mass"][0] = 0.007 * ball["mass"].sum()
    naive = _com(ball, 1)
    centre, mass, radius = oracle.body_bulk(ball, 1)
    true = _com(ball[1:], 1)
    assert np.linalg.norm(naive - true) > 0.1 * R_M
    assert np.linalg.norm(centre - true) < 0.02 * R_M
    assert 0.8 * R_M < radius < 1.05 * R_M
    assert mass == pytest.approx(float(ball["mass"].astype(np.float64).sum()), rel=1e-12)
    empty = oracle.body_bulk(ball, 5)
    assert empty[1] == 0.0 and empty[2] == 0.0 and not empty[0].any()


# ---- device parity -------------------------------------------------------------------------------------------
def _solver(n):
    from botheadstudios_b200 import ic, materials
    from botheadstudios_b200.gpusph import GpuSph
    return GpuSph(n, h_mode=1, h_neighbours=48.0, max_neighbours=192, **ic.config_kwargs(materials.SI))


def _same_assembly(got, ref):
    assert len(got) == len(ref)
    for f in ("h", "u", "mass", "mat", "rho", "prov"):
        assert np.array_equal(got[f], ref[f]), f
    for f in ("pos", "vel"):  # the f32 rounding of the same f64 sums, associated differently: within an ulp
        a, b = got[f].astype(np.float64), ref[f].astype(np.float64)
        assert (np.abs(a - b) <= np.spacing(np.abs(ref[f])).astype(np.float64)).all(), f


@pytest.mark.gpu
def test_gpu_body_bulk_matches_oracle():
    p = bodies()
    with _solver(len(p)) as s:
        s.upload(p, eos_table(), 1.0e4)
        for prov in (0, 1, 2, 7, 9):
            c, m, r = s.body_bulk(prov)
            rc, rm, rr = oracle.body_bulk(p, prov)
            assert np.allclose(c, rc, rtol=0, atol=1e-9 * R_E), prov
            assert m == pytest.approx(rm, rel=1e-12) and r == pytest.approx(rr, rel=1e-12), prov


@pytest.mark.gpu
def test_gpu_assemble_matches_oracle():
    p = bodies(1)
    with _solver(len(p)) as s:
        s.upload(p, eos_table(), 1.0e4)
        soft, dt = s.assemble(PLACEMENTS)
        got = s.readback()
    ref, rsoft, rdt = oracle.assemble(p, PLACEMENTS)
    _same_assembly(got, ref)
    assert soft == rsoft and dt == rdt


@pytest.mark.gpu
def test_gpu_relax_then_assemble_then_step():
    """The reference's flow: relax the bodies, assemble them on the live geometry, run the impact. The assembly
    reads the relaxed state where it lies (sorted on the device), with no host round trip."""
    p = bodies(2)
    with _solver(len(p)) as s:
        s.upload(p, eos_table(), 1.0e4)
        s.set_dt(1.0, 0.9)
        s.set_omega(1.0e-4)
        s.encode_relax(3)
        relaxed = s.readback()
        soft, dt = s.assemble(PLACEMENTS[:2])
        got = s.readback()
        assert s.count() == len(got)
        s.set_dt(float(dt), 1.0)
        s.encode_kdk(1)
        after = s.readback()
    ref, rsoft, rdt = oracle.assemble(relaxed, PLACEMENTS[:2])
    _same_assembly(got, ref)
    assert soft == rsoft and dt == rdt
    assert len(after) == len(ref) and np.isfinite(after["pos"]).all()


@pytest.mark.gpu
def test_gpu_assemble_rejects():
    from botheadstudios_b200.gpusph import SphError
    p = bodies(3)
    with _solver(len(p)) as s:
        s.upload(p, eos_table(), 1.0e4)
        with pytest.raises(SphError):
            s.assemble([])  # nothing kept
        with pytest.raises(SphError):
            s.assemble([((np.nan, 0, 0), (0, 0, 0), (0, 0, 0))])
        assert s.count() == len(p)  # a rejected assembly leaves the state alone
