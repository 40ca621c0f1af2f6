"""Disk measurement and the Moon candidate (impact-run `measure` + `moon_candidate`, main.rs:732-878; the engine's
`disk_stats_json` + `find_clumps`, gpu_sph.rs:399-469 and accretion.rs:73-160).

CPU: the oracle restatement is pinned by an independent numpy/scipy restatement (KD-tree pairs + connected
components) on seeded scenes, and by the engine's own accretion cases (accretion.rs:261-310: the Roche gate and
the hot unbound group) rebuilt around a remnant. GPU: sph_measure_disk against the oracle on the same particles —
single impacts, every impact of a batch, the state after KDK steps (sorted on the device), and a 200k-particle
scene. Counts must agree exactly; masses and radii within 1e-9 relative (the device sums the same f64 terms in a
different association)."""
import math

import numpy as np
import pytest
from scipy.sparse import coo_matrix
from scipy.sparse.csgraph import connected_components
from scipy.spatial import cKDTree

import oracle
import disk_scene as ds

COUNTS = ("clump_n", "n_clumps", "n_bound", "n_disk")
FLOATS = ("earth_frac", "disk_mass", "disk_target", "disk_impactor", "remnant_target", "remnant_impactor",
          "escaped_target", "escaped_impactor", "r_remnant", "m_remnant", "clump_mass", "clump_target_frac")


def _numpy_measure(p, variant, G=ds.G):
    """Second restatement: vectorised classification, KD-tree friends-of-friends, per-group energies."""
    x = p["pos"].astype(np.float64)
    v = p["vel"].astype(np.float64)
    m = p["mass"].astype(np.float64)
    M = m.sum()
    com = (x * m[:, None]).sum(0) / M
    vcom = (v * m[:, None]).sum(0) / M
    rad = np.linalg.norm(x - com, axis=1)
    o = np.argsort(rad, kind="stable")
    cum = np.cumsum(m[o])
    k = int(np.argmax(cum >= 0.85 * M))
    r_rem, m_rem = rad[o][k], cum[k]
    mu = G * m_rem
    rp, rv = x - com, v - vcom
    r = np.linalg.norm(rp, axis=1)
    energy = 0.5 * (rv * rv).sum(1) - mu / r
    h2 = (np.cross(rp, rv) ** 2).sum(1)
    e = np.sqrt(np.maximum(1.0 + 2.0 * energy * h2 / mu**2, 0.0))
    bound = energy < 0
    peri = np.where(bound, -mu / (2.0 * energy) * (1.0 - e), 0.0)
    disk = bound & (peri > r_rem)
    idx = np.nonzero(disk)[0]
    link = 2.0 * (p["h"][idx].astype(np.float64).mean() if variant == 0 else p["h"].astype(np.float64).mean())
    pairs = cKDTree(x[idx]).query_pairs(link * (1 + 1e-6), output_type="ndarray")
    # exact predicate of the variant on the candidate pairs
    a, b = pairs[:, 0], pairs[:, 1]
    if variant == 0:
        d = (p["pos"][idx][a] - p["pos"][idx][b]).astype(np.float64)
    else:
        d = x[idx][a] - x[idx][b]
    keep = (d * d).sum(1) <= link * link
    a, b = a[keep], b[keep]
    n = len(idx)
    ncomp, lab = connected_components(coo_matrix((np.ones(len(a)), (a, b)), shape=(n, n)), directed=False)
    rho_rem = m_rem / (4.0 / 3.0 * math.pi * r_rem**3)
    best, n_cl, n_bound = 0.0, 0, 0
    for g in range(ncomp):
        mem = idx[lab == g]
        if len(mem) < 2:
            continue
        n_cl += 1
        mg = m[mem].sum()
        cv = (v[mem] * m[mem, None]).sum(0) / mg
        cp = (x[mem] * m[mem, None]).sum(0) / mg
        rho = p["rho"][mem].astype(np.float64) if variant == 0 else np.maximum(p["rho"][mem], 1.0).astype(np.float64)
        vol = (m[mem] / rho).sum()
        ke = 0.5 * (m[mem] * ((v[mem] - cv) ** 2).sum(1)).sum()
        dd = x[mem][:, None, :] - x[mem][None, :, :]
        rr = np.sqrt((dd * dd).sum(2))
        rr = np.maximum(rr, 1.0) if variant == 0 else np.sqrt(rr * rr + 1.0e8)
        iu = np.triu_indices(len(mem), 1)
        pe = -(G * np.outer(m[mem], m[mem])[iu] / rr[iu]).sum()
        ok = ke + pe < 0
        n_bound += int(ok)
        d_roche = 2.44 * r_rem * np.cbrt(rho_rem / (mg / vol))
        if ok and np.linalg.norm(cp - com) > d_roche:
            best = max(best, mg)
    return dict(r_remnant=r_rem, n_disk=len(idx), n_clumps=n_cl, n_bound=n_bound, clump_mass=best,
                disk_mass=m[idx].sum())


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_agrees_with_kdtree_restatement(seed, variant):
    p = ds.scene(seed)
    a = oracle.measure_disk(p, ds.G, variant=variant)
    b = _numpy_measure(p, variant)
    for k in ("n_disk", "n_clumps", "n_bound"):
        assert a[k] == b[k], k
    for k in ("r_remnant", "clump_mass", "disk_mass"):
        assert a[k] == pytest.approx(b[k], rel=1e-9), k


def test_oracle_scene_known_answers():
    """The scene's bound clump outside Roche (40 members at 4.5 R) is the candidate; the 25-member one outside
    and the 30-member one inside Roche are bound; the hot group is not."""
    p = ds.scene(0)
    r = oracle.measure_disk(p, ds.G, variant=0)
    assert r["clump_n"] == 40 and r["clump_mass"] == pytest.approx(40 * 1.0e18, rel=1e-6)
    assert r["n_bound"] == 3
    assert 0.9 * ds.R < r["r_remnant"] < ds.R
    esc = (r["escaped_target"] + r["escaped_impactor"]) / 1.0e18  # the 100 launched, plus a few hot members
    assert 99.99 < esc < 130.01
    total = sum(r[k] for k in ("disk_mass", "remnant_target", "remnant_impactor", "escaped_target",
                                "escaped_impactor"))
    assert total == pytest.approx(float(p["mass"].astype(np.float64).sum()), rel=1e-12)


def _remnant_with(clump_at_R, sigma, m_i=1.0e19, seed=0, n=30):
    """A remnant plus one clump on a circular orbit (accretion.rs:195 cold_blob, here a random ball)."""
    return ds.scene(seed, n_ring=0, n_esc=0, clumps=((n, clump_at_R, sigma, 0.0),), m_debris=m_i)


@pytest.mark.parametrize("variant", [0, 1])
def test_oracle_roche_gate(variant):
    """accretion.rs:261-277: the same cold clump does not count inside the Roche limit and does outside it."""
    inside = oracle.measure_disk(_remnant_with(1.8, 1.0), ds.G, variant=variant)
    outside = oracle.measure_disk(_remnant_with(5.0, 1.0), ds.G, variant=variant)
    assert inside["n_bound"] == 1 and inside["clump_mass"] == 0.0
    assert outside["n_bound"] == 1 and outside["clump_mass"] == pytest.approx(30 * 1.0e19, rel=1e-6)


@pytest.mark.parametrize("variant", [0, 1])
def test_oracle_hot_group_is_unbound(variant):
    """accretion.rs:279-310: a tight group with internal speeds far above its binding is one group, not bound."""
    r = oracle.measure_disk(_remnant_with(5.0, 400.0, m_i=1.0e15), ds.G, variant=variant)
    assert r["n_clumps"] >= 1 and r["n_bound"] == 0 and r["clump_mass"] == 0.0


def test_oracle_edge_cases():
    p = ds.scene(0)
    assert oracle.measure_disk(p[:0], ds.G)["n_disk"] == 0
    one = oracle.measure_disk(p[:1], ds.G)
    assert one["n_disk"] == 0 and one["r_remnant"] == 0.0 and one["clump_mass"] == 0.0
    no_disk = oracle.measure_disk(ds.scene(0, n_ring=0, n_esc=0, clumps=()), ds.G)
    assert no_disk["n_disk"] == 0 and no_disk["earth_frac"] == 0.0 and no_disk["n_clumps"] == 0


# ---- device parity -------------------------------------------------------------------------------------------
def _check(gpu, ref):
    for k in COUNTS:
        assert gpu[k] == int(ref[k]), (k, gpu[k], ref[k])
    for k in FLOATS:
        assert gpu[k] == pytest.approx(ref[k], rel=1e-9, abs=1e-300), (k, gpu[k], ref[k])


def _solver(n, **kw):
    from botheadstudios_b200 import ic, materials
    from botheadstudios_b200.gpusph import GpuSph
    return GpuSph(n, **ic.config_kwargs(materials.SI), **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_gpu_measure_matches_oracle(seed, variant):
    p = ds.scene(seed)
    with _solver(len(p)) as s:
        s.upload(p, ds.eos(), 1.0e4)
        got = s.measure_disk(0, variant=variant)
    _check(got, oracle.measure_disk(p, ds.G, variant=variant))


@pytest.mark.gpu
def test_gpu_measure_each_impact_of_a_batch():
    scenes = [ds.scene(s, n_rem=3000 + 1000 * s) for s in range(3)]
    parts = np.concatenate(scenes)
    offs = np.cumsum([0] + [len(x) for x in scenes]).astype(np.uint32)
    with _solver(len(parts)) as s:
        s.upload_batch(parts, offs, ds.eos(), np.full(3, 1.0e4, np.float32))
        for k, sc in enumerate(scenes):
            _check(s.measure_disk(k, variant=0), oracle.measure_disk(sc, ds.G, variant=0))


@pytest.mark.gpu
def test_gpu_measure_after_steps_reads_the_sorted_state():
    p = ds.scene(3)
    with _solver(len(p), h_mode=1, h_neighbours=48.0, max_neighbours=192) as s:
        s.upload(p, ds.eos(), 1.0e4)
        s.set_dt(2.0, 1.0)
        s.encode_kdk(2)
        state = s.readback()
        got = [s.measure_disk(0, variant=v) for v in (0, 1)]
    for v in (0, 1):
        _check(got[v], oracle.measure_disk(state, ds.G, variant=v))


@pytest.mark.gpu
def test_gpu_measure_large_scene():
    clumps = tuple((200 + 40 * k, 3.0 + 0.4 * k, 5.0, 0.55 * k) for k in range(8)) + ds.CLUMPS
    p = ds.scene(7, n_rem=200_000, n_ring=15_000, n_esc=2000, clumps=clumps, h_rem=2.2e5, h_debris=1.2e5,
                 clump_radius=4.0e5, m_rem=3.0e19)
    with _solver(len(p)) as s:
        s.upload(p, ds.eos(), 1.0e4)
        got = s.measure_disk(0, variant=0)
    ref = oracle.measure_disk(p, ds.G, variant=0)
    _check(got, ref)
    assert got["n_clumps"] > 8 and got["clump_mass"] > 0.0


@pytest.mark.gpu
def test_gpu_measure_edge_cases():
    from botheadstudios_b200.gpusph import SphError
    p = ds.scene(0)
    with _solver(len(p)) as s:
        s.upload(p[:1], ds.eos(), 1.0e4)
        _check(s.measure_disk(0), oracle.measure_disk(p[:1], ds.G))
        nd = ds.scene(0, n_ring=0, n_esc=0, clumps=())
        s.upload(nd, ds.eos(), 1.0e4)
        _check(s.measure_disk(0), oracle.measure_disk(nd, ds.G))
        with pytest.raises(SphError):
            s.measure_disk(1)
        with pytest.raises(SphError):
            s.measure_disk(0, variant=2)
        with pytest.raises(SphError):
            s.measure_disk(0, remnant_frac=1.5)
