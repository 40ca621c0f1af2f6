"""GPU tests of the tree build on degenerate inputs, the group walk, and size-independent properties of the
full 1,048,576-particle workload (sortedness, permutation, tree validity, conservation, gravity accuracy)."""
import math

import numpy as np
import pytest

import oracle
from botheadstudios_b200 import materials as M
from botheadstudios_b200 import workloads
from botheadstudios_b200.gpusph import GpuSph, particles_from_arrays
from refcases import cloud

pytestmark = pytest.mark.gpu
G = M.G_SI


def _dup_bodies(seed, n=1500):
    rng = np.random.default_rng(seed)
    b = rng.random((n, 4)).astype(np.float32)
    b[:, :3] = np.floor(b[:, :3] * 5.0) / 8.0  # many coincident points: long runs of equal Morton codes
    b[:, 3] = 1.0 + b[:, 3]
    return b


def _ctx(b, K, mac, theta=0.5, quad=0):
    n = len(b)
    p = particles_from_arrays(b[:, :3], np.full(n, 1e-3, np.float32), np.zeros((n, 3), np.float32),
                              np.zeros(n, np.float32), b[:, 3], np.zeros(n, np.uint32))
    s = GpuSph(n, G=1.0, theta=theta, leaf_size=K, mac=mac, multipole=quad, max_neighbours=512)
    s.upload(p, M.eos_table(), softening=1e-2)
    s.eval_forces()
    s.sync()
    return s


@pytest.mark.parametrize("K", [1, 16])
def test_duplicate_codes_reference_split_reproduced(K):
    """PARTICLE mode reproduces the reference's Karras split for runs of equal codes (even where it is invalid)."""
    b = _dup_bodies(3)
    t = oracle.tree_pipeline32(b, K=K, exact_dups=False)
    with _ctx(b, K, mac=1) as s:
        assert np.array_equal(s.inspect("LEFT"), t["left"]) and np.array_equal(s.inspect("RIGHT"), t["right"])
        # where the reference split makes an invalid tree a node is claimed by two parents and its parent
        # entry depends on write order; compare the nodes claimed exactly once
        refs = np.bincount(np.concatenate([t["left"], t["right"]]), minlength=len(t["parent"]))
        once = refs == 1
        assert np.array_equal(s.inspect("PARENT")[once], t["parent"][once])


@pytest.mark.parametrize("K", [1, 16])
def test_duplicate_codes_group_mode_builds_valid_tree(K):
    b = _dup_bodies(4)
    t = oracle.tree_pipeline32(b, K=K, exact_dups=True)
    assert oracle.verify_tree(t["left"], t["right"], t["parent"], t["L"])
    with _ctx(b, K, mac=0) as s:
        left, right, parent = s.inspect("LEFT"), s.inspect("RIGHT"), s.inspect("PARENT")
        assert np.array_equal(left, t["left"]) and np.array_equal(right, t["right"])
        assert oracle.verify_tree(left, right, parent, s.n_leaves())
        # every particle is still summed exactly once: θ -> 0 reproduces the direct sum
    with _ctx(b, K, mac=0, theta=1e-6) as s:
        a = s.inspect("ACC_GRAV")[:, :3].astype(np.float64)
    ref = oracle.gravity_direct64(b[:, :3].astype(np.float64), b[:, 3].astype(np.float64), 1e-2, 1.0)
    assert math.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum()) < 1e-5


@pytest.mark.parametrize("K,quad", [(1, 0), (16, 0), (16, 1)])
def test_group_walk_gravity_bounds(K, quad):
    """Group MAC: the reference's 1 % RMS bound (gpu-bh-verify main.rs:546-568; bhtree.rs:239) and θ → 0
    exactness. θ is side-based here, so the monopole case is held to the bound at θ = 0.4."""
    bodies, pos, mass = cloud(1500, 0xABCD1234)
    ref = oracle.gravity_direct64(pos, mass, 5.0e3, G)
    for theta, bound in ((0.5 if quad else 0.4, 1e-2), (0.25, 1e-2), (1e-4, 1e-5)):
        n = len(bodies)
        p = particles_from_arrays(bodies[:, :3], np.full(n, 1.0, np.float32), np.zeros((n, 3), np.float32),
                                  np.zeros(n, np.float32), bodies[:, 3], np.zeros(n, np.uint32))
        with GpuSph(n, G=G, theta=theta, leaf_size=K, multipole=quad, mac=0, max_neighbours=64) as s:
            s.upload(p, M.eos_table(), softening=5.0e3)
            s.eval_forces()
            a = s.inspect("ACC_GRAV")[:, :3].astype(np.float64)
        rms = math.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum())
        assert rms < bound, (theta, rms)


@pytest.mark.parametrize("mac", [0, 1])
def test_gravity_and_sph_bitwise_repeatable(mac):
    """gpu_gravity.rs:655-880 asks for bitwise repeatability: the same input gives the same bits, in a fresh
    context and on a second evaluation in the same context (no order-dependent atomics on the force path)."""
    bodies, pos, mass = cloud(3000, 11)
    n = len(bodies)
    p = particles_from_arrays(bodies[:, :3], np.full(n, 2.0e5, np.float32), np.zeros((n, 3), np.float32),
                              np.full(n, 1.0e5, np.float32), bodies[:, 3], np.zeros(n, np.uint32))
    runs = []
    for _ in range(2):
        with GpuSph(n, G=G, theta=0.6, leaf_size=16 if mac == 0 else 1, multipole=1 if mac == 0 else 0, mac=mac,
                    max_neighbours=256) as s:
            s.upload(p, M.eos_table(), softening=5.0e3)
            for _ in range(2):
                s.eval_forces()
                runs.append([s.inspect(q).copy() for q in ("ACC_GRAV", "RHO", "ACC_SPH")])
    for r in runs[1:]:
        for a, b in zip(runs[0], r):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_point_set_gravity_api_matches_direct():
    """sph_gravity (GravityField::accelerations): tree and direct modes against the f64 direct sum."""
    _, pos, mass = cloud(3000, 11)
    ref = oracle.gravity_direct64(pos, mass, 5.0e3, G)
    with GpuSph(3000, G=G, theta=0.5, leaf_size=8, multipole=1) as s:
        for mode, bound in (("tree", 1e-2), ("direct", 1e-5)):
            a = s.gravity(pos, mass, 5.0e3, mode)
            assert math.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum()) < bound, mode
        a64 = s.gravity_direct64(pos, mass, 5.0e3, targets=np.arange(0, 3000, 7))
        assert np.allclose(a64, ref[::7], rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.fixture(scope="module")
def impact1m():
    wl = workloads.WORKLOADS["impact_1m"]
    I = workloads.build(wl)
    s = workloads.solver(wl, I)
    s.upload(I.particles, I.eos, I.softening)
    s.encode_kdk(2)
    s.sync()
    yield wl, I, s
    s.close()


def test_full_size_sort_permutation_tree(impact1m):
    wl, I, s = impact1m
    n = len(I.particles)
    codes, order = s.inspect("CODES"), s.inspect("ORDER")
    assert np.all(np.diff(codes.astype(np.int64)) >= 0)
    # ties in the code are ordered by original index
    same = np.diff(codes.astype(np.int64)) == 0
    assert np.all(np.diff(order.astype(np.int64))[same] > 0)
    assert np.array_equal(np.sort(order), np.arange(n, dtype=np.uint32))
    L = s.n_leaves()
    assert L == (n + wl["leaf"] - 1) // wl["leaf"]
    assert oracle.verify_tree(s.inspect("LEFT"), s.inspect("RIGHT"), s.inspect("PARENT"), L)
    com = s.inspect("NODE_COM")
    assert np.isclose(com[0, 3], I.particles["mass"].astype(np.float64).sum(), rtol=1e-5)


def test_full_size_conservation_and_accuracy(impact1m):
    wl, I, s = impact1m
    d0 = s.diag()
    s.encode_kdk(3)
    d1 = s.diag()
    assert d1["overflow_flags"] == 0 and d1["steps"] == d0["steps"] + 3
    pscale = (I.particles["mass"].astype(np.float64) * np.linalg.norm(I.particles["vel"], axis=1)).sum()
    assert np.abs(np.array(d1["momentum"]) - np.array(d0["momentum"])).max() / pscale < 1e-4
    e0 = d0["kinetic"] + d0["internal"] + d0["potential"]
    e1 = d1["kinetic"] + d1["internal"] + d1["potential"]
    assert abs(e1 - e0) / abs(d0["potential"]) < 1e-3
    assert d1["h_residual"] < 2e-3
    st = s.readback()
    g = s.inspect("ACC_GRAV")[:, :3].astype(np.float64)
    tg = np.random.default_rng(5).choice(len(st), 2048, replace=False).astype(np.uint32)
    ref = s.gravity_direct64(st["pos"].astype(np.float64), st["mass"].astype(np.float64), I.softening, targets=tg)
    rms = math.sqrt(((g[tg] - ref) ** 2).sum() / (ref ** 2).sum())
    assert rms < 1e-3, rms


@pytest.mark.parametrize("graph", [0, 1])
def test_potential_on_demand_after_steps(graph):
    """KDK walks leave the potential out; sph_diag sums it in a potential-only walk over the last evaluation's
    tree. Its PE agrees with the FP64 direct sum of the state, repeated calls agree exactly, the per-particle φ
    of the inspection is what it summed, and a diagnostic between steps changes nothing: the trajectory and the
    final PE equal those of a run without it, bit for bit (eager steps and graph replays)."""
    from botheadstudios_b200 import ic
    I = ic.impact(16_000, 2_000, n_ngb=48, seed=4)
    kw = dict(kernel="wendland", multipole=1, leaf_size=16, theta=0.6, h_mode=1, h_neighbours=48, cfl=0.3,
              graph=graph, **ic.config_kwargs(I.units))
    n = len(I.particles)
    with GpuSph(n, **kw) as a, GpuSph(n, **kw) as b:
        for s in (a, b):
            s.upload(I.particles, I.eos, I.softening)
        a.encode_kdk(2)
        d1, d2 = a.diag(), a.diag()
        g1 = a.inspect("ACC_GRAV")
        st = a.readback()
        a.encode_kdk(2)
        b.encode_kdk(4)
        assert np.array_equal(a.readback().view(np.uint8), b.readback().view(np.uint8))
        assert a.diag()["potential"] == b.diag()["potential"]
    assert d1["potential"] == d2["potential"] and d1["potential"] < 0.0
    assert 0.5 * (st["mass"].astype(np.float64) * g1[:, 3]).sum() == pytest.approx(d1["potential"], rel=1e-6)
    pe = oracle.conservation64(st["pos"], st["vel"], st["mass"], st["u"], soft=I.softening, G=I.units.G)[2]
    assert d1["potential"] == pytest.approx(pe, rel=1e-3)
