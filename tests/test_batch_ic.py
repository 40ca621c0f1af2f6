"""The batched-impact generator (host side, no GPU): seeded, sizes log-uniform in range, collision parameters in
range, impacts contiguous, each impact a zero-momentum pair."""
import math

import numpy as np

from botheadstudios_b200 import ic, workloads


def test_batch_is_seeded_and_in_range():
    a = ic.batch(12, 300, 3000, n_ngb=16.0, seed=7)
    b = ic.batch(12, 300, 3000, n_ngb=16.0, seed=7)
    assert np.array_equal(a.particles, b.particles) and np.array_equal(a.offsets, b.offsets)
    sizes = np.diff(a.offsets)
    assert a.n_impacts == 12 and (sizes >= 300).all() and (sizes <= 3000).all()
    assert [p["n"] for p in a.params] == sizes.tolist()
    for p in a.params:
        assert 0.05 <= p["mass_ratio"] <= 0.15 and 0.0 <= p["angle_deg"] <= 75.0 and 1.0 <= p["v_factor"] <= 1.5
    for k in range(a.n_impacts):
        imp = a.impact(k)
        mom = (imp["mass"][:, None].astype(np.float64) * imp["vel"]).sum(0)
        assert np.abs(mom).max() < 1e-5
        assert set(np.unique(imp["prov"])) == {0, 1}  # target and impactor
    assert (a.softening > 0).all()


def test_batch_sizes_are_log_uniform():
    d = ic.batch_draws(4000, 20_000, 200_000, seed=3)
    x = np.log(np.array([v["n"] for v in d], np.float64))
    lo, hi = math.log(20_000), math.log(200_000)
    # uniform in log: mean at the centre, quartiles at the quarter points
    assert abs(x.mean() - 0.5 * (lo + hi)) < 0.03 * (hi - lo)
    q = np.quantile(x, [0.25, 0.75])
    assert np.allclose(q, [lo + 0.25 * (hi - lo), lo + 0.75 * (hi - lo)], atol=0.03 * (hi - lo))


def test_batch_workload_counts():
    wl = workloads.WORKLOADS["batch_256"]
    n = workloads.n_particles(wl)
    assert 1.5e7 < n < 2.6e7  # 256 × the log-uniform mean (~78k)
    assert sum(d["n"] for d in ic.batch_draws(256, 20_000, 200_000, 11)) == n
