"""Named benchmark workloads (synthetic giant impacts) and the solver configuration each one runs with."""
from __future__ import annotations

from . import ic

WORKLOADS = {
    # the 1M single impact: Wendland C2, 64 neighbours with the smoothing-length solve, θ = 0.6 with
    # quadrupoles, 16-particle leaves
    "impact_1m": dict(n_target=953_250, n_impactor=95_326, n_ngb=64.0, kernel="wendland", theta=0.6, quad=1, leaf=16,
                      h_solve=1, max_nbr=192),
    # the 4M impact shape (same method)
    "impact_4m": dict(n_target=3_813_004, n_impactor=381_300, n_ngb=64.0, kernel="wendland", theta=0.6, quad=1,
                      leaf=16, h_solve=1, max_nbr=192),
    # the small plain-method impact: cubic spline, 48 neighbours, monopole θ = 0.5, one particle per leaf
    "impact_10k": dict(n_target=8_192, n_impactor=2_048, n_ngb=48.0, kernel="cubic", theta=0.5, quad=0, leaf=1,
                       h_solve=0, max_nbr=256),
    # the precision-sweep body: a 4,194,304-particle differentiated planet at rest (θ swept by the caller)
    "planet_4m": dict(kind="planet", n_target=4_194_304, n_impactor=0, n_ngb=64.0, kernel="wendland", theta=0.5,
                      quad=1, leaf=16, h_solve=1, max_nbr=192),
    # the learned smoothing-length form of the 4M and 1M impacts: the network (trained on the 10k impact and the
    # planet) proposes h, one residual check, Newton only for the rejected particles
    "learned_4m": dict(n_target=3_813_004, n_impactor=381_300, n_ngb=64.0, kernel="wendland", theta=0.6, quad=1,
                       leaf=16, h_solve=2, max_nbr=192),
    "learned_1m": dict(n_target=953_250, n_impactor=95_326, n_ngb=64.0, kernel="wendland", theta=0.6, quad=1,
                       leaf=16, h_solve=2, max_nbr=192),
    # 256 independent impacts, total particle counts log-uniform in [20k, 200k] (about 2.0e7 particles), mass
    # ratio 0.05-0.15, angle 0-75°, v_imp 1.0-1.5 v_esc; the 1M impact's method; one context per size bucket
    # (launch configuration autotuned per bucket) advancing its impacts with one launch per phase, steady steps
    # replayed from a captured CUDA graph
    "batch_256": dict(kind="batch", n_impacts=256, n_min=20_000, n_max=200_000, n_ngb=64.0, kernel="wendland",
                      theta=0.6, quad=1, leaf=16, h_solve=1, max_nbr=192, graph=1, autotune=1),
    # the learned smoothing-length form of the same 256 impacts (the network proposes h, Newton only where the
    # proposal's residual check fails), batched and graphed as above
    "batch_256_learned": dict(kind="batch", n_impacts=256, n_min=20_000, n_max=200_000, n_ngb=64.0,
                              kernel="wendland", theta=0.6, quad=1, leaf=16, h_solve=2, max_nbr=192, graph=1,
                              autotune=1),
    # the same draw with 16 impacts (a quick check of the batched path)
    "batch_16": dict(kind="batch", n_impacts=16, n_min=20_000, n_max=200_000, n_ngb=64.0, kernel="wendland",
                     theta=0.6, quad=1, leaf=16, h_solve=1, max_nbr=192, graph=1, autotune=1),
}

# Post-impact fields for the disk measurement (SI): a remnant of n_rem particles, a debris ring, escaping
# particles and clumps (eight cold ones of 200-480 members between 3 and 5.8 R plus the four gate cases). The
# 1M field's ring is 2 % of the particles, the share of a giant-impact disk at this resolution.
_MEASURE_CLUMPS = tuple((200 + 40 * k, 3.0 + 0.4 * k, 5.0, 0.55 * k) for k in range(8)) + ic.SCENE_CLUMPS
MEASURE_WORKLOADS = {
    "post_impact_1m": dict(n_rem=1_000_000, n_ring=20_000, n_esc=2_000, clumps=_MEASURE_CLUMPS, m_rem=6.0e18,
                           h_rem=2.5e5, h_debris=1.2e5, clump_radius=4.0e5),
    "post_impact_4m": dict(n_rem=4_000_000, n_ring=80_000, n_esc=8_000, clumps=_MEASURE_CLUMPS, m_rem=1.5e18,
                           h_rem=1.6e5, h_debris=0.8e5, clump_radius=2.6e5),
    "post_impact_200k": dict(n_rem=200_000, n_ring=15_000, n_esc=2000, clumps=_MEASURE_CLUMPS, m_rem=3.0e19,
                             h_rem=2.2e5, h_debris=1.2e5, clump_radius=4.0e5),
}


def impactor_fraction(wl: dict) -> float:
    """Fraction of a workload's particles in the impactor (the batch: mass ratio 0.1 at the range centre)."""
    if wl.get("kind") == "batch":
        return 0.1 / 1.1
    return wl["n_impactor"] / (wl["n_target"] + wl["n_impactor"])


def n_particles(wl: dict, seed: int = 1) -> int:
    """Particles of the workload build(wl, seed) makes, without building it."""
    if wl.get("kind") == "batch":
        return sum(d["n"] for d in ic.batch_draws(wl["n_impacts"], wl["n_min"], wl["n_max"], 10 + seed))
    return wl["n_target"] + wl["n_impactor"]


def upload(s, I) -> int:
    """Upload a built workload (one impact, or a batch) into a solver."""
    if isinstance(I, ic.Batch):
        return s.upload_batch(I.particles, I.offsets, I.eos, I.softening)
    return s.upload(I.particles, I.eos, I.softening)


def build(wl: dict, seed: int = 1):
    if wl.get("kind") == "batch":
        return ic.batch(wl["n_impacts"], wl["n_min"], wl["n_max"], n_ngb=wl["n_ngb"], seed=10 + seed)
    if wl.get("kind") == "planet":
        return ic.planet(wl["n_target"], n_ngb=wl["n_ngb"], seed=seed)
    return ic.impact(wl["n_target"], wl["n_impactor"], n_ngb=wl["n_ngb"], seed=seed)


def config(wl: dict, I, **over) -> dict:
    """The solver configuration (sph_config fields) a workload runs with."""
    kw = dict(theta=wl["theta"], leaf_size=wl["leaf"], kernel=wl["kernel"], multipole=wl["quad"],
              h_mode=wl["h_solve"], h_neighbours=wl["n_ngb"], h_iters=2, max_neighbours=wl["max_nbr"], cfl=0.3,
              graph=wl.get("graph", 0), **ic.config_kwargs(I.units))
    kw.update(over)
    return kw


def solver(wl: dict, I, device: int = -1, **over):
    """A context for the workload; the learned form gets the trained network (progress held at 0.5)."""
    from .gpusph import GpuSph
    s = GpuSph(len(I.particles), device=device, **config(wl, I, **over))
    if config(wl, I, **over)["h_mode"] == 2:
        from . import learned_h
        s.mlp_set(learned_h.load())
        s.set_progress(0.5)
    return s
