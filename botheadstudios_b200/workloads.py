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
}


def build(wl: dict, seed: int = 1) -> ic.Impact:
    if wl.get("kind") == "planet":
        return ic.planet(wl["n_target"], n_ngb=wl["n_ngb"], seed=seed)
    return ic.impact(wl["n_target"], wl["n_impactor"], n_ngb=wl["n_ngb"], seed=seed)


def solver(wl: dict, I: ic.Impact, device: int = -1, **over):
    from .gpusph import GpuSph
    kw = dict(theta=wl["theta"], leaf_size=wl["leaf"], kernel=wl["kernel"], multipole=wl["quad"],
              h_mode=wl["h_solve"], h_neighbours=wl["n_ngb"], h_iters=2, max_neighbours=wl["max_nbr"], cfl=0.3,
              device=device, **ic.config_kwargs(I.units))
    kw.update(over)
    return GpuSph(len(I.particles), **kw)
