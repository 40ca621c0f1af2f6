"""Profiling driver: run a named workload for a few KDK steps and print per-phase device times and the
tree-walk counters. Small and deterministic, so it can run under ncu:

    python -m botheadstudios_b200.profile_step --workload impact_1m --warmup 1 --steps 1
"""
from __future__ import annotations

import argparse
import json

from . import workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="impact_1m", choices=sorted(workloads.WORKLOADS))
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--mac", type=int, default=0)
    args = ap.parse_args()
    wl = workloads.WORKLOADS[args.workload]
    I = workloads.build(wl)
    with workloads.solver(wl, I, mac=args.mac) as s:
        s.upload(I.particles, I.eos, I.softening)
        s.encode_kdk(args.warmup)
        s.sync()
        d0 = s.diag()
        s.profile_enable(True)
        s.encode_kdk(args.steps)
        prof = s.profile_read()
        d1 = s.diag()
    n = len(I.particles)
    walks = max(prof["calls"]["gravity"], 1)
    stats = {k: (d1[k] - d0[k]) / walks for k in ("walk_nodes", "walk_pops", "m2p_interactions", "p2p_interactions")}
    print(json.dumps(dict(workload=args.workload, particles=n, steps=args.steps, phases_ms=prof["ms"],
                          calls=prof["calls"], launches=prof["kernel_launches"], per_walk=stats,
                          per_particle={k: v / n for k, v in stats.items()})))


if __name__ == "__main__":
    main()
