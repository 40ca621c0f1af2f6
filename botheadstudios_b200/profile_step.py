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
    ap.add_argument("--theta", type=float, default=None)
    ap.add_argument("--local-theta", type=float, default=None,
                    help="group walk: the local expansion's opening parameter (0 = off; default: the library's)")
    ap.add_argument("--precision", type=int, default=0, help="1 = node-relative hi/lo + compensated sums")
    ap.add_argument("--leaf", type=int, default=None, help="LBVH leaf size (default: the workload's)")
    ap.add_argument("--walk-warps", type=int, default=0, help="warps per walk block (2, 4, 8; 0 = 4)")
    ap.add_argument("--block", type=int, default=0, help="threads per block of the gather kernels (0 = 256)")
    ap.add_argument("--gravity", default=None, choices=["tree", "direct", "none"], help="override the gravity mode")
    ap.add_argument("--accuracy", type=int, default=0,
                    help="targets for an FP64 direct-sum check of the tree gravity (0 = skip)")
    args = ap.parse_args()
    wl = workloads.WORKLOADS[args.workload]
    I = workloads.build(wl)
    over = dict(mac=args.mac, precision=args.precision, walk_warps=args.walk_warps, block_threads=args.block)
    if args.leaf is not None:
        over["leaf_size"] = args.leaf
    if args.gravity is not None:
        over["gravity"] = args.gravity
    if args.theta is not None:
        over["theta"] = args.theta
    if args.local_theta is not None:
        over["local_theta"] = args.local_theta
    acc_err = None
    with workloads.solver(wl, I, **over) as s:
        workloads.upload(s, I)
        s.encode_kdk(args.warmup)
        s.sync()
        d0 = s.diag()
        s.profile_enable(True)
        s.encode_kdk(args.steps)
        prof = s.profile_read()
        d1 = s.diag()
        if args.accuracy:
            import numpy as np
            state = s.readback()
            g = s.inspect("ACC_GRAV")[:, :3].astype(np.float64)
            pos = state["pos"].astype(np.float64)
            mass = state["mass"].astype(np.float64)
            tg = np.random.default_rng(7).choice(len(mass), args.accuracy, replace=False).astype(np.uint32)
            ref = s.gravity_direct64(pos, mass, I.softening, targets=tg)
            e = np.linalg.norm(g[tg] - ref, axis=1) / np.linalg.norm(ref, axis=1)
            acc_err = dict(targets=args.accuracy, rms_rel=float(np.sqrt(np.mean(e * e))),
                           p99_rel=float(np.quantile(e, 0.99)), max_rel=float(e.max()),
                           global_rms=float(np.sqrt(((g[tg] - ref) ** 2).sum() / (ref ** 2).sum())))
    n = len(I.particles)
    walks = max(prof["calls"]["gravity"], prof["calls"]["neighbours"], 1)
    stats = {k: (d1[k] - d0[k]) / walks for k in ("walk_nodes", "walk_pops", "m2p_interactions", "p2p_interactions",
                                                "local_expansions", "p2p_slots")}
    print(json.dumps(dict(workload=args.workload, particles=n, steps=args.steps, config=over, phases_ms=prof["ms"],
                          calls=prof["calls"], launches=prof["kernel_launches"], per_walk=stats,
                          per_particle={k: v / n for k, v in stats.items()}, gravity_error=acc_err)))


if __name__ == "__main__":
    main()
