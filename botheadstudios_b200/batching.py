"""Batched impacts by size bucket, with a launch-configuration autotuner.

A batch of impacts of uneven size is split into size buckets, each tuned on its own; buckets whose tuned launch
configurations agree share one context, which advances all of their impacts with one launch per phase (with one
configuration for every bucket, the whole batch is one context), and contexts of different configurations run
concurrently on their own streams. The autotuner picks, per bucket, the LBVH leaf size, the block size of the
per-particle gather kernels (density, h-solve, forces) and the traversal tile of the fused walk (warps per
block) by timing candidates on a probe batch drawn from that bucket. Choices are cached in a JSON file keyed
by the GPU name and the bucket.

The reference has no counterpart: its offline driver runs impacts one after another
(tools/impact-run/src/main.rs:645-671).
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import ic
from .gpusph import GpuSph

# particle-count buckets [lo, hi)
BUCKETS = ((0, 45_000), (45_000, 100_000), (100_000, 1 << 31))
CANDIDATES = dict(leaf_size=(8, 16, 32), walk_warps=(2, 4, 8), block_threads=(128, 256, 512))
DEFAULT_CHOICE = dict(leaf_size=16, walk_warps=2, block_threads=256)


def bucket_of(n: int) -> int:
    for b, (lo, hi) in enumerate(BUCKETS):
        if lo <= n < hi:
            return b
    raise ValueError(n)


def subset(B: ic.Batch, idx) -> ic.Batch:
    """The impacts `idx` of a batch, in that order, as a batch of their own."""
    parts = [B.impact(k) for k in idx]
    offs = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.uint32)
    return ic.Batch(particles=np.concatenate(parts), offsets=offs, softening=B.softening[list(idx)].copy(),
                    eos=B.eos, units=B.units, params=[B.params[k] for k in idx])


def _time_steps(s: GpuSph, steps: int) -> float:
    """Device time (ms) of `steps` KDK steps on the context's stream (CUDA events)."""
    import torch
    ext = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    s.encode_kdk(steps)
    e1.record(ext)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _load_network(s, cfg: dict):
    """The learned smoothing-length form needs the trained network in every context (progress held at 0.5)."""
    if cfg.get("h_mode") in (2, "learned"):
        from . import learned_h
        s.mlp_set(learned_h.load())
        s.set_progress(0.5)


class Autotuner:
    """Coordinate search over CANDIDATES (leaf size, then walk tile, then block size), each candidate timed on
    the same probe batch: a fresh context, one warm-up step (the full rebuild), `steps` timed steps."""

    def __init__(self, base: dict, cache_path: str | None = None, steps: int = 2, device: int = -1):
        self.base = dict(base)
        self.cache_path = cache_path
        self.steps = steps
        self.device = device
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            self.cache = json.load(open(cache_path))
        self.log = []
        self.bucket_logs = {}  # bucket → the measurements its own tuning made (none for a cached choice)

    def _key(self, bucket: int) -> str:
        import torch
        name = torch.cuda.get_device_name(self.device if self.device >= 0 else None)
        return f"{name}|bucket{bucket}|{json.dumps(self.base, sort_keys=True, default=str)}"

    def measure(self, probe: ic.Batch, choice: dict) -> float:
        """Particle-steps/s of `choice` on the probe batch."""
        cfg = dict(self.base, **choice)
        with GpuSph(len(probe.particles), device=self.device, **cfg) as s:
            _load_network(s, cfg)
            s.upload_batch(probe.particles, probe.offsets, probe.eos, probe.softening)
            s.encode_kdk(1)
            s.sync()
            ms = _time_steps(s, self.steps)
        rate = len(probe.particles) * self.steps / (ms / 1000.0)
        self.log.append(dict(choice=choice, rate=rate))
        return rate

    def tune(self, bucket: int, probe: ic.Batch) -> dict:
        key = self._key(bucket)
        if key in self.cache:
            return dict(self.cache[key])
        start = len(self.log)
        best = dict(DEFAULT_CHOICE)
        best_rate = self.measure(probe, best)
        timed = [dict(best)]  # each configuration is timed once (a coordinate's first value may already be)
        for name in ("leaf_size", "walk_warps", "block_threads"):
            for v in CANDIDATES[name]:
                trial = dict(best, **{name: v})
                if trial in timed:
                    continue
                timed.append(trial)
                r = self.measure(probe, trial)
                if r > best_rate:
                    best, best_rate = trial, r
        self.bucket_logs[bucket] = self.log[start:]
        self.cache[key] = best
        if self.cache_path:
            json.dump(self.cache, open(self.cache_path, "w"), indent=1)
        return dict(best)


# The choices that shape the tree and the walk; buckets that agree on them share one context.
TREE_KEYS = ("leaf_size", "walk_warps")


def context_groups(bucket_ids, choices: dict) -> list:
    """Buckets that share a context: those whose tuned leaf size and walk tile agree (in bucket order). The
    gather kernels' block size, the one choice left, is taken from the group's bucket with the most particles
    (group_choice); its measured effect is within 2 % on the 256-impact batch."""
    groups = []
    for b in sorted(bucket_ids):
        ch = choices.get(b, DEFAULT_CHOICE)
        for g in groups:
            if all(choices.get(g[0], DEFAULT_CHOICE)[k] == ch[k] for k in TREE_KEYS):
                g.append(b)
                break
        else:
            groups.append([b])
    return groups


# Unify unconditionally by default: on the 256-impact batch one context with the largest bucket's tree ran at
# 193.2M particle-steps/s against 191.4M for per-bucket choices in two contexts (the small-impact bucket alone
# prefers 8-particle leaves by more than 3 %).
UNIFY_TOL = None


def unify_tree_choices(choices: dict, bucket_logs: dict, particles: dict, tol: float | None = UNIFY_TOL) -> dict:
    """One context (one launch per phase) for the whole batch. Every bucket takes the tree choice (leaf size,
    walk tile) of the bucket with the most particles. With a tolerance `tol`, only a bucket whose own
    measurements put that tree choice within `tol` of its best rate takes it (with the block size it measured
    best under it), and a bucket with no such measurement (a cached choice, or the tree never timed on it)
    keeps its own choice."""
    if not choices:
        return {}
    lead = max(choices, key=lambda b: particles.get(b, 0))
    tree = {k: choices[lead][k] for k in TREE_KEYS}
    out = {}
    for b, ch in choices.items():
        out[b] = dict(ch)
        if all(ch[k] == tree[k] for k in TREE_KEYS):
            continue
        if tol is None:
            out[b] = dict(ch, **tree)
            continue
        log = bucket_logs.get(b) or []
        if not log:
            continue
        best = max(e["rate"] for e in log)
        same = [e for e in log if all(e["choice"][k] == tree[k] for k in TREE_KEYS)]
        if same:
            e = max(same, key=lambda e: e["rate"])
            if e["rate"] >= (1.0 - tol) * best:
                out[b] = dict(e["choice"])
    return out


def group_choice(group, choices: dict, particles: dict) -> dict:
    """The configuration of a context holding `group`: the choice of its bucket with the most particles."""
    b = max(group, key=lambda k: particles.get(k, 0))
    return dict(choices.get(b, DEFAULT_CHOICE))


class BucketedBatch:
    """A batch of impacts advanced as one context per group of buckets with equal tuned choices (impacts
    reordered so that each context holds a contiguous range of the particle array; `order` maps back to the
    caller's impact order)."""

    def __init__(self, B: ic.Batch, base: dict, choices: dict | None = None, device: int = -1):
        sizes = np.diff(B.offsets).astype(np.int64)
        buckets = np.array([bucket_of(int(n)) for n in sizes])
        choices = choices or {}
        self.bucket_ids = sorted(set(buckets.tolist()))
        self.groups = context_groups(self.bucket_ids, choices)
        group_of = {b: gi for gi, g in enumerate(self.groups) for b in g}
        per_bucket = {int(b): int(sizes[buckets == b].sum()) for b in self.bucket_ids}
        self.group_choices = [group_choice(g, choices, per_bucket) for g in self.groups]
        gidx = np.array([group_of[int(b)] for b in buckets])
        self.order = np.argsort(gidx, kind="stable")
        self.batch = subset(B, self.order)
        self.ranges, self.ctxs, self.sub = [], [], []
        k0 = 0
        for gi, g in enumerate(self.groups):
            k1 = k0 + int((gidx == gi).sum())
            sub = subset(self.batch, range(k0, k1))
            cfg = dict(base, **self.group_choices[gi])
            s = GpuSph(len(sub.particles), device=device, **cfg)
            _load_network(s, cfg)
            self.ctxs.append(s)
            self.sub.append(sub)
            self.ranges.append((int(self.batch.offsets[k0]), int(self.batch.offsets[k1])))
            k0 = k1
        self.n = len(self.batch.particles)

    def upload(self, particles: np.ndarray | None = None):
        """Upload every bucket (from `particles`, a bucket-ordered array such as a pinned copy, or the batch)."""
        p = self.batch.particles if particles is None else particles
        for s, sub, (a, b) in zip(self.ctxs, self.sub, self.ranges):
            s.upload_batch(p[a:b], sub.offsets, sub.eos, sub.softening)

    def encode_kdk(self, substeps: int):
        for s in self.ctxs:
            s.encode_kdk(substeps)

    def sync(self):
        for s in self.ctxs:
            s.sync()

    def readback_into(self, out: np.ndarray):
        for s, (a, b) in zip(self.ctxs, self.ranges):
            s.readback_into(out[a:b])

    def profile_enable(self, on: bool):
        for s in self.ctxs:
            s.profile_enable(on)

    def profile_read(self) -> list:
        return [s.profile_read() for s in self.ctxs]

    def diag(self, check: bool = True) -> list:
        return [s.diag(check) for s in self.ctxs]

    def close(self):
        for s in self.ctxs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def tune_buckets(B: ic.Batch, base: dict, cache_path: str | None = None, probe_particles: int = 600_000,
                 device: int = -1) -> tuple[dict, list]:
    """Autotune every bucket that `B` populates, on a probe of that bucket's impacts (about probe_particles
    particles, the bucket's first impacts), then unify the tree choices where the measurements allow one
    context (unify_tree_choices). Returns ({bucket: choice}, measurement log)."""
    tuner = Autotuner(base, cache_path=cache_path, device=device)
    sizes = np.diff(B.offsets).astype(np.int64)
    choices = {}
    particles = {}
    for n in sizes:
        particles[bucket_of(int(n))] = particles.get(bucket_of(int(n)), 0) + int(n)
    for b in sorted({bucket_of(int(n)) for n in sizes}):
        idx, tot = [], 0
        for k, n in enumerate(sizes):
            if bucket_of(int(n)) == b and tot < probe_particles:
                idx.append(k)
                tot += int(n)
        choices[b] = tuner.tune(b, subset(B, idx))
    return unify_tree_choices(choices, getattr(tuner, "bucket_logs", {}), particles), tuner.log
