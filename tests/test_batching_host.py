"""Host logic of the batched form (botheadstudios_b200/batching.py), on the CPU: size buckets, impact subsets,
the autotuner's coordinate search and its cache, and the probe each bucket is tuned on. Timings are replaced
by a fake rate function; the GPU measurement itself is covered by tests/test_gpu_batch.py."""
import json

import numpy as np
import pytest

from botheadstudios_b200 import batching, ic


def test_bucket_edges():
    assert [batching.bucket_of(n) for n in (0, 44_999, 45_000, 99_999, 100_000, 21_000_000)] == [0, 0, 1, 1, 2, 2]
    with pytest.raises(ValueError):
        batching.bucket_of(-1)


def test_subset_keeps_each_impact_whole_and_in_the_given_order():
    B = ic.batch(5, 600, 2_000, seed=3)
    sub = batching.subset(B, [3, 0, 4])
    sizes = np.diff(B.offsets)
    assert np.array_equal(np.diff(sub.offsets), sizes[[3, 0, 4]])
    for j, k in enumerate((3, 0, 4)):
        a, b = int(sub.offsets[j]), int(sub.offsets[j + 1])
        assert np.array_equal(sub.particles[a:b], B.impact(k))
        assert sub.softening[j] == B.softening[k]
        assert sub.params[j] == B.params[k]


class _FakeTuner(batching.Autotuner):
    """Rates from a fixed table instead of GPU timings; every measurement is recorded."""

    def __init__(self, rate, **kw):
        super().__init__(dict(kernel="wendland"), **kw)
        self.rate = rate
        self.calls = []

    def _key(self, bucket):
        return f"fake|bucket{bucket}"

    def measure(self, probe, choice):
        self.calls.append(dict(choice))
        r = self.rate(choice)
        self.log.append(dict(choice=choice, rate=r))
        return r


def _rate(choice):
    # best: leaf 8, 2 warps, 512 threads; each coordinate matters on its own
    return (100.0 + {8: 30, 16: 10, 32: 0}[choice["leaf_size"]] + {2: 5, 4: 3, 8: 0}[choice["walk_warps"]]
            + {128: 0, 256: 1, 512: 2}[choice["block_threads"]])


def test_autotuner_coordinate_search_and_cache(tmp_path):
    cache = str(tmp_path / "tune.json")
    t = _FakeTuner(_rate, cache_path=cache)
    best = t.tune(1, probe=None)
    assert best == dict(leaf_size=8, walk_warps=2, block_threads=512)
    # the default first, then each other value of each coordinate once: 1 + 2 + 2 + 2 measurements
    assert t.calls[0] == batching.DEFAULT_CHOICE and len(t.calls) == 7
    assert [c["leaf_size"] for c in t.calls[1:3]] == [8, 32]
    assert all(c["leaf_size"] == 8 for c in t.calls[3:])  # later coordinates start from the better leaf size
    # cached: a second tune measures nothing, and a new tuner reads the choice back from the file
    assert t.tune(1, probe=None) == best and len(t.calls) == 7
    t2 = _FakeTuner(_rate, cache_path=cache)
    assert t2.tune(1, probe=None) == best and t2.calls == []
    assert json.load(open(cache)) == {"fake|bucket1": best}
    # a bucket not in the cache is tuned on its own
    t2.tune(2, probe=None)
    assert len(t2.calls) == 7


def test_autotuner_keeps_the_default_when_nothing_beats_it():
    t = _FakeTuner(lambda c: 1.0 if c == batching.DEFAULT_CHOICE else 0.5)
    assert t.tune(0, probe=None) == batching.DEFAULT_CHOICE


@pytest.mark.parametrize("probe_particles", [1, 10**9])
def test_tune_buckets_probes_each_populated_bucket_with_its_first_impacts(monkeypatch, probe_particles):
    """A bucket's probe is its impacts in batch order, taken until the probe holds probe_particles: the first
    impact alone for a budget of 1, all of them for an unbounded one."""
    B = ic.batch(6, 600, 2_000, seed=5)
    sizes = np.diff(B.offsets).astype(np.int64)
    m = int(np.median(sizes)) + 1
    monkeypatch.setattr(batching, "BUCKETS", ((0, m), (m, 1 << 31)))
    members = {b: [k for k in range(6) if (sizes[k] >= m) == bool(b)] for b in (0, 1)}
    assert members[0] and members[1]
    probes = {}

    class Recording(_FakeTuner):
        def __init__(self, base, cache_path=None, device=-1):
            super().__init__(_rate)

        def tune(self, bucket, probe):
            probes[bucket] = probe
            return super().tune(bucket, probe)

    monkeypatch.setattr(batching, "Autotuner", Recording)
    choices, log = batching.tune_buckets(B, dict(kernel="wendland"), probe_particles=probe_particles)
    assert sorted(choices) == [0, 1] and all(c["leaf_size"] == 8 for c in choices.values())
    for b, ks in members.items():
        want = ks[:1] if probe_particles == 1 else ks
        p = probes[b]
        assert len(p.offsets) - 1 == len(want)
        for j, k in enumerate(want):
            assert np.array_equal(p.particles[int(p.offsets[j]):int(p.offsets[j + 1])], B.impact(k))
    assert len(log) == 7 * 2


def test_buckets_with_equal_walk_choices_share_one_context():
    """One launch per phase for the whole batch when every bucket is tuned to the same leaf size and walk tile;
    buckets tuned to another tree or walk keep contexts of their own; the merged context takes the gather block
    size of its bucket with the most particles."""
    same = dict(leaf_size=8, walk_warps=2, block_threads=256)
    assert batching.context_groups([0, 1, 2], {0: same, 1: dict(same), 2: dict(same)}) == [[0, 1, 2]]
    blk = {0: dict(same, block_threads=128), 1: same, 2: dict(same, block_threads=512)}
    assert batching.context_groups([0, 1, 2], blk) == [[0, 1, 2]]
    assert batching.group_choice([0, 1, 2], blk, {0: 10, 1: 50, 2: 30})["block_threads"] == 256
    other = dict(same, leaf_size=16)
    assert batching.context_groups([0, 1, 2], {0: same, 1: other, 2: dict(same)}) == [[0, 2], [1]]
    assert batching.context_groups([0, 1, 2], {0: same, 1: dict(same, walk_warps=4), 2: same}) == [[0, 2], [1]]
    assert batching.context_groups([1], {}) == [[1]]
    assert batching.context_groups([0, 2], {}) == [[0, 2]]  # both untuned: the default choice


def test_unify_takes_the_largest_buckets_tree_where_the_measurements_allow():
    """With a tolerance, a bucket takes the tree choice (leaf size, walk tile) of the bucket with the most
    particles when its own measurements put that choice within 3 % of its best, so the batch runs as one
    context; otherwise, and for a bucket without measurements, it keeps its own. Without one (the default)
    every bucket takes it."""
    a = dict(leaf_size=8, walk_warps=2, block_threads=256)
    b = dict(leaf_size=16, walk_warps=2, block_threads=256)

    def log(*entries):
        return [dict(choice=c, rate=r) for c, r in entries]

    choices = {0: dict(a), 1: dict(b), 2: dict(b)}
    particles = {0: 100, 1: 500, 2: 50}
    logs = {0: log((a, 100.0), (b, 98.0), (dict(b, block_threads=512), 99.5)),
            1: log((b, 200.0), (a, 190.0)),
            2: log((b, 100.0), (a, 90.0))}
    out = batching.unify_tree_choices(choices, logs, particles, tol=0.03)
    # bucket 1 leads; bucket 0 measured its tree within 3 % (99.5 with 512 threads), bucket 2 already has it
    assert out == {0: dict(b, block_threads=512), 1: b, 2: b}
    assert batching.context_groups([0, 1, 2], out) == [[0, 1, 2]]
    # 5 % slower than its best: bucket 0 keeps its own choice
    logs[0] = log((a, 100.0), (b, 95.0))
    assert batching.unify_tree_choices(choices, logs, particles, tol=0.03)[0] == a
    # no measurements (a cached choice) or the lead's tree never timed on it: kept
    assert batching.unify_tree_choices(choices, {}, particles, tol=0.03) == choices
    logs[0] = log((a, 100.0), (dict(a, walk_warps=4), 99.0))
    assert batching.unify_tree_choices(choices, logs, particles, tol=0.03)[0] == a
    assert batching.unify_tree_choices({}, {}, {}) == {}
    # the default: unconditional, every bucket on the lead's tree (its own block size kept)
    out = batching.unify_tree_choices(choices, {}, particles)
    assert out == {0: dict(a, leaf_size=16), 1: b, 2: b}
    assert batching.context_groups([0, 1, 2], out) == [[0, 1, 2]]


def test_tune_buckets_unifies_when_rates_tie(monkeypatch):
    """Through tune_buckets: with a rate table that does not depend on the bucket, every bucket tunes to the same
    tree, and the result is one context."""
    B = ic.batch(6, 600, 2_000, seed=5)
    sizes = np.diff(B.offsets).astype(np.int64)
    m = int(np.median(sizes)) + 1
    monkeypatch.setattr(batching, "BUCKETS", ((0, m), (m, 1 << 31)))

    class Fake(_FakeTuner):
        def __init__(self, base, cache_path=None, device=-1):
            super().__init__(_rate)

    monkeypatch.setattr(batching, "Autotuner", Fake)
    choices, _ = batching.tune_buckets(B, dict(kernel="wendland"))
    assert batching.context_groups(sorted(choices), choices) == [sorted(choices)]
