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
