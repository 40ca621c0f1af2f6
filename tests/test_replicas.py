"""Multi-GPU is replicas only: each rank advances its own seeded workload, there is no collective on the data path,
and the job's throughput is the units all ranks processed over the slowest rank's device time. The host logic of
that (bench.py's reductions over ranks, the per-rank seeds) runs here as two gloo ranks on the CPU."""
import json
import math
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from botheadstudios_b200 import ic
        draws = ic.batch_draws(4, 20_000, 200_000, seed=11 + rank)  # each replica's own draw
        n_local = sum(d["n"] for d in draws)
        res = dict(
            max=bench.max_over_ranks(dist, float(rank + 1), rank),
            sum=bench.sum_over_ranks(dist, float(10 * (rank + 1)), rank),
            value=bench.replica_value(dist, 100.0 * (rank + 1), 10.0 * (rank + 1), rank),
            n_local=n_local,
            n_total=bench.sum_over_ranks(dist, float(n_local), rank),
        )
        bench.barrier(dist)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


def test_replica_reductions_over_two_gloo_ranks(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["max"] == 2.0                       # the slowest rank's time
        assert r["sum"] == 30.0
        assert r["value"] == pytest.approx(300.0 / 0.020)  # all units ÷ the slowest time (20 ms)
        assert r["n_total"] == res[0]["n_local"] + res[1]["n_local"]
    assert res[0]["n_local"] != res[1]["n_local"]  # the replicas are different draws


def _diag(ke, ie, pe, p, L, m=2.0):
    return dict(kinetic=ke, internal=ie, potential=pe, momentum=list(p), angular_momentum=list(L), mass=m)


def test_conservation_drifts_over_contexts():
    """The drifts bench.py reports: energy change over |PE|, |ΔP| over sqrt(2 M KE), |ΔL| over |L|, each summed
    over the contexts (isolated impacts) before the ratio."""
    sys.path.insert(0, ROOT)
    import bench
    start = [_diag(1.0, 2.0, -4.0, (1.0, 0.0, 0.0), (0.0, 0.0, 3.0)),
             _diag(1.0, 1.0, -4.0, (-1.0, 0.0, 0.0), (0.0, 0.0, 1.0))]
    end = [_diag(1.5, 2.0, -4.0, (1.0, 0.3, 0.0), (0.0, 0.0, 3.0)),
           _diag(1.0, 0.9, -4.0, (-1.0, 0.1, 0.0), (0.0, 0.04, 1.0))]
    d = bench.conservation_drifts(start, end)
    assert d["energy_drift"] == pytest.approx(0.4 / 8.0)
    assert d["momentum_drift"] == pytest.approx(0.4 / math.sqrt(2.0 * 4.0 * 2.0))
    assert d["angular_momentum_drift"] == pytest.approx(0.04 / 4.0)
    still = bench.conservation_drifts(start, start)
    assert still == dict(energy_drift=0.0, momentum_drift=0.0, angular_momentum_drift=0.0)
    zero = [_diag(0.0, 0.0, 0.0, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))]
    assert bench.conservation_drifts(zero, zero) == dict(energy_drift=None, momentum_drift=None,
                                                         angular_momentum_drift=None)


def test_cpu_legs_on_a_small_impact():
    """The CPU baseline legs on a small impact of the benchmark's generator: full KDK steps on all cores, the
    sampled single-thread estimate, the host record, and one config dict shared by both arms."""
    import argparse
    sys.path.insert(0, ROOT)
    import bench
    wl = dict(bench.WORKLOADS["impact_1m"], n_target=3000, n_impactor=300)
    leg = bench.cpu_baseline_leg(wl, budget_s=5.0, max_steps=1)
    assert leg["value"] > 0 and leg["single_thread"]["value"] > 0 and leg["single_thread"]["cores"] == 1
    assert leg["cores"] >= 1 and leg["host"]["nproc"] >= 1
    assert "3,300-particle" in leg["sample"]
    args = argparse.Namespace(workload="impact_1m", gpus=1)
    cfg = bench.bench_config(args, wl, 3300, 1)
    assert cfg["particles"] == 3300 and cfg["workload"] == "impact_1m" and cfg["leaf"] == 16
