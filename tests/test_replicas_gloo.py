"""Multi-process path of ``bench.py`` on CPU: two ``gloo`` ranks.

A single case does not shard (every CG iteration reduces over all edges), so
``--gpus N`` runs N independent replicas.  The only cross-rank steps are the
barrier around the timed region and the max (time) / sum (work) reductions;
the reference arm runs on rank 0 alone and the other ranks exit without work.
"""
import json
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    w, r, local = bench.dist_env()
    dist = bench.maybe_init_dist(w, local, backend="gloo")
    bench.barrier(dist)
    t_max = bench.reduce_max(dist, 1.0 + rank)          # per-rank "device times"
    total = bench.reduce_sum(dist, 10.0 * (rank + 1))   # per-rank work
    res = {"rank": r, "world": w, "max": t_max, "sum": total}
    (Path(out_dir) / f"rank{rank}.json").write_text(json.dumps(res))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_barrier(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, d in enumerate(res):
        assert d["rank"] == r and d["world"] == world
        assert d["max"] == pytest.approx(2.0)       # max over ranks, every rank sees it
        assert d["sum"] == pytest.approx(30.0)


def test_reference_arm_other_ranks_exit_without_work(capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    class Args:
        workload = "d32_oscillating_sphere"
        warmup, steps, gpus = 3, 1, 2

    assert bench.run_reference(Args, world=2, rank=1) == 0
    assert capsys.readouterr().out == ""


def _batch_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    w, r, local = bench.dist_env()
    dist = bench.maybe_init_dist(w, local, backend="gloo")
    agg = bench.aggregate_batch(dist, seconds_concurrent=2.0 + rank, seconds_sequential=5.0 - rank,
                                cells=1000 * (rank + 1), launches=7, cg_iterations=100 + rank,
                                max_case_iterations=40 + 10 * rank)
    (Path(out_dir) / f"batch{rank}.json").write_text(json.dumps(agg))
    dist.destroy_process_group()


def test_sharded_sweep_reductions_on_two_gloo_ranks(tmp_path):
    """The sharded batched sweep's whole-job figures: the slowest rank's times and the
    summed work, identical on every rank."""
    world = 2
    mp.start_processes(_batch_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    res = [json.loads((tmp_path / f"batch{r}.json").read_text()) for r in range(world)]
    assert res[0] == res[1]
    a = res[0]
    assert a["seconds_concurrent"] == 3.0 and a["seconds_sequential"] == 5.0
    assert a["cells"] == 3000 and a["launches"] == 14
    assert a["cg_iterations"] == 201 and a["max_case_iterations"] == 50
