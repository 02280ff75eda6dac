"""The benchmark's multi-rank logic on CPU: world size 2 over gloo.

Each rank builds its own seeded design (a population member, no data-path
collective), the step times reduce to the slowest rank, and the reference
arm runs on rank 0 only. The population workload splits one population over
the ranks longest-first; every problem lands on exactly one rank."""

import os
import socket

import numpy as np

import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = bench.workload(rank, 128, 40)
        t = bench.max_over_ranks(dist, [1.0 + rank, 5.0 - rank], "cpu")
        args = type("A", (), {})()
        world_, rank_, local_ = bench.dist_setup(args)
        out[rank] = (float(w["sigma_d"].sum()), t, (world_, rank_, local_))
    finally:
        dist.destroy_process_group()


def test_two_ranks_seeded_designs_and_max_timing():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    (s0, t0, ids0), (s1, t1, ids1) = res[0], res[1]
    assert s0 != s1  # rank-seeded population members differ
    assert t0 == t1 == [2.0, 5.0]  # max over ranks, element-wise
    assert ids0 == (2, 0, 0) and ids1 == (2, 1, 1)


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    a = type("A", (), dict(grid=128, time_steps=40, dtype="f32", warmup=3, steps=1, gpus=2))()
    assert bench.run_reference(a) == 0
    assert capsys.readouterr().out == ""


def test_lpt_partition_covers_every_problem_once():
    import numpy as np

    import bench

    rng = np.random.default_rng(0)
    costs = list(rng.integers(1, 1000, size=64).astype(float))
    for n in (1, 2, 3, 8):
        parts = bench.lpt_partition(costs, n)
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = [sum(costs[i] for i in p) for p in parts]
        # Graham's bound: within 4/3 of the optimum, which is at least the
        # mean load and the largest item.
        lower = max(sum(costs) / n, max(costs))
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9
    assert bench.lpt_partition([5.0, 1.0, 1.0], 2) == [[0], [1, 2]]


def _pop_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        specs = bench.population(0, n_problems=12, max_steps=50)
        share = bench.lpt_partition([bench.pop_cells([sp]) for sp in specs], world)[rank]
        out[rank] = (share, [float(np.asarray(specs[q]["design_sigma"]).sum()) for q in share])
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_one_population():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_pop_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    (s0, d0), (s1, d1) = res[0], res[1]
    assert sorted(s0 + s1) == list(range(12)) and not set(s0) & set(s1)
    assert d0 and d1
