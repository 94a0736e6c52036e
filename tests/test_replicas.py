"""Multi-GPU host logic on CPU: scene sharding, request routing and the
rank reductions, including a world-size-2 run over the gloo backend in
which each rank steps its own scenes (the oracle stands in for the GPU
replica) and the sharded traces equal the unsharded ones."""
import os
import socket

import numpy as np
import pytest

from naga_b200 import replicas


def test_partition_covers_every_scene_once_and_balances():
    rng = np.random.default_rng(0)
    sizes = np.exp(rng.uniform(np.log(2e3), np.log(1e5), 256)).astype(int)
    for world in (1, 2, 3, 4, 8):
        parts = replicas.partition_by_size(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [int(sizes[p].sum()) for p in parts]
        # greedy LPT bound: no rank exceeds another by more than one scene
        assert max(loads) - min(loads) <= sizes.max()
        assert parts == replicas.partition_by_size(list(sizes), world)  # deterministic
        assert replicas.shard(sizes, world - 1, world) == parts[world - 1]


def test_partition_edge_cases():
    assert replicas.partition_by_size([], 3) == [[], [], []]
    assert replicas.partition_by_size([5], 2) == [[0], []]
    assert replicas.partition_by_size([4, 4, 4, 4], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        replicas.partition_by_size([1], 0)


def test_router_places_on_least_loaded_rank():
    r = replicas.Router(2)
    assert r.place(100, 10) == 0
    assert r.place(10, 10) == 1
    assert r.place(10, 10) == 1
    r.done(0, 100, 10)
    assert r.place(1, 1) == 0


def test_reductions_without_process_group():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.sum_over_ranks(2.0) == 2.0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scene_sizes():
    return [18, 26, 22, 30, 20]  # 2-D grid sides


def _run_scene(n_side):
    from oracle import oracle
    import naga_b200 as naga

    g = naga.generate_grid(2, n_side, 3, n_side)
    probes = np.array([[0.3, 0.5], [0.7, 0.5]], np.float32)
    s = oracle.Scene(2, g["points"], g["n_bulk"], g["n_layer"], g["n_boundary"], g["normals"], g["sigma"], g["h"],
                     k=16, shape=1, probes=probes)
    s.set_density(naga.gaussian_pulse(g["points"], [0.5, 0.5], 1e-3, 0.08))
    return s.step(6), len(g["points"])


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sides = _scene_sizes()
        mine = replicas.shard([s * s for s in sides], rank, world)
        nodes = 0
        for i in mine:
            trace, n = _run_scene(sides[i])
            nodes += n
            np.save(os.path.join(outdir, f"scene{i}_rank{rank}.npy"), trace)
        total = replicas.sum_over_ranks(nodes, dist)
        slowest = replicas.max_over_ranks(float(rank + 1), dist)
        with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{total} {slowest}\n")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo_shard_scenes(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    sides = _scene_sizes()
    parts = replicas.partition_by_size([s * s for s in sides], world)
    total_nodes = 0
    for i, side in enumerate(sides):
        owner = next(r for r in range(world) if i in parts[r])
        files = [f for f in os.listdir(tmp_path) if f.startswith(f"scene{i}_")]
        assert files == [f"scene{i}_rank{owner}.npy"]  # stepped once, by its owner
        ref, n = _run_scene(side)
        total_nodes += n
        assert np.array_equal(np.load(os.path.join(tmp_path, files[0])), ref)
    for r in range(world):
        total, slowest = open(os.path.join(tmp_path, f"rank{r}.txt")).read().split()
        assert float(total) == total_nodes
        assert float(slowest) == world
