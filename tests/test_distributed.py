"""CPU tests of the multi-rank plumbing with gloo, world size 2."""

import os

import numpy as np
import torch.multiprocessing as mp

from rfx_b200.distributed import shard_instances


def test_shard_instances_balances_cells():
    rng = np.random.default_rng(0)
    cells = [(int(n) + 17) ** 3 for n in rng.integers(64, 161, 64)]
    for world in (1, 2, 4, 8):
        parts = shard_instances(cells, world)
        assert sorted(q for p in parts for q in p) == list(range(64))
        loads = [sum(cells[q] for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells)


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from rfx_b200.distributed import gather_objects, max_over_ranks, shard_instances
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v = max_over_ranks(10.0 + rank)
        cells = [100, 90, 80, 70, 60]
        mine = shard_instances(cells, world)[rank]
        allparts = gather_objects(mine)
        out.put((rank, v, allparts))
    finally:
        dist.destroy_process_group()


def test_gloo_world_size_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, v, parts in res:
        assert v == 11.0
        assert sorted(parts[0] + parts[1]) == [0, 1, 2, 3, 4]


def test_sharded_sweep_reassembles_the_global_sweep():
    """The bench's multi-GPU workload: each rank builds only its share of one
    global sweep (same random stream), the shares partition it, and the cells
    of the shares add up to the whole."""
    from rfx_b200.workloads import batched_sweep, batched_sweep_instance_cells
    n_all, world = 6, 2
    cells = batched_sweep_instance_cells(seed=0, n_inst=n_all, n_lo=8, n_hi=20)
    parts = shard_instances(cells, world)
    whole = batched_sweep(seed=0, n_inst=n_all, n_steps=8, n_lo=8, n_hi=20)
    got = {}
    for part in parts:
        for q, inst in zip(part, batched_sweep(seed=0, n_inst=n_all, n_steps=8, n_lo=8, n_hi=20, subset=part)):
            got[q] = inst
    assert sorted(got) == list(range(n_all))
    for q, inst in got.items():
        assert np.array_equal(inst.eps_r, whole[q].eps_r) and inst.box == whole[q].box
        assert int(np.prod(inst.grid.shape)) == cells[q]
    assert sum(cells[q] for p in parts for q in p) == sum(cells)
