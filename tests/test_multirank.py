"""The multi-GPU host path on CPU: two gloo ranks split the batched
workload's sites (LPT by pixels, no data crosses ranks) and reduce their
step times to the max, as bench.py does over NCCL."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from solweig_project_b200 import batch as B
from solweig_project_b200 import synthetic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = synthetic.multi_site_specs()
        costs = [s["side"] ** 2 for s in specs]
        mine = B.partition_sites(costs, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = torch.tensor([float(sum(costs[i] for i in mine))], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            out.put((gathered, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_the_sites_and_reduce_the_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    specs = synthetic.multi_site_specs()
    costs = [s["side"] ** 2 for s in specs]
    assert sorted(i for part in gathered for i in part) == list(range(len(specs)))
    loads = [sum(costs[i] for i in part) for part in gathered]
    assert tmax == max(loads)
    # LPT bound: the heavier rank carries at most 4/3 of the ideal share
    assert max(loads) <= 4 / 3 * sum(costs) / 2 + max(costs)


@pytest.mark.parametrize("n", [1, 2, 3, 8])
def test_partition_is_a_balanced_cover(n):
    costs = [s["side"] ** 2 for s in synthetic.multi_site_specs()]
    parts = B.partition_sites(costs, n)
    assert len(parts) == n and sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
