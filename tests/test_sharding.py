"""Host side of the multi-GPU path: independent systems are shared out by
LPT with no data-path collective; results are gathered once.  Exercised with
world_size-2 gloo process groups on CPU."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from sdddst_b200 import sharding, workloads


def test_lpt_partition_is_complete_disjoint_and_balanced():
    sizes = workloads.batch_sizes(512, 3)
    for ranks in (1, 2, 4, 8):
        parts = sharding.lpt_partition(sizes, ranks)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(int(sizes[k]) ** 2 for k in p) for p in parts]
        assert max(loads) - min(loads) <= int(max(sizes)) ** 2
    assert sharding.lpt_partition(sizes, 4) == sharding.lpt_partition(sizes, 4)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = sharding.rank_share(sizes, rank, world)
    # stand-in per-system result: a deterministic function of the system
    local = {k: float(np.sum(workloads.dislocations(int(sizes[k]), 1000 + k)[0][:, 0])) for k in mine}
    gathered = [None] * world
    dist.all_gather_object(gathered, local)
    if rank == 0:
        merged = {}
        for g in gathered:
            assert not (set(g) & set(merged))
            merged.update(g)
        out.put(sorted(merged.items()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_share_and_gather():
    sizes = [int(s) for s in workloads.batch_sizes(24, 3)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    expect = sorted((k, float(np.sum(workloads.dislocations(n, 1000 + k)[0][:, 0]))) for k, n in enumerate(sizes))
    assert res == expect
