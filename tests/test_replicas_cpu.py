"""Host logic of the multi-GPU replica path on two gloo ranks (CPU only):
each rank draws its own key stream, timing is reduced with MAX over ranks,
and the aggregate throughput counts the work of every rank."""
import os
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import importlib

    import torch

    import bench
    from oracle import OracleLSM

    dist.init_process_group("gloo", rank=rank, world_size=world)
    W = importlib.import_module("gpu-lsm-tree_b200.workloads")
    w = bench.make_workload(W, "lsm_scale", 8, rank)
    o = OracleLSM()
    for op in w.ops:
        o.insert(op[1], op[2]) if op[0] == "insert" else o.erase(op[1])
    answers = o.lookup(w.lookups)
    ms = torch.tensor([10.0 + rank])
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    first = torch.from_numpy(w.ops[0][1][:4].astype(np.int64))
    gathered = [torch.zeros_like(first) for _ in range(world)]
    dist.all_gather(gathered, first)
    q.put((rank, float(ms.item()), [g.tolist() for g in gathered], int((answers != 0xFFFFFFFF).sum())))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ms0, g0, hits0), (r1, ms1, g1, hits1) = res
    assert ms0 == ms1 == 11.0  # max over ranks
    assert g0[0] != g0[1]  # ranks insert different keys
    assert hits0 > 0 and hits1 > 0
