"""Multi-GPU runs are independent replicas (no data-path collective).  The
host logic bench.py uses for them — per-rank work, max-over-ranks timing and
whole-job throughput — is exercised here with two gloo ranks on CPU.  Each
rank's work is the product's host-side path for its own replica (the seeded
generator and the verifier of the library; the partition itself needs a GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    import time
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "tests"))
    from conftest import _load_package
    import numpy as np
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    gp = _load_package()
    t = time.perf_counter()
    g = gp.rmat(12 + rank, 8, 0.57, 0.19, 0.19, rank)
    labels = (np.arange(g.n) * 4 // g.n).astype(np.int32)
    verdict = gp.verify(g, labels, 4, 1.03)
    cut = gp.edge_cut(g, labels)
    elapsed = torch.tensor([time.perf_counter() - t], dtype=torch.float64)
    dist.all_reduce(elapsed, op=dist.ReduceOp.MAX)
    cuts = [None] * world
    dist.all_gather_object(cuts, (rank, cut, verdict["cut"], verdict["capacity_ok"], float(elapsed.item())))
    if rank == 0:
        out.put(cuts)
    dist.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    result = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in result] == [0, 1]
    for rank, cut, vcut, ok, elapsed in result:
        assert cut == vcut
    assert result[0][4] == result[1][4]  # both ranks see the max-over-ranks time
