"""Graph-level placement of the batched form across GPUs, exercised with two
gloo ranks on CPU: every rank computes the product's placement plan
(gp_plan_placement, host code, no device) for the same seeded batch, takes
its own share, runs the product's host verifier on each of its graphs as the
per-graph work, and the ranks gather their results.  No collective touches
the data path besides that gather of results."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _jobs(gp):
    rng = np.random.default_rng(5)
    jobs = []
    for i in range(24):
        n = int(10 ** rng.uniform(2.5, 4.5))
        if i % 3 == 0:
            g = gp.rmat(max(8, int(np.log2(n))), 8, 0.57, 0.19, 0.19, i)
        elif i % 3 == 1:
            w = max(2, int(n ** 0.5))
            g = gp.grid2d(w, max(2, n // w))
        else:
            g = gp.with_weights(gp.grid2d(max(2, n // 50), 50), i, (1, 4), (1, 9))
        jobs.append((g, int(rng.choice([2, 4, 8, 16]))))
    return jobs


def _worker(rank, world, port, out):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "tests"))
    from conftest import _load_package
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    gp = _load_package()
    jobs = _jobs(gp)
    work = np.array([gp.batch_work(g) for g, _ in jobs], np.uint64)
    device_of, device_work = gp.plan_placement(work, world)
    mine = {}
    for i, (g, k) in enumerate(jobs):
        if device_of[i] == rank:
            labels = (np.arange(g.n) * k // g.n).astype(np.int32)
            mine[i] = gp.verify(g, labels, k, 1.5)["cut"]
    gathered = [None] * world
    dist.all_gather_object(gathered, (rank, device_of.tolist(), device_work.tolist(), mine))
    if rank == 0:
        out.put(gathered)
    dist.destroy_process_group()


def test_two_rank_placement_covers_every_graph_once(gp):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    result = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    plans = [r[1] for r in result]
    assert plans[0] == plans[1], "ranks computed different plans"
    done = {}
    for rank, plan, device_work, mine in result:
        for i, cut in mine.items():
            assert i not in done, "graph placed twice"
            assert plan[i] == rank
            done[i] = cut
    jobs = _jobs(gp)
    assert sorted(done) == list(range(len(jobs)))
    for i, (g, k) in enumerate(jobs):  # the same host work done in this process
        labels = (np.arange(g.n) * k // g.n).astype(np.int32)
        assert done[i] == gp.verify(g, labels, k, 1.5)["cut"]
    work = [gp.batch_work(g) for g, _ in jobs]
    loads = result[0][2]
    assert sum(loads) == sum(work)
    assert max(loads) - min(loads) <= max(work)  # longest-processing-time bound


def test_placement_is_longest_processing_time(gp):
    """The plan equals a restatement of LPT: decreasing work, ties by index,
    each item to the least-loaded device, ties to the lower device."""
    rng = np.random.default_rng(3)
    work = rng.integers(1, 1000, 57).astype(np.uint64)
    work[10] = work[11] = work[12]  # ties
    for devices in (1, 2, 3, 8):
        device_of, device_work = gp.plan_placement(work, devices)
        loads = [0] * devices
        expected = [0] * len(work)
        for i in sorted(range(len(work)), key=lambda i: (-int(work[i]), i)):
            d = min(range(devices), key=lambda d: (loads[d], d))
            expected[i] = d
            loads[d] += int(work[i])
        assert device_of.tolist() == expected
        assert device_work.tolist() == loads
    with pytest.raises(gp.GpartError):
        gp.plan_placement(work, 0)
