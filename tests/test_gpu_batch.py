"""Many graphs on one GPU: gp_partition_batch and the partition server.

Every result must equal the same request partitioned alone (the same
deterministic single-graph path runs on each worker context), and the
verifier must accept it."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mixed_graphs(gp):
    """Uneven sizes and kinds: grids, meshes, R-MAT (one weighted)."""
    return [
        (gp.grid2d(40, 30), 4, 1.03, 0),
        (gp.rmat(14, 8, 0.57, 0.19, 0.19, 1), 64, 1.03, 0),
        (gp.mesh3d(12, 10, 9), 16, 1.05, 3),
        (gp.rmat(16, 16, 0.57, 0.19, 0.19, 2), 128, 1.03, 0),
        (gp.grid2d(256, 256), 8, 1.03, 0),
        (gp.with_weights(gp.rmat(13, 12, 0.57, 0.19, 0.19, 4), 5, (1, 16), (1, 64)), 37, 1.01, 9),
        (gp.rmat(12, 16, 0.57, 0.19, 0.19, 7), 2, 1.03, 1),
        (gp.mesh3d(30, 30, 30), 32, 1.03, 0),
        (gp.grid2d(7, 500), 8, 1.03, 2),
        (gp.rmat(17, 10, 0.57, 0.19, 0.19, 8), 64, 1.03, 0),
    ]


def test_batch_equals_single_calls(gp, ctx):
    jobs = mixed_graphs(gp)
    alone = [ctx.partition(g, k, eps, seed) for g, k, eps, seed in jobs]
    batched = ctx.partition_batch(jobs, concurrency=6)
    for (g, k, eps, _), (labels, st), (blabels, bst, run_s) in zip(jobs, alone, batched):
        np.testing.assert_array_equal(blabels, labels)
        assert bst.edge_cut == st.edge_cut and run_s > 0
        verdict = gp.verify(g, blabels, k, eps)
        assert verdict["capacity_ok"] and verdict["cut"] == bst.edge_cut


def test_batch_reports_failed_request(gp, ctx):
    jobs = [(gp.grid2d(20, 20), 4, 1.03, 0), (gp.grid2d(3, 3), 16, 2.0, 0)]
    with pytest.raises(gp.GpartError) as e:
        ctx.partition_batch(jobs, concurrency=2)
    assert "request 1" in str(e.value)


def test_server_results_same_alone_and_in_mix(gp, ctx):
    jobs = mixed_graphs(gp)
    alone = [ctx.partition(g, k, eps, seed)[0] for g, k, eps, seed in jobs]
    with gp.Server(0, workers=4) as server:
        resident = server.add_graph(jobs[3][0])
        tickets = []

        def arrive():
            rng = np.random.default_rng(0)
            for i, (g, k, eps, seed) in enumerate(jobs):
                graph = resident if i == 3 else g
                tickets.append((i, server.submit(graph, k, eps, seed)))
                time.sleep(float(rng.exponential(0.004)))

        producer = threading.Thread(target=arrive)
        producer.start()
        producer.join()
        for i, ticket in tickets:
            labels, st, queued, run = server.wait(ticket)
            np.testing.assert_array_equal(labels, alone[i])
            assert run > 0 and queued >= 0


def test_server_footprint_budget_still_completes(gp, ctx):
    """With a budget smaller than any request, requests run one at a time
    (an idle server always admits the next one) and all complete."""
    jobs = mixed_graphs(gp)[:4]
    alone = [ctx.partition(g, k, eps, seed)[0] for g, k, eps, seed in jobs]
    with gp.Server(0, workers=3, hbm_budget_bytes=1) as server:
        tickets = [server.submit(g, k, eps, seed) for g, k, eps, seed in jobs]
        for t, expect in zip(tickets, alone):
            labels, _, _, _ = server.wait(t, timeout=300.0)
            np.testing.assert_array_equal(labels, expect)


def test_batch_mixed_part_counts_equal_single_calls(gp, ctx):
    """Concurrent workers launch the same kernels with different shared-memory
    sizes (the part-matching table grows with k, the large-row tables with
    the row class, the exchange's one-block move sort with the number of
    moves); every result must still equal the graph partitioned alone."""
    jobs = []
    for i in range(48):
        k = (8, 128, 32, 64, 16, 4)[i % 6]
        g = gp.rmat(12 + i % 4, 12, 0.57, 0.19, 0.19, 100 + i) if i % 2 else gp.grid2d(90 + 3 * i, 70)
        jobs.append((g, k, 1.03, i % 5))
    alone = [ctx.partition(g, k, eps, seed)[0] for g, k, eps, seed in jobs]
    for labels_batched, expect in zip(ctx.partition_batch(jobs, concurrency=16), alone):
        np.testing.assert_array_equal(labels_batched[0], expect)


def test_batch_over_devices_equals_single_calls(gp, ctx):
    """gp_partition_batch_devices places the graphs over the listed devices
    by longest processing time.  One GPU is listed twice here (two workers'
    pools on it), so the placement, the per-device queues and the gather run
    as they would on two GPUs; every result equals the graph alone."""
    jobs = mixed_graphs(gp)
    alone = [ctx.partition(g, k, eps, seed)[0] for g, k, eps, seed in jobs]
    out = ctx.partition_batch(jobs, concurrency=3, devices=[0, 0])
    for (labels, st, run_s), expect in zip(out, alone):
        np.testing.assert_array_equal(labels, expect)


def test_server_over_devices_and_measured_footprint(gp, ctx):
    """A server over a device list (the one GPU twice) gives the same labels
    as single calls, and after a resident graph has run its admission
    estimate comes from the measured device peak of that request."""
    jobs = mixed_graphs(gp)
    alone = [ctx.partition(g, k, eps, seed)[0] for g, k, eps, seed in jobs]
    with gp.Server([0, 0], workers=2, hbm_budget_bytes=64 << 30) as server:
        gid = server.add_graph(jobs[3][0])
        static = server.footprint(gid, 128)
        tickets = [server.submit(gid if i == 3 else g, k, eps, seed) for i, (g, k, eps, seed) in enumerate(jobs)]
        peaks = {}
        for i, t in enumerate(tickets):
            labels, st, _, _ = server.wait(t)
            np.testing.assert_array_equal(labels, alone[i])
            peaks[i] = st.device_peak_bytes
        g = jobs[3][0]
        measured = server.footprint(gid, 128)
        assert peaks[3] > 0 and measured != static
        used, cache = peaks[3] + 4 * g.n, 4 * g.n * 128
        base = used - cache if used > cache else used
        expected = base + cache + 4 * g.n
        assert measured == expected + expected // 8


def test_server_keeps_hierarchies(gp, ctx):
    """With kept hierarchies, a request that repeats a resident graph's
    (k, seed) skips coarsening and still returns exactly the labels of the
    request alone, whatever its epsilon; a different k or seed coarsens anew.
    The unit-weight grid checks that the vertex weights the first request
    materialised live with the kept hierarchy.  A one-byte budget keeps
    nothing once the request that made a hierarchy is done."""
    weighted = gp.with_weights(gp.rmat(15, 12, 0.57, 0.19, 0.19, 21), 3, (1, 8), (1, 20))
    grid = gp.grid2d(200, 150)
    plan = [(weighted, 32, 1.03, 5), (weighted, 32, 1.05, 5), (weighted, 32, 1.03, 5), (weighted, 16, 1.03, 5),
            (weighted, 32, 1.03, 6), (grid, 8, 1.03, 0), (grid, 8, 1.01, 0)]
    expect_reused = [0, 1, 1, 0, 0, 0, 1]
    alone = [ctx.partition(g, k, eps, seed)[0] for g, k, eps, seed in plan]
    with gp.Server(0, workers=2) as server:
        server.keep_hierarchies(8 << 30)
        ids = {id(weighted): server.add_graph(weighted), id(grid): server.add_graph(grid)}
        for (g, k, eps, seed), expect, reused in zip(plan, alone, expect_reused):
            labels, st, _, _ = server.wait(server.submit(ids[id(g)], k, eps, seed))
            np.testing.assert_array_equal(labels, expect)
            assert st.hierarchy_reused == reused
        assert server.kept_bytes() > 0
    with gp.Server(0, workers=1) as server:
        server.keep_hierarchies(1)
        gid = server.add_graph(weighted)
        for eps in (1.03, 1.05):
            labels, st, _, _ = server.wait(server.submit(gid, 32, eps, 5))
            assert st.hierarchy_reused == 0
        assert server.kept_bytes() == 0
