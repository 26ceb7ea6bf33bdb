"""gp_refine (the reference's refine_partition, include/refine.hpp:84-88) on
the GPU, through the C ABI: identical to the CPU oracle on every case (labels
and every move statistic, capacity repair included, since both order repair
deterministically), and compared with the reference's own refine_partition
(tests/golden/refine_cases.json) wherever the reference is reproducible."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, assert_refine_parity

pytestmark = pytest.mark.gpu

RECORDS = json.load(open(os.path.join(GOLDEN, "refine_cases.json"))) if os.path.exists(
    os.path.join(GOLDEN, "refine_cases.json")) else {}
ORACLE_FIELDS = ("rounds", "admission_iterations", "checkpoint_updates", "proposals", "accepted", "initial_cut",
                 "final_cut", "final_max_part_weight", "capacity", "lp_cut_gain", "lp_cut_loss",
                 "rebalance_cut_gain", "rebalance_cut_loss", "group_cut_gain", "group_accepted")


@pytest.fixture(scope="module")
def graphs(gp, cases):
    CASES, build = cases
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = build(gp, CASES[name])
        return cache[name]
    return get


@pytest.mark.parametrize("name", sorted(RECORDS))
def test_gpu_refine_matches_oracle_and_reference(name, gp, ctx, oracle, graphs):
    from cases import refine_start
    record = RECORDS[name]
    spec = record["spec"]
    g = graphs(spec["graph"])
    start = refine_start(gp, oracle, spec, g)
    labels, stats = ctx.refine(g, start, spec["k"], spec["eps"], spec["rounds"], spec["exchange"])
    expected, ostats = oracle.refine(g, start, spec["k"], spec["eps"], spec["rounds"], spec["exchange"])
    np.testing.assert_array_equal(labels, expected, err_msg=name)
    for key in ORACLE_FIELDS:
        assert stats[key] == ostats[key], f"{name}: {key} {stats[key]} != oracle {ostats[key]}"
    verdict = gp.verify(g, labels, spec["k"], spec["eps"])
    assert verdict["cut"] == stats["final_cut"]
    assert verdict["capacity_ok"]
    assert_refine_parity(name, record, labels, stats, verdict["cut"], np.array(verdict["loads"], np.uint64))


def test_gpu_refine_verify_mode(gp, ctx, oracle, graphs):
    """GP_FLAG_VERIFY checks the incremental cut and cache after every batch."""
    from cases import CASES, swapped_start
    g = graphs("rmat14_k16")
    start = swapped_start(g, 16, 0.08)
    a, _ = ctx.refine(g, start, 16, 1.10, 32, 2, gp.FLAG_QUIET | gp.FLAG_VERIFY)
    b, _ = ctx.refine(g, start, 16, 1.10, 32, 2)
    np.testing.assert_array_equal(a, b)


def test_gpu_refine_rejects(gp, ctx, graphs):
    g = graphs("g2_k8")
    bad = np.zeros(g.n, np.int32)
    bad[5] = 8
    with pytest.raises(gp.GpartError, match="invalid part id"):
        ctx.refine(g, bad, 8, 1.03)
    with pytest.raises(gp.GpartError, match="invalid refinement options"):
        ctx.refine(g, np.zeros(g.n, np.int32), 8, 1.03, max_rounds=65)
    with pytest.raises(gp.GpartError, match="imbalanced") as e:
        ctx.refine(g, np.zeros(g.n, np.int32), 8, 1.03, flags=gp.FLAG_QUIET | gp.FLAG_REQUIRE_BALANCED)
    assert e.value.status == 1
