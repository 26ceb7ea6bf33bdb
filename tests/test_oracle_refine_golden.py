"""The CPU oracle's single-level refinement against the reference's own
refinement (its run_incremental_refinement, driven through the resident
refine_hierarchy_device on a one-level hierarchy) run on a B200 on the same
graph and start labels (tests/golden/refine_cases.json, made by
tests/golden/make_golden.py --refine)."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, assert_refine_parity, reference_repaired

RECORDS = json.load(open(os.path.join(GOLDEN, "refine_cases.json"))) if os.path.exists(
    os.path.join(GOLDEN, "refine_cases.json")) else {}


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
def test_oracle_refine_matches_reference(name, gp, oracle, graphs):
    from cases import refine_start
    record = RECORDS[name]
    spec = record["spec"]
    g = graphs(spec["graph"])
    start = refine_start(gp, oracle, spec, g)
    assert hashlib.sha256(start.tobytes()).hexdigest() == record["start"], "start labelling changed"
    labels, stats = oracle.refine(g, start, spec["k"], spec["eps"], spec["rounds"], spec["exchange"])
    w = np.ones(g.n, np.uint64) if g.vertex_weights is None else g.vertex_weights.astype(np.uint64)
    loads = np.bincount(labels, weights=w, minlength=spec["k"]).astype(np.uint64)
    assert_refine_parity(name, record, labels, stats, gp.edge_cut(g, labels), loads)


def test_refine_goldens_cover_the_kernels():
    """Bit-exact cases exist for propagation, the priority filter and the
    exchange, at k = 8 and k = 128, above and below 65,536 vertices."""
    assert RECORDS and all("stats" in r for r in RECORDS.values()), "reference runs missing or failed"
    exact = {n: r for n, r in RECORDS.items() if not reference_repaired(r)}
    assert any(r["stats"]["group_accepted"] > 0 for r in exact.values()), "no exact exchange case"
    assert any(r["spec"]["k"] == 8 for r in exact.values())
    assert any(r["spec"]["k"] == 128 for r in exact.values())
    assert any(r["spec"]["graph"] in ("g512_k16", "mesh48_k64") for r in exact.values())
    first = [r for r in RECORDS.values() if r["spec"]["rounds"] == 1 and r["spec"]["graph"].startswith("rmat")]
    assert first, "no R-MAT first-round case"
