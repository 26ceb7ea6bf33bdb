"""GPU parity: the CUDA path against the reference's golden vectors (every
level of the hierarchy, METIS labels) and against the CPU oracle (final
labels identical in the deterministic mode), through the C ABI."""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

CASE_NAMES = ["g2_k8", "g512_k16", "rmat14_k16", "rmat16_k64", "rmat18_k64", "mesh16w_k32", "mesh48_k64",
              "mesh32w_k128", "odd_k32"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", CASE_NAMES)
def test_hierarchy_bit_exact_with_reference(name, gp, ctx, cases):
    CASES, build = cases
    spec, fx = CASES[name], golden(name)
    g = build(gp, spec)
    labels, st = ctx.partition(g, spec["k"], spec["eps"], spec["seed"], gp.FLAG_QUIET | gp.FLAG_KEEP_HIERARCHY)
    levels = ctx.levels()
    assert len(levels) == len(fx["levels"]) == st.levels
    for i, (a, b) in enumerate(zip(levels, fx["levels"])):
        assert (a["offsets"].shape[0] - 1, a["neighbors"].shape[0]) == (b["n"], b["m"]), f"level {i}"
        for key in ("maximum_degree", "has_heavy_rows", "incident_weight_bound"):
            assert a[key] == b[key], f"level {i} {key}"
        for key in ("offsets", "neighbors", "edge_weights", "vertex_weights", "map"):
            if b[key] is None:
                assert a[key] is None
            else:
                assert digest(a[key]) == b[key], f"level {i} {key}"
    assert digest(ctx.initial_labels(fx["coarsest_n"])) == fx["metis_labels"]


@pytest.mark.parametrize("name", CASE_NAMES)
def test_labels_identical_to_oracle(name, gp, ctx, oracle, cases):
    CASES, build = cases
    spec, fx = CASES[name], golden(name)
    g = build(gp, spec)
    labels, st = ctx.partition(g, spec["k"], spec["eps"], spec["seed"])
    expected, cut = oracle.partition(g, spec["k"], spec["eps"], spec["seed"])
    np.testing.assert_array_equal(labels, expected)
    verdict = gp.verify(g, labels, spec["k"], spec["eps"])
    assert st.edge_cut == cut == verdict["cut"]
    assert verdict["capacity_ok"] and st.max_part_weight == verdict["max_load"]


def test_cut_geomean_within_one_percent_of_reference(gp, ctx, cases):
    """The partition quality bar: over every golden case the geometric mean of
    (our cut / the reference build's cut) is at most 1.01, and no case breaks
    the capacity floor(total * eps / k)."""
    CASES, build = cases
    ratios = []
    for name in CASE_NAMES:
        spec, fx = CASES[name], golden(name)
        g = build(gp, spec)
        labels, st = ctx.partition(g, spec["k"], spec["eps"], spec["seed"])
        assert gp.verify(g, labels, spec["k"], spec["eps"])["capacity_ok"], name
        ratios.append(st.edge_cut / fx["reference_final_cut"])
    geomean = float(np.exp(np.mean(np.log(ratios))))
    assert geomean <= 1.01, (geomean, ratios)


HEADLINE = [name for name in ("rmat22_k64", "m3_k128")
            if os.path.exists(os.path.join(GOLDEN, f"{name}.json"))]


@pytest.mark.parametrize("name", HEADLINE)
def test_headline_hierarchy_bit_exact_with_reference(name, gp, ctx, cases):
    """R-MAT scale 22 at k=64 and the 256^3 weighted mesh at k=128: every
    level's CSR, weights, map and metadata, and the METIS labels, equal the
    reference build's (SHA-256 digests); the cut is within 1% of the
    reference run's and the capacity holds; the final labels and cut equal
    the serial oracle's (digest recorded by make_golden.py --oracle-labels)."""
    CASES, build = cases
    spec, fx = CASES[name], golden(name)
    g = build(gp, spec)
    labels, st = ctx.partition(g, spec["k"], spec["eps"], spec["seed"], gp.FLAG_QUIET | gp.FLAG_KEEP_HIERARCHY)
    levels = ctx.levels()
    assert len(levels) == len(fx["levels"]) == st.levels
    for i, (a, b) in enumerate(zip(levels, fx["levels"])):
        assert (a["offsets"].shape[0] - 1, a["neighbors"].shape[0]) == (b["n"], b["m"]), f"level {i}"
        for key in ("maximum_degree", "has_heavy_rows", "incident_weight_bound"):
            assert a[key] == b[key], f"level {i} {key}"
        for key in ("offsets", "neighbors", "edge_weights", "vertex_weights", "map"):
            if b[key] is None:
                assert a[key] is None
            else:
                assert digest(a[key]) == b[key], f"level {i} {key}"
    assert digest(ctx.initial_labels(fx["coarsest_n"])) == fx["metis_labels"]
    verdict = gp.verify(g, labels, spec["k"], spec["eps"])
    assert verdict["capacity_ok"] and verdict["cut"] == st.edge_cut
    assert st.edge_cut <= 1.01 * fx["reference_final_cut"]
    if "oracle_final_labels" in fx:
        assert st.edge_cut == fx["oracle_final_cut"]
        assert digest(labels) == fx["oracle_final_labels"]


def test_reference_failure_reproduced(gp, ctx, cases):
    CASES, build = cases
    g = build(gp, CASES["odd_k4"])
    with pytest.raises(gp.GpartError, match="odd directed edge weight") as e:
        ctx.partition(g, 4, 1.03, 11)
    assert e.value.status == 5
