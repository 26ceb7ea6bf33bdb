"""Seeded parity cases shared by make_golden.py and the tests.

Each case names a generator and its parameters, so the same input graph is
rebuilt bit-for-bit wherever the fixture is checked.
"""
from __future__ import annotations

import numpy as np

CASES = {
    # 256x256 5-point grid, k=8 (the G2 configuration).
    "g2_k8": dict(kind="grid2d", width=256, height=256, k=8, eps=1.03, seed=0),
    # 512x512 grid: n >= 65536, degree <= 4, so seed matching runs.
    "g512_k16": dict(kind="grid2d", width=512, height=512, k=16, eps=1.03, seed=3),
    "rmat14_k16": dict(kind="rmat", scale=14, ef=16, gseed=0, k=16, eps=1.03, seed=0),
    "rmat16_k64": dict(kind="rmat", scale=16, ef=16, gseed=0, k=64, eps=1.03, seed=0),
    "rmat18_k64": dict(kind="rmat", scale=18, ef=16, gseed=1, k=64, eps=1.03, seed=1),
    "mesh16w_k32": dict(kind="mesh3d", x=16, y=16, z=16, weighted=True, gseed=0, k=32, eps=1.03, seed=0),
    "mesh48_k64": dict(kind="mesh3d", x=48, y=48, z=48, weighted=False, gseed=0, k=64, eps=1.05, seed=2),
    "mesh32w_k128": dict(kind="mesh3d", x=32, y=32, z=32, weighted=True, gseed=5, k=128, eps=1.01, seed=7),
    # Self loops, parallel edges, unsorted rows, isolated vertices, weights.
    "odd_k4": dict(kind="odd", scale=11, ef=8, gseed=4, k=4, eps=1.03, seed=11),
    "odd_k32": dict(kind="odd", scale=13, ef=6, gseed=9, k=32, eps=1.05, seed=5),
    # The headline configurations (hierarchy digests only; GPU tests).
    "rmat22_k64": dict(kind="rmat", scale=22, ef=16, gseed=0, k=64, eps=1.03, seed=0, headline=True),
    "m3_k128": dict(kind="mesh3d", x=256, y=256, z=256, weighted=True, gseed=0, k=128, eps=1.03, seed=0,
                    headline=True),
}


# Single-level refinement cases: a graph case, a start labelling, and the
# round budgets of refine_partition.  "projected": the oracle pipeline's
# refined level-1 labels projected onto level 0 (the input the pipeline's
# last refinement sees); "swapped": balanced blocks of vertex ids in which a
# fraction of equal-weight vertex pairs swap labels, so every part keeps its
# load exactly and label propagation has moves to make.
REFINE_CASES = {}
for _name in ("g2_k8", "g512_k16", "rmat14_k16", "rmat16_k64", "rmat18_k64", "mesh16w_k32", "mesh48_k64",
              "mesh32w_k128", "odd_k32"):
    _k = CASES[_name]["k"]
    REFINE_CASES[f"{_name}_projected"] = dict(graph=_name, start="projected", k=_k, eps=CASES[_name]["eps"],
                                              rounds=32, exchange=2)
    REFINE_CASES[f"{_name}_swap_round"] = dict(graph=_name, start="swapped", frac=0.08, k=_k, eps=1.10,
                                               rounds=1, exchange=0)
    REFINE_CASES[f"{_name}_swap_round_x"] = dict(graph=_name, start="swapped", frac=0.08, k=_k, eps=1.10,
                                                 rounds=1, exchange=2)
    REFINE_CASES[f"{_name}_swap"] = dict(graph=_name, start="swapped", frac=0.08, k=_k, eps=1.10,
                                         rounds=32, exchange=2)
    REFINE_CASES[f"{_name}_swap_tight"] = dict(graph=_name, start="swapped", frac=0.03, k=_k, eps=1.03,
                                               rounds=32, exchange=2)


def swapped_start(graph, k, frac, seed=0):
    """Balanced blocks by vertex-weight prefix, then a seeded fraction of
    vertices paired up inside each weight class and their labels swapped."""
    w = np.ones(graph.n, np.int64) if graph.vertex_weights is None else graph.vertex_weights.astype(np.int64)
    total = int(w.sum())
    prefix = np.cumsum(w) - w
    labels = (prefix * k // total).astype(np.int32)
    rng = np.random.default_rng(seed + 12345)
    for value in np.unique(w):
        members = np.flatnonzero(w == value)
        pick = members[rng.random(members.shape[0]) < frac]
        rng.shuffle(pick)
        half = pick.shape[0] // 2
        a, b = pick[:half], pick[half:2 * half]
        labels[a], labels[b] = labels[b].copy(), labels[a].copy()
    return labels


def refine_start(gp, oracle, spec, graph):
    """The start labelling of a refinement case (numpy int32, length n)."""
    if spec["start"] == "swapped":
        return swapped_start(graph, spec["k"], spec["frac"])
    base = CASES[spec["graph"]]
    oracle.partition(graph, base["k"], base["eps"], base["seed"])
    levels = oracle.levels()
    coarse = oracle.level_labels(1, levels[1]["n"])
    return coarse[levels[0]["map"]].astype(np.int32)


def _odd_graph(gp, spec):
    base = gp.rmat(spec["scale"], spec["ef"], 0.57, 0.19, 0.19, spec["gseed"])
    n0 = base.n
    rows = np.repeat(np.arange(n0, dtype=np.int64), np.diff(base.offsets))
    cols = base.neighbors.astype(np.int64)
    upper = rows < cols
    u, v = rows[upper], cols[upper]
    dup = ((u + v) % 11) == 0
    u = np.concatenate([u, u[dup]])
    v = np.concatenate([v, v[dup]])
    loops = np.arange(0, n0, 17, dtype=np.int64)
    isolated = 37
    n = n0 + isolated
    src = np.concatenate([u, v, loops])
    dst = np.concatenate([v, u, loops])
    rng = np.random.default_rng(spec["gseed"] + 1000)
    order = np.lexsort((rng.random(src.shape[0]), src))  # rows grouped, shuffled inside
    src, dst = src[order], dst[order]
    offsets = np.zeros(n + 1, np.int64)
    np.add.at(offsets, src + 1, 1)
    offsets = np.cumsum(offsets)
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    ew = (1 + (lo * 7919 + hi * 104729 + spec["gseed"]) % 5).astype(np.uint32)
    vw = (1 + (np.arange(n) * 2654435761 + spec["gseed"]) % 9).astype(np.uint32)
    return gp.Graph(offsets.astype(np.int32), dst.astype(np.int32), vw, ew)


def build_case(gp, spec):
    kind = spec["kind"]
    if kind == "grid2d":
        return gp.grid2d(spec["width"], spec["height"])
    if kind == "rmat":
        return gp.rmat(spec["scale"], spec["ef"], 0.57, 0.19, 0.19, spec["gseed"])
    if kind == "mesh3d":
        return gp.mesh3d(spec["x"], spec["y"], spec["z"], spec["weighted"], spec["gseed"])
    if kind == "odd":
        return _odd_graph(gp, spec)
    raise ValueError(kind)
