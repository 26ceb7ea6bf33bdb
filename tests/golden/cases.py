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
}


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
