"""Host-side utilities of the C ABI (no GPU): generators, the int64 on-disk
CSR format, capacity arithmetic and the independent verifier."""
import os
import subprocess

import numpy as np
import pytest


def test_grid_sizes_and_symmetry(gp):
    g = gp.grid2d(256, 256)
    assert (g.n, g.m) == (65536, 261120)  # the G2 configuration
    assert gp.verify(g, np.zeros(g.n, np.int32) + (np.arange(g.n) % 2), 2, 1.03, check_symmetry=True)["cut"] > 0


def test_mesh_weights_symmetric_and_in_range(gp):
    g = gp.mesh3d(6, 5, 4, weighted=True, seed=3)
    assert g.n == 120
    assert g.vertex_weights.min() >= 1 and g.vertex_weights.max() <= 4
    assert g.edge_weights.min() >= 1 and g.edge_weights.max() <= 16
    gp.verify(g, np.arange(g.n) % 4, 4, 1.5, check_symmetry=True)  # raises on asymmetric weights


def test_rmat_deterministic_sorted_unique_no_loops(gp):
    a = gp.rmat(12, 16, 0.57, 0.19, 0.19, 7)
    b = gp.rmat(12, 16, 0.57, 0.19, 0.19, 7)
    np.testing.assert_array_equal(a.offsets, b.offsets)
    np.testing.assert_array_equal(a.neighbors, b.neighbors)
    rows = np.repeat(np.arange(a.n), np.diff(a.offsets))
    assert not np.any(rows == a.neighbors)
    for v in range(0, a.n, 97):
        seg = a.neighbors[a.offsets[v]:a.offsets[v + 1]]
        assert np.all(np.diff(seg) > 0)
    gp.verify(a, np.zeros(a.n, np.int32), 2, 2.0, check_symmetry=True)
    c = gp.rmat(12, 16, 0.57, 0.19, 0.19, 8)
    assert not np.array_equal(a.neighbors[:1000], c.neighbors[:1000])


@pytest.mark.parametrize("total,k,eps", [(65536, 8, 1.03), (4194304, 64, 1.03), (1001, 7, 1.0), (123457, 128, 1.05)])
def test_partition_capacity_formula(gp, total, k, eps):
    import math
    cap = gp.partition_capacity(total, k, eps)
    assert cap == math.floor(total * eps / k) or abs(cap - total * eps / k) < 1
    assert cap * k >= total


def test_partition_capacity_infeasible(gp):
    with pytest.raises(gp.GpartError) as e:
        gp.partition_capacity(10, 3, 1.0)  # floor(10/3)=3 cannot hold 10 in 3 parts
    assert e.value.status == 2
    with pytest.raises(gp.GpartError):
        gp.partition_capacity(100, 1, 1.03)
    with pytest.raises(gp.GpartError):
        gp.partition_capacity(100, 129, 1.03)


def test_int64_csr_round_trip_and_validation(gp, tmp_path):
    g = gp.rmat(10, 8, 0.57, 0.19, 0.19, 1)
    ip, ix = str(tmp_path / "a.indptr"), str(tmp_path / "a.indices")
    gp.write_csr_int64(g, ip, ix)
    assert os.path.getsize(ip) == 8 * (g.n + 1) and os.path.getsize(ix) == 8 * g.m
    h = gp.read_csr_int64(ip, ix)
    np.testing.assert_array_equal(g.offsets, h.offsets)
    np.testing.assert_array_equal(g.neighbors, h.neighbors)
    bad = np.fromfile(ix, dtype=np.int64)
    bad[3] = g.n  # neighbour out of range
    bad.tofile(ix)
    with pytest.raises(gp.GpartError, match="invalid neighbor"):
        gp.read_csr_int64(ip, ix)
    off = np.fromfile(ip, dtype=np.int64)
    off[5], off[6] = off[6], off[5] - 1  # non-monotone
    off.tofile(ip)
    with pytest.raises(gp.GpartError):
        gp.read_csr_int64(ip, ix)


def test_verifier_matches_numpy(gp):
    g = gp.with_weights(gp.mesh3d(8, 8, 8), 5, (1, 4), (1, 9))
    rng = np.random.default_rng(0)
    labels = rng.integers(0, 8, g.n).astype(np.int32)
    out = gp.verify(g, labels, 8, 1.2)
    rows = np.repeat(np.arange(g.n), np.diff(g.offsets))
    cut = int(g.edge_weights[labels[rows] != labels[g.neighbors]].sum()) // 2
    loads = np.bincount(labels, weights=g.vertex_weights, minlength=8)
    assert out["cut"] == cut == gp.edge_cut(g, labels)
    assert out["loads"] == [int(x) for x in loads]
    assert out["capacity"] == gp.partition_capacity(int(g.vertex_weights.sum()), 8, 1.2)


def test_verifier_cli_reference_contract(gp, tmp_path):
    """gpart_verify_csr: JSON line, exit 0 / 1 (capacity) / 2 (error),
    capacity n*103/(100k) with unit loads (tools/verify_csr.cpp:97-109)."""
    import json
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "acc-gp_b200", "bin", "gpart_verify_csr")
    if not os.path.exists(exe):
        pytest.skip("CLI not built")
    g = gp.grid2d(10, 10)
    ip, ix, part = str(tmp_path / "g.indptr"), str(tmp_path / "g.indices"), str(tmp_path / "g.part")
    gp.write_csr_int64(g, ip, ix)
    (np.arange(100) // 50).astype(np.int32).tofile(part)
    r = subprocess.run([exe, ip, ix, "2", part, "binary", "--symmetric"], capture_output=True, text=True)
    assert r.returncode == 0
    out = json.loads(r.stdout)
    assert out["cut"] == 10 and out["capacity"] == 100 * 103 // 200 and out["capacity_ok"]
    (np.zeros(100)).astype(np.int32).tofile(part)
    r = subprocess.run([exe, ip, ix, "2", part, "binary"], capture_output=True, text=True)
    assert r.returncode == 1 and json.loads(r.stdout)["capacity_ok"] is False
    r = subprocess.run([exe, ip, ix, "200", part, "binary"], capture_output=True, text=True)
    assert r.returncode == 2


def test_partition_cli_usage_errors():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "acc-gp_b200", "bin", "gpart_partition_standard")
    if not os.path.exists(exe):
        pytest.skip("CLI not built")
    r = subprocess.run([exe, "a"], capture_output=True, text=True)
    assert r.returncode == 2 and "Usage" in r.stderr
    env = dict(os.environ, GPART_REFINE_MODE="x")
    r = subprocess.run([exe, "a", "b", "4", "c"], capture_output=True, text=True, env=env)
    assert r.returncode == 1 and r.stderr.startswith("gpart_partition:")


def test_write_hierarchy_layout(gp, tmp_path):
    """write_hierarchy's int32 layout (include/hierarchy.hpp:38-123): level
    count, then n, m, offsets, neighbors, edge weights, vertex weights and the
    previous level's map; unit weights are written as ones."""
    fine = gp.grid2d(4, 4)
    mp = (np.arange(16) // 2).astype(np.int32)  # pairs along rows
    coarse = gp.Graph(np.arange(9, dtype=np.int32), np.array([1, 0, 3, 2, 5, 4, 7, 6], np.int32),
                      vertex_weights=np.full(8, 2, np.uint32), edge_weights=np.arange(1, 9, dtype=np.uint32))
    path = tmp_path / "h.bin"
    gp.write_hierarchy([(fine, mp), (coarse, None)], path)
    assert not (tmp_path / "h.bin.tmp").exists()
    raw = np.fromfile(path, np.int32)
    expected = np.concatenate([[2, fine.n, fine.m], fine.offsets, fine.neighbors, np.ones(fine.m), np.ones(fine.n),
                               [coarse.n, coarse.m], coarse.offsets, coarse.neighbors, coarse.edge_weights,
                               coarse.vertex_weights, mp]).astype(np.int32)
    np.testing.assert_array_equal(raw, expected)
    levels = gp.read_hierarchy(path)
    assert len(levels) == 2
    np.testing.assert_array_equal(levels[1]["map_from_previous"], mp)
    np.testing.assert_array_equal(levels[1]["edge_weights"], coarse.edge_weights)


@pytest.mark.parametrize("defect, message", [
    ("map", "hierarchy map contains an invalid coarse id"),
    ("edge_weight", "hierarchy edge weight exceeds int32"),
    ("vertex_weight", "hierarchy vertex weight exceeds int32"),
    ("missing_map", "cannot write an incomplete hierarchy"),
])
def test_write_hierarchy_rejects_like_the_reference(gp, tmp_path, defect, message):
    fine = gp.grid2d(3, 3)
    mp = np.zeros(9, np.int32)
    coarse = gp.Graph(np.zeros(2, np.int32), np.zeros(0, np.int32))
    if defect == "map":
        mp[4] = 1  # the coarse level has one vertex
    if defect == "edge_weight":
        fine = gp.Graph(fine.offsets, fine.neighbors, edge_weights=np.full(fine.m, 1 << 31, np.uint32))
    if defect == "vertex_weight":
        fine = gp.Graph(fine.offsets, fine.neighbors, vertex_weights=np.full(fine.n, 1 << 31, np.uint32))
    levels = [(fine, None if defect == "missing_map" else mp), (coarse, None)]
    path = tmp_path / "h.bin"
    with pytest.raises(gp.GpartError) as e:
        gp.write_hierarchy(levels, path)
    assert message in str(e.value)
    assert not path.exists() and not (tmp_path / "h.bin.tmp").exists()
