"""GPU edge cases and size-independent properties: tiny and disconnected
graphs, k at both ends, exact balance, invalid inputs, the device-pointer
entry point, determinism, and a large R-MAT checked by the verifier."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def check(gp, g, labels, st, k, eps):
    verdict = gp.verify(g, labels, k, eps)
    assert verdict["capacity_ok"], verdict
    assert verdict["cut"] == st.edge_cut
    assert labels.min() >= 0 and labels.max() < k
    return verdict


@pytest.mark.parametrize("k", [2, 3, 8, 64, 128])
def test_k_range_matches_oracle(gp, ctx, oracle, k):
    g = gp.mesh3d(24, 24, 24)
    labels, st = ctx.partition(g, k, 1.03, 5)
    check(gp, g, labels, st, k, 1.03)
    expected, cut = oracle.partition(g, k, 1.03, 5)
    np.testing.assert_array_equal(labels, expected)


def test_graph_below_cutoff_skips_coarsening(gp, ctx, oracle):
    g = gp.grid2d(12, 12)  # n=144 <= 64*8: METIS on the input, then refinement
    labels, st = ctx.partition(g, 8, 1.03, 0)
    assert st.levels == 1
    check(gp, g, labels, st, 8, 1.03)
    np.testing.assert_array_equal(labels, oracle.partition(g, 8, 1.03, 0)[0])


def test_isolated_vertices_and_components(gp, ctx, oracle):
    base = gp.grid2d(60, 60)
    n = base.n + 500  # 500 isolated vertices
    off = np.concatenate([base.offsets, np.full(500, base.offsets[-1], np.int32)])
    g = gp.Graph(off, base.neighbors)
    labels, st = ctx.partition(g, 4, 1.03, 1)
    check(gp, g, labels, st, 4, 1.03)
    np.testing.assert_array_equal(labels, oracle.partition(g, 4, 1.03, 1)[0])


def test_exact_balance(gp, ctx, oracle):
    g = gp.grid2d(64, 64)
    labels, st = ctx.partition(g, 4, 1.0, 2)
    v = check(gp, g, labels, st, 4, 1.0)
    assert v["max_load"] == 1024
    np.testing.assert_array_equal(labels, oracle.partition(g, 4, 1.0, 2)[0])


def test_weighted_rmat(gp, ctx, oracle):
    g = gp.with_weights(gp.rmat(15, 12, 0.57, 0.19, 0.19, 3), 9, (1, 16), (1, 64))
    labels, st = ctx.partition(g, 50, 1.05, 4)
    check(gp, g, labels, st, 50, 1.05)
    np.testing.assert_array_equal(labels, oracle.partition(g, 50, 1.05, 4)[0])


def test_row_weight_sums_beyond_32_bits(gp, ctx, oracle):
    """Edge weights of 2^20..2^21 on hubs of thousands of entries: row weight
    sums exceed 32 bits, so the coarsening affinity tables keep clusters and
    connections apart instead of packing both into one 64-bit slot.  (Coarse
    edge weights are 32-bit sums of parallel edges, as in the reference, so the
    weights stay small enough for those sums.)"""
    g = gp.with_weights(gp.rmat(16, 16, 0.57, 0.19, 0.19, 6), 13, (1, 8), (1 << 20, 1 << 21))
    degree = np.diff(g.offsets)
    assert int(degree.max()) > 2048  # heavy rows: global tables too
    row_sums = np.add.reduceat(g.edge_weights.astype(np.uint64), g.offsets[:-1][degree > 0])
    assert int(row_sums.max()) >= 1 << 32
    labels, st = ctx.partition(g, 64, 1.03, 2)
    check(gp, g, labels, st, 64, 1.03)
    np.testing.assert_array_equal(labels, oracle.partition(g, 64, 1.03, 2)[0])


@pytest.mark.parametrize("side, k, seed", [(64, 128, 2), (48, 64, 5)])
def test_weighted_mesh_levels_without_cache_match_oracle(gp, ctx, oracle, side, k, seed):
    """Levels above 65,536 vertices whose rows are short next to k keep no
    affinity cache, and their LP proposals visit only the frontier of rows
    that have been boundary rows; capacity repair runs with prices (weighted
    vertices).  The labels must still equal the oracle's full scan."""
    g = gp.mesh3d(side, side, side, weighted=True, seed=1)
    labels, st = ctx.partition(g, k, 1.03, seed)
    check(gp, g, labels, st, k, 1.03)
    np.testing.assert_array_equal(labels, oracle.partition(g, k, 1.03, seed)[0])


def test_fewer_vertices_than_parts_is_rejected(gp, ctx):
    g = gp.grid2d(3, 3)
    with pytest.raises(gp.GpartError) as e:
        ctx.partition(g, 16, 2.0, 0)
    assert e.value.status in (1, 2)


@pytest.mark.parametrize("defect", ["neighbor", "offsets", "zero_weight", "k"])
def test_invalid_inputs_raise(gp, ctx, defect):
    g = gp.grid2d(20, 20)
    off, nbr = g.offsets.copy(), g.neighbors.copy()
    vw = None
    k = 4
    if defect == "neighbor":
        nbr[7] = g.n + 3
    elif defect == "offsets":
        off[10], off[11] = off[11], off[10]
    elif defect == "zero_weight":
        vw = np.ones(g.n, np.uint32)
        vw[5] = 0
    else:
        k = 200
    with pytest.raises(gp.GpartError) as e:
        ctx.partition(gp.Graph(off, nbr, vw), k, 1.03, 0)
    assert e.value.status == 1


def test_device_entry_point_equals_host(gp, ctx):
    import torch
    g = gp.rmat(16, 16, 0.57, 0.19, 0.19, 2)
    host_labels, st = ctx.partition(g, 32, 1.03, 7)
    off = torch.from_numpy(g.offsets).cuda()
    nbr = torch.from_numpy(g.neighbors).cuda()
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    st2 = ctx.partition_device(off.data_ptr(), nbr.data_ptr(), g.n, g.m, None, None, 32, 1.03, 7, out.data_ptr(),
                               stream.cuda_stream)
    np.testing.assert_array_equal(out.cpu().numpy(), host_labels)
    assert st2.edge_cut == st.edge_cut


def test_deterministic_and_independent_of_context(gp, ctx):
    g = gp.rmat(18, 16, 0.57, 0.19, 0.19, 5)
    a, sa = ctx.partition(g, 64, 1.03, 0)
    b, sb = ctx.partition(g, 64, 1.03, 0)
    with gp.Context(0) as other:
        c, sc = other.partition(g, 64, 1.03, 0)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)
    check(gp, g, a, sa, 64, 1.03)


def test_rmat20_properties(gp, ctx):
    """Full-size-class property check: reported cut == independent recount,
    capacity respected, repeatable."""
    g = gp.rmat(20, 16, 0.57, 0.19, 0.19, 0)
    labels, st = ctx.partition(g, 64, 1.03, 0)
    check(gp, g, labels, st, 64, 1.03)
    assert st.levels >= 5 and st.kernel_launches > 0


def test_evaluate_device_matches_verifier(gp, ctx):
    import torch
    g = gp.with_weights(gp.rmat(14, 16, 0.57, 0.19, 0.19, 6), 2, (1, 5), (1, 7))
    k = 37
    labels = (np.arange(g.n) * 7919 % k).astype(np.int32)
    dev = [torch.from_numpy(a).cuda() for a in (g.offsets, g.neighbors, g.vertex_weights, g.edge_weights, labels)]
    cut = torch.zeros(1, dtype=torch.int64, device="cuda")
    loads = torch.zeros(k, dtype=torch.int64, device="cuda")
    ctx.evaluate_device(dev[0].data_ptr(), dev[1].data_ptr(), g.n, g.m, dev[2].data_ptr(), dev[3].data_ptr(),
                        dev[4].data_ptr(), k, cut.data_ptr(), loads.data_ptr())
    verdict = gp.verify(g, labels, k, 2.0)
    assert int(cut.item()) == verdict["cut"]
    assert [int(x) for x in loads.cpu()] == verdict["loads"]


@pytest.mark.parametrize("case", ["rmat", "weighted_mesh"])
def test_verify_flag_checks_pass_and_change_nothing(gp, ctx, case):
    """GP_FLAG_VERIFY (the reference's --verify) runs every strict check and
    leaves the result unchanged."""
    if case == "rmat":
        g, k = gp.rmat(16, 16, 0.57, 0.19, 0.19, 3), 64
    else:
        g, k = gp.with_weights(gp.mesh3d(20, 20, 20), 9, (1, 4), (1, 16)), 32
    plain, sp = ctx.partition(g, k, 1.03, 0)
    checked, sc = ctx.partition(g, k, 1.03, 0, gp.FLAG_QUIET | gp.FLAG_VERIFY)
    np.testing.assert_array_equal(plain, checked)
    assert sc.edge_cut == sp.edge_cut


def test_verify_flag_rejects_one_way_edges(gp, ctx):
    g = gp.grid2d(20, 20)
    off, nbr = g.offsets.copy(), g.neighbors.copy()
    # Redirect one directed entry of vertex 0 to another valid vertex: the
    # reverse entry is missing, which only the strict check detects.
    nbr[off[0]] = 399
    bad = gp.Graph(off, nbr, None)
    with pytest.raises(gp.GpartError) as e:
        ctx.partition(bad, 4, 1.03, 0, gp.FLAG_QUIET | gp.FLAG_VERIFY)
    assert e.value.status == 1 and "bidirectional" in str(e.value)


def test_verify_flag_rejects_unequal_reverse_weights(gp, ctx):
    g = gp.with_weights(gp.grid2d(16, 16), 1, (1, 1), (1, 9))
    ew = g.edge_weights.copy()
    ew[g.offsets[5]] += 1
    bad = gp.Graph(g.offsets, g.neighbors, g.vertex_weights, ew)
    with pytest.raises(gp.GpartError) as e:
        ctx.partition(bad, 4, 1.03, 0, gp.FLAG_QUIET | gp.FLAG_VERIFY)
    assert e.value.status == 1 and "reverse edge weights differ" in str(e.value)


def test_kept_hierarchy_written_like_write_hierarchy(gp, ctx, tmp_path):
    """gp_write_kept_hierarchy writes the levels and maps of the last call
    kept with FLAG_KEEP_HIERARCHY in write_hierarchy's int32 layout."""
    g = gp.with_weights(gp.rmat(14, 8, 0.57, 0.19, 0.19, 2), 3, (1, 4), (1, 9))
    ctx.partition(g, 16, 1.03, 0, gp.FLAG_QUIET | gp.FLAG_KEEP_HIERARCHY)
    kept = ctx.levels()
    assert len(kept) > 2
    path = tmp_path / "hierarchy.bin"
    ctx.write_kept_hierarchy(path)
    written = gp.read_hierarchy(path)
    assert len(written) == len(kept)
    for i, (w, k) in enumerate(zip(written, kept)):
        for name in ("offsets", "neighbors", "edge_weights", "vertex_weights"):
            np.testing.assert_array_equal(w[name], k[name].astype(np.int32), err_msg=f"level {i} {name}")
        if i:
            np.testing.assert_array_equal(w["map_from_previous"], kept[i - 1]["map"])


def test_out_of_memory_request_does_not_fail_the_next(gp):
    """A request whose device allocation fails reports GP_OUT_OF_MEMORY and
    leaves no error behind: the next request on the same context succeeds
    with the same labels as a fresh context.  The failure is a real
    cudaMalloc refusal (a 4 TB arena block), not a fault."""
    g = gp.grid2d(96, 80)
    with gp.Context(0) as fresh:
        expected, _ = fresh.partition(g, 8, 1.03, 0)
    with gp.Context(0) as c:
        c.set_option("arena_chunk_mb", 1 << 22)
        with pytest.raises(gp.GpartError) as e:
            c.partition(g, 8, 1.03, 0)
        assert e.value.status == 3
        c.set_option("arena_chunk_mb", 256)
        labels, st = c.partition(g, 8, 1.03, 0)
    np.testing.assert_array_equal(labels, expected)
