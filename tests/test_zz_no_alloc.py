"""The allocation-free evaluation entry point, gp_evaluate_device_static.

It exists for callers that cannot let the library allocate device memory (a
framework allocator that owns the memory budget, a serving loop that must not
call cudaMalloc/cudaFree).  Its scratch is a fixed device array shared by all
calls, so this test calls it twice in a row with different labels and checks
both results against the allocating gp_evaluate_device, exactly (integer
cut and loads).  The file sorts last so a failure here comes after every
other test has run; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_scratch_entry_matches_allocating_entry(gp):
    import torch
    g = gp.with_weights(gp.rmat(16, 16, 0.57, 0.19, 0.19, 11), 3, (1, 9), (1, 20))
    k = 96
    dev = {name: torch.from_numpy(a).cuda() for name, a in
           (("off", g.offsets), ("nbr", g.neighbors), ("vw", g.vertex_weights), ("ew", g.edge_weights))}
    stream = torch.cuda.current_stream()
    with gp.Context(0) as ctx:
        for call in range(2):
            labels = torch.from_numpy(((np.arange(g.n) * (7919 + call * 104729)) % k).astype(np.int32)).cuda()
            cut_a = torch.zeros(1, dtype=torch.int64, device="cuda")
            loads_a = torch.zeros(k, dtype=torch.int64, device="cuda")
            cut_b = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            loads_b = torch.full((k,), -1, dtype=torch.int64, device="cuda")
            ptrs = (dev["off"].data_ptr(), dev["nbr"].data_ptr(), g.n, g.m, dev["vw"].data_ptr(), dev["ew"].data_ptr(),
                    labels.data_ptr(), k)
            ctx.evaluate_device(*ptrs, cut_a.data_ptr(), loads_a.data_ptr(), stream.cuda_stream)
            gp.evaluate_device_static(*ptrs, cut_b.data_ptr(), loads_b.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
            assert int(cut_b.item()) == int(cut_a.item()) > 0
            np.testing.assert_array_equal(loads_b.cpu().numpy(), loads_a.cpu().numpy())
            assert int(loads_b.sum().item()) == int(g.vertex_weights.sum())
            # And against the host verifier, which shares no code with either.
            verdict = gp.verify(g, labels.cpu().numpy(), k, 2.0)
            assert int(cut_b.item()) == verdict["cut"]
            assert [int(x) for x in loads_b.cpu().numpy()] == verdict["loads"]


def test_out_of_range_labels_are_skipped_not_dereferenced(gp):
    """A label outside [0,k) is never used as an index: the allocating entry
    returns GP_INVALID_ARGUMENT, the static entry (which does not wait for
    its results) writes UINT64_MAX as the cut, and both stay usable."""
    import torch
    g = gp.grid2d(40, 30)
    k = 6
    off = torch.from_numpy(g.offsets).cuda()
    nbr = torch.from_numpy(g.neighbors).cuda()
    good = (np.arange(g.n) % k).astype(np.int32)
    bad = good.copy()
    bad[[3, 500, 1199]] = [k, -1, 1 << 20]
    cut = torch.zeros(1, dtype=torch.int64, device="cuda")
    loads = torch.zeros(k, dtype=torch.int64, device="cuda")
    with gp.Context(0) as ctx:
        for labels, ok in ((bad, False), (good, True)):
            d = torch.from_numpy(labels).cuda()
            ptrs = (off.data_ptr(), nbr.data_ptr(), g.n, g.m, None, None, d.data_ptr(), k)
            gp.evaluate_device_static(*ptrs, cut.data_ptr(), loads.data_ptr())
            torch.cuda.synchronize()
            if ok:
                assert int(cut.item()) == gp.verify(g, labels, k, 2.0)["cut"]
            else:
                assert int(cut.item()) == -1  # UINT64_MAX read as int64
                with pytest.raises(gp.GpartError) as e:
                    ctx.evaluate_device(*ptrs, cut.data_ptr(), loads.data_ptr())
                assert e.value.status == 1 and "out of range" in e.value.message


def test_static_scratch_entry_rejects_k_beyond_capacity(gp):
    import torch
    g = gp.grid2d(8, 8)
    off = torch.from_numpy(g.offsets).cuda()
    nbr = torch.from_numpy(g.neighbors).cuda()
    labels = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    out = torch.zeros(256, dtype=torch.int64, device="cuda")
    with pytest.raises(gp.GpartError) as e:
        gp.evaluate_device_static(off.data_ptr(), nbr.data_ptr(), g.n, g.m, None, None, labels.data_ptr(), 129,
                                  out.data_ptr(), out[1:].data_ptr())
    assert e.value.status == 1 and "k must be" in e.value.message
