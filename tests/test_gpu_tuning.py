"""Thread-mapping thresholds and the autotuner: a threshold decides which
kernel and how many threads handle a row, never a value, so every setting
must give the same labels."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EXTREMES = {
    "medium_degree": [8, 64, 256],
    "large_narrow": [256, 2048],
    "build_short": [8, 32, 2048],
    "rebuild_divisor": [1, 100000],
    "on_demand_degree": [0, 8, 32],
    "refine_heavy_small": [64, 8192],
    "refine_heavy_mid": [64, 8192],
    "refine_heavy_large": [64, 1024, 8192],
}


@pytest.fixture(scope="module")
def graphs(gp):
    # R-MAT: every coarsening degree class and hubs above 2048 entries;
    # mesh: levels above 65536 vertices with maximum degree 6 < k / 3 (on-demand rows).
    return [(gp.rmat(16, 16, 0.57, 0.19, 0.19, 5), 64), (gp.mesh3d(48, 48, 40), 64)]


@pytest.mark.parametrize("name", sorted(EXTREMES))
def test_mapping_thresholds_do_not_change_labels(gp, graphs, name):
    with gp.Context(0) as base:
        expected = [base.partition(g, k, 1.03, 1)[0] for g, k in graphs]
    for value in EXTREMES[name]:
        with gp.Context(0) as c:
            c.set_option(name, value)
            for (g, k), want in zip(graphs, expected):
                labels, _ = c.partition(g, k, 1.03, 1)
                np.testing.assert_array_equal(labels, want, err_msg=f"{name}={value}")


def test_set_option_rejects_out_of_range(gp, ctx):
    for name, bad in [("medium_degree", 300), ("large_narrow", 4096), ("build_short", 4),
                      ("rebuild_divisor", 0), ("on_demand_degree", 64), ("refine_heavy_large", 32)]:
        with pytest.raises(gp.GpartError):
            ctx.set_option(name, bad)


def test_autotune_keeps_labels_and_reports(gp):
    g = gp.rmat(15, 16, 0.57, 0.19, 0.19, 2)
    with gp.Context(0) as c:
        before, _ = c.partition(g, 64, 1.03, 0)
        t = c.autotune(g, 64, 1.03, 0, repeats=1)
        assert t["medium_degree"] in (64, 128, 256) and t["large_narrow"] in (512, 1024, 2048)
        assert t["build_short"] in (32, 64, 128) and t["rebuild_divisor"] in (25, 50, 100, 200, 400)
        assert t["on_demand_degree"] in (0, 32)
        assert t["refine_heavy_small"] in (128, 256, 512) and t["refine_heavy_mid"] in (256, 512, 1024)
        assert t["refine_heavy_large"] in (1024, 2048, 4096)
        assert t["trials"] == 18 and 0 < t["tuned_ms"] <= t["default_ms"]
        after, _ = c.partition(g, 64, 1.03, 0)  # the chosen thresholds stay on the context
        np.testing.assert_array_equal(after, before)
