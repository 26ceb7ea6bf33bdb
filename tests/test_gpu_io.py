"""The reference's file formats on the GPU path: int64 CSR files streamed
into device memory (gp_load_csr_int64, load_weighted_graph's checks) and the
drop-in command line on them."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def write(gp, g, tmp_path, name="g"):
    ip, ix = str(tmp_path / f"{name}.indptr"), str(tmp_path / f"{name}.indices")
    gp.write_csr_int64(g, ip, ix)
    return ip, ix


def test_loaded_graph_partitions_like_host_input(gp, ctx, tmp_path):
    """R-MAT scale 20: 31M index values, four 8 Mi-value chunks through the
    two pinned buffers."""
    g = gp.rmat(20, 16, 0.57, 0.19, 0.19, 0)
    ip, ix = write(gp, g, tmp_path)
    n, m = ctx.load_csr_int64(ip, ix)
    assert (n, m) == (g.n, g.m) and m > 3 * (1 << 23)
    labels, st = ctx.partition_loaded(64, 1.03, 0)
    expected, est = ctx.partition(g, 64, 1.03, 0)
    np.testing.assert_array_equal(labels, expected)
    assert st.edge_cut == est.edge_cut
    again, st2 = ctx.partition_loaded(64, 1.03, 0)  # the loaded graph stays resident
    np.testing.assert_array_equal(again, expected)


@pytest.mark.parametrize("defect, message", [
    ("neighbor", "CSR contains an invalid neighbor"),
    ("monotone", "CSR offsets are not monotone"),
    ("ends", "CSR offsets do not match indices"),
])
def test_load_rejects_like_load_weighted_graph(gp, ctx, tmp_path, defect, message):
    g = gp.grid2d(30, 20)
    ip, ix = write(gp, g, tmp_path)
    if defect == "neighbor":
        nbr = np.fromfile(ix, np.int64)
        nbr[17] = g.n
        nbr.tofile(ix)
    else:
        off = np.fromfile(ip, np.int64)
        if defect == "monotone":
            off[5], off[6] = off[6], off[5] - 1
        else:
            off[-1] -= 1
        off.tofile(ip)
    with pytest.raises(gp.GpartError) as e:
        ctx.load_csr_int64(ip, ix)
    assert message in str(e.value)
    with pytest.raises(gp.GpartError):  # nothing stays loaded after a failure
        ctx.partition_loaded(4)


@pytest.mark.parametrize("verify", [False, True])
def test_partition_cli_end_to_end(gp, ctx, tmp_path, verify):
    """gpart_partition_standard on int64 files: labels, cut and stdout keys
    of app/partition_main.cu."""
    g = gp.mesh3d(20, 18, 16)
    ip, ix = write(gp, g, tmp_path)
    out = str(tmp_path / "labels.part")
    exe = os.path.join(ROOT, "acc-gp_b200", "bin", "gpart_partition_standard")
    args = [exe, ip, ix, "16", out, "1.03", "3"] + (["--verify"] if verify else [])
    run = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    labels = np.fromfile(out, np.int32)
    expected, st = ctx.partition(g, 16, 1.03, 3)
    np.testing.assert_array_equal(labels, expected)
    lines = run.stdout
    assert f"vertices={g.n} edge_entries={g.m}" in lines
    assert f"verify={int(verify)}" in lines and "coarsen_mode=regret" in lines
    assert f"final_edge_cut={st.edge_cut}" in lines
    assert "algorithm_total_seconds=" in lines and "wall_total_seconds=" in lines
