"""Checks against the reference's own CPU-side tools, built from its sources
into oracle/_ref by oracle/ref/Makefile (skipped where they were not built):
* the drop-in verifier prints byte-identical JSON to tools/verify_csr.cpp;
* the warm timing harness (oracle/ref/ref_bench.cu) generates the same R-MAT
  graph as the library, so both bench arms partition one input."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
OURS = os.path.join(ROOT, "acc-gp_b200", "bin", "gpart_verify_csr")


def _need(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path, ROOT)} was not built")


@pytest.mark.parametrize("graph, k, mode, symmetric", [
    ("rmat", 16, "binary", False), ("rmat", 16, "binary", True), ("grid", 7, "text", True),
    ("grid", 128, "binary", False)])
def test_verifier_json_identical_to_reference(gp, tmp_path, graph, k, mode, symmetric):
    _need(OURS)
    _need(os.path.join(REF, "gpart_verify_csr"))
    g = gp.rmat(12, 16, 0.57, 0.19, 0.19, 3) if graph == "rmat" else gp.grid2d(61, 37)
    ip, ix, part = str(tmp_path / "g.indptr"), str(tmp_path / "g.indices"), str(tmp_path / "g.part")
    gp.write_csr_int64(g, ip, ix)
    rng = np.random.default_rng(k)
    labels = (np.arange(g.n) * k // g.n).astype(np.int32)
    flip = rng.random(g.n) < 0.1
    labels[flip] = rng.integers(0, k, int(flip.sum()))
    if mode == "binary":
        labels.tofile(part)
    else:
        with open(part, "w") as f:
            f.write("\n".join(str(x) for x in labels) + "\n")
    args = [ip, ix, str(k), part, mode] + (["--symmetric"] if symmetric else [])
    a = subprocess.run([OURS] + args, capture_output=True, text=True)
    b = subprocess.run([os.path.join(REF, "gpart_verify_csr")] + args, capture_output=True, text=True)
    assert a.returncode == b.returncode
    assert a.stdout == b.stdout and a.stdout.strip()


@pytest.mark.parametrize("scale, ef, seed", [(12, 16, 0), (14, 8, 5)])
def test_bench_harness_generator_matches_library(gp, tmp_path, scale, ef, seed):
    exe = os.path.join(REF, "gpart_ref_bench")
    _need(exe)
    ip, ix = str(tmp_path / "r.indptr"), str(tmp_path / "r.indices")
    r = subprocess.run([exe, "write-rmat", str(scale), str(ef), "0.57", "0.19", "0.19", str(seed), ip, ix],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    g = gp.rmat(scale, ef, 0.57, 0.19, 0.19, seed)
    np.testing.assert_array_equal(np.fromfile(ip, np.int64), g.offsets)
    np.testing.assert_array_equal(np.fromfile(ix, np.int64), g.neighbors)
