"""Generate the golden fixtures in tests/golden/ from the reference build.

Runs the reference partitioner compiled for sm_100a (oracle/_ref, built by
oracle/ref/Makefile) on seeded synthetic inputs and records, for every level
of its hierarchy, the sizes, metadata and SHA-256 digests of the coarse CSR,
weights and fine-to-coarse map, then the METIS labels of the coarsest graph
and the final cut.  Needs a CUDA GPU (the reference is GPU code).

    python tests/golden/make_golden.py [--out DIR] [--cases a,b,...] [--baseline]
    python tests/golden/make_golden.py --refine [--out DIR]
    python tests/golden/make_golden.py --digests-only --cases rmat22_k64,m3_k128
    python tests/golden/make_golden.py --oracle-labels --cases rmat22_k64,m3_k128

--refine runs the reference's single-level refinement (oracle/_ref/
gpart_ref_refine: its run_incremental_refinement on a one-level resident
hierarchy) on every case of cases.REFINE_CASES and writes refine_cases.json:
per case the SHA-256 of the refined labels, the part loads, and the
RefineStats fields the reference reports for that run (-1 where it reports
none).  --digests-only records hierarchy
digests and the METIS digest without the final-label checks (for the
headline-size cases, whose full arrays are too large to keep).
--oracle-labels needs no GPU: it adds the serial oracle's final-label digest
and cut to existing case files, for the label-identity check of the
headline-size cases.

--baseline additionally times the unmodified reference CLI on R-MAT scale 22
(k=64, seeds 0-2) and writes baseline_rmat22.json.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref")


def load_package():
    pkg = os.path.join(ROOT, "acc-gp_b200")
    spec = importlib.util.spec_from_file_location("acc_gp_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["acc_gp_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


gp = load_package()
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from cases import CASES, REFINE_CASES, build_case, refine_start  # noqa: E402

sys.path.insert(0, os.path.join(ROOT, "oracle"))
STAT_FIELDS = ["rounds", "proposals", "accepted", "initial_cut", "final_cut", "final_max_part_weight",
               "admission_iterations", "admission_fallbacks", "lp_cut_gain", "lp_cut_loss", "rebalance_cut_gain",
               "rebalance_cut_loss", "checkpoint_updates", "group_cut_gain", "group_accepted",
               "frontier_vertices_initial"]


def digest(array) -> str:
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def parse_dump(path: str) -> dict:
    data = open(path, "rb").read()
    assert data[:8] == b"GPDUMP01", "bad dump magic"
    pos = 8

    def take(dtype, count):
        nonlocal pos
        arr = np.frombuffer(data, dtype=dtype, count=count, offset=pos)
        pos += arr.nbytes
        return arr

    levels_count = int(take(np.int32, 1)[0])
    levels = []
    for i in range(levels_count):
        n = int(take(np.int64, 1)[0]); m = int(take(np.int64, 1)[0])
        maxdeg = int(take(np.uint64, 1)[0]); heavy = int(take(np.uint8, 1)[0])
        bound = int(take(np.uint64, 1)[0])
        level = dict(n=n, m=m, maximum_degree=maxdeg, has_heavy_rows=heavy, incident_weight_bound=bound,
                     offsets=take(np.int32, n + 1), neighbors=take(np.int32, m),
                     edge_weights=take(np.uint32, m), vertex_weights=take(np.uint32, n))
        level["map"] = take(np.int32, n) if i + 1 < levels_count else None
        levels.append(level)
    nc = int(take(np.int64, 1)[0])
    metis = take(np.int32, nc)
    n0 = int(take(np.int64, 1)[0])
    final = take(np.int32, n0)
    cut = int(take(np.uint64, 1)[0])
    seconds = float(take(np.float64, 1)[0])
    return dict(levels=levels, metis=metis, final=final, cut=cut, seconds=seconds)


def run_reference(graph, k, eps, seed, workdir):
    ip, ix = os.path.join(workdir, "g.indptr"), os.path.join(workdir, "g.indices")
    gp.write_csr_int64(graph, ip, ix)
    vw = ew = "-"
    if graph.vertex_weights is not None:
        vw = os.path.join(workdir, "g.vw"); graph.vertex_weights.tofile(vw)
    if graph.edge_weights is not None:
        ew = os.path.join(workdir, "g.ew"); graph.edge_weights.tofile(ew)
    out = os.path.join(workdir, "g.dump")
    proc = subprocess.run([os.path.join(REF, "gpart_ref_dump"), ip, ix, vw, ew, str(k), repr(eps), str(seed), out],
                          capture_output=True, text=True)
    if proc.returncode != 0:
        return None, proc.stderr.strip()[-400:]
    return parse_dump(out), proc.stdout


def summarise(name, spec, dump, graph):
    levels = []
    for lv in dump["levels"]:
        levels.append(dict(
            n=lv["n"], m=lv["m"], maximum_degree=lv["maximum_degree"], has_heavy_rows=lv["has_heavy_rows"],
            incident_weight_bound=lv["incident_weight_bound"],
            offsets=digest(lv["offsets"]), neighbors=digest(lv["neighbors"]),
            edge_weights=digest(lv["edge_weights"]), vertex_weights=digest(lv["vertex_weights"]),
            map=None if lv["map"] is None else digest(lv["map"])))
    verdict = gp.verify(graph, dump["final"], spec["k"], spec["eps"])
    return dict(case=name, spec=spec, levels=levels, coarsest_n=int(dump["metis"].shape[0]),
                metis_labels=digest(dump["metis"]), metis_cut=None, reference_final_cut=dump["cut"],
                reference_verifier=dict(cut=verdict["cut"], max_load=verdict["max_load"],
                                        capacity=verdict["capacity"], capacity_ok=verdict["capacity_ok"]),
                reference_seconds=dump["seconds"])


def write_inputs(graph, workdir):
    ip, ix = os.path.join(workdir, "g.indptr"), os.path.join(workdir, "g.indices")
    gp.write_csr_int64(graph, ip, ix)
    vw = ew = "-"
    if graph.vertex_weights is not None:
        vw = os.path.join(workdir, "g.vw"); graph.vertex_weights.tofile(vw)
    if graph.edge_weights is not None:
        ew = os.path.join(workdir, "g.ew"); graph.edge_weights.tofile(ew)
    return ip, ix, vw, ew


def refine_goldens(out_dir, names, arrays_dir=None):
    """The reference's refine_partition on every refinement case."""
    import oracle
    records = {}
    graphs = {}
    for name in names:
        spec = REFINE_CASES[name]
        g = graphs.get(spec["graph"])
        if g is None:
            g = graphs[spec["graph"]] = build_case(gp, CASES[spec["graph"]])
        start = refine_start(gp, oracle, spec, g)
        with tempfile.TemporaryDirectory() as tmp:
            ip, ix, vw, ew = write_inputs(g, tmp)
            lp = os.path.join(tmp, "start.i32")
            start.astype(np.int32).tofile(lp)
            out = os.path.join(tmp, "refined.dump")
            proc = subprocess.run([os.path.join(REF, "gpart_ref_refine"), ip, ix, vw, ew, lp, str(spec["k"]),
                                   repr(spec["eps"]), str(spec["rounds"]), str(spec["exchange"]), out],
                                  capture_output=True, text=True)
            if proc.returncode != 0:
                records[name] = dict(spec=spec, error=proc.stderr.strip()[-400:])
                print(name, "REFERENCE FAILED", proc.stderr.strip()[-300:], flush=True)
                continue
            data = open(out, "rb").read()
        assert data[:8] == b"GPREF002"
        n = int(np.frombuffer(data, np.int64, 1, 8)[0])
        labels = np.frombuffer(data, np.int32, n, 16)
        fields = np.frombuffer(data, np.int64, 16, 16 + 4 * n)
        stats = {key: int(v) for key, v in zip(STAT_FIELDS, fields)}
        w = np.ones(n, np.uint64) if g.vertex_weights is None else g.vertex_weights.astype(np.uint64)
        loads = np.bincount(labels, weights=w, minlength=spec["k"]).astype(np.uint64)
        records[name] = dict(spec=spec, start=digest(start.astype(np.int32)), labels=digest(labels),
                             loads=[int(x) for x in loads], cut=gp.edge_cut(g, labels), stats=stats)
        if arrays_dir:
            np.save(os.path.join(arrays_dir, f"refine_{name}.npy"), labels)
        print(name, "cut", stats["initial_cut"], "->", stats["final_cut"], "rounds", stats["rounds"],
              "repair_iterations", stats["admission_iterations"], flush=True)
    with open(os.path.join(out_dir, "refine_cases.json"), "w") as f:
        json.dump(records, f, indent=1, sort_keys=True)


def baseline(out_dir):
    g = gp.rmat(22, 16, 0.57, 0.19, 0.19, 0)
    rows = []
    with tempfile.TemporaryDirectory() as tmp:
        ip, ix = os.path.join(tmp, "r22.indptr"), os.path.join(tmp, "r22.indices")
        gp.write_csr_int64(g, ip, ix)
        for seed in (0, 1, 2):
            part = os.path.join(tmp, f"r22.{seed}.part")
            proc = subprocess.run([os.path.join(REF, "gpart_partition_standard"), ip, ix, "64", part, "1.03",
                                   str(seed)], capture_output=True, text=True)
            t = re.search(r"algorithm_total_seconds=([0-9.eE+-]+)", proc.stdout)
            c = re.search(r"final_edge_cut=(\d+)", proc.stdout)
            ver = subprocess.run([os.path.join(REF, "gpart_verify_csr"), ip, ix, "64", part, "binary"],
                                 capture_output=True, text=True)
            rows.append(dict(seed=seed, rc=proc.returncode, algorithm_total_seconds=float(t.group(1)) if t else None,
                             final_edge_cut=int(c.group(1)) if c else None, verifier=ver.stdout.strip()[:400],
                             stderr=proc.stderr.strip()[-300:]))
            print(rows[-1], flush=True)
    with open(os.path.join(out_dir, "baseline_rmat22.json"), "w") as f:
        json.dump(dict(graph=dict(n=g.n, m=g.m), k=64, eps=1.03, runs=rows), f, indent=1)


def oracle_labels(out_dir, names):
    """Adds to each named case file the SHA-256 of the serial oracle's final
    labels and its cut, so a GPU test can require identical labels on graphs
    whose full label arrays are too large to keep (the headline cases).  Runs
    on the CPU only; R-MAT scale 22 takes a few minutes on one core."""
    import oracle  # CPU restatement of the reference's rules
    for name in names:
        path = os.path.join(out_dir, f"{name}.json")
        with open(path) as f:
            record = json.load(f)
        spec = CASES[name]
        graph = build_case(gp, spec)
        labels, cut = oracle.partition(graph, spec["k"], spec["eps"], spec["seed"])
        record["oracle_final_labels"] = digest(labels)
        record["oracle_final_cut"] = int(cut)
        with open(path, "w") as f:
            json.dump(record, f, indent=1)
        print(name, "oracle cut", cut, flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--cases", default="")
    ap.add_argument("--baseline", action="store_true")
    ap.add_argument("--keep-arrays", action="store_true", help="also save full small-level arrays (npz)")
    ap.add_argument("--refine", action="store_true", help="refinement goldens (refine_cases.json)")
    ap.add_argument("--arrays-dir", default="", help="--refine: also save each refined labelling here (.npy)")
    ap.add_argument("--oracle-labels", action="store_true",
                    help="add the CPU oracle's final-label digest and cut to existing case files (no GPU)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    if args.oracle_labels:
        oracle_labels(args.out, [c for c in args.cases.split(",") if c])
        return
    if args.refine:
        names = [c for c in args.cases.split(",") if c] or list(REFINE_CASES)
        if args.arrays_dir:
            os.makedirs(args.arrays_dir, exist_ok=True)
        refine_goldens(args.out, names, args.arrays_dir or None)
        return
    names = [c for c in args.cases.split(",") if c] or list(CASES)
    for name in names:
        spec = CASES[name]
        graph = build_case(gp, spec)
        with tempfile.TemporaryDirectory() as tmp:
            dump, log = run_reference(graph, spec["k"], spec["eps"], spec["seed"], tmp)
        if dump is None:
            record = dict(case=name, spec=spec, error=log)
            print(name, "REFERENCE FAILED", log, flush=True)
        else:
            record = summarise(name, spec, dump, graph)
            print(name, "levels", len(record["levels"]), "cut", dump["cut"], "sec", round(dump["seconds"], 4), flush=True)
            if args.keep_arrays:
                arrays = {"metis": dump["metis"], "final": dump["final"]}
                for i, lv in enumerate(dump["levels"]):
                    if lv["n"] <= 70000:
                        for key in ("offsets", "neighbors", "edge_weights", "vertex_weights", "map"):
                            if lv[key] is not None:
                                arrays[f"l{i}_{key}"] = lv[key]
                np.savez_compressed(os.path.join(args.out, f"{name}.npz"), **arrays)
        with open(os.path.join(args.out, f"{name}.json"), "w") as f:
            json.dump(record, f, indent=1)
    if args.baseline:
        baseline(args.out)


if __name__ == "__main__":
    main()
