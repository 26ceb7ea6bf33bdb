"""ctypes binding of liboracle.so — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module.  It runs the serial CPU restatement of the reference partitioner and
exposes its hierarchy, METIS labels and per-level refined labels.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "liboracle.so")
FLAG_NO_SEED_MATCHING = 0x4
FLAG_COARSEN_ONLY = 0x10

_lib = None


class _Csr(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("offsets", C.c_void_p), ("neighbors", C.c_void_p),
                ("vertex_weights", C.c_void_p), ("edge_weights", C.c_void_p)]


class OracleError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"oracle status {status}: {message}")
        self.status = status
        self.message = message


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(PATH)
        _lib.orc_last_error.restype = C.c_char_p
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def partition(graph, k, epsilon=1.03, seed=0, flags=0):
    """Run the oracle; returns (labels or None, cut or None, levels list)."""
    L = lib()
    g = _Csr(graph.n, graph.m, _p(graph.offsets), _p(graph.neighbors), _p(graph.vertex_weights),
             _p(graph.edge_weights))
    labels = np.empty(graph.n, np.int32)
    cut = C.c_uint64()
    status = L.orc_partition(C.byref(g), C.c_int32(k), C.c_double(epsilon), C.c_uint32(seed), C.c_uint32(flags),
                             _p(labels), C.byref(cut))
    if status != 0:
        raise OracleError(status, L.orc_last_error().decode())
    if flags & FLAG_COARSEN_ONLY:
        return None, None
    return labels, cut.value


class _RefineStats(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("admission_iterations", C.c_int32), ("checkpoint_updates", C.c_int32),
                ("reserved", C.c_int32), ("proposals", C.c_uint64), ("accepted", C.c_uint64),
                ("initial_cut", C.c_uint64), ("final_cut", C.c_uint64), ("final_max_part_weight", C.c_uint64),
                ("capacity", C.c_uint64), ("lp_cut_gain", C.c_uint64), ("lp_cut_loss", C.c_uint64),
                ("rebalance_cut_gain", C.c_uint64), ("rebalance_cut_loss", C.c_uint64),
                ("group_cut_gain", C.c_uint64), ("group_accepted", C.c_uint64)]


def refine(graph, labels, k, epsilon=1.03, max_rounds=32, exchange_rounds=2):
    """refine_partition restated: one level of refinement of `labels`;
    returns (refined labels, dict of RefineStats)."""
    L = lib()
    g = _Csr(graph.n, graph.m, _p(graph.offsets), _p(graph.neighbors), _p(graph.vertex_weights),
             _p(graph.edge_weights))
    out = np.array(labels, dtype=np.int32, copy=True)
    st = _RefineStats()
    status = L.orc_refine(C.byref(g), C.c_int32(k), C.c_double(epsilon), C.c_int32(max_rounds),
                          C.c_int32(exchange_rounds), _p(out), C.byref(st))
    if status != 0:
        raise OracleError(status, L.orc_last_error().decode())
    return out, {name: getattr(st, name) for name, _ in _RefineStats._fields_ if name != "reserved"}


def levels():
    L = lib()
    out = []
    count = L.orc_level_count()
    for i in range(count):
        n, m = C.c_int64(), C.c_int64()
        L.orc_level_size(C.c_int32(i), C.byref(n), C.byref(m))
        off = np.empty(n.value + 1, np.int32)
        nbr = np.empty(m.value, np.int32)
        ew = np.empty(m.value, np.uint32)
        vw = np.empty(n.value, np.uint32)
        mp = np.empty(n.value, np.int32) if i + 1 < count else None
        meta = np.zeros(4, np.uint64)
        L.orc_level_copy(C.c_int32(i), _p(off), _p(nbr), _p(ew), _p(vw), _p(mp), _p(meta))
        out.append(dict(n=n.value, m=m.value, offsets=off, neighbors=nbr, edge_weights=ew, vertex_weights=vw, map=mp,
                        maximum_degree=int(meta[0]), has_heavy_rows=int(meta[1]),
                        incident_weight_bound=int(meta[2])))
    return out


def initial_labels(n):
    out = np.empty(n, np.int32)
    if lib().orc_initial_labels(_p(out), C.c_int64(n)) != 0:
        raise OracleError(1, "no initial labels")
    return out


def level_labels(level, n):
    out = np.empty(n, np.int32)
    if lib().orc_level_labels(C.c_int32(level), _p(out)) != 0:
        raise OracleError(1, "no labels for level")
    return out


def level_result(level):
    cut, refined = C.c_uint64(), C.c_int32()
    lib().orc_level_result(C.c_int32(level), C.byref(cut), C.byref(refined))
    return cut.value, bool(refined.value)
