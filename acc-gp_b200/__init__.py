"""Python host mirror of the gpart_b200 partitioner.

The reference (Acc-GPart) exposes its hot path as a C++ pipeline driven by
``app/partition_main.cu`` and an independent verifier ``tools/verify_csr.cpp``.
This module mirrors that operator surface over the C ABI declared in
``include/gpart_b200.h``: CSR arrays in (int32 offsets/neighbors, uint32
vertex/edge weights, ``None`` meaning unit weights), ``k`` in 2..128, an
imbalance ratio ``epsilon`` and a ``seed``; int32 labels out.  Errors raise
:class:`GpartError` carrying the library's status and message, the way the
reference's ``gpart_partition`` reports a failed run (exit 1 with a message).

The compute path is the CUDA library ``libgpart_b200.so`` built in-tree for
sm_100a.  There is no CPU fallback: if the library cannot be loaded, or no
CUDA device is present, partitioning raises.
"""
from __future__ import annotations

import ctypes as _C
import os as _os
from dataclasses import dataclass

import numpy as _np

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIBRARY_PATH = _os.path.join(_HERE, "libgpart_b200.so")

STATUS_NAMES = {
    0: "GP_OK", 1: "GP_INVALID_ARGUMENT", 2: "GP_CAPACITY_INFEASIBLE",
    3: "GP_OUT_OF_MEMORY", 4: "GP_DEVICE_TIMEOUT", 5: "GP_INTERNAL",
    6: "GP_CUDA_ERROR", 7: "GP_NO_DEVICE", 8: "GP_IO_ERROR",
}

FLAG_VERIFY = 0x1
FLAG_KEEP_HIERARCHY = 0x2
FLAG_NO_SEED_MATCHING = 0x4
FLAG_QUIET = 0x8
FLAG_COARSEN_ONLY = 0x10
FLAG_REQUIRE_BALANCED = 0x20


class GpartError(RuntimeError):
    """A gp_status other than GP_OK, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class _Csr(_C.Structure):
    _fields_ = [("n", _C.c_int64), ("m", _C.c_int64),
                ("offsets", _C.c_void_p), ("neighbors", _C.c_void_p),
                ("vertex_weights", _C.c_void_p), ("edge_weights", _C.c_void_p)]


class _Stats(_C.Structure):
    _fields_ = [("edge_cut", _C.c_uint64), ("max_part_weight", _C.c_uint64),
                ("capacity", _C.c_uint64), ("initial_cut", _C.c_uint64),
                ("levels", _C.c_int32), ("coarsest_vertices", _C.c_int32),
                ("coarsen_seconds", _C.c_double), ("initial_seconds", _C.c_double),
                ("uncoarsen_seconds", _C.c_double), ("algorithm_seconds", _C.c_double),
                ("h2d_seconds", _C.c_double), ("d2h_seconds", _C.c_double),
                ("kernel_launches", _C.c_uint64), ("algorithmic_bytes", _C.c_uint64),
                ("device_peak_bytes", _C.c_uint64), ("hierarchy_reused", _C.c_uint32), ("reserved", _C.c_uint32)]


class _RefineStats(_C.Structure):
    _fields_ = [("rounds", _C.c_int32), ("admission_iterations", _C.c_int32),
                ("checkpoint_updates", _C.c_int32), ("reserved", _C.c_int32),
                ("proposals", _C.c_uint64), ("accepted", _C.c_uint64), ("initial_cut", _C.c_uint64),
                ("final_cut", _C.c_uint64), ("final_max_part_weight", _C.c_uint64), ("capacity", _C.c_uint64),
                ("lp_cut_gain", _C.c_uint64), ("lp_cut_loss", _C.c_uint64),
                ("rebalance_cut_gain", _C.c_uint64), ("rebalance_cut_loss", _C.c_uint64),
                ("group_cut_gain", _C.c_uint64), ("group_accepted", _C.c_uint64),
                ("seconds", _C.c_double), ("kernel_launches", _C.c_uint64)]


class _Level(_C.Structure):
    _fields_ = [("graph", _Csr), ("map", _C.c_void_p)]


class _Tuning(_C.Structure):
    _fields_ = [("medium_degree", _C.c_int32), ("large_narrow", _C.c_int32), ("build_short", _C.c_int32),
                ("rebuild_divisor", _C.c_int32), ("on_demand_degree", _C.c_int32), ("default_ms", _C.c_double),
                ("tuned_ms", _C.c_double), ("trials", _C.c_int32), ("refine_heavy_small", _C.c_int32),
                ("refine_heavy_mid", _C.c_int32), ("refine_heavy_large", _C.c_int32)]


class _Request(_C.Structure):
    _fields_ = [("graph", _Csr), ("k", _C.c_int32), ("epsilon", _C.c_double), ("seed", _C.c_uint32),
                ("flags", _C.c_uint32), ("labels_out", _C.c_void_p), ("stats", _Stats), ("status", _C.c_int),
                ("queue_seconds", _C.c_double), ("run_seconds", _C.c_double)]


_lib_handle = None


def library() -> _C.CDLL:
    """Load libgpart_b200.so (raises OSError when it has not been built)."""
    global _lib_handle
    if _lib_handle is None:
        if not _os.path.exists(LIBRARY_PATH):
            raise OSError(f"{LIBRARY_PATH} is missing; run `make -C acc-gp_b200`")
        lib = _C.CDLL(LIBRARY_PATH)
        lib.gp_last_error.restype = _C.c_char_p
        lib.gp_version.restype = _C.c_char_p
        _lib_handle = lib
    return _lib_handle


def _check(status: int) -> None:
    if status != 0:
        raise GpartError(status, library().gp_last_error().decode(errors="replace"))


def _ptr(array):
    return None if array is None else array.ctypes.data_as(_C.c_void_p)


@dataclass
class Graph:
    """A CSR graph. ``vertex_weights``/``edge_weights`` of None mean unit."""
    offsets: _np.ndarray
    neighbors: _np.ndarray
    vertex_weights: _np.ndarray | None = None
    edge_weights: _np.ndarray | None = None

    def __post_init__(self):
        self.offsets = _np.ascontiguousarray(self.offsets, dtype=_np.int32)
        self.neighbors = _np.ascontiguousarray(self.neighbors, dtype=_np.int32)
        if self.vertex_weights is not None:
            self.vertex_weights = _np.ascontiguousarray(self.vertex_weights, dtype=_np.uint32)
        if self.edge_weights is not None:
            self.edge_weights = _np.ascontiguousarray(self.edge_weights, dtype=_np.uint32)

    @property
    def n(self) -> int:
        return int(self.offsets.shape[0]) - 1

    @property
    def m(self) -> int:
        return int(self.neighbors.shape[0])

    def total_vertex_weight(self) -> int:
        return self.n if self.vertex_weights is None else int(self.vertex_weights.sum(dtype=_np.uint64))

    def as_c(self) -> _Csr:
        return _Csr(self.n, self.m, _ptr(self.offsets), _ptr(self.neighbors),
                    _ptr(self.vertex_weights), _ptr(self.edge_weights))


# ---------------------------------------------------------------- host utilities

def partition_capacity(total: int, k: int, epsilon: float) -> int:
    """floor(total*epsilon/k); include/partition_capacity.hpp:14-25."""
    out = _C.c_uint64()
    _check(library().gp_partition_capacity(_C.c_uint64(total), _C.c_int32(k),
                                           _C.c_double(epsilon), _C.byref(out)))
    return out.value


def grid2d(width: int, height: int) -> Graph:
    lib = library()
    n, m = _C.c_int64(), _C.c_int64()
    _check(lib.gp_generate_grid2d(width, height, _C.byref(n), _C.byref(m), None, None))
    off = _np.empty(n.value + 1, _np.int32)
    nbr = _np.empty(m.value, _np.int32)
    _check(lib.gp_generate_grid2d(width, height, _C.byref(n), _C.byref(m), _ptr(off), _ptr(nbr)))
    return Graph(off, nbr)


def mesh3d(x: int, y: int, z: int, weighted: bool = False, seed: int = 0) -> Graph:
    lib = library()
    n, m = _C.c_int64(), _C.c_int64()
    _check(lib.gp_generate_mesh3d(x, y, z, int(weighted), _C.c_uint64(seed), _C.byref(n), _C.byref(m),
                                  None, None, None, None))
    off = _np.empty(n.value + 1, _np.int32)
    nbr = _np.empty(m.value, _np.int32)
    vw = _np.empty(n.value, _np.uint32) if weighted else None
    ew = _np.empty(m.value, _np.uint32) if weighted else None
    _check(lib.gp_generate_mesh3d(x, y, z, int(weighted), _C.c_uint64(seed), _C.byref(n), _C.byref(m),
                                  _ptr(off), _ptr(nbr), _ptr(vw), _ptr(ew)))
    return Graph(off, nbr, vw, ew)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 0) -> Graph:
    lib = library()
    n, m = _C.c_int64(), _C.c_int64()
    args = (_C.c_int32(scale), _C.c_int32(edge_factor), _C.c_double(a), _C.c_double(b), _C.c_double(c),
            _C.c_uint64(seed))
    _check(lib.gp_generate_rmat(*args, _C.byref(n), _C.byref(m), None, None))
    off = _np.empty(n.value + 1, _np.int32)
    nbr = _np.empty(m.value, _np.int32)
    _check(lib.gp_generate_rmat(*args, _C.byref(n), _C.byref(m), _ptr(off), _ptr(nbr)))
    return Graph(off, nbr)


def with_weights(graph: Graph, seed: int, vw=(1, 1), ew=(1, 1)) -> Graph:
    """Copy of ``graph`` with seeded uniform weights in the given ranges."""
    vws = _np.empty(graph.n, _np.uint32)
    ews = _np.empty(graph.m, _np.uint32)
    g = graph.as_c()
    _check(library().gp_generate_weights(_C.byref(g), _C.c_uint64(seed), vw[0], vw[1], ew[0], ew[1],
                                         _ptr(vws), _ptr(ews)))
    return Graph(graph.offsets, graph.neighbors, vws, ews)


def write_hierarchy(levels: list, path: str) -> None:
    """write_hierarchy (include/hierarchy.hpp:38-123): ``levels`` is a list of
    (Graph, map) pairs, map (int32, length n of its level) for every level but
    the last, None for the last."""
    arr = (_Level * max(1, len(levels)))()
    keep = []
    for i, (graph, mp) in enumerate(levels):
        mp = None if mp is None else _np.ascontiguousarray(mp, dtype=_np.int32)
        keep.append(mp)
        arr[i] = _Level(graph.as_c(), _ptr(mp))
    _check(library().gp_write_hierarchy(arr, _C.c_int32(len(levels)), str(path).encode()))


def read_hierarchy(path: str) -> list[dict]:
    """Parse a file of write_hierarchy: per level offsets, neighbors, edge and
    vertex weights (int32) and the map of the previous level to this one."""
    data = _np.fromfile(path, dtype=_np.int32)
    pos = 1
    out = []
    for i in range(int(data[0])):
        n, m = int(data[pos]), int(data[pos + 1])
        pos += 2
        level = {}
        for name, size in (("offsets", n + 1), ("neighbors", m), ("edge_weights", m), ("vertex_weights", n)):
            level[name] = data[pos:pos + size].copy()
            pos += size
        if i:
            fine = out[-1]["offsets"].shape[0] - 1
            level["map_from_previous"] = data[pos:pos + fine].copy()
            pos += fine
        out.append(level)
    if pos != data.shape[0]:
        raise ValueError(f"{path}: {data.shape[0] - pos} trailing int32 values")
    return out


def read_csr_int64(indptr_path: str, indices_path: str) -> Graph:
    """load_weighted_graph (src/graph.cpp:47-116) with unit weights."""
    lib = library()
    n, m = _C.c_int64(), _C.c_int64()
    a, b = indptr_path.encode(), indices_path.encode()
    _check(lib.gp_read_csr_int64(a, b, _C.byref(n), _C.byref(m), None, None))
    off = _np.empty(n.value + 1, _np.int32)
    nbr = _np.empty(m.value, _np.int32)
    _check(lib.gp_read_csr_int64(a, b, _C.byref(n), _C.byref(m), _ptr(off), _ptr(nbr)))
    return Graph(off, nbr)


def write_csr_int64(graph: Graph, indptr_path: str, indices_path: str) -> None:
    g = graph.as_c()
    _check(library().gp_write_csr_int64(indptr_path.encode(), indices_path.encode(), _C.byref(g)))


def edge_cut(graph: Graph, labels) -> int:
    labels = _np.ascontiguousarray(labels, dtype=_np.int32)
    out = _C.c_uint64()
    g = graph.as_c()
    _check(library().gp_edge_cut(_C.byref(g), _ptr(labels), _C.byref(out)))
    return out.value


def verify(graph: Graph, labels, k: int, epsilon: float = 1.03, check_symmetry: bool = False) -> dict:
    """Independent verifier (tools/verify_csr.cpp) with weights; returns its JSON as a dict."""
    import json
    labels = _np.ascontiguousarray(labels, dtype=_np.int32)
    cut = _C.c_uint64()
    ok = _C.c_int32()
    loads = _np.zeros(k, _np.uint64)
    buf = _C.create_string_buffer(64 + 24 * (k + 16))
    g = graph.as_c()
    _check(library().gp_verify(_C.byref(g), _ptr(labels), _C.c_int32(k), _C.c_double(epsilon),
                               _C.c_int32(int(check_symmetry)), _C.byref(cut), _ptr(loads), _C.byref(ok),
                               buf, _C.c_size_t(len(buf))))
    return json.loads(buf.value.decode())


# ---------------------------------------------------------------- partitioning

@dataclass
class Stats:
    edge_cut: int
    max_part_weight: int
    capacity: int
    initial_cut: int
    levels: int
    coarsest_vertices: int
    coarsen_seconds: float
    initial_seconds: float
    uncoarsen_seconds: float
    algorithm_seconds: float
    h2d_seconds: float
    d2h_seconds: float
    kernel_launches: int
    algorithmic_bytes: int
    device_peak_bytes: int = 0
    hierarchy_reused: int = 0

    @classmethod
    def _from(cls, s: _Stats) -> "Stats":
        return cls(**{name: getattr(s, name) for name, _ in _Stats._fields_ if name != "reserved"})


class Context:
    """A device context (arena + stream); gp_context_create/destroy."""

    def __init__(self, device: int = 0):
        lib = library()
        self._lib = lib
        self._handle = _C.c_void_p()
        _check(lib.gp_context_create(_C.c_int(device), _C.byref(self._handle)))

    def close(self) -> None:
        if self._handle:
            self._lib.gp_context_destroy(self._handle)
            self._handle = _C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def partition(self, graph: Graph, k: int, epsilon: float = 1.03, seed: int = 0, flags: int = FLAG_QUIET):
        """Partition a host graph; returns (labels, Stats)."""
        labels = _np.empty(graph.n, _np.int32)
        stats = _Stats()
        g = graph.as_c()
        _check(self._lib.gp_partition(self._handle, _C.byref(g), _C.c_int32(k), _C.c_double(epsilon),
                                      _C.c_uint32(seed), _C.c_uint32(flags), _ptr(labels), _C.byref(stats)))
        return labels, Stats._from(stats)

    def refine(self, graph: Graph, labels, k: int, epsilon: float = 1.03, max_rounds: int = 32,
               exchange_rounds: int = 2, flags: int = FLAG_QUIET):
        """gp_refine (the reference's refine_partition): one level of refinement
        of `labels` on `graph`; returns (refined labels, dict of RefineStats)."""
        out = _np.array(labels, dtype=_np.int32, copy=True)
        if out.shape != (graph.n,):
            raise GpartError(1, "refinement partition has the wrong length")
        stats = _RefineStats()
        g = graph.as_c()
        _check(self._lib.gp_refine(self._handle, _C.byref(g), _C.c_int32(k), _C.c_double(epsilon),
                                   _C.c_int32(max_rounds), _C.c_int32(exchange_rounds), _C.c_uint32(flags),
                                   _ptr(out), _C.byref(stats)))
        return out, {name: getattr(stats, name) for name, _ in _RefineStats._fields_ if name != "reserved"}

    def load_csr_int64(self, indptr_path: str, indices_path: str) -> tuple[int, int]:
        """gp_load_csr_int64: the reference's int64 files streamed into device memory; returns (n, m)."""
        n, m = _C.c_int64(), _C.c_int64()
        _check(self._lib.gp_load_csr_int64(self._handle, str(indptr_path).encode(), str(indices_path).encode(),
                                           _C.byref(n), _C.byref(m)))
        self._loaded_n = n.value
        return n.value, m.value

    def partition_loaded(self, k: int, epsilon: float = 1.03, seed: int = 0, flags: int = FLAG_QUIET):
        """gp_partition_loaded: partition the graph of the last load_csr_int64; returns (labels, Stats)."""
        labels = _np.empty(getattr(self, "_loaded_n", 0), _np.int32)
        stats = _Stats()
        _check(self._lib.gp_partition_loaded(self._handle, _C.c_int32(k), _C.c_double(epsilon), _C.c_uint32(seed),
                                             _C.c_uint32(flags), _ptr(labels), _C.byref(stats)))
        return labels, Stats._from(stats)

    def partition_device(self, offsets_ptr: int, neighbors_ptr: int, n: int, m: int, vertex_weights_ptr,
                         edge_weights_ptr, k: int, epsilon: float, seed: int, labels_ptr: int,
                         stream_ptr=None, flags: int = FLAG_QUIET) -> Stats:
        """Partition a graph already resident on the device (raw pointers)."""
        stats = _Stats()
        g = _Csr(n, m, offsets_ptr, neighbors_ptr, vertex_weights_ptr, edge_weights_ptr)
        _check(self._lib.gp_partition_device(self._handle, _C.byref(g), _C.c_int32(k), _C.c_double(epsilon),
                                             _C.c_uint32(seed), _C.c_uint32(flags), _C.c_void_p(labels_ptr),
                                             _C.c_void_p(stream_ptr) if stream_ptr else None, _C.byref(stats)))
        return Stats._from(stats)

    def partition_host_ptrs(self, offsets_ptr: int, neighbors_ptr: int, n: int, m: int, vertex_weights_ptr,
                            edge_weights_ptr, k: int, epsilon: float, seed: int, labels_ptr: int,
                            flags: int = FLAG_QUIET) -> Stats:
        """gp_partition on raw host pointers (e.g. pinned buffers)."""
        stats = _Stats()
        g = _Csr(n, m, offsets_ptr, neighbors_ptr, vertex_weights_ptr, edge_weights_ptr)
        _check(self._lib.gp_partition(self._handle, _C.byref(g), _C.c_int32(k), _C.c_double(epsilon),
                                      _C.c_uint32(seed), _C.c_uint32(flags), _C.c_void_p(labels_ptr), _C.byref(stats)))
        return Stats._from(stats)

    def partition_batch(self, jobs, concurrency: int = 8, flags: int = FLAG_QUIET, devices=None):
        """gp_partition_batch over (graph, k, epsilon, seed) tuples; returns a
        list of (labels, Stats, run_seconds) in input order.  Raises on the
        first failed request.  With `devices` (device ordinals), the graphs
        are placed over those GPUs (gp_partition_batch_devices)."""
        jobs = list(jobs)
        requests = (_Request * max(1, len(jobs)))()
        keep = []
        outs = []
        for r, (graph, k, eps, seed) in zip(requests, jobs):
            g = graph.as_c()
            labels = _np.empty(graph.n, _np.int32)
            keep.append((graph, g))
            outs.append(labels)
            r.graph = g
            r.k, r.epsilon, r.seed, r.flags = k, eps, seed, flags
            r.labels_out = labels.ctypes.data_as(_C.c_void_p)
        if devices is None:
            _check(self._lib.gp_partition_batch(self._handle, requests, _C.c_int32(len(jobs)),
                                                _C.c_int32(concurrency)))
        else:
            devs = (_C.c_int32 * len(devices))(*devices)
            _check(self._lib.gp_partition_batch_devices(self._handle, devs, _C.c_int32(len(devices)), requests,
                                                        _C.c_int32(len(jobs)), _C.c_int32(concurrency)))
        return [(outs[i], Stats._from(requests[i].stats), requests[i].run_seconds) for i in range(len(jobs))]

    def evaluate_device(self, offsets_ptr: int, neighbors_ptr: int, n: int, m: int, vertex_weights_ptr,
                        edge_weights_ptr, labels_ptr: int, k: int, cut_ptr: int, loads_ptr: int,
                        stream_ptr=None) -> None:
        """gp_evaluate_device: cut and part loads of device labels into device outputs."""
        g = _Csr(n, m, offsets_ptr, neighbors_ptr, vertex_weights_ptr, edge_weights_ptr)
        _check(self._lib.gp_evaluate_device(self._handle, _C.byref(g), _C.c_void_p(labels_ptr), _C.c_int32(k),
                                            _C.c_void_p(cut_ptr), _C.c_void_p(loads_ptr),
                                            _C.c_void_p(stream_ptr) if stream_ptr else None))

    def profile_begin(self, kernel_substring: str) -> None:
        """Time every launch of kernels whose name contains the substring."""
        _check(self._lib.gp_profile_begin(self._handle, kernel_substring.encode()))

    def profile_end(self) -> tuple[int, float, float]:
        """(launches, total device milliseconds, algorithmic bytes) since profile_begin."""
        launches, ms, nbytes = _C.c_uint64(), _C.c_double(), _C.c_double()
        _check(self._lib.gp_profile_end(self._handle, _C.byref(launches), _C.byref(ms), _C.byref(nbytes)))
        return launches.value, ms.value, nbytes.value

    def autotune(self, graph: Graph, k: int, epsilon: float = 1.03, seed: int = 0, repeats: int = 2) -> dict:
        """gp_autotune: choose the thread-mapping thresholds for this workload
        (kept on the context); returns them with the default and tuned times."""
        t = _Tuning()
        g = graph.as_c()
        _check(self._lib.gp_autotune(self._handle, _C.byref(g), _C.c_int32(k), _C.c_double(epsilon),
                                     _C.c_uint32(seed), _C.c_int32(repeats), _C.byref(t)))
        return {name: getattr(t, name) for name, _ in _Tuning._fields_}

    def set_option(self, name: str, value: int) -> None:
        _check(self._lib.gp_set_option(self._handle, name.encode(), _C.c_int64(value)))

    def levels(self) -> list[dict]:
        """Host copies of the hierarchy kept by FLAG_KEEP_HIERARCHY."""
        lib = self._lib
        count = _C.c_int32()
        _check(lib.gp_level_count(self._handle, _C.byref(count)))
        out = []
        for i in range(count.value):
            n, m = _C.c_int64(), _C.c_int64()
            _check(lib.gp_level_size(self._handle, _C.c_int32(i), _C.byref(n), _C.byref(m)))
            off = _np.empty(n.value + 1, _np.int32)
            nbr = _np.empty(m.value, _np.int32)
            ew = _np.empty(m.value, _np.uint32)
            vw = _np.empty(n.value, _np.uint32)
            mp = _np.empty(n.value, _np.int32) if i + 1 < count.value else None
            meta = _np.zeros(4, _np.uint64)
            _check(lib.gp_level_copy(self._handle, _C.c_int32(i), _ptr(off), _ptr(nbr), _ptr(ew), _ptr(vw),
                                     _ptr(mp), _ptr(meta)))
            out.append(dict(offsets=off, neighbors=nbr, edge_weights=ew, vertex_weights=vw, map=mp,
                            maximum_degree=int(meta[0]), has_heavy_rows=int(meta[1]),
                            incident_weight_bound=int(meta[2])))
        return out

    def write_kept_hierarchy(self, path: str) -> None:
        """gp_write_kept_hierarchy: the hierarchy kept by FLAG_KEEP_HIERARCHY, as write_hierarchy writes it."""
        _check(self._lib.gp_write_kept_hierarchy(self._handle, str(path).encode()))

    def initial_labels(self, n: int) -> _np.ndarray:
        out = _np.empty(n, _np.int32)
        _check(self._lib.gp_initial_labels(self._handle, _ptr(out), _C.c_int64(n)))
        return out


def evaluate_device_static(offsets_ptr: int, neighbors_ptr: int, n: int, m: int, vertex_weights_ptr,
                           edge_weights_ptr, labels_ptr: int, k: int, cut_ptr: int, loads_ptr: int,
                           stream_ptr=None) -> None:
    """gp_evaluate_device_static: the allocation-free twin of Context.evaluate_device.

    For callers that must not let the library allocate device memory (a
    framework allocator that owns the memory budget, an allocation-free
    serving loop).  Scratch is a fixed 616 KB device array shared by all
    calls on a device; overlapping calls race, k must be <= 128, and the
    first call on a device should precede any stream capture.  Does not wait
    for the results.
    """
    g = _Csr(n, m, offsets_ptr, neighbors_ptr, vertex_weights_ptr, edge_weights_ptr)
    _check(library().gp_evaluate_device_static(_C.byref(g), _C.c_void_p(labels_ptr), _C.c_int32(k),
                                               _C.c_void_p(cut_ptr), _C.c_void_p(loads_ptr),
                                               _C.c_void_p(stream_ptr) if stream_ptr else None))


def batch_work(graph: Graph) -> int:
    """The batched form's placement estimate of one partition (bytes of one
    CSR sweep with its neighbour gathers)."""
    return 4 * (graph.n + 1) + 8 * graph.m + (4 * graph.m if graph.edge_weights is not None else 0)


def plan_placement(work, devices: int):
    """gp_plan_placement: longest-processing-time placement of work items on
    `devices` devices; returns (device_of, device_work) as numpy arrays."""
    work = _np.ascontiguousarray(work, dtype=_np.uint64)
    device_of = _np.empty(work.shape[0], _np.int32)
    device_work = _np.empty(devices, _np.uint64)
    _check(library().gp_plan_placement(_ptr(work), _C.c_int32(work.shape[0]), _C.c_int32(devices),
                                       _ptr(device_of), _ptr(device_work)))
    return device_of, device_work


class Server:
    """gp_server_*: worker contexts taking requests as they arrive, admitted
    by estimated device footprint; resident graphs via add_graph.  `device`
    may be a list of device ordinals (gp_server_create_devices; `workers`
    per device, `hbm_budget_bytes` per device)."""

    def __init__(self, device=0, workers: int = 8, hbm_budget_bytes: int = 0):
        self._lib = library()
        self._handle = _C.c_void_p()
        self._pending = {}
        if isinstance(device, (list, tuple)):
            devs = (_C.c_int32 * len(device))(*device)
            _check(self._lib.gp_server_create_devices(devs, _C.c_int32(len(device)), _C.c_int32(workers),
                                                      _C.c_uint64(hbm_budget_bytes), _C.byref(self._handle)))
        else:
            _check(self._lib.gp_server_create(_C.c_int(device), _C.c_int32(workers), _C.c_uint64(hbm_budget_bytes),
                                              _C.byref(self._handle)))
        self._graphs = []

    def keep_hierarchies(self, bytes_per_device: int) -> None:
        """gp_server_keep_hierarchies: keep coarsened hierarchies of resident
        graphs (per graph, k, seed) for later requests, within this budget."""
        _check(self._lib.gp_server_keep_hierarchies(self._handle, _C.c_uint64(bytes_per_device)))

    def kept_bytes(self) -> int:
        out = _C.c_uint64()
        _check(self._lib.gp_server_kept_bytes(self._handle, _C.byref(out)))
        return out.value

    def footprint(self, graph_id: int, k: int) -> int:
        """gp_server_footprint: the admission estimate of a request, in bytes."""
        out = _C.c_uint64()
        _check(self._lib.gp_server_footprint(self._handle, _C.c_int32(graph_id), _C.c_int32(k), _C.byref(out)))
        return out.value

    def add_graph(self, graph: Graph) -> int:
        gid = _C.c_int32()
        g = graph.as_c()
        _check(self._lib.gp_server_add_graph(self._handle, _C.byref(g), _C.byref(gid)))
        self._graphs.append(graph)
        return gid.value

    def submit(self, graph: Graph | int, k: int, epsilon: float = 1.03, seed: int = 0,
               flags: int = FLAG_QUIET) -> int:
        """Queue a request for a host graph or a resident graph id; returns a ticket."""
        req = _Request()
        resident = isinstance(graph, int)
        host = self._graphs[graph] if resident else graph
        g = host.as_c()
        if not resident:
            req.graph = g
        labels = _np.empty(host.n, _np.int32)
        req.k, req.epsilon, req.seed, req.flags = k, epsilon, seed, flags
        req.labels_out = labels.ctypes.data_as(_C.c_void_p)
        ticket = _C.c_uint64()
        _check(self._lib.gp_server_submit(self._handle, _C.byref(req), _C.c_int32(graph if resident else -1),
                                          _C.byref(ticket)))
        self._pending[ticket.value] = (req, labels, host, g)
        return ticket.value

    def wait(self, ticket: int, timeout: float = -1.0):
        """Returns (labels, Stats, queue_seconds, run_seconds); raises on failure."""
        _check(self._lib.gp_server_wait(self._handle, _C.c_uint64(ticket), _C.c_double(timeout)))
        req, labels, _, _ = self._pending.pop(ticket)
        if req.status != 0:
            raise GpartError(req.status, "request failed")
        return labels, Stats._from(req.stats), req.queue_seconds, req.run_seconds

    def close(self) -> None:
        if self._handle:
            self._lib.gp_server_destroy(self._handle)
            self._handle = _C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def partition(graph: Graph, k: int, epsilon: float = 1.03, seed: int = 0, flags: int = FLAG_QUIET):
    """One-shot partition on device 0; returns (labels, Stats)."""
    with Context(0) as ctx:
        return ctx.partition(graph, k, epsilon, seed, flags)


def version() -> str:
    return library().gp_version().decode()
