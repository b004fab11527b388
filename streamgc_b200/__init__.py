"""streamgc_b200 -- B200-native streaming graph coloring (single GPU).

Python binding of libstreamgc_b200.so (C ABI in include/streamgc_b200.h). The
library owns every computation; this module only moves numpy arrays across
the ABI. There is no fallback: without the built library (streamgc_b200/lib/)
every call raises.

The reference program (algorithms/streamgc/src/streamgc.cu main) maps onto:
    Graph.load_mtx / rmat / chung_lu / delaunay     graph input
    Graph.init_stream / churn_stream / kcore_stream the update streams
    StreamGC(graph, ...)                            allocate_gpu_partition
    StreamGC.apply / epoch / publish / repair       process_stream pieces
    StreamGC.process_stream                         process_stream
    StreamGC.validate                               check_coloring_valid
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libstreamgc_b200.so")

MODE_DETERMINISTIC = 0
MODE_CONCURRENT = 1
ADD, DEL = 0, 1

EDGE_UPDATE = np.dtype([("u", "<u4"), ("v", "<u4"), ("type", "u1"), ("_pad", "u1", (7,))], align=True)
assert EDGE_UPDATE.itemsize == 16

DL = dict(states=0, colors=1, bitmaps=2, hist=3, row_ptr=4, col=5, snapshot=6, highwater=7, hdmap=8, overflow=9,
          base_run=10, holes=11)


ABLATIONS = {"force_bitmap": 16, "no_overflow": 32, "live_deg": 64}  # SGC_OPT_ABL_*


class StreamGCError(RuntimeError):
    pass


class _Config(C.Structure):
    _fields_ = [("num_gpus", C.c_uint32), ("num_vertices", C.c_uint32), ("num_edges", C.c_uint64),
                ("stream_buffer_size", C.c_uint32), ("epoch_size", C.c_uint32),
                ("priority_refresh_interval", C.c_uint32), ("histogram_threshold", C.c_uint32),
                ("rebalance_threshold", C.c_float)]


class _Options(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("slack_pct", C.c_uint32), ("max_hist_colors", C.c_uint32),
                ("max_batch", C.c_uint32), ("device", C.c_int32), ("flags", C.c_uint32),
                ("full_repair_every", C.c_uint32), ("repair_tile", C.c_uint32)]


class RepairReport(C.Structure):
    _fields_ = [("tier1_iterations", C.c_uint32), ("tier1_last_count", C.c_uint32), ("tier2_ran", C.c_uint32),
                ("tier2_fixed", C.c_uint32), ("tier2_gave_up", C.c_uint32), ("drained", C.c_uint32),
                ("drain_failed", C.c_uint64), ("proper", C.c_uint32), ("incremental", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("_")}


class Stats(C.Structure):
    _fields_ = [("updates_submitted", C.c_uint64), ("updates_skipped", C.c_uint64), ("epochs", C.c_uint64),
                ("overflow_pending", C.c_uint64), ("overflow_lost", C.c_uint64), ("drain_failed", C.c_uint64),
                ("tier1_sweeps", C.c_uint64), ("tier2_runs", C.c_uint64), ("tier2_fixed", C.c_uint64),
                ("device_error", C.c_uint32), ("num_vertices", C.c_uint32), ("num_high_degree", C.c_uint32),
                ("max_hist_colors", C.c_uint32), ("total_slots", C.c_uint64), ("device_bytes", C.c_uint64),
                ("sweep_ms", C.c_double), ("sweep_count", C.c_uint64), ("sweep_bytes", C.c_uint64),
                ("live_entries", C.c_uint64), ("kernel_launches", C.c_uint64), ("h2d_bytes", C.c_uint64),
                ("d2h_bytes", C.c_uint64), ("sweep_phase_ms", C.c_double * 4),
                ("hub_deferred", C.c_uint64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["sweep_phase_ms"] = list(d["sweep_phase_ms"])
        return d


class Validation(C.Structure):
    _fields_ = [("violations", C.c_uint64), ("uncolored_with_edges", C.c_uint64), ("edges", C.c_uint64),
                ("max_color", C.c_uint64), ("out_of_range", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StateReport(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("bad_rows", C.c_uint64), ("flags", C.c_uint32), ("first_bad", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# sgc_state_report.flags bits
STATE_HW, STATE_TAIL, STATE_ID, STATE_RUN, STATE_HOLES, STATE_COLOR = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20


class _CSR(C.Structure):
    _fields_ = [("n", C.c_uint32), ("nnz", C.c_uint64), ("row_ptr", C.POINTER(C.c_uint64)),
                ("col_idx", C.POINTER(C.c_uint32)), ("degree", C.POINTER(C.c_uint32))]


_u8p, _u16p, _u32p, _u64p, _vp = (C.POINTER(C.c_uint8), C.POINTER(C.c_uint16), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint64), C.c_void_p)
_lib = None

# every exported entry point of include/streamgc_b200.h and csrc/sgc_host.h
class BatchGraph(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("epoch_size", C.c_uint32), ("histogram_threshold", C.c_uint32),
                ("_reserved", C.c_uint32), ("row_ptr", _u64p), ("col_idx", _u32p), ("degree", _u32p)]


class BatchOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("slack_pct", C.c_uint32), ("max_tick_updates", C.c_uint32),
                ("device", C.c_int32), ("flags", C.c_uint32), ("repair_tile", C.c_uint32),
                ("apply_blocks_per_sm", C.c_uint32), ("_reserved", C.c_uint32)]


class TickReport(C.Structure):
    _fields_ = [("updates", C.c_uint32), ("published", C.c_uint32), ("tier1_iterations", C.c_uint32),
                ("tier2_ran", C.c_uint32), ("proper", C.c_uint32), ("tier2_reason", C.c_uint32),
                ("device_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("_")}


class BatchTuning(C.Structure):
    _fields_ = [("repair_tile", C.c_uint32), ("apply_blocks_per_sm", C.c_uint32)]


BATCH_FEED = C.CFUNCTYPE(C.c_int, _vp, _vp)


class ServerOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("flags", C.c_uint32), ("hbm_budget_bytes", C.c_uint64),
                ("max_tick_updates", C.c_uint32), ("max_staleness_us", C.c_uint32), ("device", C.c_int32),
                ("slack_pct", C.c_uint32), ("regrow", C.c_uint32)]


class StepReport(C.Structure):
    _fields_ = [("admitted", C.c_uint32), ("groups_ticked", C.c_uint32), ("updates", C.c_uint32),
                ("published", C.c_uint32), ("requests_visible", C.c_uint32), ("proper", C.c_uint32),
                ("step_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("tenants_resident", C.c_uint64), ("tenants_queued", C.c_uint64), ("groups", C.c_uint64),
                ("resident_bytes", C.c_uint64), ("budget_bytes", C.c_uint64), ("update_requests", C.c_uint64),
                ("updates_applied", C.c_uint64), ("requests_visible", C.c_uint64), ("queries", C.c_uint64),
                ("query_vertices", C.c_uint64), ("visible_p50_ms", C.c_double), ("visible_p99_ms", C.c_double),
                ("query_p50_ms", C.c_double), ("query_p99_ms", C.c_double), ("ticks", C.c_uint64),
                ("tier1_sweeps", C.c_uint64), ("tier2_ticks", C.c_uint64), ("tier2_mirror_ticks", C.c_uint64),
                ("tick_device_ms", C.c_double), ("overflows", C.c_uint64), ("drain_failed", C.c_uint64),
                ("device_errors", C.c_uint64), ("tenants_regrown", C.c_uint64), ("requests_tracked", C.c_uint64),
                ("requests_dropped", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

SIGNATURES = {
    "sgc_default_options": (C.c_int, [C.POINTER(_Options)]),
    "sgc_create": (C.c_int, [C.POINTER(_Config), _u32p, _u32p, _u32p, C.POINTER(_vp)]),
    "sgc_create_ex": (C.c_int, [C.POINTER(_Config), C.POINTER(_Options), _u64p, _u32p, _u32p, C.POINTER(_vp)]),
    "sgc_destroy": (C.c_int, [_vp]),
    "sgc_apply": (C.c_int, [_vp, _vp, C.c_uint32, C.c_int]),
    "sgc_stage": (C.c_int, [_vp, C.c_void_p, C.c_uint32]),
    "sgc_apply_staged": (C.c_int, [_vp, C.c_int]),
    "sgc_epoch": (C.c_int, [_vp]),
    "sgc_drain_and_compact": (C.c_int, [_vp, C.POINTER(RepairReport)]),
    "sgc_repair": (C.c_int, [_vp, C.POINTER(RepairReport)]),
    "sgc_publish": (C.c_int, [_vp, C.POINTER(RepairReport)]),
    "sgc_process_stream": (C.c_int, [_vp, _vp, C.c_uint64, C.c_int, _u32p]),
    "sgc_query": (C.c_int, [_vp, _u32p, _u16p, C.c_uint32]),
    "sgc_query_noalloc": (C.c_int, [_vp, _u32p, _u16p, C.c_uint32]),
    "sgc_download": (C.c_int, [_vp, C.c_int, _vp, C.c_uint64]),
    "sgc_upload": (C.c_int, [_vp, C.c_int, _vp, C.c_uint64]),
    "sgc_color_core": (C.c_int, [_vp, C.c_uint32, _u32p]),
    "sgc_ring_create": (C.c_int, [_vp, C.c_uint32]),
    "sgc_ring_push": (C.c_int, [_vp, _vp, C.c_uint32, _u32p]),
    "sgc_ring_apply": (C.c_int, [_vp, C.c_uint32, C.c_int, _u32p]),
    "sgc_find_color": (C.c_int, [_vp, C.c_uint32, _u16p]),
    "sgc_validate": (C.c_int, [_vp, C.POINTER(Validation)]),
    "sgc_check_state": (C.c_int, [_vp, C.POINTER(StateReport)]),
    "sgc_get_stats": (C.c_int, [_vp, C.POINTER(Stats)]),
    "sgc_synchronize": (C.c_int, [_vp]),
    "sgc_cuda_stream": (_vp, [_vp]),
    "sgc_last_error": (C.c_char_p, []),
    "sgc_version": (C.c_char_p, []),
    "sgc_load_mtx": (C.c_int, [C.c_char_p, C.POINTER(_CSR)]),
    "sgc_csr_from_edges": (C.c_int, [C.c_uint32, _u32p, C.c_uint64, C.POINTER(_CSR)]),
    "sgc_csr_symmetrize": (C.c_int, [C.c_uint32, _u64p, _u32p, C.POINTER(_CSR)]),
    "sgc_csr_free": (None, [C.POINTER(_CSR)]),
    "sgc_write_mtx": (C.c_int, [C.c_char_p, C.POINTER(_CSR)]),
    "sgc_gen_init_stream": (C.c_uint64, [C.POINTER(_CSR), _u32p]),
    "sgc_gen_churn_stream": (C.c_int, [C.POINTER(_CSR), C.c_uint64, C.c_uint32, C.c_uint64, _u32p, _u8p]),
    "sgc_gen_kcore_stream": (C.c_int, [C.POINTER(_CSR), C.c_uint64, C.c_double, C.c_uint64, _u32p, _u8p, _u32p,
                                       _u32p]),
    "sgc_core_numbers": (C.c_int, [C.POINTER(_CSR), _u32p]),
    "sgc_gen_rmat": (C.c_int, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                               C.POINTER(_CSR)]),
    "sgc_gen_chung_lu": (C.c_int, [C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.POINTER(_CSR)]),
    "sgc_static_greedy": (C.c_uint32, [C.POINTER(_CSR)]),
    "sgc_write_coloring": (C.c_int, [C.c_char_p, _u16p, C.c_uint32]),
    "sgc_batch_default_options": (C.c_int, [C.POINTER(BatchOptions)]),
    "sgc_batch_create": (C.c_int, [C.POINTER(BatchGraph), C.c_uint32, C.POINTER(BatchOptions), C.POINTER(_vp)]),
    "sgc_batch_destroy": (C.c_int, [_vp]),
    "sgc_batch_num_graphs": (C.c_uint32, [_vp]),
    "sgc_batch_epoch_size": (C.c_uint32, [_vp, C.c_uint32]),
    "sgc_batch_submit": (C.c_int, [_vp, C.c_uint32, _vp, C.c_uint32]),
    "sgc_batch_pending": (C.c_uint64, [_vp]),
    "sgc_batch_tick": (C.c_int, [_vp, C.POINTER(TickReport)]),
    "sgc_batch_close_epochs": (C.c_int, [_vp]),
    "sgc_batch_query": (C.c_int, [_vp, C.c_uint32, _u32p, _u16p, C.c_uint32]),
    "sgc_batch_snapshot": (C.c_int, [_vp, C.c_uint32, _u16p]),
    "sgc_batch_rows": (C.c_int, [_vp, C.c_uint32, _u64p, _u32p, C.c_uint64]),
    "sgc_batch_color_core": (C.c_int, [_vp, C.c_uint32, _u32p]),
    "sgc_batch_validate": (C.c_int, [_vp, C.POINTER(Validation)]),
    "sgc_batch_check_state": (C.c_int, [_vp, C.POINTER(StateReport)]),
    "sgc_batch_dropped": (C.c_int, [_vp, _u8p]),
    "sgc_batch_set_thresholds": (C.c_int, [_vp, C.c_uint32]),
    "sgc_batch_get_tuning": (C.c_int, [_vp, C.POINTER(BatchTuning)]),
    "sgc_batch_set_tuning": (C.c_int, [_vp, C.POINTER(BatchTuning)]),
    "sgc_batch_autotune": (C.c_int, [_vp, BATCH_FEED, _vp, C.c_uint32, C.POINTER(BatchTuning)]),
    "sgc_batch_stats": (C.c_int, [_vp, C.POINTER(Stats)]),
    "sgc_batch_tick_begin": (C.c_int, [_vp]),
    "sgc_batch_tick_end": (C.c_int, [_vp, C.POINTER(TickReport)]),
    "sgc_batch_close_epoch": (C.c_int, [_vp, C.c_uint32]),
    "sgc_batch_publish_count": (C.c_uint64, [_vp, C.c_uint32]),
    "sgc_server_default_options": (C.c_int, [C.POINTER(ServerOptions)]),
    "sgc_server_create": (C.c_int, [C.POINTER(ServerOptions), C.POINTER(_vp)]),
    "sgc_server_destroy": (C.c_int, [_vp]),
    "sgc_tenant_footprint": (C.c_uint64, [C.c_uint32, C.c_uint64, C.c_uint32]),
    "sgc_server_add_tenant": (C.c_int, [_vp, C.POINTER(BatchGraph), _u32p]),
    "sgc_server_remove_tenant": (C.c_int, [_vp, C.c_uint32]),
    "sgc_server_tenant_state": (C.c_int, [_vp, C.c_uint32]),
    "sgc_server_submit": (C.c_int, [_vp, C.c_uint32, _vp, C.c_uint32, C.POINTER(C.c_uint64)]),
    "sgc_server_query": (C.c_int, [_vp, C.c_uint32, _u32p, _u16p, C.c_uint32]),
    "sgc_server_step": (C.c_int, [_vp, C.POINTER(StepReport)]),
    "sgc_server_request_visible": (C.c_int, [_vp, C.c_uint64]),
    "sgc_server_snapshot": (C.c_int, [_vp, C.c_uint32, _u16p]),
    "sgc_server_get_stats": (C.c_int, [_vp, C.POINTER(ServerStats)]),
    "sgc_server_rows": (C.c_int, [_vp, C.c_uint32, _u64p, _u32p, C.c_uint64]),
}


def lib():
    """Loads libstreamgc_b200.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise StreamGCError(f"{LIB_PATH} is missing: run __graft_entry__.build() (make -C streamgc_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        msg = lib().sgc_last_error().decode(errors="replace")
        raise StreamGCError(f"{what} failed ({rc}): {msg}")


def _p(a, t):
    return a.ctypes.data_as(t)


def updates_from(pairs, types=None):
    """(k,2) uint32 pairs + uint8 types (0=ADD, 1=DEL; default ADD) -> EdgeUpdate records."""
    pairs = np.asarray(pairs, dtype=np.uint32).reshape(-1, 2)
    ups = np.zeros(len(pairs), dtype=EDGE_UPDATE)
    ups["u"] = pairs[:, 0]
    ups["v"] = pairs[:, 1]
    if types is not None:
        ups["type"] = np.asarray(types, dtype=np.uint8)
    return ups


class Graph:
    """Host CSR (64-bit row offsets, ascending rows, symmetric, no self loops)."""

    def __init__(self, row_ptr, col_idx, degree=None):
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.uint64)
        self.col_idx = np.ascontiguousarray(col_idx, dtype=np.uint32)
        self.n = len(self.row_ptr) - 1
        self.degree = (np.ascontiguousarray(degree, dtype=np.uint32) if degree is not None
                       else np.diff(self.row_ptr).astype(np.uint32))

    @property
    def nnz(self):
        return int(self.row_ptr[-1])

    def _c(self):
        c = _CSR()
        c.n = self.n
        c.nnz = self.nnz
        c.row_ptr = _p(self.row_ptr, _u64p)
        c.col_idx = _p(self.col_idx, _u32p)
        c.degree = _p(self.degree, _u32p)
        return c

    @staticmethod
    def _take(c):
        g = Graph(np.ctypeslib.as_array(c.row_ptr, (c.n + 1,)).copy(),
                  np.ctypeslib.as_array(c.col_idx, (max(c.nnz, 1),))[: c.nnz].copy(),
                  np.ctypeslib.as_array(c.degree, (max(c.n, 1),))[: c.n].copy())
        lib().sgc_csr_free(C.byref(c))
        return g

    @staticmethod
    def load_mtx(path):
        c = _CSR()
        _check(lib().sgc_load_mtx(path.encode(), C.byref(c)), f"load_mtx({path})")
        return Graph._take(c)

    @staticmethod
    def from_edges(n, pairs):
        pairs = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1, 2)
        c = _CSR()
        _check(lib().sgc_csr_from_edges(n, _p(pairs, _u32p), len(pairs), C.byref(c)), "csr_from_edges")
        return Graph._take(c)

    @staticmethod
    def symmetrized(row_ptr, col):
        """The graph of rows that may miss mirror entries: an edge is kept when
        either direction is present."""
        rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
        cl = np.ascontiguousarray(col, dtype=np.uint32)
        c = _CSR()
        _check(lib().sgc_csr_symmetrize(len(rp) - 1, _p(rp, _u64p), _p(cl, _u32p), C.byref(c)), "csr_symmetrize")
        return Graph._take(c)

    @staticmethod
    def rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=42):
        cs = _CSR()
        _check(lib().sgc_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(cs)), "gen_rmat")
        return Graph._take(cs)

    @staticmethod
    def chung_lu(n, exponent=2.1, avg_degree=17.0, max_degree=100000.0, seed=42):
        cs = _CSR()
        _check(lib().sgc_gen_chung_lu(n, exponent, avg_degree, max_degree, seed, C.byref(cs)), "gen_chung_lu")
        return Graph._take(cs)

    @staticmethod
    def delaunay(n, seed=42):
        """Delaunay triangulation of n uniform points in the unit square (scipy/Qhull)."""
        from scipy.spatial import Delaunay
        pts = np.random.default_rng(seed).random((n, 2))
        tri = Delaunay(pts).simplices.astype(np.uint32)
        e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [0, 2]]])
        return Graph.from_edges(n, e)

    def write_mtx(self, path):
        c = self._c()
        _check(lib().sgc_write_mtx(path.encode(), C.byref(c)), "write_mtx")

    def init_stream(self):
        out = np.zeros(max(self.nnz, 2), dtype=np.uint32)
        c = self._c()
        k = lib().sgc_gen_init_stream(C.byref(c), _p(out, _u32p))
        return updates_from(out[: 2 * k].reshape(-1, 2))

    def churn_stream(self, size, insert_pct=50, seed=42):
        pairs = np.zeros(2 * size, dtype=np.uint32)
        types = np.zeros(size, dtype=np.uint8)
        c = self._c()
        _check(lib().sgc_gen_churn_stream(C.byref(c), size, insert_pct, seed, _p(pairs, _u32p), _p(types, _u8p)),
               "gen_churn_stream")
        return updates_from(pairs.reshape(-1, 2), types)

    def kcore_stream(self, size, percentile=90.0, seed=42):
        pairs = np.zeros(2 * size, dtype=np.uint32)
        types = np.zeros(size, dtype=np.uint8)
        k = np.zeros(1, dtype=np.uint32)
        cs = np.zeros(1, dtype=np.uint32)
        c = self._c()
        _check(lib().sgc_gen_kcore_stream(C.byref(c), size, percentile, seed, _p(pairs, _u32p), _p(types, _u8p),
                                          _p(k, _u32p), _p(cs, _u32p)), "gen_kcore_stream")
        return updates_from(pairs.reshape(-1, 2), types), int(k[0]), int(cs[0])

    def core_numbers(self):
        out = np.zeros(self.n, dtype=np.uint32)
        c = self._c()
        _check(lib().sgc_core_numbers(C.byref(c), _p(out, _u32p)), "core_numbers")
        return out

    def static_greedy(self):
        c = self._c()
        return int(lib().sgc_static_greedy(C.byref(c)))


def write_coloring(path, colors):
    colors = np.ascontiguousarray(colors, dtype=np.uint16)
    _check(lib().sgc_write_coloring(path.encode(), _p(colors, _u16p), len(colors)), "write_coloring")


class StreamGC:
    """One graph resident on one GPU (a handle of the C ABI)."""

    def __init__(self, graph: Graph, epoch_size=32768, histogram_threshold=64, slack_pct=300,
                 max_hist_colors=1024, max_batch=32768, device=0, profile=False, exact_select=False,
                 full_repair_every=None, repair_tile=None, graph_publish=False, sorted_rows=False, ablations=()):
        """ablations: names among "force_bitmap", "no_overflow", "live_deg" -- the
        reference's ablation builds, with its rules (not with exact_select)."""
        L = lib()
        cfg = _Config(1, graph.n, graph.nnz, 1 << 20, epoch_size, 100, histogram_threshold, 0.2)
        opt = _Options()
        L.sgc_default_options(C.byref(opt))
        opt.slack_pct, opt.max_hist_colors, opt.max_batch, opt.device = slack_pct, max_hist_colors, max_batch, device
        opt.flags = (1 if profile else 0) | (2 if exact_select else 0) | (4 if graph_publish else 0) | \
            (8 if sorted_rows else 0) | sum(ABLATIONS[a] for a in ablations)
        if full_repair_every is not None:
            opt.full_repair_every = full_repair_every
        if repair_tile is not None:
            opt.repair_tile = repair_tile
        self.h = _vp()
        self.graph = graph
        self.n = graph.n
        self.max_batch = max_batch
        self.epoch_size = epoch_size
        _check(L.sgc_create_ex(C.byref(cfg), C.byref(opt), _p(graph.row_ptr, _u64p), _p(graph.col_idx, _u32p),
                               _p(graph.degree, _u32p), C.byref(self.h)), "sgc_create_ex")
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            lib().sgc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- stepping ----
    def apply(self, ups, mode=MODE_DETERMINISTIC):
        """Host EdgeUpdate array (numpy) or a device pointer (int) with an explicit count via apply_ptr."""
        ups = np.ascontiguousarray(ups, dtype=EDGE_UPDATE)
        for s in range(0, len(ups), self.max_batch):
            part = ups[s: s + self.max_batch]
            _check(lib().sgc_apply(self.h, part.ctypes.data, len(part), mode), "sgc_apply")

    def stage(self, ups):
        """Copies a host batch (<= max_batch updates) into the next ingest slot
        without waiting for the GPU; apply it later with apply_staged()."""
        ups = np.ascontiguousarray(ups, dtype=EDGE_UPDATE)
        _check(lib().sgc_stage(self.h, ups.ctypes.data, len(ups)), "sgc_stage")

    def stage_ptr(self, ptr, n):
        """stage() for updates at a pinned host or device address (unchanged until applied)."""
        _check(lib().sgc_stage(self.h, C.c_void_p(ptr), n), "sgc_stage")

    def apply_staged(self, mode=MODE_CONCURRENT):
        """Applies the oldest staged batch once its copy is done."""
        _check(lib().sgc_apply_staged(self.h, mode), "sgc_apply_staged")

    def ring_create(self, log2_slots):
        """A pinned, device-mapped ingest ring of 2**log2_slots update slots."""
        _check(lib().sgc_ring_create(self.h, log2_slots), "ring_create")

    def ring_push(self, ups, offset=0):
        """Appends ups[offset:] to the ring (any one producer thread; no CUDA
        call); returns how many fit."""
        out = np.zeros(1, dtype=np.uint32)
        _check(lib().sgc_ring_push(self.h, ups.ctypes.data + 16 * offset, len(ups) - offset, _p(out, _u32p)),
               "ring_push")
        return int(out[0])

    def ring_push_ptr(self, ptr, n):
        out = np.zeros(1, dtype=np.uint32)
        _check(lib().sgc_ring_push(self.h, ptr, n, _p(out, _u32p)), "ring_push")
        return int(out[0])

    def ring_apply(self, max_updates, mode=MODE_CONCURRENT):
        """The GPU copies up to max_updates published slots from the ring and
        applies them; returns how many."""
        out = np.zeros(1, dtype=np.uint32)
        _check(lib().sgc_ring_apply(self.h, max_updates, mode, _p(out, _u32p)), "ring_apply")
        return int(out[0])

    def apply_ptr(self, ptr, n, mode=MODE_CONCURRENT):
        """Updates already in device (or pinned host) memory at address `ptr`."""
        _check(lib().sgc_apply(self.h, C.c_void_p(ptr), n, mode), "sgc_apply")

    def epoch(self):
        _check(lib().sgc_epoch(self.h), "sgc_epoch")

    def drain_and_compact(self):
        r = RepairReport()
        _check(lib().sgc_drain_and_compact(self.h, C.byref(r)), "sgc_drain_and_compact")
        return r.as_dict()

    def repair(self):
        r = RepairReport()
        _check(lib().sgc_repair(self.h, C.byref(r)), "sgc_repair")
        return r.as_dict()

    def publish(self):
        r = RepairReport()
        _check(lib().sgc_publish(self.h, C.byref(r)), "sgc_publish")
        return r.as_dict()

    def process_stream(self, ups, mode=MODE_DETERMINISTIC):
        ups = np.ascontiguousarray(ups, dtype=EDGE_UPDATE)
        ne = np.zeros(1, dtype=np.uint32)
        _check(lib().sgc_process_stream(self.h, ups.ctypes.data, len(ups), mode, _p(ne, _u32p)),
               "sgc_process_stream")
        return int(ne[0])

    def synchronize(self):
        _check(lib().sgc_synchronize(self.h), "sgc_synchronize")

    def cuda_stream(self):
        return lib().sgc_cuda_stream(self.h)

    # ---- reads ----
    def query(self, vertices):
        v = np.ascontiguousarray(vertices, dtype=np.uint32)
        out = np.zeros(len(v), dtype=np.uint16)
        _check(lib().sgc_query(self.h, _p(v, _u32p), _p(out, _u16p), len(v)), "sgc_query")
        return out

    def query_noalloc(self, vertices):
        """Like query(), without any device allocation (fixed scratch, at most
        65536 vertices per call; calls overlapping on the GPU race)."""
        v = np.ascontiguousarray(vertices, dtype=np.uint32)
        out = np.zeros(len(v), dtype=np.uint16)
        _check(lib().sgc_query_noalloc(self.h, _p(v, _u32p), _p(out, _u16p), len(v)), "sgc_query_noalloc")
        return out

    def stats(self):
        s = Stats()
        rc = lib().sgc_get_stats(self.h, C.byref(s))
        d = s.as_dict()
        if rc not in (0, -4):
            _check(rc, "sgc_get_stats")
        return d

    def _dl(self, what, dtype, count):
        out = np.zeros(count, dtype=dtype)
        _check(lib().sgc_download(self.h, DL[what], out.ctypes.data, out.nbytes), f"download {what}")
        return out

    def download_into(self, what, ptr, nbytes):
        """Copies a device array (see DL) into caller memory at address `ptr`."""
        _check(lib().sgc_download(self.h, DL[what], ptr, nbytes), f"download {what}")

    def base_runs(self):
        return self._dl("base_run", np.uint32, self.n)

    def holes(self):
        return self._dl("holes", np.uint32, self.n)

    def states(self):
        return self._dl("states", np.uint32, self.n)

    def colors(self):
        return self._dl("colors", np.uint16, self.n)

    def bitmaps(self):
        return self._dl("bitmaps", np.uint64, self.n)

    def hist(self):
        s = self.stats()
        rows = s["num_high_degree"] if s["max_hist_colors"] else 0
        return self._dl("hist", np.uint32, rows * s["max_hist_colors"])

    def row_ptr(self):
        return self._dl("row_ptr", np.uint64, self.n + 1)

    def col(self):
        return self._dl("col", np.uint32, self.stats()["total_slots"])

    def snapshot(self):
        return self._dl("snapshot", np.uint16, self.n)

    def highwater(self):
        return self._dl("highwater", np.uint32, self.n)

    def hdmap(self):
        return self._dl("hdmap", np.uint32, self.n)

    def overflow(self):
        pend = self.stats()["overflow_pending"]
        return self._dl("overflow", np.uint32, 2 * min(pend, 262144)).reshape(-1, 2)

    def upload(self, what, arr):
        arr = np.ascontiguousarray(arr)
        _check(lib().sgc_upload(self.h, DL[what], arr.ctypes.data, arr.nbytes), f"upload {what}")

    def color_core(self, min_degree):
        """Colors the uncolored vertices of degree >= min_degree one at a time in
        descending degree order (first free color); returns how many."""
        out = np.zeros(1, dtype=np.uint32)
        _check(lib().sgc_color_core(self.h, min_degree, _p(out, _u32p)), "color_core")
        return int(out[0])

    def find_color(self, x):
        c = np.zeros(1, dtype=np.uint16)
        _check(lib().sgc_find_color(self.h, x, _p(c, _u16p)), "sgc_find_color")
        return int(c[0])

    def validate(self):
        v = Validation()
        _check(lib().sgc_validate(self.h, C.byref(v)), "sgc_validate")
        return v.as_dict()

    def check_state(self):
        """Layout invariants of every row (STATE_* bits in `flags`)."""
        r = StateReport()
        _check(lib().sgc_check_state(self.h, C.byref(r)), "sgc_check_state")
        return r.as_dict()


def version():
    return lib().sgc_version().decode()


BATCH_CUDA_GRAPH = 1
BATCH_STREAM_ORDER = 2
BATCH_PROFILE = 4
BATCH_SORTED_ROWS = 8


class Batch:
    """Many graphs resident on one GPU (include/streamgc_batch.h): updates are
    submitted per graph in the graph's own ids; tick() applies everything
    submitted in one persistent launch, repairs, and publishes each graph whose
    epoch closed."""

    def __init__(self, graphs, epoch_sizes=None, thresholds=None, max_tick_updates=1 << 20, slack_pct=300,
                 device=0, cuda_graph=True, stream_order=False, profile=False, repair_tile=0, apply_blocks_per_sm=0,
                 sorted_rows=False):
        L = lib()
        self.graphs = list(graphs)
        G = len(self.graphs)
        arr = (BatchGraph * G)()
        for k, g in enumerate(self.graphs):
            arr[k].num_vertices = g.n
            arr[k].epoch_size = int(epoch_sizes[k]) if epoch_sizes is not None else 0
            arr[k].histogram_threshold = int(thresholds[k]) if thresholds is not None else 0
            arr[k].row_ptr = _p(g.row_ptr, _u64p)
            arr[k].col_idx = _p(g.col_idx, _u32p)
            arr[k].degree = _p(g.degree, _u32p)
        opt = BatchOptions()
        L.sgc_batch_default_options(C.byref(opt))
        opt.slack_pct, opt.max_tick_updates, opt.device = slack_pct, max_tick_updates, device
        opt.flags = (BATCH_CUDA_GRAPH if cuda_graph else 0) | (BATCH_STREAM_ORDER if stream_order else 0) | \
            (BATCH_PROFILE if profile else 0) | (BATCH_SORTED_ROWS if sorted_rows else 0)
        opt.repair_tile, opt.apply_blocks_per_sm = repair_tile, apply_blocks_per_sm
        self.b = _vp()
        _check(L.sgc_batch_create(arr, G, C.byref(opt), C.byref(self.b)), "sgc_batch_create")
        self.G = G

    def close(self):
        if getattr(self, "b", None):
            lib().sgc_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def epoch_size(self, k):
        return lib().sgc_batch_epoch_size(self.b, k)

    def submit(self, k, ups):
        ups = np.ascontiguousarray(ups, dtype=EDGE_UPDATE)
        _check(lib().sgc_batch_submit(self.b, k, ups.ctypes.data, len(ups)), "sgc_batch_submit")

    def pending(self):
        return lib().sgc_batch_pending(self.b)

    def tick(self):
        r = TickReport()
        _check(lib().sgc_batch_tick(self.b, C.byref(r)), "sgc_batch_tick")
        return r.as_dict()

    def tick_begin(self):
        """Launches the tick and returns; submits for the next tick may follow."""
        _check(lib().sgc_batch_tick_begin(self.b), "sgc_batch_tick_begin")

    def tick_end(self):
        r = TickReport()
        _check(lib().sgc_batch_tick_end(self.b, C.byref(r)), "sgc_batch_tick_end")
        return r.as_dict()

    def close_epochs(self):
        _check(lib().sgc_batch_close_epochs(self.b), "sgc_batch_close_epochs")

    def query(self, k, vertices):
        v = np.ascontiguousarray(vertices, dtype=np.uint32)
        out = np.zeros(len(v), dtype=np.uint16)
        _check(lib().sgc_batch_query(self.b, k, _p(v, _u32p), _p(out, _u16p), len(v)), "sgc_batch_query")
        return out

    def snapshot(self, k):
        out = np.zeros(self.graphs[k].n, dtype=np.uint16)
        _check(lib().sgc_batch_snapshot(self.b, k, _p(out, _u16p)), "sgc_batch_snapshot")
        return out

    def rows(self, k):
        """The graph's live rows (its own ids): (row_ptr, col)."""
        n = self.graphs[k].n
        rp = np.zeros(n + 1, dtype=np.uint64)
        _check(lib().sgc_batch_rows(self.b, k, _p(rp, _u64p), None, 0), "sgc_batch_rows")
        col = np.zeros(max(int(rp[-1]), 1), dtype=np.uint32)
        _check(lib().sgc_batch_rows(self.b, k, _p(rp, _u64p), _p(col, _u32p), len(col)), "sgc_batch_rows")
        return rp, col[: int(rp[-1])]

    def color_core(self, min_degree):
        """sgc_color_core over every graph (before the first tick); returns how many were colored."""
        out = np.zeros(1, dtype=np.uint32)
        _check(lib().sgc_batch_color_core(self.b, min_degree, _p(out, _u32p)), "sgc_batch_color_core")
        return int(out[0])

    def validate(self):
        v = Validation()
        _check(lib().sgc_batch_validate(self.b, C.byref(v)), "sgc_batch_validate")
        return v.as_dict()

    def check_state(self):
        r = StateReport()
        _check(lib().sgc_batch_check_state(self.b, C.byref(r)), "sgc_batch_check_state")
        return r.as_dict()

    def dropped(self):
        """Per graph: 1 when the graph has dropped an entry (full row / full overflow buffer)."""
        out = np.zeros(len(self.graphs), dtype=np.uint8)
        _check(lib().sgc_batch_dropped(self.b, _p(out, _u8p)), "sgc_batch_dropped")
        return out

    def set_thresholds(self, thr):
        _check(lib().sgc_batch_set_thresholds(self.b, thr), "sgc_batch_set_thresholds")

    def tuning(self):
        t = BatchTuning()
        _check(lib().sgc_batch_get_tuning(self.b, C.byref(t)), "sgc_batch_get_tuning")
        return {"repair_tile": t.repair_tile, "apply_blocks_per_sm": t.apply_blocks_per_sm}

    def set_tuning(self, repair_tile, apply_blocks_per_sm):
        t = BatchTuning(repair_tile, apply_blocks_per_sm)
        _check(lib().sgc_batch_set_tuning(self.b, C.byref(t)), "sgc_batch_set_tuning")

    def autotune(self, feed, ticks_per_candidate=2):
        """feed(): stages one tick's updates. Returns the chosen tuning."""
        def _cb(_b, _ctx):
            try:
                feed()
                return 0
            except Exception:
                return -1
        cb = BATCH_FEED(_cb)
        t = BatchTuning()
        _check(lib().sgc_batch_autotune(self.b, cb, None, ticks_per_candidate, C.byref(t)), "sgc_batch_autotune")
        return {"repair_tile": t.repair_tile, "apply_blocks_per_sm": t.apply_blocks_per_sm}

    def stats(self):
        st = Stats()
        _check(lib().sgc_batch_stats(self.b, C.byref(st)), "sgc_batch_stats")
        return st.as_dict()


TENANT_QUEUED, TENANT_RESIDENT, TENANT_REMOVED = 0, 1, 2


class Server:
    """Request loop over many tenant graphs on one GPU (include/streamgc_server.h).
    submit() and query() may be called from other threads while step() runs."""

    def __init__(self, hbm_budget_bytes=150 << 30, max_tick_updates=1 << 20, max_staleness_us=0, device=0,
                 slack_pct=300, cuda_graph=True, stream_order=False, profile=False, regrow=False, sorted_rows=False):
        L = lib()
        opt = ServerOptions()
        L.sgc_server_default_options(C.byref(opt))
        opt.regrow = 1 if regrow else 0
        opt.hbm_budget_bytes = hbm_budget_bytes
        opt.max_tick_updates = max_tick_updates
        opt.max_staleness_us = max_staleness_us
        opt.device, opt.slack_pct = device, slack_pct
        opt.flags = (BATCH_CUDA_GRAPH if cuda_graph else 0) | (BATCH_STREAM_ORDER if stream_order else 0) | \
            (BATCH_PROFILE if profile else 0) | (BATCH_SORTED_ROWS if sorted_rows else 0)
        self.s = _vp()
        _check(L.sgc_server_create(C.byref(opt), C.byref(self.s)), "sgc_server_create")
        self.n = {}

    def close(self):
        if getattr(self, "s", None):
            lib().sgc_server_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def footprint(n, entries, slack_pct=300):
        return lib().sgc_tenant_footprint(n, entries, slack_pct)

    def add_tenant(self, graph, epoch_size=0, histogram_threshold=0):
        g = BatchGraph(graph.n, epoch_size, histogram_threshold, 0, _p(graph.row_ptr, _u64p),
                       _p(graph.col_idx, _u32p), _p(graph.degree, _u32p))
        t = np.zeros(1, dtype=np.uint32)
        _check(lib().sgc_server_add_tenant(self.s, C.byref(g), _p(t, _u32p)), "sgc_server_add_tenant")
        self.n[int(t[0])] = graph.n
        return int(t[0])

    def remove_tenant(self, t):
        _check(lib().sgc_server_remove_tenant(self.s, t), "sgc_server_remove_tenant")

    def state(self, t):
        return lib().sgc_server_tenant_state(self.s, t)

    def submit(self, t, ups):
        ups = np.ascontiguousarray(ups, dtype=EDGE_UPDATE)
        rid = C.c_uint64(0)
        _check(lib().sgc_server_submit(self.s, t, ups.ctypes.data, len(ups), C.byref(rid)), "sgc_server_submit")
        return rid.value

    def query(self, t, vertices):
        v = np.ascontiguousarray(vertices, dtype=np.uint32)
        out = np.zeros(len(v), dtype=np.uint16)
        _check(lib().sgc_server_query(self.s, t, _p(v, _u32p), _p(out, _u16p), len(v)), "sgc_server_query")
        return out

    def step(self):
        r = StepReport()
        _check(lib().sgc_server_step(self.s, C.byref(r)), "sgc_server_step")
        return r.as_dict()

    def visible(self, request):
        return lib().sgc_server_request_visible(self.s, request) == 1

    def snapshot(self, t):
        out = np.zeros(self.n[t], dtype=np.uint16)
        _check(lib().sgc_server_snapshot(self.s, t, _p(out, _u16p)), "sgc_server_snapshot")
        return out

    def rows(self, t):
        """A resident tenant's live rows (its own ids): (row_ptr, col). Between steps."""
        n = self.n[t]
        rp = np.zeros(n + 1, dtype=np.uint64)
        _check(lib().sgc_server_rows(self.s, t, _p(rp, _u64p), None, 0), "sgc_server_rows")
        col = np.zeros(max(int(rp[-1]), 1), dtype=np.uint32)
        _check(lib().sgc_server_rows(self.s, t, _p(rp, _u64p), _p(col, _u32p), len(col)), "sgc_server_rows")
        return rp, col[: int(rp[-1])]

    def stats(self):
        st = ServerStats()
        _check(lib().sgc_server_get_stats(self.s, C.byref(st)), "sgc_server_get_stats")
        return st.as_dict()
