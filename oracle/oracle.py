"""CPU oracle binding -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over oracle/lib/liboracle.so (the C++ restatement of the
reference's single-GPU coloring path, oracle/sgc_oracle.cpp) and over
oracle/_ref/libref_host.so (the reference's own stream generator and .mtx
loader compiled from its sources). Only tests, the smoke entry point and the
bench's CPU-baseline leg import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liboracle.so")
REF_HOST_PATH = os.path.join(HERE, "_ref", "libref_host.so")

EDGE_UPDATE = np.dtype([("u", "<u4"), ("v", "<u4"), ("type", "u1"), ("_pad", "u1", (7,))], align=True)
assert EDGE_UPDATE.itemsize == 16

_u8p = C.POINTER(C.c_uint8)
_u16p = C.POINTER(C.c_uint16)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_vp = C.c_void_p


def _p(arr, ct):
    return arr.ctypes.data_as(ct)


def build():
    """Compile the oracle (and, when the reference sources exist here, the
    reference-built checkers) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "lib/liboracle.so"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        sig = {
            "og_create": (_vp, [C.c_uint32, _u64p, _u32p, _u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]),
            "og_destroy": (None, [_vp]),
            "og_num_vertices": (C.c_uint32, [_vp]),
            "og_total_slots": (C.c_uint64, [_vp]),
            "og_num_high_degree": (C.c_uint32, [_vp]),
            "og_max_hist_colors": (C.c_uint32, [_vp]),
            "og_apply": (None, [_vp, _vp, C.c_uint64]),
            "og_epoch": (None, [_vp]),
            "og_drain_and_compact": (C.c_uint64, [_vp]),
            "og_snapshot": (None, [_vp]),
            "og_compact": (None, [_vp]),
            "og_drain_pending": (C.c_uint64, [_vp]),
            "og_rebuild_bitmaps": (None, [_vp]),
            "og_tier1_sweep": (C.c_uint32, [_vp]),
            "og_tier1": (C.c_int, [_vp, _u32p, C.c_int, _u32p]),
            "og_tier2": (C.c_uint32, [_vp]),
            "og_process_stream": (C.c_uint32, [_vp, _vp, C.c_uint64, C.c_uint32, C.c_uint32]),
            "og_process_stream_repaired": (C.c_uint32, [_vp, _vp, C.c_uint64, C.c_uint32, C.c_uint32]),
            "og_phase_end": (C.c_uint32, [_vp, C.POINTER(C.c_int), _u32p]),
            "og_load_state": (None, [_vp, _u32p, _u32p, _u64p, _u32p]),
            "og_col_data": (C.c_void_p, [_vp]),
            "og_load_rows_model": (None, [_vp, _u32p, _u32p, _u32p]),
            "og_color_greedy": (C.c_uint16, [_vp]),
            "og_color_core": (C.c_uint32, [_vp, C.c_uint32]),
            "og_load_state_inplace": (None, [_vp, _u64p, _u32p, _u32p, _u64p, _u32p]),
            "og_publish_repair": (None, [_vp, C.c_int, _u32p]),
            "og_set_full_repair_every": (None, [_vp, C.c_uint32]),
            "og_set_repair_state": (None, [_vp, C.c_int, C.c_int]),
            "og_get_states": (None, [_vp, _u32p]),
            "og_set_states": (None, [_vp, _u32p]),
            "og_get_bitmaps": (None, [_vp, _u64p]),
            "og_get_hdmap": (None, [_vp, _u32p]),
            "og_get_hist": (None, [_vp, _u32p]),
            "og_get_row_ptr": (None, [_vp, _u64p]),
            "og_get_col": (None, [_vp, _u32p]),
            "og_get_snapshot": (None, [_vp, _u16p]),
            "og_overflow_count": (C.c_uint32, [_vp]),
            "og_get_overflow": (None, [_vp, _u32p, C.c_uint32]),
            "og_counters": (None, [_vp, _u64p]),
            "og_reset_bytes": (None, [_vp]),
            "og_fac": (C.c_uint16, [_vp, C.c_uint32]),
            "og_set_bitmap": (None, [_vp, C.c_uint32, C.c_uint64]),
            "og_set_hist_row": (None, [_vp, C.c_uint32, _u32p, C.c_uint32]),
            "og_validate": (None, [_vp, _u64p]),
            "og_validate_colors": (None, [C.c_uint32, _u64p, _u32p, _u16p, _u64p]),
            "og_static_greedy": (C.c_uint16, [C.c_uint32, _u64p, _u32p]),
            "og_gen_init_stream": (C.c_uint64, [C.c_uint32, _u64p, _u32p, _u32p, _u32p]),
            "og_gen_bench_stream": (None, [C.c_uint32, _u64p, _u32p, C.c_uint64, C.c_uint32, C.c_uint64,
                                           _u32p, _u8p]),
            "og_load_mtx": (_vp, [C.c_char_p]),
            "og_loaded_n": (C.c_uint32, [_vp]),
            "og_loaded_nnz": (C.c_uint64, [_vp]),
            "og_loaded_copy": (None, [_vp, _u64p, _u32p, _u32p]),
            "og_loaded_free": (None, [_vp]),
            "og_num_threads": (C.c_int, []),
            "og_set_threads": (None, [C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


ABLATIONS = {"force_bitmap": 4, "no_overflow": 8, "live_deg": 16}


def updates_from(pairs, types=None):
    """Pack (k,2) uint32 pairs and uint8 types (0=ADD,1=DEL) into EdgeUpdate records."""
    pairs = np.asarray(pairs, dtype=np.uint32).reshape(-1, 2)
    ups = np.zeros(len(pairs), dtype=EDGE_UPDATE)
    ups["u"] = pairs[:, 0]
    ups["v"] = pairs[:, 1]
    if types is not None:
        ups["type"] = np.asarray(types, dtype=np.uint8)
    return ups


class Oracle:
    """Single-GPU StreamGC state restated on the CPU (sequential, stream order)."""

    def __init__(self, row_ptr, col, degree, hist_threshold=64, slack_pct=300, max_hist_colors=1024,
                 exact=False, conc=False, ablations=()):
        """exact: exact color selection above the threshold and the independent-set
        Tier-1 (the concurrent configuration's rules); default: the reference's.
        conc (with exact): also the concurrent apply's row layout and update
        rules (sorted base runs with tombstones, tail inserts, scans bounded by
        the high-water mark, lazy compaction, early-exit color reduction), so
        that the byte counters count what those rules read and write.
        ablations: names among "force_bitmap", "no_overflow", "live_deg" (the
        reference's ablation builds; reference rules only)."""
        self.L = lib()
        rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
        col = np.ascontiguousarray(col, dtype=np.uint32)
        deg = np.ascontiguousarray(degree, dtype=np.uint32)
        self.n = len(rp) - 1
        self.h = self.L.og_create(self.n, _p(rp, _u64p), _p(col, _u32p), _p(deg, _u32p),
                                  hist_threshold, slack_pct, max_hist_colors,
                                  (1 if exact else 0) | (2 if exact and conc else 0) |
                                  sum(ABLATIONS[a] for a in ablations))

    def close(self):
        if self.h:
            self.L.og_destroy(self.h)
            self.h = None

    __del__ = close

    # --- stepping ---
    def apply(self, ups):
        ups = np.ascontiguousarray(ups, dtype=EDGE_UPDATE)
        self.L.og_apply(self.h, ups.ctypes.data, len(ups))

    def epoch(self):
        self.L.og_epoch(self.h)

    def drain_and_compact(self):
        return self.L.og_drain_and_compact(self.h)

    def tier1(self):
        hist = np.zeros(20, dtype=np.uint32)
        last = np.zeros(1, dtype=np.uint32)
        it = self.L.og_tier1(self.h, _p(hist, _u32p), 20, _p(last, _u32p))
        return it, hist[:it].tolist()

    def tier2(self):
        return self.L.og_tier2(self.h)

    def phase_end(self):
        it = C.c_int(0)
        last = np.zeros(1, dtype=np.uint32)
        fixed = self.L.og_phase_end(self.h, C.byref(it), _p(last, _u32p))
        return it.value, int(last[0]), fixed

    def publish_repair(self, force_full=False):
        """Compact, drain, repair, snapshot as the library's sgc_publish does under
        exact selection (incremental when allowed)."""
        out = np.zeros(6, dtype=np.uint32)
        self.L.og_publish_repair(self.h, 1 if force_full else 0, _p(out, _u32p))
        keys = ("tier1_iterations", "tier1_last_count", "incremental", "tier2_ran", "proper", "tier2_fixed")
        return {k: int(v) for k, v in zip(keys, out)}

    def set_full_repair_every(self, every):
        self.L.og_set_full_repair_every(self.h, every)

    def set_repair_state(self, clean, asym):
        self.L.og_set_repair_state(self.h, 1 if clean else 0, 1 if asym else 0)

    def process_stream(self, ups, epoch_size, batch=32768):
        ups = np.ascontiguousarray(ups, dtype=EDGE_UPDATE)
        return self.L.og_process_stream(self.h, ups.ctypes.data, len(ups), epoch_size, batch)

    def process_stream_repaired(self, ups, epoch_size, batch=32768):
        ups = np.ascontiguousarray(ups, dtype=EDGE_UPDATE)
        return self.L.og_process_stream_repaired(self.h, ups.ctypes.data, len(ups), epoch_size, batch)

    # --- state ---
    def states(self):
        a = np.zeros(self.n, dtype=np.uint32)
        self.L.og_get_states(self.h, _p(a, _u32p))
        return a

    def load_state(self, col, states, bitmaps, hist):
        col = np.ascontiguousarray(col, dtype=np.uint32)
        states = np.ascontiguousarray(states, dtype=np.uint32)
        bitmaps = np.ascontiguousarray(bitmaps, dtype=np.uint64)
        hist = np.ascontiguousarray(hist, dtype=np.uint32)
        self.L.og_load_state(self.h, _p(col, _u32p), _p(states, _u32p), _p(bitmaps, _u64p), _p(hist, _u32p))

    def col_data(self):
        """Address and byte size of the oracle's slot slab (filled in place by
        load_state_inplace's caller)."""
        return int(self.L.og_col_data(self.h)), int(self.L.og_total_slots(self.h)) * 4

    def load_state_inplace(self, row_ptr, col_idx, states, bitmaps, hist=None):
        """After the slab was written through col_data(): rows that differ from
        their base rows are marked edited; states, bitmaps (and histograms)
        are copied in."""
        rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
        col = np.ascontiguousarray(col_idx, dtype=np.uint32)
        states = np.ascontiguousarray(states, dtype=np.uint32)
        bitmaps = np.ascontiguousarray(bitmaps, dtype=np.uint64)
        hp = None if hist is None else _p(np.ascontiguousarray(hist, dtype=np.uint32), _u32p)
        self.L.og_load_state_inplace(self.h, _p(rp, _u64p), _p(col, _u32p), _p(states, _u32p), _p(bitmaps, _u64p),
                                     hp)

    def load_rows_model(self, highwater, base_runs, holes):
        """Concurrent rules: each row's high-water mark, base-run length and
        hole count (the library's, after load_state)."""
        a = [np.ascontiguousarray(x, dtype=np.uint32) for x in (highwater, base_runs, holes)]
        self.L.og_load_rows_model(self.h, *[_p(x, _u32p) for x in a])

    def color_core(self, min_degree):
        """The library's sgc_color_core restated; returns how many were colored."""
        return int(self.L.og_color_core(self.h, min_degree))

    def color_greedy(self):
        """First-fit coloring of the live rows in id order; returns the largest color."""
        return int(self.L.og_color_greedy(self.h))

    def set_states(self, a):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        self.L.og_set_states(self.h, _p(a, _u32p))

    def colors(self):
        return (self.states() & 0xFFFF).astype(np.uint16)

    def bitmaps(self):
        a = np.zeros(self.n, dtype=np.uint64)
        self.L.og_get_bitmaps(self.h, _p(a, _u64p))
        return a

    def hdmap(self):
        a = np.zeros(self.n, dtype=np.uint32)
        self.L.og_get_hdmap(self.h, _p(a, _u32p))
        return a

    def hist(self):
        a = np.zeros(self.L.og_num_high_degree(self.h) * self.L.og_max_hist_colors(self.h), dtype=np.uint32)
        self.L.og_get_hist(self.h, _p(a, _u32p))
        return a

    def row_ptr(self):
        a = np.zeros(self.n + 1, dtype=np.uint64)
        self.L.og_get_row_ptr(self.h, _p(a, _u64p))
        return a

    def col(self):
        a = np.zeros(self.L.og_total_slots(self.h), dtype=np.uint32)
        self.L.og_get_col(self.h, _p(a, _u32p))
        return a

    def snapshot(self):
        a = np.zeros(self.n, dtype=np.uint16)
        self.L.og_get_snapshot(self.h, _p(a, _u16p))
        return a

    def overflow_count(self):
        return self.L.og_overflow_count(self.h)

    def overflow(self):
        cnt = min(self.overflow_count(), 262144)
        a = np.zeros(2 * cnt, dtype=np.uint32)
        if cnt:
            self.L.og_get_overflow(self.h, _p(a, _u32p), cnt)
        return a.reshape(-1, 2)

    def counters(self):
        a = np.zeros(9, dtype=np.uint64)
        self.L.og_counters(self.h, _p(a, _u64p))
        keys = ["updates_applied", "skipped", "recolors", "overflow_lost", "drain_failed",
                "bytes_update", "bytes_epoch", "bytes_tier1", "bytes_tier2"]
        return dict(zip(keys, a.tolist()))

    def reset_bytes(self):
        self.L.og_reset_bytes(self.h)

    def fac(self, x):
        return int(self.L.og_fac(self.h, x))

    def set_bitmap(self, x, v):
        self.L.og_set_bitmap(self.h, x, v)

    def set_hist_row(self, x, vals):
        vals = np.ascontiguousarray(vals, dtype=np.uint32)
        self.L.og_set_hist_row(self.h, x, _p(vals, _u32p), len(vals))

    def validate(self):
        a = np.zeros(5, dtype=np.uint64)
        self.L.og_validate(self.h, _p(a, _u64p))
        return dict(zip(["violations", "uncolored_with_edges", "edges", "max_color", "out_of_range"], a.tolist()))


# ---------------- free functions ----------------

def static_greedy(row_ptr, col):
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    return int(lib().og_static_greedy(len(rp) - 1, _p(rp, _u64p), _p(col, _u32p)))


def validate_colors(row_ptr, col, colors):
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    colors = np.ascontiguousarray(colors, dtype=np.uint16)
    out = np.zeros(3, dtype=np.uint64)
    lib().og_validate_colors(len(rp) - 1, _p(rp, _u64p), _p(col, _u32p), _p(colors, _u16p), _p(out, _u64p))
    return dict(zip(["violations", "uncolored_with_edges", "max_color"], out.tolist()))


def init_stream(row_ptr, col, degree):
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    deg = np.ascontiguousarray(degree, dtype=np.uint32)
    out = np.zeros(len(col), dtype=np.uint32)
    k = lib().og_gen_init_stream(len(rp) - 1, _p(rp, _u64p), _p(col, _u32p), _p(deg, _u32p), _p(out, _u32p))
    return out[: 2 * k].reshape(-1, 2)


def bench_stream(row_ptr, col, size, insert_pct=50, seed=42):
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    pairs = np.zeros(2 * size, dtype=np.uint32)
    types = np.zeros(size, dtype=np.uint8)
    lib().og_gen_bench_stream(len(rp) - 1, _p(rp, _u64p), _p(col, _u32p), size, insert_pct, seed,
                              _p(pairs, _u32p), _p(types, _u8p))
    return pairs.reshape(-1, 2), types


def load_mtx(path):
    L = lib()
    h = L.og_load_mtx(path.encode())
    if not h:
        raise IOError(f"cannot load {path}")
    n = L.og_loaded_n(h)
    nnz = L.og_loaded_nnz(h)
    rp = np.zeros(n + 1, dtype=np.uint64)
    col = np.zeros(nnz, dtype=np.uint32)
    deg = np.zeros(n, dtype=np.uint32)
    L.og_loaded_copy(h, _p(rp, _u64p), _p(col, _u32p), _p(deg, _u32p))
    L.og_loaded_free(h)
    return rp, col, deg


# ---------------- the reference's own host code (oracle/_ref) ----------------

_ref = None


def ref_host_available():
    return os.path.exists(REF_HOST_PATH)


def ref_host():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_HOST_PATH)
        L.ref_init_stream.restype = C.c_uint64
        L.ref_init_stream.argtypes = [C.c_uint32, _u32p, _u32p, _u32p, _u32p]
        L.ref_bench_stream.restype = None
        L.ref_bench_stream.argtypes = [C.c_uint32, _u32p, _u32p, _u32p, C.c_uint64, C.c_uint32, C.c_uint64,
                                       _u32p, _u8p]
        L.ref_load_mtx.restype = C.c_int
        L.ref_load_mtx.argtypes = [C.c_char_p, _u32p, _u64p]
        L.ref_loaded_copy.restype = None
        L.ref_loaded_copy.argtypes = [_u32p, _u32p, _u32p]
        _ref = L
    return _ref


def ref_init_stream(row_ptr, col, degree):
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    deg = np.ascontiguousarray(degree, dtype=np.uint32)
    out = np.zeros(len(col), dtype=np.uint32)
    k = ref_host().ref_init_stream(len(rp) - 1, _p(rp, _u32p), _p(col, _u32p), _p(deg, _u32p), _p(out, _u32p))
    return out[: 2 * k].reshape(-1, 2)


def ref_bench_stream(row_ptr, col, degree, size, insert_pct=50, seed=42):
    rp = np.ascontiguousarray(row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    deg = np.ascontiguousarray(degree, dtype=np.uint32)
    pairs = np.zeros(2 * size, dtype=np.uint32)
    types = np.zeros(size, dtype=np.uint8)
    ref_host().ref_bench_stream(len(rp) - 1, _p(rp, _u32p), _p(col, _u32p), _p(deg, _u32p), size, insert_pct,
                                seed, _p(pairs, _u32p), _p(types, _u8p))
    return pairs.reshape(-1, 2), types


def ref_load_mtx(path):
    L = ref_host()
    n = np.zeros(1, dtype=np.uint32)
    nnz = np.zeros(1, dtype=np.uint64)
    L.ref_load_mtx(path.encode(), _p(n, _u32p), _p(nnz, _u64p))
    rp = np.zeros(int(n[0]) + 1, dtype=np.uint32)
    col = np.zeros(int(nnz[0]), dtype=np.uint32)
    deg = np.zeros(int(n[0]), dtype=np.uint32)
    L.ref_loaded_copy(_p(rp, _u32p), _p(col, _u32p), _p(deg, _u32p))
    return rp, col, deg
