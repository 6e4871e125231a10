"""ctypes binding of the B200 MOSP update library (include/mosp_b200.h,
include/mosp_b200_host.h).

The library is the product: sm_100a kernels behind a C ABI. This module only
loads it and converts arguments; it raises if the shared library is missing
(there is no fallback path). Device arrays are passed as raw pointers, so any
owner of device memory works (torch tensors are used by the tests and the
benchmark).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# MOSP_B200_LIBRARY loads another build of the library (e.g. one compiled
# with other build constants) in place of the in-tree one
LIB_PATH = os.environ.get("MOSP_B200_LIBRARY") or os.path.join(os.path.dirname(_HERE), "lib", "libmosp_b200.so")
BIN_DIR = os.path.join(os.path.dirname(_HERE), "bin")

OK, ERR_INVALID, ERR_OVERFLOW, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_UNSUPPORTED = range(7)
DISTANCE_INF = 0x7FFFFFFFFFFFFFFF // 4
MODES = {"uniform": 0, "targeted": 1, "reweight": 2, "increase": 3}

_p = C.c_void_p
_i = C.c_int
_ll = C.c_longlong
_ip = C.POINTER(C.c_int)
_llp = C.POINTER(C.c_longlong)


class MospError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} [status {status}]")
        self.status = status


class SospStats(C.Structure):
    _fields_ = [("invalidated", C.c_int), ("jump_rounds", C.c_int), ("iterations", C.c_int),
                ("epochs", C.c_int), ("pushes", C.c_longlong), ("packed_parents", C.c_int),
                ("reserved", C.c_int)]


class CombineStats(C.Structure):
    _fields_ = [("edges", C.c_int), ("reserved", C.c_int), ("scale", C.c_longlong),
                ("delta", C.c_longlong), ("search", SospStats)]


class ServerResult(C.Structure):
    _fields_ = [("status", C.c_int), ("graph", C.c_int), ("version", C.c_longlong), ("coalesced", C.c_int),
                ("reserved", C.c_int), ("queue_us", C.c_double), ("latency_us", C.c_double),
                ("checksum", C.c_ulonglong)]


class ServerStats(C.Structure):
    _fields_ = [("requests", C.c_longlong), ("passes", C.c_longlong), ("changes", C.c_longlong),
                ("deferred", C.c_longlong), ("applies", C.c_longlong), ("max_coalesced", C.c_int),
                ("overlapped", C.c_int),
                ("busy_us", C.c_double), ("apply_us", C.c_double), ("engine_us", C.c_double),
                ("result_us", C.c_double)]


class Timings(C.Structure):
    _fields_ = [("apply_batch", C.c_double), ("upload", C.c_double), ("objectives", C.c_double),
                ("combined", C.c_double), ("costs", C.c_double), ("download", C.c_double)]


_SIGS = {
    "mosp_abi_version": (_i, []),
    "mosp_last_error": (C.c_char_p, []),
    "mosp_status_name": (C.c_char_p, [_i]),
    "mosp_default_delta": (_ll, [_ll, _i, _ll]),
    "mosp_choose_packing": (_i, [_i, _ll, _ip, C.POINTER(C.c_ulonglong)]),
    "mosp_preference_scale": (_ll, [_ip, _i]),
    "mosp_workspace_create": (_i, [C.POINTER(_p)]),
    "mosp_workspace_destroy": (None, [_p]),
    "mosp_workspace_reserve": (_i, [_p, _i, _i]),
    "mosp_workspace_reserve_graph": (_i, [_p, _i, _ll, _i]),
    "mosp_workspace_set_timeout_ms": (_i, [_p, _ll]),
    "mosp_workspace_set_ctas_per_sm": (_i, [_p, _i]),
    "mosp_workspace_set_sources": (_i, [_p, _ip, _i]),
    "mosp_workspace_set_combined_delta": (_i, [_p, _ll]),
    "mosp_workspace_use_graphs": (_i, [_p, _i]),
    "mosp_workspace_set_local_rounds": (_i, [_p, _i, _i]),
    "mosp_workspace_set_narrow": (_i, [_p, _i, _i]),
    "mosp_workspace_set_async": (_i, [_p, _i, _ll]),
    "mosp_workspace_set_canonical_trees": (_i, [_p, _i]),
    "mosp_workspace_set_grid": (_i, [_p, _i, _i]),
    "mosp_workspace_tuning": (_i, [_p, _ip, _ip, _ip]),
    "mosp_workspace_graph_launches": (_i, [_p, _ip]),
    "mosp_autotune_update": (_i, [_p, _i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _ip, _p, _i, _i,
                                  _llp, _llp, _ip, _p, _p, _p, _p, _llp, _llp, _ip, C.POINTER(C.c_float), _p]),
    "mosp_workspace_grid": (_i, [_p, _ip]),
    "mosp_workspace_buffer": (_i, [_p, _i, C.c_ulonglong, C.POINTER(_p)]),
    "mosp_workspace_enable_timing": (_i, [_p, _i]),
    "mosp_workspace_last_timing": (_i, [_p, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "mosp_workspace_last_phases": (_i, [_p, _i, C.POINTER(C.c_ulonglong)]),
    "mosp_workspace_loop_profile": (_i, [_p, _i, C.POINTER(C.c_ulonglong), _llp, _llp]),
    "mosp_build_device_graph": (_i, [_p, _i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _p]),
    "mosp_apply_batch_device": (_i, [_p, _i, _i, _i, _p, _p, _p, _i, _p, _p, _p, _i, _p, _p, _p, _p, _p,
                                     _ll, _ip, _p, _llp, _llp, _p]),
    "mosp_sosp_update": (_i, [_p, _i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _i, _i, _ll, _ll,
                              _p, _p, C.POINTER(SospStats), _p]),
    "mosp_sosp_update_multi": (_i, [_p, _i, _i, _i, _p, _p, C.POINTER(_p), _p, _p, C.POINTER(_p),
                                    C.POINTER(_p), C.POINTER(_p), _ip, _p, _i, _i, _llp, _llp,
                                    C.POINTER(_p), C.POINTER(_p), C.POINTER(SospStats), _p]),
    "mosp_sosp_from_scratch": (_i, [_p, _i, _i, _p, _p, _p, _i, _ll, _ll, _p, _p,
                                    C.POINTER(SospStats), _p]),
    "mosp_sosp_from_scratch_static": (_i, [_i, _i, _p, _p, _p, _i, _ll, _ll, _p, _p,
                                           C.POINTER(SospStats), _p]),
    "mosp_combined_sosp": (_i, [_p, _i, _i, _p, _ip, _i, _ll, _p, _p, C.POINTER(CombineStats), _p]),
    "mosp_path_costs": (_i, [_p, _i, _i, _i, _p, _p, _p, _p, _i, _p, _p]),
    "mosp_update_device": (_i, [_p, _i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _ip, _p, _i, _i,
                                _llp, _llp, _ip, _p, _p, _p, _p, C.POINTER(SospStats),
                                C.POINTER(CombineStats), _p]),
    "mosp_update_host": (_i, [_p, _i, _i, _i, _p, _p, _p, _i, _p, _p, _p, _i, _p, _p, _p, _p, _i,
                              _i, _ip, _ll, _p, _p, _p, _p, _p, C.POINTER(Timings)]),
    "mosp_debug_barrier_timeout": (_i, [_p, _ll, _ip]),
    "mosp_debug_barrier_cost": (_i, [_p, _i, _i, C.POINTER(C.c_double)]),
    "mosp_server_create": (_i, [_i, _ll, _i, C.POINTER(_p)]),
    "mosp_server_destroy": (None, [_p]),
    "mosp_server_set_overlap": (_i, [_p, _i]),
    "mosp_server_add_graph": (_i, [_p, _i, _i, _i, _p, _p, _p, _i, _i, _ip, _ip]),
    "mosp_server_submit": (_i, [_p, _i, _i, _p, _p, _p, _i, _p, _p, _llp]),
    "mosp_server_wait": (_i, [_p, _ll, _p, _p, C.POINTER(ServerResult)]),
    "mosp_server_read_graph": (_i, [_p, _i, _llp, _p, _p, _p, _p]),
    "mosp_server_get_stats": (_i, [_p, C.POINTER(ServerStats)]),
    # host side
    "mosp_graph_read": (_i, [C.c_char_p, C.c_char_p, C.POINTER(_p)]),
    "mosp_graph_write": (_i, [_p, C.c_char_p]),
    "mosp_graph_save_cache": (_i, [_p, C.c_char_p, C.c_char_p]),
    "mosp_graph_from_arrays": (_i, [_i, _i, _p, _p, _p, C.POINTER(_p)]),
    "mosp_graph_grid_road": (_i, [_i, _i, C.c_double, C.c_double, _i, _i, _i, C.c_uint,
                                  C.POINTER(_p)]),
    "mosp_graph_rmat": (_i, [_i, _i, C.c_double, C.c_double, C.c_double, _i, _i, _i, _i, C.c_uint,
                             C.POINTER(_p)]),
    "mosp_graph_info": (_i, [_p, _ip, _ip, _llp]),
    "mosp_graph_arrays": (_i, [_p, C.POINTER(_ip), C.POINTER(_ip), C.POINTER(_ip)]),
    "mosp_graph_free": (None, [_p]),
    "mosp_batch_generate": (_i, [_p, _i, C.c_double, _i, _i, _i, C.c_uint, _i, _i, _i,
                                 C.POINTER(_p)]),
    "mosp_batch_near": (_i, [_p, _i, _i, _i, _i, _i, C.c_uint, _i, _i, _i, C.POINTER(_p)]),
    "mosp_batch_read": (_i, [C.c_char_p, C.c_char_p, _i, _i, C.POINTER(_p)]),
    "mosp_batch_write": (_i, [_p, C.c_char_p, C.c_char_p]),
    "mosp_batch_from_arrays": (_i, [_i, _i, _p, _p, _p, _i, _p, _p, C.POINTER(_p)]),
    "mosp_batch_info": (_i, [_p, _ip, _ip, _ip]),
    "mosp_batch_arrays": (_i, [_p, C.POINTER(_ip), C.POINTER(_ip), C.POINTER(_ip), C.POINTER(_ip),
                               C.POINTER(_ip), C.POINTER(C.POINTER(C.c_uint))]),
    "mosp_batch_free": (None, [_p]),
    "mosp_apply_batch": (_i, [_p, _p, C.POINTER(_p)]),
    "mosp_host_dijkstra": (_i, [_p, _i, _i, _p, _p]),
    "mosp_canonicalize_tree": (_i, [_p, _i, _i, _p, _p]),
    "mosp_read_tree": (_i, [C.c_char_p, C.c_char_p, _i, _p, _p]),
    "mosp_write_tree": (_i, [C.c_char_p, C.c_char_p, _i, _p, _p]),
    "mosp_algorithmic_bytes": (_i, [_p, _p, _i, _i, _p, _p, _p, _p, _ll, _llp, _llp, _llp, _llp]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C mosp-cuda_b200`")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def exported_names() -> list[str]:
    return sorted(_SIGS)


def check(status: int) -> None:
    if status != OK:
        raise MospError(status, lib().mosp_last_error().decode(errors="replace"))


def _ptr(a) -> int | None:
    """Raw address of a numpy array, a torch tensor or an int; None for None."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


# ---------------------------------------------------------------------------
# Host graphs and batches
# ---------------------------------------------------------------------------
class HostGraph:
    """A CSR graph owned by the library (reference CsrGraph)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        n, K, m = C.c_int(), C.c_int(), C.c_longlong()
        check(lib().mosp_graph_info(self._h, C.byref(n), C.byref(K), C.byref(m)))
        self.n, self.K, self.m = n.value, K.value, m.value

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.mosp_graph_free(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def arrays(self):
        """(row[n+1], col[m], w[m, K]) as numpy copies."""
        row, col, w = _ip(), _ip(), _ip()
        check(lib().mosp_graph_arrays(self._h, C.byref(row), C.byref(col), C.byref(w)))
        r = np.ctypeslib.as_array(row, (self.n + 1,)).copy()
        if self.m == 0:  # no edges: the column and weight arrays may be NULL
            return r, np.zeros(0, np.int32), np.zeros((0, self.K), np.int32)
        c = np.ctypeslib.as_array(col, (self.m,)).copy()
        ww = np.ctypeslib.as_array(w, (self.m * self.K,)).copy()
        return r, c, ww.reshape(self.m, self.K)

    @classmethod
    def from_arrays(cls, row, col, w):
        row, col = _i32(row), _i32(col)
        w = _i32(w)
        K = w.shape[1] if w.ndim == 2 else 1
        h = C.c_void_p()
        check(lib().mosp_graph_from_arrays(len(row) - 1, K, _ptr(row), _ptr(col), _ptr(w), C.byref(h)))
        return cls(h)

    @classmethod
    def read(cls, prefix: str, cache: str | None = None):
        h = C.c_void_p()
        check(lib().mosp_graph_read(prefix.encode(), cache.encode() if cache else None, C.byref(h)))
        return cls(h)

    @classmethod
    def grid_road(cls, width, height, keep, shortcut, K, wmin, wmax, seed):
        h = C.c_void_p()
        check(lib().mosp_graph_grid_road(width, height, keep, shortcut, K, wmin, wmax, seed, C.byref(h)))
        return cls(h)

    @classmethod
    def rmat(cls, scale, edge_factor, a, b, c, K, wmin, wmax, log_uniform, seed):
        h = C.c_void_p()
        check(lib().mosp_graph_rmat(scale, edge_factor, a, b, c, K, wmin, wmax, int(log_uniform), seed,
                                    C.byref(h)))
        return cls(h)

    def write(self, prefix: str):
        check(lib().mosp_graph_write(self._h, prefix.encode()))

    def dijkstra(self, k: int, source: int):
        d = np.empty(self.n, np.int64)
        p = np.empty(self.n, np.int32)
        check(lib().mosp_host_dijkstra(self._h, k, source, _ptr(d), _ptr(p)))
        return d, p


class HostBatch:
    """A change batch owned by the library (reference ChangeBatch)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        K, ni, nd = C.c_int(), C.c_int(), C.c_int()
        check(lib().mosp_batch_info(self._h, C.byref(K), C.byref(ni), C.byref(nd)))
        self.K, self.n_ins, self.n_del = K.value, ni.value, nd.value

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.mosp_batch_free(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def arrays(self):
        """dict of numpy copies: ins_from, ins_to, ins_w[n_ins, K], del_from,
        del_to, mask (after apply; zeros before)."""
        a = [_ip() for _ in range(5)]
        mk = C.POINTER(C.c_uint)()
        check(lib().mosp_batch_arrays(self._h, *[C.byref(x) for x in a], C.byref(mk)))

        def get(ptr, count):
            if count == 0 or not ptr:
                return np.zeros(0, np.int32)
            return np.ctypeslib.as_array(ptr, (count,)).copy()

        out = {
            "ins_from": get(a[0], self.n_ins), "ins_to": get(a[1], self.n_ins),
            "ins_w": get(a[2], self.n_ins * self.K).reshape(self.n_ins, self.K),
            "del_from": get(a[3], self.n_del), "del_to": get(a[4], self.n_del),
        }
        out["mask"] = (np.ctypeslib.as_array(mk, (self.n_ins,)).copy().astype(np.uint32)
                       if (mk and self.n_ins) else np.zeros(self.n_ins, np.uint32))
        return out

    @classmethod
    def from_arrays(cls, K, ins_from, ins_to, ins_w, del_from, del_to):
        ins_from, ins_to, ins_w = _i32(ins_from), _i32(ins_to), _i32(ins_w)
        del_from, del_to = _i32(del_from), _i32(del_to)
        h = C.c_void_p()
        check(lib().mosp_batch_from_arrays(K, len(ins_from), _ptr(ins_from), _ptr(ins_to), _ptr(ins_w),
                                           len(del_from), _ptr(del_from), _ptr(del_to), C.byref(h)))
        return cls(h)

    @classmethod
    def generate(cls, g: HostGraph, changes, ins_pct=50.0, mode="uniform", local=0, safe=False,
                 seed=1, source=0, wmin=1, wmax=100):
        h = C.c_void_p()
        check(lib().mosp_batch_generate(g.handle, changes, ins_pct, MODES[mode], local, int(safe), seed,
                                        source, wmin, wmax, C.byref(h)))
        return cls(h)

    @classmethod
    def near(cls, g: HostGraph, grid_width, n_ins, n_del, max_manhattan=3, safe=True, seed=777,
             source=0, wmin=1, wmax=100):
        h = C.c_void_p()
        check(lib().mosp_batch_near(g.handle, grid_width, n_ins, n_del, max_manhattan, int(safe), seed,
                                    source, wmin, wmax, C.byref(h)))
        return cls(h)

    @classmethod
    def read(cls, insert_path, delete_path, K, n):
        h = C.c_void_p()
        check(lib().mosp_batch_read(insert_path.encode(), delete_path.encode(), K, n, C.byref(h)))
        return cls(h)

    def write(self, insert_path, delete_path):
        check(lib().mosp_batch_write(self._h, insert_path.encode(), delete_path.encode()))


def apply_batch(g: HostGraph, b: HostBatch) -> HostGraph:
    """Reference applyChangeBatch; fills the batch's increase masks."""
    h = C.c_void_p()
    check(lib().mosp_apply_batch(g.handle, b.handle, C.byref(h)))
    return HostGraph(h)


def default_delta(m, n, weight_sum) -> int:
    return int(lib().mosp_default_delta(int(m), int(n), int(weight_sum)))


def choose_packing(n, max_weight):
    bits, maxd = C.c_int(), C.c_ulonglong()
    check(lib().mosp_choose_packing(n, max_weight, C.byref(bits), C.byref(maxd)))
    return bits.value, maxd.value


def preference_scale(pref, K) -> int:
    if pref is None:
        return int(lib().mosp_preference_scale(None, K))
    arr = (C.c_int * K)(*pref)
    return int(lib().mosp_preference_scale(arr, K))


def changed_lists(batch_arrays: dict, K: int):
    """Per objective (changed_from, changed_to): every deletion plus the
    insertions whose weight-increase mask has bit k (reference
    src/mospUpdate.cu:124-136)."""
    out = []
    for k in range(K):
        sel = (batch_arrays["mask"] >> np.uint32(k)) & np.uint32(1)
        sel = sel.astype(bool)
        out.append((np.concatenate([batch_arrays["del_from"], batch_arrays["ins_from"][sel]]).astype(np.int32),
                    np.concatenate([batch_arrays["del_to"], batch_arrays["ins_to"][sel]]).astype(np.int32)))
    return out


def algorithmic_bytes(g: HostGraph, b: HostBatch, K, source, old_d, old_p, new_d, new_p, comb_edges):
    bu, bc, inv, exp = C.c_longlong(), C.c_longlong(), C.c_longlong(), C.c_longlong()
    check(lib().mosp_algorithmic_bytes(g.handle, b.handle, K, source, _ptr(_i64(old_d)), _ptr(_i32(old_p)),
                                       _ptr(_i64(new_d)), _ptr(_i32(new_p)), int(comb_edges),
                                       C.byref(bu), C.byref(bc), C.byref(inv), C.byref(exp)))
    return {"update": bu.value, "combined": bc.value, "invalidated": inv.value, "expanded": exp.value}


# ---------------------------------------------------------------------------
# Device side
# ---------------------------------------------------------------------------
class Workspace:
    """Engine workspace on the current CUDA device (mosp_workspace)."""

    def __init__(self, timeout_ms: int | None = None, ctas_per_sm: int = 0):
        self._h = C.c_void_p()
        check(lib().mosp_workspace_create(C.byref(self._h)))
        if timeout_ms is not None:
            check(lib().mosp_workspace_set_timeout_ms(self._h, int(timeout_ms)))
        if ctas_per_sm:
            check(lib().mosp_workspace_set_ctas_per_sm(self._h, int(ctas_per_sm)))

    def close(self):
        if self._h is not None and _lib is not None and self._h.value:
            _lib.mosp_workspace_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self):
        return self._h

    def enable_timing(self, on=True):
        check(lib().mosp_workspace_enable_timing(self._h, int(on)))

    def last_timing(self):
        """(update_ms, combined_ms) of the last launches (CUDA events)."""
        a, b = C.c_float(), C.c_float()
        check(lib().mosp_workspace_last_timing(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    PHASES = ("packed", "roots", "jumped", "candidates", "pulled", "loop", "end")

    def last_phases(self, which=0):
        """Milliseconds spent in each phase of the last update (which=0) or
        combined (which=1) launch, from the device clock."""
        ns = (C.c_ulonglong * 8)()
        check(lib().mosp_workspace_last_phases(self._h, which, ns))
        out, prev = {}, ns[0]
        for name, t in zip(self.PHASES, list(ns)[1:]):
            if t:
                out[name] = round((t - prev) / 1e6, 4)
                prev = t
        return out

    def loop_profile(self, which=0, asynchronous=False):
        """Near-far loop of the last launch. Bulk loop: {split|push: (ms,
        iterations, items)} and the parts of a push iteration; asynchronous
        loop: its time and phases, the durations of the first four phases
        (the rest summed), warp rounds and the entries taken from the queue
        and from the warps' local buffers."""
        ns = (C.c_ulonglong * 7)()
        it = (C.c_longlong * 2)()
        items = (C.c_longlong * 2)()
        check(lib().mosp_workspace_loop_profile(self._h, which, ns, it, items))
        if asynchronous:
            return {"ms": round(ns[0] / 1e6, 4), "phases": it[0],
                    "phase_ms": [round(ns[2 + q] / 1e6, 4) for q in range(5)],
                    "warp_rounds": it[1], "local_rounds": ns[1], "queue_entries": items[0],
                    "local_entries": items[1]}
        out = {name: (round(ns[q] / 1e6, 4), it[q], items[q]) for q, name in enumerate(("split", "push"))}
        out["push_parts_ms"] = {name: round(ns[2 + q] / 1e6, 4) for q, name in
                                enumerate(("decide", "own_items", "wait_cta", "flush", "barrier"))}
        return out

    def grid(self) -> int:
        c = C.c_int()
        check(lib().mosp_workspace_grid(self._h, C.byref(c)))
        return c.value

    def build_device_graph(self, n, m, K, d_row, d_col, d_edge_w, d_out_w, d_in_row, d_in_col, d_in_w,
                           stream=None):
        check(lib().mosp_build_device_graph(self._h, n, m, K, _ptr(d_row), _ptr(d_col), _ptr(d_edge_w),
                                            _ptr(d_out_w), _ptr(d_in_row), _ptr(d_in_col), _ptr(d_in_w),
                                            stream))

    def sosp_update(self, n, m, out_row, out_col, out_w, in_row, in_col, in_w, ch_from, ch_to, n_changed,
                    heads, n_heads, source, delta, max_weight, dist, parent, stream=None) -> SospStats:
        st = SospStats()
        check(lib().mosp_sosp_update(self._h, n, m, _ptr(out_row), _ptr(out_col), _ptr(out_w),
                                     _ptr(in_row), _ptr(in_col), _ptr(in_w), _ptr(ch_from), _ptr(ch_to),
                                     n_changed, _ptr(heads), n_heads, source, int(delta), int(max_weight),
                                     _ptr(dist), _ptr(parent), C.byref(st), stream))
        return st

    def sosp_update_multi(self, n, m, K, out_row, out_col, out_w_list, in_row, in_col, in_w_list,
                          ch_from_list, ch_to_list, n_changed, heads, n_heads, source, deltas, max_weights,
                          dist_list, parent_list, stream=None):
        arr = lambda xs: (C.c_void_p * K)(*[_ptr(x) for x in xs])  # noqa: E731
        stats = (SospStats * K)()
        nc = (C.c_int * K)(*n_changed)
        dl = (C.c_longlong * K)(*[int(x) for x in deltas])
        mw = (C.c_longlong * K)(*[int(x) for x in max_weights])
        check(lib().mosp_sosp_update_multi(self._h, n, m, K, _ptr(out_row), _ptr(out_col), arr(out_w_list),
                                           _ptr(in_row), _ptr(in_col), arr(in_w_list), arr(ch_from_list),
                                           arr(ch_to_list), nc, _ptr(heads), n_heads, source, dl, mw,
                                           arr(dist_list), arr(parent_list), stats, stream))
        return list(stats)

    def apply_batch_device(self, n, K, m, row, col, w, ins_from, ins_to, ins_w, del_from, del_to,
                           new_row, new_col, new_w, mask, stream=None):
        """mosp_apply_batch_device: Step 1 on device buffers (edge-major
        weights). Returns (new_m, max_weight[K], weight_sum[K])."""
        nm = C.c_int()
        mx = (C.c_longlong * K)()
        sm = (C.c_longlong * K)()
        n_ins = int(ins_from.numel()) if hasattr(ins_from, "numel") else len(ins_from)
        n_del = int(del_from.numel()) if hasattr(del_from, "numel") else len(del_from)
        cap = int(new_col.numel()) if hasattr(new_col, "numel") else len(new_col)
        check(lib().mosp_apply_batch_device(self._h, n, K, m, _ptr(row), _ptr(col), _ptr(w), n_ins,
                                            _ptr(ins_from), _ptr(ins_to), _ptr(ins_w), n_del, _ptr(del_from),
                                            _ptr(del_to), _ptr(new_row), _ptr(new_col), _ptr(new_w), cap,
                                            C.byref(nm), _ptr(mask), mx, sm, stream))
        return nm.value, list(mx), list(sm)

    def set_combined_delta(self, delta):
        check(lib().mosp_workspace_set_combined_delta(self._h, int(delta)))

    def set_local_rounds(self, update_rounds, scratch_rounds):
        check(lib().mosp_workspace_set_local_rounds(self._h, int(update_rounds), int(scratch_rounds)))

    def set_narrow(self, max_items, rounds):
        check(lib().mosp_workspace_set_narrow(self._h, int(max_items), int(rounds)))

    def set_grid(self, ctas=0, hub_edges=0):
        """Grid CTAs of the engine launches (0: all SMs) and hub-row threshold (0: default)."""
        check(lib().mosp_workspace_set_grid(self._h, int(ctas), int(hub_edges)))

    def tuning(self):
        """(grid CTAs, hub threshold, asynchronous loop on) of the workspace."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().mosp_workspace_tuning(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, bool(c.value)

    def set_async(self, on=True, queue_slots=0):
        """Asynchronous near-far loop (default) or the bulk-synchronous one;
        queue_slots bounds the asynchronous near queue (0: default size)."""
        check(lib().mosp_workspace_set_async(self._h, 1 if on else 0, int(queue_slots)))

    def set_canonical_trees(self, on=True):
        """Declare that update inputs follow the lowest-id tie rule: the
        distance-only objectives then recover parents only where the batch
        reaches (same result for such trees)."""
        check(lib().mosp_workspace_set_canonical_trees(self._h, 1 if on else 0))

    def use_graphs(self, on=True):
        check(lib().mosp_workspace_use_graphs(self._h, int(bool(on))))

    def graph_launches(self) -> int:
        c = C.c_int()
        check(lib().mosp_workspace_graph_launches(self._h, C.byref(c)))
        return c.value

    def autotune_update(self, n, m, K, out_row, out_col, out_w, in_row, in_col, in_w, ch_from, ch_to,
                        ch_offset, heads, n_heads, source, deltas, max_weights, pref, dist, parent,
                        comb_dist, comb_parent, stream=None):
        """mosp_autotune_update: returns (best deltas[K], best combined
        delta, best summed launch ms, best local rounds (update, combined));
        the trees are left unchanged."""
        off = (C.c_int * (K + 1))(*[int(x) for x in ch_offset])
        dl = (C.c_longlong * K)(*[int(x) for x in deltas])
        mw = (C.c_longlong * K)(*[int(x) for x in max_weights])
        pa = None if pref is None else (C.c_int * K)(*pref)
        bd = (C.c_longlong * K)()
        bc = C.c_longlong()
        bm = C.c_float()
        br = (C.c_int * 2)()
        check(lib().mosp_autotune_update(self._h, n, m, K, _ptr(out_row), _ptr(out_col), _ptr(out_w),
                                         _ptr(in_row), _ptr(in_col), _ptr(in_w), _ptr(ch_from), _ptr(ch_to),
                                         off, _ptr(heads), n_heads, source, dl, mw, pa, _ptr(dist),
                                         _ptr(parent), _ptr(comb_dist), _ptr(comb_parent), bd, C.byref(bc), br,
                                         C.byref(bm), stream))
        return list(bd), bc.value, bm.value, (br[0], br[1])

    def set_sources(self, sources):
        """Roots of a batched run (one per instance of a disjoint union);
        an empty list or one root returns to single-source runs."""
        arr = (C.c_int * max(len(sources), 1))(*[int(x) for x in sources])
        check(lib().mosp_workspace_set_sources(self._h, arr, len(sources)))

    def sosp_from_scratch(self, n, m, out_row, out_col, out_w, source, delta, max_weight, dist, parent,
                          stream=None) -> SospStats:
        st = SospStats()
        check(lib().mosp_sosp_from_scratch(self._h, n, m, _ptr(out_row), _ptr(out_col), _ptr(out_w), source,
                                           int(delta), int(max_weight), _ptr(dist), _ptr(parent),
                                           C.byref(st), stream))
        return st

    def combined_sosp(self, n, K, parents, pref, source, delta, dist, parent, stream=None) -> CombineStats:
        st = CombineStats()
        pa = None if pref is None else (C.c_int * K)(*pref)
        check(lib().mosp_combined_sosp(self._h, n, K, _ptr(parents), pa, source, int(delta), _ptr(dist),
                                       _ptr(parent), C.byref(st), stream))
        return st

    def path_costs(self, n, m, KG, out_row, out_col, out_w, parent, source, costs, stream=None):
        check(lib().mosp_path_costs(self._h, n, m, KG, _ptr(out_row), _ptr(out_col), _ptr(out_w),
                                    _ptr(parent), source, _ptr(costs), stream))

    def update_device(self, n, m, K, out_row, out_col, out_w, in_row, in_col, in_w, ch_from, ch_to,
                      ch_offset, heads, n_heads, source, deltas, max_weights, pref, dist, parent,
                      comb_dist, comb_parent, stream=None, want_stats=True):
        off = (C.c_int * (K + 1))(*[int(x) for x in ch_offset])
        dl = (C.c_longlong * K)(*[int(x) for x in deltas])
        mw = (C.c_longlong * K)(*[int(x) for x in max_weights])
        pa = None if pref is None else (C.c_int * K)(*pref)
        stats = (SospStats * K)() if want_stats else None
        cst = CombineStats() if want_stats else None
        check(lib().mosp_update_device(self._h, n, m, K, _ptr(out_row), _ptr(out_col), _ptr(out_w),
                                       _ptr(in_row), _ptr(in_col), _ptr(in_w), _ptr(ch_from), _ptr(ch_to),
                                       off, _ptr(heads), n_heads, source, dl, mw, pa, _ptr(dist),
                                       _ptr(parent), _ptr(comb_dist), _ptr(comb_parent),
                                       stats, C.byref(cst) if cst is not None else None, stream))
        return (list(stats) if stats is not None else None), cst

    def update_host(self, graph_arrays, batch_arrays, init_dist, init_parent, K, source, pref=None,
                    delta=0, costs=True, out=None):
        """mosp_update_host: host buffers in, host buffers out. `out` may hold
        preallocated (e.g. pinned) result arrays (dist[K*n], parent[K*n],
        comb_dist[n], comb_parent[n], costs[n*KG] or None)."""
        row, col, w = (_i32(x) for x in graph_arrays)
        n = len(row) - 1
        KG = w.shape[1]
        m = len(col)
        b = {k: _i32(v) for k, v in batch_arrays.items() if k != "mask"}
        init_dist, init_parent = _i64(init_dist), _i32(init_parent)
        if out is not None:
            dist, par, cd, cp, cost = out
            costs = cost is not None
        else:
            dist = np.empty(K * n, np.int64)
            par = np.empty(K * n, np.int32)
            cd = np.empty(n, np.int64)
            cp = np.empty(n, np.int32)
            cost = np.empty(n * KG, np.int64) if costs else None
        pa = None if pref is None else (C.c_int * K)(*pref)
        t = Timings()
        check(lib().mosp_update_host(self._h, n, KG, m, _ptr(row), _ptr(col), _ptr(w), len(b["ins_from"]),
                                     _ptr(b["ins_from"]), _ptr(b["ins_to"]), _ptr(b["ins_w"]),
                                     len(b["del_from"]), _ptr(b["del_from"]), _ptr(b["del_to"]),
                                     _ptr(init_dist), _ptr(init_parent), K, source, pa, int(delta),
                                     _ptr(dist), _ptr(par), _ptr(cd), _ptr(cp), _ptr(cost), C.byref(t)))
        return dist.reshape(K, n), par.reshape(K, n), cd, cp, (cost.reshape(n, KG) if costs else None), t

    def barrier_cost_ns(self, rounds=2000, reads=False) -> float:
        x = C.c_double()
        check(lib().mosp_debug_barrier_cost(self._h, rounds, int(reads), C.byref(x)))
        return x.value

    def barrier_timeout_probe(self, timeout_ms: int) -> int:
        st = C.c_int(-1)
        check(lib().mosp_debug_barrier_timeout(self._h, int(timeout_ms), C.byref(st)))
        return st.value


class Server:
    """mosp_server_*: resident graphs served by worker threads; change
    batches from any thread, coalesced per graph, admitted by free device
    memory."""

    def __init__(self, workers=2, reserve_bytes=1 << 30, max_coalesce=64, overlap=True):
        h = C.c_void_p()
        check(lib().mosp_server_create(int(workers), int(reserve_bytes), int(max_coalesce), C.byref(h)))
        self._h = h
        self._n = {}
        check(lib().mosp_server_set_overlap(self._h, 1 if overlap else 0))

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().mosp_server_destroy(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.close()

    def add_graph(self, graph_arrays, K, source=0, pref=None) -> int:
        row, col, w = (_i32(x) for x in graph_arrays)
        n, KG, m = len(row) - 1, w.shape[1], len(col)
        gid = C.c_int()
        pa = None if pref is None else (C.c_int * K)(*pref)
        check(lib().mosp_server_add_graph(self._h, n, KG, m, _ptr(row), _ptr(col), _ptr(w), K, source, pa,
                                          C.byref(gid)))
        self._n[gid.value] = (n, K)
        return gid.value

    def submit(self, graph_id, batch_arrays) -> int:
        b = {k: _i32(v) for k, v in batch_arrays.items() if k != "mask"}
        t = C.c_longlong()
        check(lib().mosp_server_submit(self._h, graph_id, len(b["ins_from"]), _ptr(b["ins_from"]), _ptr(b["ins_to"]),
                                       _ptr(b["ins_w"]), len(b["del_from"]), _ptr(b["del_from"]), _ptr(b["del_to"]),
                                       C.byref(t)))
        return t.value

    def wait(self, ticket, graph_id=None, want_result=True):
        """(combined distances, combined parents, ServerResult); the arrays
        are None when want_result is False."""
        info = ServerResult()
        cd = cp = None
        if want_result:
            n = self._n[graph_id][0]
            cd = np.empty(n, np.int64)
            cp = np.empty(n, np.int32)
        check(lib().mosp_server_wait(self._h, int(ticket), _ptr(cd), _ptr(cp), C.byref(info)))
        return cd, cp, info

    def read_graph(self, graph_id):
        n, K = self._n[graph_id]
        v = C.c_longlong()
        d = np.empty(K * n, np.int64)
        p = np.empty(K * n, np.int32)
        cd = np.empty(n, np.int64)
        cp = np.empty(n, np.int32)
        check(lib().mosp_server_read_graph(self._h, graph_id, C.byref(v), _ptr(d), _ptr(p), _ptr(cd), _ptr(cp)))
        return v.value, d.reshape(K, n), p.reshape(K, n), cd, cp

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(lib().mosp_server_get_stats(self._h, C.byref(st)))
        return st


@dataclass
class DeviceGraph:
    """Out- and in-CSR with objective-major weight columns on the GPU
    (torch tensors), built by mosp_build_device_graph."""
    n: int
    m: int
    K: int
    out_row: object
    out_col: object
    out_w: object
    in_row: object
    in_col: object
    in_w: object

    @classmethod
    def upload(cls, ws: Workspace, g: HostGraph, device="cuda"):
        import torch
        row, col, w = g.arrays()
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        out_row, out_col, edge_w = t(row), t(col), t(w.reshape(-1))
        n, m, K = g.n, g.m, g.K
        out_w = torch.empty(max(m * K, 1), dtype=torch.int32, device=device)
        in_row = torch.empty(n + 1, dtype=torch.int32, device=device)
        in_col = torch.empty(max(m, 1), dtype=torch.int32, device=device)
        in_w = torch.empty(max(m * K, 1), dtype=torch.int32, device=device)
        ws.build_device_graph(n, m, K, out_row, out_col, edge_w, out_w, in_row, in_col, in_w)
        return cls(n, m, K, out_row, out_col, out_w, in_row, in_col, in_w)

    def out_w_col(self, k):
        return self.out_w.data_ptr() + 4 * k * self.m

    def in_w_col(self, k):
        return self.in_w.data_ptr() + 4 * k * self.m
