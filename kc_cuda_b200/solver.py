"""Python handle on the B200 kmax-truss solver (ctypes over libkt.so).

This is a thin host-side mirror of the C ABI in include/kt.h; all work runs
in the CUDA library.  There is no CPU fallback: if libkt.so is missing or no
CUDA device is present, constructing a Context raises.

Names follow the reference's entry points:
  kmax_truss(path)        -> (kmax, edges)   the `-f` path (src/kc_gpu.cpp:209-347)
  Graph.kmax_core(k)      -> k-core members  (kmax_core_gpu, src/kc.cu:770)
  Graph.tricount()        -> per-edge support (tricount_direct, src/kc.cu:584)
  Graph.kmax_truss()      -> (kmax, edges)   (kmax_truss, src/kc_gpu.cpp:129)
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkt.so")

KT_OK = 0
STATUS = {0: "KT_OK", 1: "KT_ERR_INVALID", 2: "KT_ERR_CUDA", 3: "KT_ERR_NOMEM", 4: "KT_ERR_PARSE",
          5: "KT_ERR_IO", 6: "KT_ERR_TIMEOUT", 7: "KT_ERR_LIMIT", 8: "KT_ERR_NODEV", 9: "KT_ERR_BUSY"}


class KtError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Stats(ctypes.Structure):
    _fields_ = [
        ("ms_parse", ctypes.c_double), ("ms_csr", ctypes.c_double), ("ms_kcore", ctypes.c_double),
        ("ms_subgraph", ctypes.c_double), ("ms_support", ctypes.c_double), ("ms_peel", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("kernel_launches", ctypes.c_uint64),
        ("core_vertices", ctypes.c_uint64), ("core_edges", ctypes.c_uint64),
        ("predict_vertices", ctypes.c_uint64), ("predict_edges", ctypes.c_uint64),
        ("cmax", ctypes.c_uint32), ("kmax_lower_bound", ctypes.c_uint32), ("levels", ctypes.c_uint32),
        ("rounds", ctypes.c_uint32),
        ("support_bytes", ctypes.c_uint64), ("peel_bytes", ctypes.c_uint64),
        ("ms_support_kernel", ctypes.c_double), ("ms_peel_kernel", ctypes.c_double),
        ("support_launches", ctypes.c_uint64), ("peel_launches", ctypes.c_uint64),
        ("device_bytes_peak", ctypes.c_uint64),
        ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
        ("peel_decrements", ctypes.c_uint64),
        ("batch_waves", ctypes.c_uint32), ("batch_graphs", ctypes.c_uint32),
        ("support_kernel_bytes", ctypes.c_uint64), ("support_row_words", ctypes.c_uint64),
        ("peel_recount_bytes", ctypes.c_uint64),
        ("csr_grouped", ctypes.c_uint32), ("pad0", ctypes.c_uint32),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class RequestResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int), ("kmax", ctypes.c_uint32), ("edges", ctypes.c_uint64),
        ("ms_wait", ctypes.c_double), ("ms_latency", ctypes.c_double),
        ("wave", ctypes.c_uint32), ("wave_graphs", ctypes.c_uint32),
        ("lane", ctypes.c_uint32), ("pad0", ctypes.c_uint32),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("pending", ctypes.c_uint64),
        ("waves", ctypes.c_uint64), ("max_wave_graphs", ctypes.c_uint64),
        ("ms_busy", ctypes.c_double), ("device_bytes_peak", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class TuneResult(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "recount_gamma", "dense_min_fill", "dense_max_n", "support_bitmap_max_n", "kcore_big_row",
        "peel_search_ratio", "dense_tile_mb", "kcore_blocks_per_sm", "kcore_window", "peel_bitset",
        "peel_split")] + [
        ("ms_first", ctypes.c_double), ("ms_best", ctypes.c_double), ("trials", ctypes.c_uint32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_LIB = None

# (name, restype, argtypes) of every entry point of include/kt.h.
_P, _U8P, _U32P, _U64P = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p
SIGNATURES = [
    ("kt_init", ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("kt_destroy", None, [_P]),
    ("kt_last_error", ctypes.c_char_p, [_P]),
    ("kt_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("kt_set_option", ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_int64]),
    ("kt_get_option", ctypes.c_int, [_P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]),
    ("kt_load_tsv", ctypes.c_int, [_P, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("kt_load_tsv_file", ctypes.c_int, [_P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("kt_load_pairs", ctypes.c_int, [_P, _U64P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("kt_graph_info", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    ("kt_graph_edges", ctypes.c_int, [_P, _P, _U64P]),
    ("kt_graph_free", None, [_P, _P]),
    ("kt_solve", ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)]),
    ("kt_solve_tsv", ctypes.c_int, [_P, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32),
                                    ctypes.POINTER(ctypes.c_uint64)]),
    ("kt_tsv_stage", ctypes.c_int, [_P, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("kt_solve_staged", ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)]),
    ("kt_tsv_free", None, [_P, _P]),
    ("kt_batch_create", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_void_p)]),
    ("kt_batch_add_pairs", ctypes.c_int, [_P, _U64P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32)]),
    ("kt_batch_add_mix", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    ("kt_batch_size", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    ("kt_batch_run", ctypes.c_int, [_P]),
    ("kt_batch_results", ctypes.c_int, [_P, _U32P, _U64P]),
    ("kt_batch_free", None, [_P]),
    ("kt_autotune", ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(TuneResult)]),
    ("kt_options_save", ctypes.c_int, [_P, ctypes.c_char_p]),
    ("kt_options_load", ctypes.c_int, [_P, ctypes.c_char_p]),
    ("kt_load_mix_graph", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("kt_kcore", ctypes.c_int, [_P, _P, ctypes.c_uint32, _U8P, ctypes.POINTER(ctypes.c_uint32)]),
    ("kt_kcore_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    ("kt_core_numbers", ctypes.c_int, [_P, _P, _U32P]),
    ("kt_edge_support", ctypes.c_int, [_P, _P, _U32P]),
    ("kt_edge_trussness", ctypes.c_int, [_P, _P, _U32P]),
    ("kt_server_create", ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]),
    ("kt_server_submit_pairs", ctypes.c_int, [_P, _U64P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("kt_server_submit_mix", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("kt_server_wait", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(RequestResult)]),
    ("kt_server_get_stats", ctypes.c_int, [_P, ctypes.POINTER(ServerStats)]),
    ("kt_server_destroy", None, [_P]),
    ("kt_get_stats", ctypes.c_int, [_P, ctypes.POINTER(Stats)]),
    ("kt_stats_reset", ctypes.c_int, [_P]),
]


def lib(path: str = LIB_PATH):
    """Loads libkt.so (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `make -C kc_cuda_b200` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(path)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def _buf(data) -> Tuple[ctypes.c_void_p, int, object]:
    if isinstance(data, np.ndarray):
        a = np.ascontiguousarray(data)
        return ctypes.c_void_p(a.ctypes.data), a.nbytes, a
    if isinstance(data, (bytes, bytearray, memoryview)):
        a = np.frombuffer(data, dtype=np.uint8)
        return ctypes.c_void_p(a.ctypes.data if a.size else 0), a.size, a
    raise TypeError("bytes or numpy array expected")


class Context:
    """One CUDA device, one stream, one HBM budget."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        L = lib()
        h = ctypes.c_void_p()
        s = L.kt_init(device, hbm_budget, ctypes.byref(h))
        if s != KT_OK:
            raise KtError(s, L.kt_status_string(s).decode())
        self._h = h
        self._L = L

    def close(self):
        if getattr(self, "_h", None):
            self._L.kt_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def check(self, s: int):
        if s != KT_OK:
            raise KtError(s, self._L.kt_last_error(self._h).decode())

    def set_option(self, name: str, value: int):
        self.check(self._L.kt_set_option(self._h, name.encode(), int(value)))

    def get_option(self, name: str) -> int:
        v = ctypes.c_int64()
        self.check(self._L.kt_get_option(self._h, name.encode(), ctypes.byref(v)))
        return v.value

    def save_options(self, path: str):
        self.check(self._L.kt_options_save(self._h, path.encode()))

    def load_options(self, path: str):
        self.check(self._L.kt_options_load(self._h, path.encode()))

    def stats(self) -> dict:
        st = Stats()
        self.check(self._L.kt_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        self.check(self._L.kt_stats_reset(self._h))

    # ---- ingest
    def load_tsv(self, data) -> "Graph":
        p, n, keep = _buf(data)
        g = ctypes.c_void_p()
        self.check(self._L.kt_load_tsv(self._h, p, n, ctypes.byref(g)))
        return Graph(self, g)

    def load_tsv_file(self, path: str) -> "Graph":
        g = ctypes.c_void_p()
        self.check(self._L.kt_load_tsv_file(self._h, path.encode(), ctypes.byref(g)))
        return Graph(self, g)

    def load_pairs(self, xy: np.ndarray) -> "Graph":
        xy = np.ascontiguousarray(xy, dtype=np.uint64)
        g = ctypes.c_void_p()
        self.check(self._L.kt_load_pairs(self._h, xy.ctypes.data if xy.size else None, xy.size, ctypes.byref(g)))
        return Graph(self, g)

    def load_edges(self, pairs: np.ndarray) -> "Graph":
        """Graph from an (m, 2) array of endpoints."""
        p = np.asarray(pairs, dtype=np.uint64).reshape(-1, 2)
        return self.load_pairs((p[:, 0] << np.uint64(32)) | p[:, 1])

    def stage_tsv(self, data) -> "StagedTsv":
        """Copies TSV bytes into device memory (inputs resident in HBM)."""
        p, n, keep = _buf(data)
        t = ctypes.c_void_p()
        self.check(self._L.kt_tsv_stage(self._h, p, n, ctypes.byref(t)))
        return StagedTsv(self, t, n)

    def load_mix_graph(self, index: int, base_seed: int = 0x4B54) -> "Graph":
        g = ctypes.c_void_p()
        self.check(self._L.kt_load_mix_graph(self._h, index, base_seed, ctypes.byref(g)))
        return Graph(self, g)

    def batch(self) -> "Batch":
        return Batch(self)

    def server(self, max_wave_graphs: int = 0) -> "Server":
        return Server(self, max_wave_graphs)

    # ---- one-call solve
    def solve_tsv(self, data) -> Tuple[int, int]:
        p, n, keep = _buf(data)
        k = ctypes.c_uint32()
        e = ctypes.c_uint64()
        self.check(self._L.kt_solve_tsv(self._h, p, n, ctypes.byref(k), ctypes.byref(e)))
        return k.value, e.value


class Batch:
    """Many graphs solved together (waves of disjoint unions)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx.check(ctx._L.kt_batch_create(ctx._h, ctypes.byref(h)))
        self._h = h

    def free(self):
        if getattr(self, "_h", None):
            self.ctx._L.kt_batch_free(self._h)
            self._h = None

    def __del__(self):
        self.free()

    def add_pairs(self, xy: np.ndarray) -> int:
        xy = np.ascontiguousarray(xy, dtype=np.uint64)
        gid = ctypes.c_uint32()
        self.ctx.check(self.ctx._L.kt_batch_add_pairs(self._h, xy.ctypes.data if xy.size else None, xy.size,
                                                      ctypes.byref(gid)))
        return gid.value

    def add_edges(self, pairs: np.ndarray) -> int:
        p = np.asarray(pairs, dtype=np.uint64).reshape(-1, 2)
        return self.add_pairs((p[:, 0] << np.uint64(32)) | p[:, 1])

    def add_mix(self, first: int, count: int, base_seed: int = 0x4B54):
        self.ctx.check(self.ctx._L.kt_batch_add_mix(self._h, first, count, base_seed))

    def size(self) -> Tuple[int, int]:
        g = ctypes.c_uint64()
        r = ctypes.c_uint64()
        self.ctx.check(self.ctx._L.kt_batch_size(self._h, ctypes.byref(g), ctypes.byref(r)))
        return g.value, r.value

    def run(self):
        self.ctx.check(self.ctx._L.kt_batch_run(self._h))

    def autotune(self, passes: int = 1) -> dict:
        """Tunes the context's kernel thresholds on this batch (a sample of
        graphs like the ones to be solved); returns the chosen settings and
        the sample's device time before and after."""
        r = TuneResult()
        self.ctx.check(self.ctx._L.kt_autotune(self._h, passes, ctypes.byref(r)))
        return r.as_dict()

    def results(self) -> Tuple[np.ndarray, np.ndarray]:
        n = self.size()[0]
        k = np.zeros(max(n, 1), dtype=np.uint32)
        e = np.zeros(max(n, 1), dtype=np.uint64)
        self.ctx.check(self.ctx._L.kt_batch_results(self._h, k.ctypes.data, e.ctypes.data))
        return k[:n], e[:n]


class Server:
    """Continuous-batching serving loop on a context (kt_server_*): submit
    graphs at any time, collect each result with its latency."""

    def __init__(self, ctx: Context, max_wave_graphs: int = 0):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx.check(ctx._L.kt_server_create(ctx._h, max_wave_graphs, ctypes.byref(h)))
        self._h = h

    def _check(self, s: int):
        if s != KT_OK:
            raise KtError(s, STATUS.get(s, str(s)))

    def submit_pairs(self, xy: np.ndarray) -> int:
        xy = np.ascontiguousarray(xy, dtype=np.uint64)
        rid = ctypes.c_uint64()
        self._check(self.ctx._L.kt_server_submit_pairs(self._h, xy.ctypes.data if xy.size else None, xy.size,
                                                       ctypes.byref(rid)))
        return rid.value

    def submit_mix(self, index: int, base_seed: int = 0x4B54) -> int:
        rid = ctypes.c_uint64()
        self._check(self.ctx._L.kt_server_submit_mix(self._h, index, base_seed, ctypes.byref(rid)))
        return rid.value

    def poll(self, rid: int) -> Optional[dict]:
        """The request's result, or None while it is pending."""
        return self.wait(rid, 0)

    def wait(self, rid: int, timeout_ms: int = 600_000) -> Optional[dict]:
        r = RequestResult()
        s = self.ctx._L.kt_server_wait(self._h, rid, timeout_ms, ctypes.byref(r))
        if s == 6:  # KT_ERR_TIMEOUT: still pending
            return None
        self._check(s)
        return r.as_dict()

    def stats(self) -> dict:
        st = ServerStats()
        self._check(self.ctx._L.kt_server_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def close(self):
        """Finishes every queued request and stops the worker."""
        if getattr(self, "_h", None):
            self.ctx._L.kt_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class StagedTsv:
    """TSV bytes held in device memory by a context."""

    def __init__(self, ctx: Context, h, nbytes: int):
        self.ctx = ctx
        self._h = h
        self.nbytes = nbytes

    def solve(self) -> Tuple[int, int]:
        k = ctypes.c_uint32()
        e = ctypes.c_uint64()
        self.ctx.check(self.ctx._L.kt_solve_staged(self.ctx._h, self._h, ctypes.byref(k), ctypes.byref(e)))
        return k.value, e.value

    def free(self):
        if getattr(self, "_h", None) and self.ctx._h:
            self.ctx._L.kt_tsv_free(self.ctx._h, self._h)
        self._h = None

    def __del__(self):
        self.free()


class Graph:
    """A cleaned graph resident on the device."""

    def __init__(self, ctx: Context, h):
        self.ctx = ctx
        self._h = h

    def free(self):
        if getattr(self, "_h", None) and self.ctx._h:
            self.ctx._L.kt_graph_free(self.ctx._h, self._h)
        self._h = None

    def __del__(self):
        self.free()

    def info(self) -> Tuple[int, int]:
        n = ctypes.c_uint64()
        m = ctypes.c_uint64()
        self.ctx.check(self.ctx._L.kt_graph_info(self._h, ctypes.byref(n), ctypes.byref(m)))
        return n.value, m.value

    @property
    def num_vertices(self) -> int:
        return self.info()[0]

    @property
    def num_edges(self) -> int:
        return self.info()[1]

    def edges(self) -> np.ndarray:
        m = self.num_edges
        out = np.zeros(max(m, 1), dtype=np.uint64)
        self.ctx.check(self.ctx._L.kt_graph_edges(self.ctx._h, self._h, out.ctypes.data))
        return out[:m]

    def kmax_truss(self) -> Tuple[int, int]:
        k = ctypes.c_uint32()
        e = ctypes.c_uint64()
        self.ctx.check(self.ctx._L.kt_solve(self.ctx._h, self._h, ctypes.byref(k), ctypes.byref(e)))
        return k.value, e.value

    def kmax_core(self, k: int) -> Tuple[np.ndarray, int]:
        """(membership of the k-core as bool[n], largest k with a non-empty core)."""
        n = self.num_vertices
        mem = np.zeros(max(n, 1), dtype=np.uint8)
        cmax = ctypes.c_uint32()
        self.ctx.check(self.ctx._L.kt_kcore(self.ctx._h, self._h, k, mem.ctypes.data, ctypes.byref(cmax)))
        return mem[:n].astype(bool), cmax.value

    def core_numbers(self) -> np.ndarray:
        n = self.num_vertices
        out = np.zeros(max(n, 1), dtype=np.uint32)
        self.ctx.check(self.ctx._L.kt_core_numbers(self.ctx._h, self._h, out.ctypes.data))
        return out[:n]

    def tricount(self) -> np.ndarray:
        """Triangles through each edge, in edges() order."""
        m = self.num_edges
        out = np.zeros(max(m, 1), dtype=np.uint32)
        self.ctx.check(self.ctx._L.kt_edge_support(self.ctx._h, self._h, out.ctypes.data))
        return out[:m]

    def trussness(self) -> np.ndarray:
        m = self.num_edges
        out = np.zeros(max(m, 1), dtype=np.uint32)
        self.ctx.check(self.ctx._L.kt_edge_trussness(self.ctx._h, self._h, out.ctypes.data))
        return out[:m]


def kmax_truss(path: str, device: int = 0) -> Tuple[int, int]:
    """The reference's `-f <path>` answer: (kmax, edges in the kmax-truss)."""
    with Context(device) as ctx:
        g = ctx.load_tsv_file(path)
        try:
            return g.kmax_truss()
        finally:
            g.free()
