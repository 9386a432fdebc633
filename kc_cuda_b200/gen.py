"""Seeded synthetic graphs for the kmax-truss solver (ctypes over libktgen.so).

The named workloads below fix every generator parameter, so a workload name
plus its seed always produces the same graph.  The random conventions are
documented in ``csrc/ktgen_core.h``.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

KTG_RMAT, KTG_ER, KTG_CHUNGLU = 0, 1, 2


class _Spec(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_uint32),
        ("scale", ctypes.c_uint32),
        ("n", ctypes.c_uint64),
        ("draws", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("a_ppm", ctypes.c_uint32),
        ("b_ppm", ctypes.c_uint32),
        ("c_ppm", ctypes.c_uint32),
        ("n_cliques", ctypes.c_uint32),
        ("clique_sizes", ctypes.c_uint32 * 8),
        ("cl_gamma", ctypes.c_double),
        ("cl_w_min", ctypes.c_double),
        ("cl_w_max", ctypes.c_double),
        ("block_size", ctypes.c_uint32),
        ("block_p_ppm", ctypes.c_uint32),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libktgen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run `make -C kc_cuda_b200`")
        L = ctypes.CDLL(path)
        L.ktg_make.restype = ctypes.c_void_p
        L.ktg_make.argtypes = [ctypes.POINTER(_Spec), ctypes.c_int]
        L.ktg_free.argtypes = [ctypes.c_void_p]
        L.ktg_num_vertices.restype = ctypes.c_uint64
        L.ktg_num_vertices.argtypes = [ctypes.c_void_p]
        L.ktg_num_edges.restype = ctypes.c_uint64
        L.ktg_num_edges.argtypes = [ctypes.c_void_p]
        L.ktg_edges.restype = ctypes.POINTER(ctypes.c_uint64)
        L.ktg_edges.argtypes = [ctypes.c_void_p]
        L.ktg_tsv_size.restype = ctypes.c_uint64
        L.ktg_tsv_size.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64]
        L.ktg_tsv_fill.restype = ctypes.c_uint64
        L.ktg_tsv_fill.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int]
        L.ktg_tsv_write.restype = ctypes.c_int
        L.ktg_tsv_write.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int]
        L.ktg_raw_draws.restype = ctypes.c_int
        L.ktg_raw_draws.argtypes = [ctypes.POINTER(_Spec), ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
        L.ktg_mix_spec.restype = ctypes.c_int
        L.ktg_mix_spec.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(_Spec)]
        L.ktg_sample_vertices.restype = ctypes.c_int
        L.ktg_sample_vertices.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p]
        _LIB = L
    return _LIB


@dataclass
class GraphSpec:
    kind: int = KTG_RMAT
    scale: int = 16
    n: int = 0
    draws: int = 0
    seed: int = 1
    a: float = 0.57
    b: float = 0.19
    c: float = 0.19
    cliques: List[int] = field(default_factory=list)
    cl_gamma: float = 2.1
    cl_w_min: float = 5.0
    cl_w_max: float = 2.0e6
    block_size: int = 0
    block_p: float = 0.0

    def to_c(self) -> _Spec:
        s = _Spec()
        s.kind, s.scale, s.n, s.draws, s.seed = self.kind, self.scale, self.n, self.draws, self.seed
        s.a_ppm, s.b_ppm, s.c_ppm = round(self.a * 1e6), round(self.b * 1e6), round(self.c * 1e6)
        if len(self.cliques) > 8:
            raise ValueError("at most 8 planted cliques")
        s.n_cliques = len(self.cliques)
        for i, c in enumerate(self.cliques):
            s.clique_sizes[i] = c
        s.cl_gamma, s.cl_w_min, s.cl_w_max = self.cl_gamma, self.cl_w_min, self.cl_w_max
        s.block_size, s.block_p_ppm = self.block_size, round(self.block_p * 1e6)
        return s

    @property
    def num_ids(self) -> int:
        if self.kind == KTG_RMAT:
            full = 1 << self.scale
            return full if self.n == 0 or self.n > full else self.n
        return self.n


class Graph:
    """A cleaned undirected simple graph held by the generator library."""

    def __init__(self, spec: GraphSpec, threads: int = 0):
        self.spec = spec
        self._c = spec.to_c()
        self._h = lib().ktg_make(ctypes.byref(self._c), threads)
        if not self._h:
            raise ValueError(f"generator rejected spec {spec}")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ktg_free(h)
            self._h = None

    @property
    def num_vertices(self) -> int:
        return int(lib().ktg_num_vertices(self._h))

    @property
    def num_edges(self) -> int:
        return int(lib().ktg_num_edges(self._h))

    def edges(self) -> np.ndarray:
        """Sorted canonical keys u << 32 | v (u < v) as uint64."""
        m = self.num_edges
        if m == 0:
            return np.zeros(0, dtype=np.uint64)
        p = lib().ktg_edges(self._h)
        return np.ctypeslib.as_array(p, shape=(m,)).copy()

    def edge_pairs(self) -> np.ndarray:
        k = self.edges()
        return np.stack([(k >> np.uint64(32)).astype(np.uint32), (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)], axis=1)

    def tsv_bytes(self, messy: bool = False, mess_seed: int = 7, threads: int = 0) -> bytes:
        mode = 1 if messy else 0
        size = int(lib().ktg_tsv_size(self._h, mode, mess_seed))
        buf = ctypes.create_string_buffer(size)
        w = int(lib().ktg_tsv_fill(self._h, mode, mess_seed, buf, threads))
        return buf.raw[:w]

    def tsv_into(self, out: np.ndarray, threads: int = 0) -> int:
        """Writes the contract-form TSV into a preallocated uint8 array."""
        size = self.tsv_size()
        if out.nbytes < size:
            raise ValueError("buffer too small")
        return int(lib().ktg_tsv_fill(self._h, 0, 0, out.ctypes.data, threads))

    def tsv_size(self, messy: bool = False, mess_seed: int = 7) -> int:
        return int(lib().ktg_tsv_size(self._h, 1 if messy else 0, mess_seed))

    def write_tsv(self, path: str, messy: bool = False, mess_seed: int = 7, threads: int = 0) -> None:
        rc = lib().ktg_tsv_write(self._h, 1 if messy else 0, mess_seed, path.encode(), threads)
        if rc != 0:
            raise OSError(f"writing {path} failed ({rc})")


def raw_draws(spec: GraphSpec, first: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    c = spec.to_c()
    if lib().ktg_raw_draws(ctypes.byref(c), first, count, out.ctypes.data) != 0:
        raise ValueError("raw draws are defined for R-MAT and Erdos-Renyi specs")
    return out


def sample_vertices(seed: int, stream: int, n: int, size: int) -> np.ndarray:
    out = np.zeros(size, dtype=np.uint32)
    if lib().ktg_sample_vertices(seed, stream, n, size, out.ctypes.data) != 0:
        raise ValueError("size > n")
    return out


# ---------------------------------------------------------------- workloads

def rmat_s16_k30() -> GraphSpec:
    """R-MAT scale 16, edge factor 16, a/b/c/d = .57/.19/.19/.05, seed 1, K30 planted."""
    return GraphSpec(kind=KTG_RMAT, scale=16, draws=16 << 16, seed=1, cliques=[30])


def rmat_s24_ef32_k80_120_200() -> GraphSpec:
    """R-MAT scale 24, edge factor 32, seed 2, cliques of 80, 120 and 200 planted."""
    return GraphSpec(kind=KTG_RMAT, scale=24, draws=32 << 24, seed=2, cliques=[80, 120, 200])


def chunglu_50m() -> GraphSpec:
    """Chung-Lu, 50M vertices, power-law exponent 2.1, expected degrees capped
    at 2M, ~1B edges, seed 3, a 150-vertex block with pair probability 0.95."""
    n = 50_000_000
    # Mean of min(w_max, w_min U^(-1/1.1)) with w_min = 5 is ~40, so the
    # draws below give ~1B undirected edges before repeats are merged.
    return GraphSpec(kind=KTG_CHUNGLU, n=n, draws=1_000_000_000, seed=3,
                     cl_gamma=2.1, cl_w_min=5.0, cl_w_max=2.0e6, block_size=150, block_p=0.95)


def rmat(scale: int, ef: int, seed: int, cliques: Optional[List[int]] = None) -> GraphSpec:
    return GraphSpec(kind=KTG_RMAT, scale=scale, draws=ef << scale, seed=seed, cliques=list(cliques or []))


def mix_graph(index: int, base_seed: int = 0x4B54) -> GraphSpec:
    """Graph `index` of the batched mix (4,096 graphs in the batched workload):
    n log-uniform over [1e3, 1e6]; R-MAT (a/b/c/d = .57/.19/.19/.05) or
    Erdos-Renyi with equal chance; edge factor uniform over 4..64; one clique
    of size uniform over 5..60.  The choices come from the C library
    (ktg_mix_spec) so host and device agree."""
    c = _Spec()
    if lib().ktg_mix_spec(index, base_seed, ctypes.byref(c)) != 0:
        raise ValueError("bad mix index")
    return GraphSpec(kind=c.kind, scale=c.scale, n=c.n, draws=c.draws, seed=c.seed,
                     cliques=[c.clique_sizes[0]])
