"""ctypes access to the CPU oracle (oracle/kt_oracle.c) and to the reference
solver kc_cpu built from the reference sources (oracle/_ref/kc_cpu).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, as the checker.  The solver package never
imports it.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")
_LIB = None


def build(ref: bool = False) -> None:
    """Compiles the restatement (and, with ref=True, the reference binaries
    from the reference sources when they are present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(BUILD, "libkt_oracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.kto_parse.restype = ctypes.c_int64
        L.kto_parse.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
        L.kto_clean.restype = ctypes.c_uint64
        L.kto_clean.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        for f in ("kto_core_numbers", "kto_support", "kto_trussness"):
            getattr(L, f).restype = None
            getattr(L, f).argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        L.kto_kmax_from_truss.restype = None
        L.kto_kmax_from_truss.argtypes = [ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)]
        L.kto_solve_tsv.restype = ctypes.c_int
        L.kto_solve_tsv.argtypes = [ctypes.c_char_p, ctypes.c_uint64,
                                    ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)]
        _LIB = L
    return _LIB


class ParseError(ValueError):
    def __init__(self, line: int):
        super().__init__(f"malformed record on line {line}")
        self.line = line


def parse(buf: bytes) -> np.ndarray:
    bad = ctypes.c_uint64(0)
    n = lib().kto_parse(buf, len(buf), None, ctypes.byref(bad))
    if n < 0:
        raise ParseError(bad.value)
    out = np.zeros(max(n, 1), dtype=np.uint64)
    lib().kto_parse(buf, len(buf), out.ctypes.data, ctypes.byref(bad))
    return out[:n]


def clean(xy: np.ndarray) -> np.ndarray:
    xy = np.ascontiguousarray(xy, dtype=np.uint64)
    out = np.zeros(max(len(xy), 1), dtype=np.uint64)
    m = lib().kto_clean(xy.ctypes.data, len(xy), out.ctypes.data)
    return out[:m].copy()


def _per_edge(fn, edges: np.ndarray, n: int = 0, size: Optional[int] = None) -> np.ndarray:
    edges = np.ascontiguousarray(edges, dtype=np.uint64)
    out = np.zeros(max(size if size is not None else len(edges), 1), dtype=np.uint32)
    fn(n, edges.ctypes.data, len(edges), out.ctypes.data)
    return out[: (size if size is not None else len(edges))]


def core_numbers(edges: np.ndarray, n: int) -> np.ndarray:
    return _per_edge(lib().kto_core_numbers, edges, n, size=n)


def support(edges: np.ndarray) -> np.ndarray:
    return _per_edge(lib().kto_support, edges)


def trussness(edges: np.ndarray) -> np.ndarray:
    return _per_edge(lib().kto_trussness, edges)


def kmax_from_truss(truss: np.ndarray) -> Tuple[int, int]:
    t = np.ascontiguousarray(truss, dtype=np.uint32)
    k = ctypes.c_uint32(0)
    c = ctypes.c_uint64(0)
    lib().kto_kmax_from_truss(t.ctypes.data, len(t), ctypes.byref(k), ctypes.byref(c))
    return int(k.value), int(c.value)


def solve_tsv(buf: bytes) -> Tuple[int, int]:
    k = ctypes.c_uint32(0)
    c = ctypes.c_uint64(0)
    rc = lib().kto_solve_tsv(buf, len(buf), ctypes.byref(k), ctypes.byref(c))
    if rc != 0:
        raise ValueError(f"oracle parse error {rc}")
    return int(k.value), int(c.value)


def solve_edges(edges: np.ndarray) -> Tuple[int, int]:
    return kmax_from_truss(trussness(edges))


# ------------------------------------------------------- reference kc_cpu

RESULT_RE = re.compile(rb"kmax = (\d+), Edges in kmax-truss = (\d+)\.")


def kc_cpu_path() -> str:
    return os.path.join(REF, "kc_cpu")


def have_kc_cpu() -> bool:
    return os.access(kc_cpu_path(), os.X_OK)


def run_kc_cpu(path: str, threads: Optional[int] = None, timeout: float = 600,
               binary: Optional[str] = None) -> Tuple[int, int]:
    """Runs the reference CPU solver on a TSV file and parses its answer.  A
    stand-in `vmtouch` (the reference shells out to it) goes first on PATH.
    binary: another build of it (e.g. oracle/_ref/kc_cpu_large)."""
    env = dict(os.environ)
    env["PATH"] = HERE + os.pathsep + env.get("PATH", "")
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    p = subprocess.run([binary or kc_cpu_path(), "-f", path], capture_output=True, env=env, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"kc_cpu failed ({p.returncode}): {p.stderr[-400:]!r}")
    m = RESULT_RE.search(p.stdout)
    if not m:
        raise RuntimeError(f"kc_cpu printed no result: {p.stdout[-400:]!r}")
    return int(m.group(1)), int(m.group(2))
