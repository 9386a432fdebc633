"""B200-native kmax-truss solver (CUDA library libkt.so behind a C ABI).

Host code lives in C++/CUDA (kc_cuda_b200/csrc); this package only loads it.
"""
from .solver import Context, Graph, KtError, kmax_truss, lib  # noqa: F401

__all__ = ["Context", "Graph", "KtError", "kmax_truss", "lib"]
