"""kt_kcore_noalloc: k-core membership with no device allocation.

It exists for callers that cannot allocate device memory when they need the
answer (a runtime whose memory pool is fully reserved, host callbacks where an
allocating CUDA call may block, latency-bound paths that cannot take the
synchronisation an allocation may imply): they pass a CSR and an output
buffer that already live on the device, and the library works in a fixed
static device array.  Its output must equal kt_kcore's, on two calls in a row
(the array keeps the previous call's contents).  This file runs last so a
failure here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

import kc_cuda_b200 as K
from kc_cuda_b200 import gen

pytestmark = pytest.mark.gpu

KT_ERR_INVALID = 1
KT_ERR_LIMIT = 7
MAX_VERTICES = 1 << 20


def host_csr(edges, n):
    u = (edges >> np.uint64(32)).astype(np.int64)
    v = (edges & np.uint64(0xFFFFFFFF)).astype(np.int64)
    src = np.concatenate([u, v])
    dst = np.concatenate([v, u])
    order = np.argsort(src, kind="stable")
    off = np.zeros(n + 1, dtype=np.int64)
    np.add.at(off, src + 1, 1)
    return np.cumsum(off), dst[order].astype(np.int32)


def test_kcore_noalloc_matches_kt_kcore():
    import torch

    L = K.lib()
    g = gen.Graph(gen.rmat(14, 16, 3, [40]))
    edges, n = g.edges(), g.num_vertices
    off, adj = host_csr(edges, n)
    # The caller owns every device buffer (allocated here through torch).
    d_off = torch.tensor(off, dtype=torch.int64, device="cuda")
    d_adj = torch.tensor(adj, dtype=torch.int32, device="cuda")
    d_mem = torch.empty(n, dtype=torch.uint8, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    with K.Context(0) as ctx:
        dg = ctx.load_edges(np.stack([edges >> np.uint64(32), edges & np.uint64(0xFFFFFFFF)], axis=1))
        _, cmax = dg.kmax_core(1)
        assert cmax > 2
        for k in sorted({1, 2, cmax // 2, cmax, cmax + 1}):
            want, _ = dg.kmax_core(k)
            for _call in range(2):
                d_mem.fill_(7)
                st = L.kt_kcore_noalloc(ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_adj.data_ptr()), n, k,
                                        ctypes.c_void_p(d_mem.data_ptr()), stream)
                assert st == 0, st
                got = d_mem.cpu().numpy()
                assert set(np.unique(got)) <= {0, 1}
                assert np.array_equal(got.astype(bool), want), k
        dg.free()
    # Beyond the fixed array: a clear refusal, nothing launched.
    st = L.kt_kcore_noalloc(ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_adj.data_ptr()), MAX_VERTICES + 1,
                            2, ctypes.c_void_p(d_mem.data_ptr()), stream)
    assert st == KT_ERR_LIMIT
    # A missing adjacency is refused, not read through.
    st = L.kt_kcore_noalloc(ctypes.c_void_p(d_off.data_ptr()), None, n, 2, ctypes.c_void_p(d_mem.data_ptr()), stream)
    assert st == KT_ERR_INVALID
    # The point of the entry point: calls take no device memory.  With the
    # solver's context closed, only this test's own buffers are held, so the
    # device's free memory must not move across repeated calls.
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _call in range(3):
        st = L.kt_kcore_noalloc(ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_adj.data_ptr()), n, 2,
                                ctypes.c_void_p(d_mem.data_ptr()), stream)
        assert st == 0, st
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
