"""The two bounds the device driver uses to skip or stop work, checked on the
oracle's trussness (tests only): a non-empty t-truss

* has at least t vertices each with at least t-1 of its edges, every one of
  support >= t-2 in the whole graph, so a level where fewer than t vertices
  have t-1 such edges is empty (the prediction phase skips it before any
  rebuild, truss_possible in kc_cuda_b200/csrc/solve.cu);
* has at least t(t-1)/2 edges, so a level tried from a snapshot whose
  cascade leaves fewer edges than that is empty (the cascade gives up,
  PeelArgs::fail_below in kc_cuda_b200/csrc/peel.cu).

Both must hold at every non-empty level of every graph; the first must also
reject no level that is non-empty."""
import numpy as np

import kt_oracle as O
from conftest import golden_bytes
from kc_cuda_b200 import gen


def graphs(golden):
    for name, e in golden.items():
        if "file" in e and "error" not in e:
            yield name, O.clean(O.parse(golden_bytes(e)))
    for spec in (gen.rmat(9, 8, 5, [10, 14]), gen.rmat(10, 16, 3, [25]),
                 gen.GraphSpec(kind=gen.KTG_ER, n=300, draws=6000, seed=4, cliques=[18])):
        yield str(spec), gen.Graph(spec).edges()


def vertices_with_support(edges, sup, t):
    """Vertices with at least t-1 incident edges of support >= t-2."""
    keep = sup >= t - 2
    u = (edges[keep] >> np.uint64(32)).astype(np.int64)
    v = (edges[keep] & np.uint64(0xFFFFFFFF)).astype(np.int64)
    deg = np.bincount(np.concatenate([u, v])) if len(u) else np.zeros(0, np.int64)
    return int((deg >= t - 1).sum())


def test_truss_levels_meet_both_bounds(golden):
    checked = 0
    for name, edges in graphs(golden):
        if len(edges) == 0:
            continue
        truss = O.trussness(edges)
        sup = O.support(edges)
        for t in range(3, int(truss.max()) + 1):
            inside = truss >= t
            if not inside.any():
                continue
            assert inside.sum() >= t * (t - 1) // 2, (name, t)
            assert vertices_with_support(edges, sup, t) >= t, (name, t)
            checked += 1
    assert checked > 100
