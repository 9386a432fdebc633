"""The per-graph bookkeeping of a batched peel (k_track, k_track_record and
k_track_init in kc_cuda_b200/csrc/peel.cu; the loop in truss_peel),
transcribed and checked on the CPU against each graph solved alone.

A wave is a disjoint union of graphs.  Edge e is removed in a cascade when
its support is below its graph's threshold gthr[g] (support units; 0 = the
graph is finished and its edges have left the alive list).  After each
cascade every running graph with alive edges records (its minimum support +
2, its alive edges) and continues at threshold minimum + 1; a graph with no
alive edge, or whose first level kept exactly stop[g] edges, finishes.  All
graphs share the cascades, so a graph's answer must not depend on the others
nor on where it starts (any first level up to its kmax)."""
import numpy as np

import kt_oracle as O
from kc_cuda_b200 import gen


def supports(edges, alive):
    nbr = {}
    for i in np.nonzero(alive)[0]:
        u, v = edges[i]
        nbr.setdefault(u, set()).add(v)
        nbr.setdefault(v, set()).add(u)
    sup = np.zeros(len(edges), np.int64)
    for i in np.nonzero(alive)[0]:
        u, v = edges[i]
        sup[i] = len(nbr[u] & nbr[v])
    return sup


def tracked_peel(edges, egr, ngroups, t0, stop):
    """(kmax, count) per graph, as the device records them."""
    gthr = np.array([max(t, 3) - 2 for t in t0], np.int64)   # k_track_init
    kmax = np.zeros(ngroups, np.int64)
    count = np.zeros(ngroups, np.int64)
    alive = np.ones(len(edges), bool)
    first = True
    while alive.any():
        while True:                                           # one cascade
            sup = supports(edges, alive)
            drop = alive & (sup < gthr[egr])
            if not drop.any():
                break
            alive &= ~drop
        sup = supports(edges, alive)
        for g in range(ngroups):                              # k_track + k_track_record
            if gthr[g] == 0:
                continue
            mine = alive & (egr == g)
            if mine.any():
                gmin = int(sup[mine].min())
                kmax[g], count[g] = gmin + 2, int(mine.sum())
                gthr[g] = 0 if (first and stop[g] and count[g] == stop[g]) else gmin + 1
            else:
                gthr[g] = 0
        alive &= gthr[egr] != 0                               # StillAlive
        first = False
    return list(zip(kmax.tolist(), count.tolist()))


def union(specs):
    parts, egr, base = [], [], 0
    for g, spec in enumerate(specs):
        e = gen.Graph(spec).edges()
        uv = np.stack([(e >> np.uint64(32)).astype(np.int64), (e & np.uint64(0xFFFFFFFF)).astype(np.int64)], 1)
        parts.append(uv + base)
        egr.append(np.full(len(uv), g))
        base += int(uv.max()) + 1 if len(uv) else 0
    return np.concatenate(parts), np.concatenate(egr), [O.solve_edges(gen.Graph(s).edges()) for s in specs]


def test_every_graph_climbs_its_own_levels():
    specs = [gen.rmat(6, 6, 1, [9]), gen.rmat(7, 4, 2, [5]), gen.rmat(6, 8, 3, []), gen.rmat(5, 3, 4, [4]),
             gen.rmat(6, 4, 5, [12])]
    edges, egr, alone = union(specs)
    G = len(specs)
    assert len({k for k, _ in alone}) >= 3
    assert tracked_peel(edges, egr, G, [3] * G, [0] * G) == alone
    # Own first levels anywhere up to each graph's kmax: same answers.
    rng = np.random.default_rng(9)
    t0 = [int(rng.integers(3, max(k, 3) + 1)) for k, _ in alone]
    assert tracked_peel(edges, egr, G, t0, [0] * G) == alone


def test_early_stop_on_the_first_level():
    """A graph whose first level keeps exactly stop[g] edges -- the phase-2
    case where the (L-1)-core's L-truss is the phase-1 truss -- finishes
    there with the same answer."""
    specs = [gen.rmat(6, 6, 1, [9]), gen.rmat(6, 4, 5, [12])]
    edges, egr, alone = union(specs)
    t0 = [k for k, _ in alone]
    stop = [c for _, c in alone]
    assert tracked_peel(edges, egr, 2, t0, stop) == alone
    # A stop count that does not match is ignored.
    assert tracked_peel(edges, egr, 2, t0, [c + 1 for c in stop]) == alone
