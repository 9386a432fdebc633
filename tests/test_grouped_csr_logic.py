"""CPU transcription of the graph build's grouped-input route
(k_grouped_rows, k_grouped_degrees, the upper-arc count check,
k_grouped_split, the stable sort of the transposed lower arcs by their first
column, and k_equal_u64 in kc_cuda_b200/csrc/csr.cu), run line by line.

The route must accept exactly the reference's input contract with ascending
rows (lines grouped by ascending second column, every edge in both
directions, no repeats, no self-loops or blank lines, ids without long gaps)
and then produce the sorting route's graph: row offsets, sorted rows, degrees
and the sorted canonical edge list.  Every broken variant must be refused
(the device then takes the sorting route)."""
import numpy as np
import pytest

import kt_oracle as O
from kc_cuda_b200 import gen
from test_gpu_csr_grouped import contract_lines, render, variants

MAX_GAP = 4096
NONE = (1 << 64) - 1


def records(data: bytes):
    """The parser's records: y << 32 | x per line, ~0 for a blank line or a
    self-loop, and n = largest id + 1."""
    out, mx = [], -1
    for ln in data.split(b"\n")[:-1] if data.endswith(b"\n") else data.split(b"\n"):
        xy = O.parse(ln + b"\n")
        if len(xy) == 0:
            out.append(NONE)
            continue
        r = int(xy[0])  # x << 32 | y
        x, y = r >> 32, r & 0xFFFFFFFF
        mx = max(mx, x, y)
        out.append(NONE if x == y else (y << 32) | x)
    return out, mx + 1


def grouped_route(keys, n):
    """Returns (off, adj, deg, edges) or None when refused."""
    nk = len(keys)
    if nk == 0 or nk % 2 or n == 0:
        return None
    bad = False
    off = [None] * (n + 1)
    up = [None] * n
    adj = [0] * nk
    for i, k in enumerate(keys):  # k_grouped_rows, one iteration per thread
        if k == NONE:
            bad = True
            continue
        y, x = k >> 32, k & 0xFFFFFFFF
        adj[i] = x
        row_start, prev_up = True, False
        if i == 0:
            if y + 1 > MAX_GAP:
                bad = True
            else:
                for v in range(0, y + 1):
                    off[v] = 0
        else:
            p = keys[i - 1]
            if p != NONE:
                py = p >> 32
                if y < py:
                    bad = True
                elif y > py:
                    if y - py > MAX_GAP:
                        bad = True
                    else:
                        for v in range(py + 1, y + 1):
                            off[v] = i
                else:
                    row_start = False
                    if (p & 0xFFFFFFFF) >= x:
                        bad = True
                    prev_up = (p & 0xFFFFFFFF) > y
        if i == nk - 1:
            if n - y > MAX_GAP:
                bad = True
            else:
                for v in range(y + 1, n + 1):
                    off[v] = nk
        if x > y and (row_start or not prev_up):
            up[y] = i
    if bad:
        return None
    assert all(o is not None for o in off)  # every row start written once the checks pass
    deg, ucnt = [], []
    for v in range(n):  # k_grouped_degrees
        u = off[v + 1] if up[v] is None else up[v]
        up[v] = u
        deg.append(off[v + 1] - off[v])
        ucnt.append(off[v + 1] - u)
    eoff = np.concatenate([[0], np.cumsum(ucnt)]).astype(np.int64)
    if 2 * int(eoff[n]) != nk:
        return None
    m = nk // 2
    edges, low = [None] * m, [None] * m
    for i, k in enumerate(keys):  # k_grouped_split
        y, x = k >> 32, k & 0xFFFFFFFF
        if x > y:
            j = int(eoff[y]) + (i - up[y])
            assert 0 <= j < m and edges[j] is None
            edges[j] = k
        else:
            j = (off[y] - int(eoff[y])) + (i - off[y])
            assert 0 <= j < m and low[j] is None
            low[j] = (x << 32) | y
    # Stable sort by the high half, then entry-by-entry equality (k_equal_u64).
    low.sort(key=lambda t: t >> 32)
    if low != edges:
        return None
    return off, adj, deg, np.array(edges, dtype=np.uint64)


@pytest.mark.parametrize("spec", [gen.rmat(7, 8, 5, [8]), gen.rmat(8, 8, 9, [10]),
                                  gen.GraphSpec(kind=gen.KTG_ER, n=300, draws=2000, seed=4, cliques=[9])])
def test_contract_form_accepted_and_graph_equal(spec):
    gr = gen.Graph(spec)
    data = gr.tsv_bytes()
    keys, n = records(data)
    r = grouped_route(keys, n)
    assert r is not None
    off, adj, deg, edges = r
    want = O.clean(O.parse(data))
    assert np.array_equal(edges, want)
    # Rows: each vertex's neighbours, ascending.
    nb = [[] for _ in range(n)]
    for k in want:
        u, v = int(k) >> 32, int(k) & 0xFFFFFFFF
        nb[u].append(v)
        nb[v].append(u)
    for v in range(n):
        assert adj[off[v]:off[v + 1]] == sorted(nb[v])
        assert deg[v] == len(nb[v])


@pytest.mark.parametrize("spec", [gen.rmat(7, 8, 5, [8]), gen.GraphSpec(kind=gen.KTG_ER, n=300, draws=2000,
                                                                        seed=4, cliques=[9])])
def test_broken_forms_refused(spec):
    lines = contract_lines(gen.Graph(spec).edges())
    for name, v in variants(lines).items():
        keys, n = records(render(v))
        assert grouped_route(keys, n) is None, name


def test_edge_cases():
    tri = contract_lines(np.array([(0 << 32) | 1, (0 << 32) | 2, (1 << 32) | 2], dtype=np.uint64))
    assert grouped_route(*records(render(tri))) is not None
    assert grouped_route(*records(render([(1, 0), (0, 1)]))) is not None
    far = contract_lines(np.array([(0 << 32) | 1, (1 << 32) | 20000, (0 << 32) | 20000], dtype=np.uint64))
    assert grouped_route(*records(render(far))) is None
    # Isolated ids inside the range: rows without lines are empty rows.
    gap = contract_lines(np.array([(0 << 32) | 5, (5 << 32) | 9, (0 << 32) | 9], dtype=np.uint64))
    r = grouped_route(*records(render(gap)))
    assert r is not None and r[2] == [2, 0, 0, 0, 0, 2, 0, 0, 0, 2]
