"""The graph build's grouped-input route (rows taken straight from TSV lines
grouped by the second column, as the reference builds them: init_graph,
src/kc_gpu.cpp:38-65) against the oracle, and its fallback to the sorting
route on inputs that break the reference's input contract.

Every variant must give the oracle's cleaned edge list and the oracle's
answer; the contract form must take the grouped route, every broken form the
sorting route."""
import numpy as np
import pytest

import kt_oracle as O
import kc_cuda_b200 as K
from kc_cuda_b200 import gen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = K.Context(0)
    yield c
    c.close()


def contract_lines(edges: np.ndarray):
    """(x, y) lines of the contract form: both directions, grouped by y
    ascending, x ascending within a group."""
    u = (edges >> np.uint64(32)).astype(np.int64)
    v = (edges & np.uint64(0xFFFFFFFF)).astype(np.int64)
    x = np.concatenate([v, u])
    y = np.concatenate([u, v])
    order = np.lexsort((x, y))
    return [(int(a), int(b)) for a, b in zip(x[order], y[order])]


def render(lines, sep="\t", tail="") -> bytes:
    out = []
    for ln in lines:
        if ln is None:
            out.append("\n")
        else:
            out.append(f"{ln[0]}{sep}{ln[1]}{tail}\n")
    return "".join(out).encode()


def groups(lines):
    """Start index of each group of equal y."""
    return [i for i in range(len(lines)) if i == 0 or lines[i][1] != lines[i - 1][1]]


def variants(lines):
    g = groups(lines)
    rng = np.random.default_rng(3)
    mid = len(lines) // 2
    lower = next(i for i in range(mid, len(lines)) if lines[i][0] < lines[i][1])
    upper = next(i for i in range(mid, len(lines)) if lines[i][0] > lines[i][1])
    # A group of three or more lines near the middle, and the group after it.
    gi = next(k for k in range(len(g) // 2, len(g) - 2) if g[k + 1] - g[k] >= 3)
    a, b, c = g[gi], g[gi + 1], g[gi + 2]
    y = lines[a][1]
    out = {
        "missing reverse (lower arc)": lines[:lower] + lines[lower + 1:],
        "missing reverse (upper arc)": lines[:upper] + lines[upper + 1:],
        "repeated line": lines[:mid] + [lines[mid]] + lines[mid:],
        "self-loop": lines[:a] + [(y, y)] + lines[a:],
        "group out of order": lines[:a] + lines[b:c] + lines[a:b] + lines[c:],
        "first line moved to the end of its group": lines[:a] + lines[a + 1:b] + [lines[a]] + lines[b:],
        "group split in two around the next": lines[:a + 1] + lines[b:c] + lines[a + 1:b] + lines[c:],
        "row not ascending": lines[:a] + [lines[a + 1], lines[a]] + lines[a + 2:],
        "blank line": lines[:mid] + [None] + lines[mid:],
    }
    # Random near-contract damage: a few swaps of whole lines.
    d = list(lines)
    for _ in range(3):
        i, j = rng.integers(0, len(d), size=2)
        d[i], d[j] = d[j], d[i]
    out["random swaps"] = d
    return out


def check(ctx, data: bytes, grouped: bool, name: str):
    want_edges = O.clean(O.parse(data))
    g = ctx.load_tsv(data)
    assert ctx.stats()["csr_grouped"] == int(grouped), name
    assert np.array_equal(g.edges(), want_edges), name
    assert g.kmax_truss() == O.solve_tsv(data), name
    g.free()


@pytest.mark.parametrize("spec", [gen.rmat(10, 8, 5, [12]), gen.rmat(12, 16, 9, [20]),
                                  gen.GraphSpec(kind=gen.KTG_ER, n=3000, draws=40000, seed=4, cliques=[15])])
def test_grouped_route_and_fallbacks(ctx, spec):
    gr = gen.Graph(spec)
    lines = contract_lines(gr.edges())
    data = render(lines)
    assert data == gr.tsv_bytes()  # the generator writes this same contract form
    check(ctx, data, True, "contract form")
    # Other separators, extra columns and CRLF keep the form.
    check(ctx, render(lines, sep=" ", tail="\t99\r"), True, "separators, extra column, CRLF")
    for name, v in variants(lines).items():
        check(ctx, render(v), False, name)


def test_grouped_route_edge_cases(ctx):
    # One edge; a triangle; ids with a gap longer than the route fills (sorting route).
    check(ctx, render([(1, 0), (0, 1)]), True, "one edge")
    tri = contract_lines(np.array([(0 << 32) | 1, (0 << 32) | 2, (1 << 32) | 2], dtype=np.uint64))
    check(ctx, render(tri), True, "triangle")
    far = contract_lines(np.array([(0 << 32) | 1, (1 << 32) | 20000, (0 << 32) | 20000], dtype=np.uint64))
    check(ctx, render(far), False, "gap of 20000 ids")
    # A first group far from id 0.
    late = contract_lines(np.array([(9000 << 32) | 9001, (9000 << 32) | 9002, (9001 << 32) | 9002],
                                   dtype=np.uint64))
    check(ctx, render(late), False, "first row at id 9000")
    # Odd line count (an arc without its reverse at the end).
    check(ctx, render(tri + [(5, 4)]), False, "odd line count")


def test_grouped_route_pipelined(ctx):
    """The chunked ingest of host bytes feeds the same route."""
    gr = gen.Graph(gen.rmat(14, 16, 11, [25]))
    data = gr.tsv_bytes()
    old = ctx.get_option("parse_pipeline_mb")
    ctx.set_option("parse_pipeline_mb", 1)
    try:
        assert len(data) >= 3 << 20
        g = ctx.load_tsv(data)
        assert ctx.stats()["csr_grouped"] == 1
        assert np.array_equal(g.edges(), gr.edges())
        assert g.kmax_truss() == O.solve_tsv(data)
        g.free()
    finally:
        ctx.set_option("parse_pipeline_mb", old)
