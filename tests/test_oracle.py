"""The CPU oracle against the reference's own answers (golden fixtures made
by running kc_cpu built from the reference sources)."""
import hashlib

import numpy as np
import pytest

import kt_oracle as O
from conftest import golden_bytes
from kc_cuda_b200 import gen


def test_fixture_hashes(golden):
    for name, e in golden.items():
        if "file" in e:
            assert hashlib.sha256(golden_bytes(e)).hexdigest() == e["sha256"], name


def test_oracle_matches_reference_on_fixtures(golden):
    checked = 0
    for name, e in golden.items():
        if "file" not in e or "error" in e:
            continue
        assert O.solve_tsv(golden_bytes(e)) == (e["kmax"], e["edges"]), name
        checked += 1
    assert checked >= 35


def test_oracle_matches_reference_on_generated_specs(golden):
    for name, e in golden.items():
        if "file" in e:
            continue
        spec = gen.GraphSpec(**e["spec"])
        g = gen.Graph(spec)
        data = g.tsv_bytes()
        # The generator is pinned too: same spec, same bytes.
        assert hashlib.sha256(data).hexdigest() == e["sha256"], name
        assert O.solve_edges(g.edges()) == (e["kmax"], e["edges"]), name


def test_messy_input_same_graph(golden):
    """Shuffled rows, one/both directions, repeats, self-loops, CRLF and other
    separators describe the same cleaned graph, so the same answer."""
    for name, e in golden.items():
        if "spec" not in e or "file" not in e:
            continue
        g = gen.Graph(gen.GraphSpec(**e["spec"]))
        assert O.solve_tsv(g.tsv_bytes(messy=True, mess_seed=3)) == (e["kmax"], e["edges"]), name


def test_parse_grammar():
    xy = O.parse(b"\n 1\t2\n3 4 5\r\n\n#\n6,7\n8\t9")
    assert [(int(v) >> 32, int(v) & 0xFFFFFFFF) for v in xy] == [(1, 2), (3, 4), (6, 7), (8, 9)]
    with pytest.raises(O.ParseError) as ei:
        O.parse(b"1\t2\n5\n3\t4\n")
    assert ei.value.line == 1
    # Bytes >= '0' count as digits (the reference's test); >= 0x80 do not.
    assert int(O.parse(b"a\t1\n")[0]) >> 32 == ord("a") - ord("0")
    assert [int(v) >> 32 for v in O.parse(b"12\xff34\t5\n")] == [12]


def test_clean_and_support_small():
    xy = np.array([(0 << 32) | 1, (1 << 32) | 0, (1 << 32) | 2, (2 << 32) | 0, (2 << 32) | 2, (0 << 32) | 1],
                  dtype=np.uint64)
    e = O.clean(xy)
    assert [(int(k) >> 32, int(k) & 0xFFFFFFFF) for k in e] == [(0, 1), (0, 2), (1, 2)]
    assert list(O.support(e)) == [1, 1, 1]
    assert list(O.trussness(e)) == [3, 3, 3]
    assert list(O.core_numbers(e, 4)) == [2, 2, 2, 0]


def test_core_numbers_against_definition():
    g = gen.Graph(gen.rmat(9, 8, 3, [12]))
    e, n = g.edges(), g.num_vertices
    core = O.core_numbers(e, n)
    # The k-core for k = max core: peel by definition and compare.
    k = int(core.max())
    alive = np.ones(n, bool)
    u = (e >> np.uint64(32)).astype(np.int64)
    v = (e & np.uint64(0xFFFFFFFF)).astype(np.int64)
    while True:
        keep = alive[u] & alive[v]
        deg = np.bincount(u[keep], minlength=n) + np.bincount(v[keep], minlength=n)
        drop = alive & (deg < k)
        if not drop.any():
            break
        alive &= ~drop
    assert alive.any()
    assert set(np.nonzero(alive)[0]) == set(np.nonzero(core >= k)[0])


def test_trussness_against_definition():
    """Every level of the oracle's per-edge trussness, not only kmax: for each
    k the k-truss found by definition (drop edges in fewer than k-2 triangles
    of the surviving graph until none is left) is the set truss >= k."""
    g = gen.Graph(gen.rmat(9, 8, 5, [10, 14]))
    e, n = g.edges(), g.num_vertices
    truss = O.trussness(e)
    u = (e >> np.uint64(32)).astype(np.int64)
    v = (e & np.uint64(0xFFFFFFFF)).astype(np.int64)
    assert int(truss.max()) >= 14
    for k in range(3, int(truss.max()) + 2):
        alive = np.ones(len(e), bool)
        while True:
            a = np.zeros((n, n), np.int64)
            a[u[alive], v[alive]] = 1
            a[v[alive], u[alive]] = 1
            sup = (a @ a)[u, v]
            drop = alive & (sup < k - 2)
            if not drop.any():
                break
            alive &= ~drop
        assert np.array_equal(alive, truss >= k), k
    assert O.kmax_from_truss(truss) == O.solve_edges(e)
