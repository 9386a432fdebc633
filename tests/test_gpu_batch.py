"""Batched solving: every graph's answer in a batch equals its answer alone
(the single-graph path) and the reference's (golden fixtures)."""
import numpy as np
import pytest

import kt_oracle as O
from conftest import golden_bytes
from kc_cuda_b200 import gen
import kc_cuda_b200 as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = K.Context(0)
    yield c
    c.close()


def small_mix_indices(limit=24, max_draws=1_500_000):
    out = []
    i = 0
    while len(out) < limit:
        if gen.mix_graph(i).draws <= max_draws:
            out.append(i)
        i += 1
    return out


def test_batch_of_golden_fixtures(ctx, golden):
    b = ctx.batch()
    want = []
    for name, e in sorted(golden.items()):
        if "file" not in e or "error" in e:
            continue
        b.add_pairs(O.parse(golden_bytes(e)))
        want.append((e["kmax"], e["edges"]))
    b.run()
    k, c = b.results()
    assert list(zip(k.tolist(), c.tolist())) == want
    assert ctx.stats()["batch_graphs"] == len(want)


def test_device_generator_matches_host_generator(ctx):
    for i in small_mix_indices(6):
        host = gen.Graph(gen.mix_graph(i))
        dev = ctx.load_mix_graph(i)
        assert np.array_equal(dev.edges(), host.edges()), i
        dev.free()


def test_batched_mix_equals_graph_alone(ctx):
    idx = small_mix_indices(24)
    alone = []
    for i in idx:
        g = ctx.load_mix_graph(i)
        alone.append(g.kmax_truss())
        g.free()
    b = ctx.batch()
    for i in idx:
        b.add_mix(i, 1)
    b.run()
    k, c = b.results()
    assert list(zip(k.tolist(), c.tolist())) == alone
    # Oracle on the smallest ones.
    for j, i in enumerate(idx[:6]):
        assert O.solve_edges(gen.Graph(gen.mix_graph(i)).edges()) == alone[j], i


@pytest.mark.parametrize("capped", [1, 0])
def test_batch_of_golden_specs_and_files(ctx, golden, capped):
    """The generated golden graphs (R-MAT with dense cores, two phases) and
    the golden files in one batch, with the capped search-phase support of
    the single-graph path switched on and off: the reference's answers."""
    graphs = []
    for name, e in sorted(golden.items()):
        if "spec" in e:
            graphs.append((gen.Graph(gen.GraphSpec(**e["spec"])).edges(), (e["kmax"], e["edges"])))
        elif "file" in e and "error" not in e:
            graphs.append((O.parse(golden_bytes(e)), (e["kmax"], e["edges"])))
    ctx.set_option("capped_support", capped)
    try:
        b = ctx.batch()
        for xy, _ in graphs:
            b.add_pairs(xy)
        b.run()
        k, cnt = b.results()
        b.free()
        assert list(zip(k.tolist(), cnt.tolist())) == [w for _, w in graphs]
    finally:
        ctx.set_option("capped_support", 1)


def test_batch_in_several_waves_same_answers(golden):
    """A small HBM budget forces many waves; answers must not change."""
    graphs = []
    for name, e in sorted(golden.items()):
        if "file" in e and "error" not in e:
            graphs.append((O.parse(golden_bytes(e)), (e["kmax"], e["edges"])))
    with K.Context(0, hbm_budget=256 << 20) as c:
        b = c.batch()
        for xy, _ in graphs:
            b.add_pairs(xy)
        b.run()
        k, cnt = b.results()
        assert list(zip(k.tolist(), cnt.tolist())) == [w for _, w in graphs]
        assert c.stats()["batch_waves"] >= 1


def test_empty_and_trivial_graphs_in_batch(ctx):
    b = ctx.batch()
    b.add_pairs(np.zeros(0, dtype=np.uint64))
    b.add_edges(np.array([[0, 1]]))
    b.add_edges(np.array([[0, 1], [1, 2], [2, 0]]))
    b.add_edges(np.array([[5, 5]]))
    b.run()
    k, c = b.results()
    assert list(zip(k.tolist(), c.tolist())) == [(0, 0), (0, 0), (3, 3), (0, 0)]


def test_batch_lanes_same_answers_as_one_lane():
    """Waves in flight on two lanes (two contexts' streams) give the answers of
    one lane, wave for wave; a small budget forces many waves."""
    idx = small_mix_indices(40, max_draws=400_000)
    with K.Context(0, hbm_budget=256 << 20) as c:
        got = {}
        for lanes in (1, 2):
            c.set_option("batch_lanes", lanes)
            b = c.batch()
            for i in idx:
                b.add_mix(i, 1)
            b.run()
            st = c.stats()
            assert st["batch_waves"] >= 2
            got[lanes] = b.results()
            b.free()
        assert np.array_equal(got[1][0], got[2][0]) and np.array_equal(got[1][1], got[2][1])
        for j, i in enumerate(idx[:8]):
            g = c.load_mix_graph(i)
            assert g.kmax_truss() == (int(got[2][0][j]), int(got[2][1][j]))
            g.free()
