"""Serving loop: requests submitted while others run are admitted into later
waves, and every request's answer is the same alone and in the mix (the
single-graph path, the oracle, the reference's golden answers)."""
import time

import numpy as np
import pytest

import kt_oracle as O
from conftest import golden_bytes
from kc_cuda_b200 import gen
import kc_cuda_b200 as K

pytestmark = pytest.mark.gpu


def small_mix_indices(limit, max_draws=1_500_000, start=0):
    out = []
    i = start
    while len(out) < limit:
        if gen.mix_graph(i).draws <= max_draws:
            out.append(i)
        i += 1
    return out


def golden_graphs(golden):
    out = []
    for name, e in sorted(golden.items()):
        if "file" in e and "error" not in e:
            out.append((O.parse(golden_bytes(e)), (e["kmax"], e["edges"])))
    return out


def test_served_equals_alone_and_reference(golden):
    idx = small_mix_indices(16)
    graphs = golden_graphs(golden)
    with K.Context(0) as ctx:
        alone = {}
        for i in idx:
            g = ctx.load_mix_graph(i)
            alone[i] = g.kmax_truss()
            g.free()
        with ctx.server() as srv:
            rids = []
            # Three bursts: the later ones arrive while earlier waves run.
            for burst in range(3):
                for j, i in enumerate(idx):
                    if j % 3 == burst:
                        rids.append(("mix", i, srv.submit_mix(i)))
                for j, (xy, want) in enumerate(graphs):
                    if j % 3 == burst:
                        rids.append(("golden", j, srv.submit_pairs(xy)))
                time.sleep(0.002)
            waves = set()
            for kind, key, rid in rids:
                r = srv.wait(rid)
                assert r is not None and r["status"] == 0
                got = (r["kmax"], r["edges"])
                want = alone[key] if kind == "mix" else graphs[key][1]
                assert got == want, (kind, key)
                assert r["ms_latency"] >= r["ms_wait"] >= 0
                waves.add(r["wave"])
            st = srv.stats()
            assert st["completed"] == len(rids) and st["pending"] == 0
            assert st["waves"] == len(waves) >= 1
    # The oracle on a few of them.
    for i in idx[:4]:
        assert O.solve_edges(gen.Graph(gen.mix_graph(i)).edges()) == alone[i]


def test_requests_join_later_waves_with_a_wave_cap():
    idx = small_mix_indices(12, max_draws=400_000, start=100)
    with K.Context(0) as ctx:
        alone = {}
        for i in idx:
            g = ctx.load_mix_graph(i)
            alone[i] = g.kmax_truss()
            g.free()
        with ctx.server(max_wave_graphs=3) as srv:
            first = srv.submit_mix(idx[0])
            r0 = srv.wait(first)
            later = [(i, srv.submit_mix(i)) for i in idx[1:]]
            rs = [(i, srv.wait(rid)) for i, rid in later]
        assert r0["wave"] == 0 and r0["wave_graphs"] == 1
        for i, r in rs:
            assert (r["kmax"], r["edges"]) == alone[i]
            assert 1 <= r["wave_graphs"] <= 3 and r["wave"] >= 1
        assert len({r["wave"] for _, r in rs}) >= (len(later) + 2) // 3


def test_oversized_request_is_refused_and_server_keeps_serving():
    with K.Context(0, hbm_budget=64 << 20) as ctx:
        with ctx.server() as srv:
            big = np.arange(2_000_000, dtype=np.uint64) << np.uint64(32) | np.uint64(1)
            with pytest.raises(K.KtError) as e:
                srv.submit_pairs(big)
            assert e.value.status == 7  # KT_ERR_LIMIT
            tri = np.array([(0 << 32) | 1, (1 << 32) | 2, (0 << 32) | 2], dtype=np.uint64)
            r = srv.wait(srv.submit_pairs(tri))
            assert (r["status"], r["kmax"], r["edges"]) == (0, 3, 3)


def test_request_submitted_mid_wave_overtakes_it():
    """With two lanes, requests submitted while a large wave is on the device
    start in the other lane at once and finish before that wave ends; every
    answer equals the graph's alone."""
    big = gen.Graph(gen.rmat(20, 32, 5, [60]))
    bigxy = big.edges()
    small = small_mix_indices(4, max_draws=60_000, start=300)
    with K.Context(0) as ctx:
        assert ctx.get_option("serve_lanes") == 2
        g = ctx.load_pairs(bigxy)
        want_big = g.kmax_truss()
        g.free()
        alone = {}
        for i in small:
            g = ctx.load_mix_graph(i)
            alone[i] = g.kmax_truss()
            g.free()
        with ctx.server() as srv:
            tb = time.perf_counter()
            rb = srv.submit_pairs(bigxy)
            time.sleep(0.005)  # the large wave has started
            sub = []
            for i in small:
                sub.append((i, time.perf_counter(), srv.submit_mix(i)))
            res = [(i, ts, srv.wait(rid)) for i, ts, rid in sub]
            r_big = srv.wait(rb)
    assert (r_big["kmax"], r_big["edges"]) == want_big
    big_end = tb + r_big["ms_latency"] / 1e3
    for i, ts, r in res:
        assert (r["kmax"], r["edges"]) == alone[i]
        assert r["lane"] != r_big["lane"]
        assert ts + r["ms_wait"] / 1e3 < big_end  # its wave started before the large one ended
        assert ts + r["ms_latency"] / 1e3 < big_end  # and ended first


def test_one_lane_keeps_waves_in_order():
    idx = small_mix_indices(6, max_draws=200_000, start=500)
    with K.Context(0) as ctx:
        ctx.set_option("serve_lanes", 1)
        with ctx.server(max_wave_graphs=2) as srv:
            rs = [srv.wait(srv.submit_mix(i)) for i in idx]
        assert {r["lane"] for r in rs} == {0}
        for i, r in zip(idx, rs):
            g = ctx.load_mix_graph(i)
            assert (r["kmax"], r["edges"]) == g.kmax_truss()
            g.free()


@pytest.mark.parametrize("partition,coop", [(1, 0), (0, 1), (1, 1)])
def test_small_lane_modes(partition, coop):
    """The small-request lane's variants: cooperative launches taking turns
    (serve_small_coop 1) and the other lanes kept to large requests
    (serve_partition 1).  Every answer equals the graph's alone; with the
    partition, small requests (estimated footprint well under serve_small_mb)
    run on the last lane and large ones (well over it) on the other."""
    small = [5, 7, 10, 17, 23]
    large = [9, 16, 18, 19]
    with K.Context(0) as ctx:
        ctx.set_option("serve_small_mb", 16)
        ctx.set_option("serve_partition", partition)
        ctx.set_option("serve_small_coop", coop)
        alone = {}
        for i in small + large:
            g = ctx.load_mix_graph(i)
            alone[i] = g.kmax_truss()
            g.free()
        with ctx.server() as srv:
            rids = [(i, srv.submit_mix(i)) for pair in zip(large + [None], small) for i in pair if i is not None]
            rs = {i: srv.wait(rid) for i, rid in rids}
        ctx.set_option("serve_partition", 0)
        ctx.set_option("serve_small_coop", 0)
        ctx.set_option("serve_small_mb", 128)
    for i, r in rs.items():
        assert r["status"] == 0 and (r["kmax"], r["edges"]) == alone[i], i
    if partition:
        assert {rs[i]["lane"] for i in small} == {1}
        assert {rs[i]["lane"] for i in large} == {0}
