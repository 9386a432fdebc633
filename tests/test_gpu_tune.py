"""Autotuner of the kernel thresholds: it times a sample batch under
candidate settings, keeps the fastest, never changes an answer, and its
choice survives a save / load round trip."""
import numpy as np
import pytest

from kc_cuda_b200 import gen
import kc_cuda_b200 as K

pytestmark = pytest.mark.gpu

TUNED = ("recount_gamma", "dense_min_fill", "dense_max_n", "support_bitmap_max_n", "kcore_big_row",
         "peel_search_ratio", "dense_tile_mb", "kcore_blocks_per_sm", "kcore_window", "peel_bitset",
         "peel_split")


def mix_indices(first, limit, max_draws=1_000_000):
    out, i = [], first
    while len(out) < limit:
        if gen.mix_graph(i).draws <= max_draws:
            out.append(i)
        i += 1
    return out


def batch_answers(ctx, indices):
    b = ctx.batch()
    for i in indices:
        b.add_mix(i, 1)
    b.run()
    k, c = b.results()
    b.free()
    return list(zip(k.tolist(), c.tolist()))


def test_autotune_keeps_answers_and_options(tmp_path):
    sample = mix_indices(200_000, 12)
    check = mix_indices(0, 16)
    with K.Context(0) as ref:
        want = batch_answers(ref, check)  # default settings
        defaults = {n: ref.get_option(n) for n in TUNED}
    with K.Context(0) as ctx:
        b = ctx.batch()
        for i in sample:
            b.add_mix(i, 1)
        r = b.autotune(passes=1)
        b.free()
        assert r["trials"] > 0 and r["ms_first"] > 0 and r["ms_best"] > 0
        for n in TUNED:
            assert ctx.get_option(n) == r[n], n
        # The tuned settings solve other graphs to the same answers.
        assert batch_answers(ctx, check) == want
        path = str(tmp_path / "tuned.txt")
        ctx.save_options(path)
        tuned = {n: ctx.get_option(n) for n in TUNED}
    with K.Context(0) as other:
        assert {n: other.get_option(n) for n in TUNED} == defaults
        other.load_options(path)
        assert {n: other.get_option(n) for n in TUNED} == tuned
        bad = tmp_path / "bad.txt"
        bad.write_text("no_such_option 3\n")
        with pytest.raises(K.KtError) as ei:
            other.load_options(str(bad))
        assert ei.value.status == 1
        assert {n: other.get_option(n) for n in TUNED} == tuned


@pytest.mark.parametrize("name,values", [
    ("kcore_big_row", [32, 100, 4096]),
    ("peel_search_ratio", [1, 3, 1000]),
    ("dense_tile_mb", [1, 500]),
    ("kcore_blocks_per_sm", [1, 2]),
    ("kcore_window", [1, 2, 7, 1000]),
    ("peel_bitset", [0, 1]),
    ("peel_split", [0, 1, 1000]),
    ("recount_gamma", [1, 1000]),
])
def test_thresholds_do_not_change_answers(name, values):
    """Every threshold the tuner may pick only selects a kernel variant:
    answers, core numbers and per-edge trussness stay the same."""
    g = gen.Graph(gen.rmat(13, 16, 11, [25]))
    pairs = g.edges()
    with K.Context(0) as ctx:
        d = ctx.load_pairs(pairs)
        want = (d.kmax_truss(), d.core_numbers(), d.trussness())
        for v in values:
            ctx.set_option(name, v)
            got = (d.kmax_truss(), d.core_numbers(), d.trussness())
            assert got[0] == want[0], (name, v)
            assert np.array_equal(got[1], want[1]), (name, v)
            assert np.array_equal(got[2], want[2]), (name, v)
        d.free()
