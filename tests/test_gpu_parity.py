"""GPU parity: the CUDA solver through the C ABI against the reference's
answers (golden fixtures from kc_cpu) and against the CPU oracle's stage
outputs, bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import kt_oracle as O
from conftest import ROOT, golden_bytes
from kc_cuda_b200 import gen
import kc_cuda_b200 as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = K.Context(0)
    yield c
    c.close()


def spec_graphs(golden):
    for name, e in golden.items():
        if "spec" in e and "file" not in e:
            yield name, e, gen.Graph(gen.GraphSpec(**e["spec"]))


def test_golden_fixtures_tsv(ctx, golden):
    for name, e in golden.items():
        if "file" not in e:
            continue
        data = golden_bytes(e)
        if "error" in e:
            continue
        assert ctx.solve_tsv(data) == (e["kmax"], e["edges"]), name


def test_golden_fixtures_file_path(ctx, golden):
    for name, e in golden.items():
        if "file" not in e:
            continue
        path = os.path.join(ROOT, "tests", "golden", e["file"])
        if "error" in e:
            with pytest.raises(K.KtError) as ei:
                ctx.load_tsv_file(path)
            assert ei.value.status == 5 and "mmap file error" in ei.value.message
            continue
        g = ctx.load_tsv_file(path)
        assert g.kmax_truss() == (e["kmax"], e["edges"]), name


def test_golden_generated_specs(ctx, golden):
    for name, e, g in spec_graphs(golden):
        assert ctx.solve_tsv(g.tsv_bytes()) == (e["kmax"], e["edges"]), name


def test_messy_input_same_answer(ctx, golden):
    for name, e in golden.items():
        if "spec" not in e or "file" not in e:
            continue
        g = gen.Graph(gen.GraphSpec(**e["spec"]))
        assert ctx.solve_tsv(g.tsv_bytes(messy=True, mess_seed=11)) == (e["kmax"], e["edges"]), name


def test_csr_matches_oracle_clean(ctx, golden):
    for name, e in golden.items():
        if "file" not in e or "error" in e:
            continue
        data = golden_bytes(e)
        want = O.clean(O.parse(data))
        g = ctx.load_tsv(data)
        assert np.array_equal(g.edges(), want), name


def random_record_bytes(seed: int, lines: int) -> bytes:
    """Lines of two digit runs in the parser's grammar with every kind of
    byte around them: runs of 1 to 12 "digits" (leading zeros, then up to 4
    significant bytes from 0x30..0x7f, so letters count as digits worth up
    to 79; values stay below 10^5), separators of 1 to 3 bytes from tab,
    space, comma, CR, control bytes, '/', NUL and bytes >= 0x80 (negative as
    signed char), optional trailing columns, CRLF endings and blank lines."""
    rng = np.random.default_rng(seed)
    seps = [b"\t", b" ", b",", b"\r", b"\x01", b"/", b"\x80", b"\xff", b"\x1f", b"\x00"]
    out = bytearray()
    for _ in range(lines):
        kind = rng.integers(0, 20)
        if kind == 0:
            out += b"".join(seps[i] for i in rng.integers(0, 5, rng.integers(0, 4))) + b"\n"
            continue
        parts = []
        for _ in range(2 + (rng.integers(0, 3) if kind == 1 else 0)):
            lead = b"".join(seps[i] for i in rng.integers(0, len(seps), rng.integers(1, 4) if parts else rng.integers(0, 3)))
            total = int(rng.choice([1, 2, 3, 5, 7, 8, 8, 8, 9, 10, 12]))
            sig = min(total, int(rng.integers(1, 5)))
            hi = 0x80 if rng.integers(0, 6) == 0 else 0x3A
            run = b"0" * (total - sig) + bytes(rng.integers(0x30, hi, sig, dtype=np.uint8))
            parts.append(lead + run)
        out += b"".join(parts) + (b"\r\n" if rng.integers(0, 5) == 0 else b"\n")
    return bytes(out)


def test_parse_random_bytes(ctx):
    """The device parser (8-byte, byte-window and byte-loop paths) against the
    oracle's restatement of the reference grammar on mixed byte soup."""
    for seed in range(4):
        data = random_record_bytes(seed, 60_000)
        want = O.clean(O.parse(data))
        g = ctx.load_tsv(data)
        assert np.array_equal(g.edges(), want), seed
        g.free()


def test_pipelined_ingest(ctx):
    """Host bytes of three or more chunks go over in chunks overlapped with
    the parse (1 MB chunks here): the same graph as the one-shot path, the
    same records on byte soup, a line longer than a chunk (parsed again once
    every byte has landed), and a parse error numbered from the first line."""
    old = ctx.get_option("parse_pipeline_mb")
    ctx.set_option("parse_pipeline_mb", 1)
    try:
        g = gen.Graph(gen.rmat(15, 16, 3, [20]))
        data = g.tsv_bytes()
        assert len(data) > 3 << 20
        d = ctx.load_tsv(data)
        assert np.array_equal(d.edges(), g.edges())
        assert d.kmax_truss() == ctx.solve_tsv(data)
        d.free()
        soup = random_record_bytes(7, 250_000)
        assert len(soup) > 3 << 20
        d = ctx.load_tsv(soup)
        assert np.array_equal(d.edges(), O.clean(O.parse(soup)))
        d.free()
        longline = b"1\t2\n" * 200_000 + b"3" + b" " * 2_500_000 + b"4\n" + b"5\t6\n4\t5\n" * 200_000
        d = ctx.load_tsv(longline)
        assert np.array_equal(d.edges(), O.clean(O.parse(longline)))
        d.free()
        bad = b"1\t2\n" * 1_000_000 + b"7\n" + b"2\t3\n" * 10
        with pytest.raises(K.KtError) as ei:
            ctx.load_tsv(bad)
        assert ei.value.status == 4 and "line 1000001" in ei.value.message
    finally:
        ctx.set_option("parse_pipeline_mb", old)


def test_csr_large_random_pairs(ctx):
    rng = np.random.default_rng(5)
    n = 1 << 18
    x = rng.integers(0, n, 3_000_000, dtype=np.uint64)
    y = (x + rng.integers(0, 64, x.size, dtype=np.uint64)) % np.uint64(n)  # repeats and self-loops
    xy = (x << np.uint64(32)) | y
    g = ctx.load_pairs(xy)
    assert np.array_equal(g.edges(), O.clean(xy))


def test_support_matches_oracle(ctx, golden):
    for name, e in golden.items():
        if "file" not in e or "error" in e:
            continue
        g = ctx.load_tsv(golden_bytes(e))
        edges = g.edges()
        assert np.array_equal(g.tricount(), O.support(edges)), name


def test_trussness_matches_oracle(ctx, golden):
    for name, e in golden.items():
        if "file" not in e or "error" in e:
            continue
        g = ctx.load_tsv(golden_bytes(e))
        edges = g.edges()
        t = g.trussness()
        assert np.array_equal(t, O.trussness(edges)), name
        if len(edges):
            assert O.kmax_from_truss(t) == (e["kmax"], e["edges"]), name


def test_core_numbers_and_kcore(ctx, golden):
    for name, e in golden.items():
        if "file" not in e or "error" in e:
            continue
        g = ctx.load_tsv(golden_bytes(e))
        n = g.num_vertices
        core = O.core_numbers(g.edges(), n)
        assert np.array_equal(g.core_numbers(), core), name
        cmax = int(core.max()) if n else 0
        for k in sorted({1, 2, max(1, cmax // 2), cmax, cmax + 1}):
            mem, cm = g.kmax_core(k)
            assert cm == cmax, name
            assert np.array_equal(mem, core >= k), (name, k)


@pytest.mark.parametrize("persistent", [1, 0])
def test_core_numbers_generated(ctx, persistent):
    """Core numbers of larger generated graphs by the one-launch level loop
    (persistent=1) and by host-stepped probes (persistent=0), and k-core
    membership by the maximum-core search: R-MAT hubs with rows above the
    big-row thresholds (512 in the rounds, 2048 in the compaction), a
    Chung-Lu graph, a mix graph, and a small graph with isolated vertex ids."""
    specs = [
        gen.rmat(15, 24, 5, [40]),
        gen.GraphSpec(kind=gen.KTG_CHUNGLU, n=200_000, draws=1_500_000, seed=9, cl_w_max=20_000.0),
        gen.mix_graph(17),
        gen.rmat(8, 2, 3),
    ]
    ctx.set_option("persistent", persistent)
    try:
        for spec in specs:
            g = gen.Graph(spec)
            d = ctx.load_pairs(g.edges())
            n = d.num_vertices
            edges = d.edges()
            want = O.core_numbers(edges, n)
            got = d.core_numbers()
            assert np.array_equal(got, want), (spec, persistent)
            # k-core membership through the maximum-core search (compacted
            # copies of the core, hub rows included).
            cmax = int(want.max()) if n else 0
            for k in sorted({2, max(1, cmax // 4), max(1, cmax // 2), cmax}):
                mem, cm = d.kmax_core(k)
                assert cm == cmax, (spec, k)
                assert np.array_equal(mem, want >= k), (spec, k)
            d.free()
    finally:
        ctx.set_option("persistent", 1)


def test_kcore_restore_from_nested_compactions(ctx, golden):
    """With a compacted copy made at almost every successful probe
    (kcore_compact 1: whenever the core has lost edges), a restore below the
    last copy's level starts from the deepest earlier copy at or below it:
    k-core membership for levels spread over 1..cmax equals the oracle's, and
    the solver's answers (whose search phase restores the (L-1)-core) equal
    the golden ones."""
    ctx.set_option("kcore_compact", 1)
    try:
        specs = [gen.GraphSpec(kind=gen.KTG_CHUNGLU, n=200_000, draws=1_500_000, seed=9, cl_w_max=20_000.0),
                 gen.rmat(15, 24, 5, [40])]
        for spec in specs:
            g = gen.Graph(spec)
            d = ctx.load_pairs(g.edges())
            want = O.core_numbers(d.edges(), d.num_vertices)
            cmax = int(want.max())
            for k in sorted(set(np.linspace(1, cmax, 12).astype(int).tolist()) | {max(1, cmax - 1)}):
                mem, cm = d.kmax_core(k)
                assert cm == cmax, (spec, k)
                assert np.array_equal(mem, want >= k), (spec, k)
            d.free()
        for name, e, gg in spec_graphs(golden):
            assert ctx.solve_tsv(gg.tsv_bytes()) == (e["kmax"], e["edges"]), name
    finally:
        ctx.set_option("kcore_compact", 4)


def test_config1_rmat_s16(ctx, golden):
    e = golden["rmat_s16_ef16_k30"]
    g = gen.Graph(gen.GraphSpec(**e["spec"]))
    assert ctx.solve_tsv(g.tsv_bytes()) == (e["kmax"], e["edges"]) == (114, 8958)
    st = ctx.stats()
    assert st["cmax"] > 0 and st["core_edges"] > 0


def test_without_prediction_same_answer(ctx, golden):
    ctx.set_option("predict", 0)
    try:
        for name, e, g in spec_graphs(golden):
            assert ctx.solve_tsv(g.tsv_bytes()) == (e["kmax"], e["edges"]), name
    finally:
        ctx.set_option("predict", 1)


@pytest.mark.parametrize("mode", ["sparse", "dense_recount_always", "dense_recount_never", "dense_uncapped",
                                  "dense_merge_only", "dense_split_always", "bisect_always_sparse",
                                  "bisect_always_dense"])
def test_modes_support_trussness_answer(ctx, golden, mode):
    """Sparse lists vs dense bitsets, dense peels that recount every round vs
    never, dense peels that intersect sorted lists instead of bitset rows, and
    peels that bisect the truss levels after the first one (undoing empty
    levels from a snapshot): all bit-identical to the oracle."""
    opts = {"sparse": {"dense_max_n": 0},
            "dense_recount_always": {"dense_min_fill": 1 << 30, "recount_gamma": 1 << 30},
            "dense_recount_never": {"dense_min_fill": 1 << 30, "recount_gamma": 1},
            "dense_uncapped": {"dense_min_fill": 1 << 30, "capped_support": 0},
            "dense_merge_only": {"dense_min_fill": 1 << 30, "recount_gamma": 1, "peel_bitset": 0},
            "dense_split_always": {"dense_min_fill": 1 << 30, "recount_gamma": 1, "peel_split": 1 << 20},
            "bisect_always_sparse": {"dense_max_n": 0, "peel_bisect_after": 1, "peel_bisect_gap": 1},
            "bisect_always_dense": {"dense_min_fill": 1 << 30, "peel_bisect_after": 1, "peel_bisect_gap": 1}}[mode]
    old = {k: ctx.get_option(k) for k in opts}
    for k, v in opts.items():
        ctx.set_option(k, v)
    try:
        for name, e in golden.items():
            if "file" not in e or "error" in e:
                continue
            g = ctx.load_tsv(golden_bytes(e))
            edges = g.edges()
            assert np.array_equal(g.tricount(), O.support(edges)), (mode, name)
            assert np.array_equal(g.trussness(), O.trussness(edges)), (mode, name)
            assert g.kmax_truss() == (e["kmax"], e["edges"]), (mode, name)
        for name, e, gg in spec_graphs(golden):
            assert ctx.solve_tsv(gg.tsv_bytes()) == (e["kmax"], e["edges"]), (mode, name)
    finally:
        for k, v in old.items():
            ctx.set_option(k, v)


def test_search_fallback_support_kernel(ctx, golden):
    """The binary-search support kernel (used above the bitmap size limit)."""
    ctx.set_option("support_bitmap_max_n", 0)
    ctx.set_option("dense_max_n", 0)
    try:
        for name, e in golden.items():
            if "file" not in e or "error" in e:
                continue
            g = ctx.load_tsv(golden_bytes(e))
            assert np.array_equal(g.tricount(), O.support(g.edges())), name
            assert g.kmax_truss() == (e["kmax"], e["edges"]), name
    finally:
        ctx.set_option("support_bitmap_max_n", 1 << 20)
        ctx.set_option("dense_max_n", 1 << 16)


def test_parse_error_reports_line(ctx):
    with pytest.raises(K.KtError) as ei:
        ctx.solve_tsv(b"1\t2\n2\t3\n5\n3\t1\n")
    assert ei.value.status == 4 and "line 3" in ei.value.message
    # The context stays usable.
    assert ctx.solve_tsv(b"0\t1\n1\t2\n2\t0\n") == (3, 3)


def test_cli_matches_reference_output(golden):
    exe = os.path.join(ROOT, "kc_cuda_b200", "kt_solve")
    for name in ("triangle", "k10", "rmat_s10_ef16_k20_k12", "empty", "square"):
        e = golden[name]
        p = subprocess.run([exe, "-f", os.path.join(ROOT, "tests", "golden", e["file"])],
                           capture_output=True, text=True)
        if "error" in e:
            assert p.returncode == 255 and "mmap file error" in p.stderr
        else:
            assert p.returncode == 0, p.stderr
            assert p.stdout == f"kmax = {e['kmax']}, Edges in kmax-truss = {e['edges']}.\n"
