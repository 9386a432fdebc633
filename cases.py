"""Small, named workloads for profiling single kernels of the solver.

    python cases.py <case> [--reps N]

Cases (each fits in a few GB of device memory, inputs larger than L2):
  dense-support   Erdos-Renyi G(n=40000, M=48,000,000 draws), seed 7: one
                  kt_edge_support call -> k_dense_support<64> on ~46M edges
                  (bitset rows of 1250 words).
  core55k-support Erdos-Renyi G(n=55455, M=95,000,000 draws), seed 7: one
                  kt_edge_support call -> k_dense_support on ~92M edges with
                  bitset rows of 1736 words (385 MB of rows, above L2): the
                  shape of the bench graph's search core (55,455 vertices,
                  92.1M edges).
  er1m-support    Erdos-Renyi G(n=1,000,000, M=64,000,000 draws), seed 7: one
                  kt_edge_support call in list mode -> k_support_bitmap
                  (average degree ~128, the shape of the mix's largest
                  Erdos-Renyi graphs).
  rmat21-solve    R-MAT scale 21, edge factor 32, seed 2, cliques 80/120/200:
                  one kt_solve_staged (every stage; peel kernel k_cascade<8>).
  rmat16-solve    config-1 graph (R-MAT scale 16, edge factor 16, seed 1, K30).
  rmat24-solve    the bench graph (R-MAT scale 24, edge factor 32, seed 2,
                  cliques 80/120/200; 15.5 GB of TSV staged on the device).
  chunglu10m-solve  Chung-Lu, 10M vertices, 200M draws, exponent 2.1, expected
                  degrees capped at 400K, seed 3, a 150-vertex block of pair
                  probability 0.95 (config 3's shape at a fifth of its size).
  chunglu50m-solve  config 3 itself (32 GB of TSV staged on the device).
  mix-batch       graphs 0..255 (--graphs; --max-draws keeps the smaller
                  ones) of the batched mix in one kt_batch_run
                  (k_core_levels on the union, grouped support and peel).
  mix-largest     the --count largest of mix graphs 0..4095 (by draws) in one
                  kt_batch_run; --alone also solves them one at a time.
--verbose prints the solver's stage decisions and per-level cascades
(--verbose-alone: also for the graphs solved one at a time).
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from kc_cuda_b200 import gen
from kc_cuda_b200.solver import Context


def dense_support(reps: int, n: int = 40000, draws: int = 48_000_000, options=()) -> None:
    spec = gen.GraphSpec(kind=gen.KTG_ER, n=n, draws=draws, seed=7)
    g = gen.Graph(spec)
    with Context(0) as ctx:
        for name, v in options:
            ctx.set_option(name, v)
        dg = ctx.load_pairs(g.edges())
        for _ in range(reps):
            t = time.perf_counter()
            sup = dg.tricount()
            st = ctx.stats()
            print(f"support of {dg.num_edges} edges: {1e3 * (time.perf_counter() - t):.1f} ms, "
                  f"kernel {st['ms_support_kernel']:.2f} ms, row words read {st['support_row_words']}, "
                  f"sum {int(sup.astype(np.uint64).sum())}", flush=True)
        dg.free()


def solve(spec: gen.GraphSpec, reps: int, verbose: bool = False, options=()) -> None:
    g = gen.Graph(spec)
    data = g.tsv_bytes()
    del g
    with Context(0) as ctx:
        ctx.set_option("pool_reserve_mb", 1 << 30)  # no memory mapped mid-solve
        for name, v in options:
            ctx.set_option(name, v)
        if verbose:
            ctx.set_option("verbose", 1)
        t = ctx.stage_tsv(data)
        for _ in range(reps):
            r = t.solve()
            st = ctx.stats()
            stages = " ".join(f"{k[3:]} {st[k]:.1f}" for k in
                              ("ms_parse", "ms_csr", "ms_kcore", "ms_subgraph", "ms_support", "ms_peel"))
            print(f"{r} in {st['ms_total']:.1f} ms device ({stages})", flush=True)
        t.free()


def mix_batch(reps: int, verbose: bool = False, indices=None, options=(), alone: bool = False,
              verbose_alone: bool = False) -> None:
    indices = list(range(256)) if indices is None else indices
    with Context(0) as ctx:
        ctx.set_option("pool_reserve_mb", 1 << 30)
        for name, v in options:
            ctx.set_option(name, v)
        if verbose:
            ctx.set_option("verbose", 1)
        for _ in range(reps):
            b = ctx.batch()
            for i in indices:
                b.add_mix(i, 1)
            b.run()
            st = ctx.stats()
            k, _ = b.results()
            b.free()
            stages = " ".join(f"{x[3:]} {st[x]:.1f}" for x in
                              ("ms_parse", "ms_csr", "ms_kcore", "ms_subgraph", "ms_support", "ms_peel"))
            print(f"{len(indices)} mix graphs, kmax sum {int(k.sum())}, {st['ms_total']:.1f} ms device "
                  f"({st['batch_waves']} waves; stage sums: {stages}; support kernel {st['ms_support_kernel']:.1f}, "
                  f"peel kernel {st['ms_peel_kernel']:.1f}, {st['levels']} levels, {st['rounds']} rounds)", flush=True)
        if alone:
            ctx.set_option("verbose", 1 if verbose_alone else 0)
            tot = {x: 0.0 for x in ("ms_parse", "ms_csr", "ms_kcore", "ms_subgraph", "ms_support", "ms_peel",
                                    "ms_total", "ms_support_kernel", "ms_peel_kernel")}
            for i in indices:
                g = ctx.load_mix_graph(i)
                st = ctx.stats()
                tot["ms_parse"] += st["ms_parse"]
                tot["ms_csr"] += st["ms_csr"]
                g.kmax_truss()
                st = ctx.stats()
                for x in ("ms_kcore", "ms_subgraph", "ms_support", "ms_peel", "ms_total", "ms_support_kernel",
                          "ms_peel_kernel"):
                    tot[x] += st[x]
                g.free()
            print("one at a time: " + " ".join(f"{x[3:]} {v:.1f}" for x, v in tot.items()), flush=True)


def largest_mix(count: int, among: int = 4096):
    """The `count` mix graphs with the most draws among graphs 0..among-1."""
    sizes = sorted(((gen.mix_graph(i).draws, i) for i in range(among)), reverse=True)
    return sorted(i for _, i in sizes[:count])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["dense-support", "core55k-support", "er1m-support", "rmat21-solve", "rmat16-solve", "rmat24-solve",
                                     "chunglu10m-solve", "chunglu50m-solve", "mix-batch", "mix-largest"])
    ap.add_argument("--count", type=int, default=64, help="mix-largest: how many of the largest graphs")
    ap.add_argument("--graphs", type=int, default=256, help="mix-batch: graphs 0..N-1")
    ap.add_argument("--max-draws", type=int, default=0, help="mix-batch: only graphs of at most this many draws")
    ap.add_argument("--alone", action="store_true", help="mix cases: also solve the graphs one at a time")
    ap.add_argument("--verbose-alone", action="store_true")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="a solver option to set first (repeatable)")
    a = ap.parse_args()
    opts = [(o.split("=")[0], int(o.split("=")[1])) for o in a.option]
    if a.case == "dense-support":
        dense_support(a.reps, options=opts)
    elif a.case == "core55k-support":
        dense_support(a.reps, n=55455, draws=95_000_000, options=opts)
    elif a.case == "er1m-support":
        dense_support(a.reps, n=1_000_000, draws=64_000_000, options=opts)
    elif a.case == "rmat21-solve":
        solve(gen.rmat(21, 32, 2, [80, 120, 200]), a.reps, a.verbose, opts)
    elif a.case == "mix-batch":
        idx = [i for i in range(a.graphs) if not a.max_draws or gen.mix_graph(i).draws <= a.max_draws]
        mix_batch(a.reps, a.verbose, indices=idx, options=opts, alone=a.alone,
                  verbose_alone=a.verbose_alone)
    elif a.case == "mix-largest":
        mix_batch(a.reps, a.verbose, indices=largest_mix(a.count), options=opts, alone=a.alone,
                  verbose_alone=a.verbose_alone)
    elif a.case == "rmat24-solve":
        solve(gen.rmat_s24_ef32_k80_120_200(), a.reps, a.verbose, opts)
    elif a.case == "chunglu10m-solve":
        solve(gen.GraphSpec(kind=gen.KTG_CHUNGLU, n=10_000_000, draws=200_000_000, seed=3, cl_gamma=2.1,
                            cl_w_min=5.0, cl_w_max=400_000.0, block_size=150, block_p=0.95), a.reps, a.verbose,
              opts)
    elif a.case == "chunglu50m-solve":
        solve(gen.chunglu_50m(), a.reps, a.verbose, opts)
    else:
        solve(gen.rmat_s16_k30(), a.reps, a.verbose, opts)


if __name__ == "__main__":
    main()
