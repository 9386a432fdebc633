"""Regenerates the golden fixtures in this directory.

Each fixture is a graph in the solvers' TSV form plus the answer printed by
the REFERENCE solver kc_cpu, compiled from the reference sources by
`make -C oracle ref` (oracle/_ref/kc_cpu).  This script needs that binary, so
it runs where the reference sources are; the fixtures it writes are committed
and the tests only read them.

    python tests/golden/make_golden.py

Outputs:
  graphs/*.tsv      small graphs (hand-made edge cases and seeded generator
                    output), each well under 200 KB
  golden.json       {name: {file | spec, sha256, kmax, edges, threads}}

Larger generated graphs are recorded by spec only (their TSV is regenerated
by the seeded generator at test time); the sha256 of the generated TSV pins
the generator as well.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import kt_oracle as O  # noqa: E402
from kc_cuda_b200 import gen  # noqa: E402

GRAPHS = os.path.join(HERE, "graphs")


def tsv_of_edges(edges):
    """Reference input form: both directions, grouped by ascending column 2."""
    rows = []
    for u, v in edges:
        if u == v:
            continue
        rows.append((u, v))
        rows.append((v, u))
    rows = sorted(set(rows), key=lambda r: (r[1], r[0]))
    return "".join(f"{x}\t{y}\n" for x, y in rows).encode()


def clique(vs):
    return [(a, b) for i, a in enumerate(vs) for b in vs[i + 1:]]


def hand_made():
    g = {}
    g["empty"] = b""
    g["blank_lines"] = b"\n\n\n"
    g["single_edge"] = tsv_of_edges([(0, 1)])
    g["triangle"] = tsv_of_edges(clique([0, 1, 2]))
    g["triangle_crlf"] = tsv_of_edges(clique([0, 1, 2])).replace(b"\n", b"\r\n")
    g["k4"] = tsv_of_edges(clique([0, 1, 2, 3]))
    g["k5_sparse_ids"] = tsv_of_edges(clique([3, 17, 99, 1000, 4242]))
    g["k10"] = tsv_of_edges(clique(list(range(10))))
    g["square"] = tsv_of_edges([(0, 1), (1, 2), (2, 3), (3, 0)])
    g["star"] = tsv_of_edges([(0, i) for i in range(1, 50)])
    g["path"] = tsv_of_edges([(i, i + 1) for i in range(100)])
    g["bipartite_k5_5"] = tsv_of_edges([(a, b) for a in range(5) for b in range(5, 10)])
    g["two_triangles_shared_edge"] = tsv_of_edges([(0, 1), (1, 2), (0, 2), (1, 3), (0, 3)])
    g["bowtie"] = tsv_of_edges(clique([0, 1, 2]) + clique([2, 3, 4]))
    g["k6_plus_k4_tail"] = tsv_of_edges(clique(list(range(6))) + clique([5, 6, 7, 8]) + [(8, 9), (9, 10)])
    g["two_k7_disjoint"] = tsv_of_edges(clique(list(range(7))) + clique(list(range(10, 17))))
    g["k8_and_k6_bridge"] = tsv_of_edges(clique(list(range(8))) + clique(list(range(20, 26))) + [(7, 20)])
    g["hub_star_plus_clique"] = tsv_of_edges([(0, i) for i in range(1, 300)] + clique(list(range(1, 13))))
    g["wheel_20"] = tsv_of_edges([(0, i) for i in range(1, 21)] + [(i, i % 20 + 1) for i in range(1, 21)])
    g["extra_columns_and_spaces"] = b"".join(
        f"{x} {y}\t7\t8\n".encode() for x, y in sorted(
            {(a, b) for e in clique([0, 1, 2, 3]) for a, b in (e, e[::-1])}, key=lambda r: (r[1], r[0])))
    return g


def generated():
    out = {}
    specs = {}
    for s in range(6, 12):
        specs[f"rmat_s{s}_ef8_k{s + 2}"] = gen.rmat(s, 8, 100 + s, [s + 2])
    specs["rmat_s10_ef16_k20_k12"] = gen.rmat(10, 16, 7, [20, 12])
    specs["rmat_s12_ef4"] = gen.rmat(12, 4, 9)
    specs["er_n500_ef3"] = gen.GraphSpec(kind=gen.KTG_ER, n=500, draws=1500, seed=11)
    specs["er_n2000_ef8_k15"] = gen.GraphSpec(kind=gen.KTG_ER, n=2000, draws=16000, seed=12, cliques=[15])
    specs["er_n300_ef20"] = gen.GraphSpec(kind=gen.KTG_ER, n=300, draws=6000, seed=13)
    specs["chunglu_n3000"] = gen.GraphSpec(kind=gen.KTG_CHUNGLU, n=3000, draws=12000, seed=14,
                                           cl_gamma=2.1, cl_w_min=3.0, cl_w_max=300.0, block_size=25, block_p=0.9)
    specs["er_n100_ef1_triangle_free_likely"] = gen.GraphSpec(kind=gen.KTG_ER, n=100, draws=60, seed=15)
    for i in range(8):
        specs[f"mix_small_{i}"] = None
    for name, spec in specs.items():
        if spec is None:
            # Small members of the batched mix's families (R-MAT / ER + clique).
            i = int(name.rsplit("_", 1)[1])
            base = gen.mix_graph(i)
            n = 1000 + 137 * i
            spec = gen.GraphSpec(kind=base.kind, scale=max(1, (n - 1).bit_length()), n=n,
                                 draws=min(base.draws, 6 * n), seed=base.seed, cliques=base.cliques)
        g = gen.Graph(spec)
        out[name] = (g.tsv_bytes(), spec)
    return out


def main():
    if not O.have_kc_cpu():
        sys.exit("oracle/_ref/kc_cpu is missing: run `make -C oracle ref` where the reference sources are")
    os.makedirs(GRAPHS, exist_ok=True)
    golden = {}
    items = [(k, v, None) for k, v in hand_made().items()]
    items += [(k, v[0], v[1]) for k, v in generated().items()]
    for name, data, spec in items:
        path = os.path.join(GRAPHS, name + ".tsv")
        with open(path, "wb") as f:
            f.write(data)
        entry = {"file": f"graphs/{name}.tsv", "sha256": hashlib.sha256(data).hexdigest()}
        try:
            answers = {t: O.run_kc_cpu(path, threads=t) for t in (1, 8)}
        except RuntimeError as e:
            # The reference refuses the input (an empty file cannot be mapped).
            entry["error"] = str(e)
            golden[name] = entry
            print(f"{name:40s} reference error: {e}")
            continue
        if len(set(answers.values())) != 1:
            print(f"{name}: kc_cpu answer depends on threads: {answers}")
        kmax, edges = answers[8]
        entry.update({"kmax": kmax, "edges": edges, "threads": sorted(answers)})
        if spec is not None:
            entry["spec"] = spec.__dict__
        golden[name] = entry
        print(f"{name:40s} kmax={kmax:4d} edges={edges}")
    # Spec-only entries (TSV regenerated at test time).
    big = {"rmat_s16_ef16_k30": gen.rmat_s16_k30(), "rmat_s14_ef32_k40": gen.rmat(14, 32, 5, [40])}
    for name, spec in big.items():
        g = gen.Graph(spec)
        data = g.tsv_bytes()
        path = os.path.join("/tmp", f"golden_{name}.tsv")
        with open(path, "wb") as f:
            f.write(data)
        kmax, edges = O.run_kc_cpu(path, threads=8)
        golden[name] = {"spec": spec.__dict__, "sha256": hashlib.sha256(data).hexdigest(),
                        "kmax": kmax, "edges": edges, "threads": [8], "num_edges": g.num_edges,
                        "tsv_bytes": len(data)}
        os.remove(path)
        print(f"{name:40s} kmax={kmax:4d} edges={edges} (spec only)")
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
