"""Benchmark: kmax-truss solve of one large graph per GPU, with the batched
and serving figures of the same run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rmat24|rmat21|rmat16|chunglu50m|mix4096|serve]
                    [--no-batched] [--no-serving] [--no-cpu-baseline]

Workload (default rmat24): undirected R-MAT, scale 24 (16.7M vertex ids), edge
factor 32 (536.9M draws), a/b/c/d = .57/.19/.19/.05, seed 2, cliques of 80,
120 and 200 planted on seeded random vertices, written as the reference's TSV
edge list (both directions, grouped by the second column).  chunglu50m is the
skewed-degree graph: Chung-Lu, 50M vertices, power-law exponent 2.1, expected
degrees capped at 2M, ~1B edge draws, seed 3, a 150-vertex block of pair
probability 0.95 (a 32 GB TSV).  Synthetic: the seeded generator in
kc_cuda_b200/csrc/ktgen.cpp.

One step = one solve of the whole graph:
  value : edges / device time of kt_solve_staged (TSV bytes already in HBM:
          parse, clean, CSR, k-core, support, peel), CUDA events on the
          library's stream.
  e2e   : edges / wall time of kt_solve_tsv from pinned host bytes (the
          host-to-device copy of the TSV and the device-to-host reads of the
          answer inside).
The TSV (16 GB) is larger than L2, so no flush is needed between steps.
`parity` compares the answer with the reference CPU solver's answer on the
same graph (kc_cpu, recorded in tests/golden/large_configs.json); a mismatch
fails the run.

`batched` (unless --no-batched): graphs/s of the batched path over graphs
0..4095 of the batched mix, against the one-graph-per-launch path over the
same 4,096 graphs (every answer compared), with a per-size-decile table.
`serving` (unless --no-serving): the serving loop under Poisson arrivals of
2,000 other mix graphs at 0.8 x the batched graphs/s; p50/p99 latency beside
the per-graph path under the same arrivals.  Both use fixed counts, not
--steps.

Under torchrun each rank solves its own replica on its own GPU (graphs are
independent units: no data-path collective); the step time is the max over
ranks and value counts the edges of all ranks.

--impl reference runs the reference's own CPU solver (kc_cpu, built from the
reference sources into oracle/_ref/) on a bounded sample of the same
workload family on all host cores; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# name: (scale, edge factor, seed, cliques) of an R-MAT graph, or a spec builder name
WORKLOADS = {
    "rmat24": (24, 32, 2, [80, 120, 200]),
    "rmat21": (21, 32, 2, [80, 120, 200]),
    "rmat16": (16, 16, 1, [30]),
    "chunglu50m": "chunglu_50m",
    "mix4096": None,  # batched alone: the 4,096-graph mix
    "serve": None,    # serving alone: Poisson arrivals of mix graphs
}
# CPU sample of the same family for the reference solver (about 10-30 s).
CPU_SAMPLE = (20, 32, 2, [80, 120, 200])
# Answers of the reference CPU solver on the single-graph workloads.
REFERENCE_ANSWERS = os.path.join(ROOT, "tests", "golden", "large_configs.json")


def workload_spec(name: str):
    """(config name, GraphSpec) of a single-graph workload."""
    from kc_cuda_b200 import gen
    w = WORKLOADS[name]
    if isinstance(w, str):
        spec = getattr(gen, w)()
        return "chunglu_n50m_g2.1_wmax2m_seed3_block150", spec
    scale, ef, seed, cliques = w
    return f"rmat{scale}_ef{ef}_seed{seed}_k" + "_".join(map(str, cliques)), gen.rmat(scale, ef, seed, cliques)


def reference_answer(config_name: str):
    """The reference CPU solver's (kmax, edges) on this workload, if recorded."""
    try:
        with open(REFERENCE_ANSWERS) as f:
            rec = json.load(f).get(config_name)
    except OSError:
        return None
    if not rec:
        return None
    return [int(rec["kmax"]), int(rec["kmax_truss_edges"])], rec


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def core_bitset_bytes(n: int) -> int:
    """Bytes of the dense support's bitset rows for an n-vertex core: one row
    of ceil(n/32) words per vertex, padded to whole 16-byte vectors."""
    words = ((n + 31) // 32 + 3) & ~3
    return n * words * 4


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def make_tsv(spec, pinned: bool):
    """Generates the workload graph and its TSV bytes (pinned host memory
    when torch can provide it)."""
    from kc_cuda_b200 import gen
    g = gen.Graph(spec)
    size = g.tsv_size()
    buf = None
    if pinned:
        try:
            import torch
            buf = torch.empty(size, dtype=torch.uint8, pin_memory=True).numpy()
        except Exception:
            buf = None
    if buf is None:
        import numpy as np
        buf = np.empty(size, dtype=np.uint8)
    g.tsv_into(buf)
    return g, buf


def cpu_baseline_run(steps: int, warmup: int, threads: int):
    """kc_cpu (reference sources, oracle/_ref) on the CPU sample.  Returns
    (edges/s, sample description, per-step seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import kt_oracle as O
    if not O.have_kc_cpu():
        return None, "oracle/_ref/kc_cpu missing", []
    from kc_cuda_b200 import gen
    scale, ef, seed, cliques = CPU_SAMPLE
    g = gen.Graph(gen.rmat(scale, ef, seed, cliques))
    m = g.num_edges
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "sample.tsv")
        g.write_tsv(path)
        with open(path, "rb") as f:  # page cache warm, as vmtouch would make it
            while f.read(1 << 26):
                pass
        times = []
        for i in range(warmup + steps):
            t0 = time.perf_counter()
            O.run_kc_cpu(path, threads=threads, timeout=900)
            dt = time.perf_counter() - t0
            if i >= warmup:
                times.append(dt)
    med = statistics.median(times)
    desc = (f"kc_cpu -f on R-MAT s{scale} ef{ef} seed {seed} + K{'/K'.join(map(str, cliques))} "
            f"({m} edges), whole-process wall time, median of {len(times)}, OMP_NUM_THREADS={threads}")
    return m / med, desc, times


def cpu_mix_sample(indices, threads: int, answers: dict):
    """kc_cpu on a seeded sample of mix graphs (the CPU baseline of the
    batched path, and the check of its answers against the reference solver):
    graphs/s of kc_cpu (whole-process wall time, one graph at a time on all
    host cores) and the mismatches against `answers`.  The reference's
    multi-threaded parse fails on some of these graphs (it crashes or never
    answers); such a graph is rerun on one thread, and the failure recorded."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import kt_oracle as O
    if not O.have_kc_cpu():
        return None
    from kc_cuda_b200 import gen
    total = 0.0
    mism, failed = [], []
    with tempfile.TemporaryDirectory() as d:
        for i in indices:
            path = os.path.join(d, f"mix{i}.tsv")
            gen.Graph(gen.mix_graph(i)).write_tsv(path)
            with open(path, "rb") as f:
                while f.read(1 << 26):
                    pass
            t0 = time.perf_counter()
            try:
                ref = O.run_kc_cpu(path, threads=threads, timeout=30)
                total += time.perf_counter() - t0
            except (RuntimeError, subprocess.TimeoutExpired) as e:
                failed.append([i, type(e).__name__])
                t0 = time.perf_counter()
                ref = O.run_kc_cpu(path, threads=1, timeout=300)
                total += time.perf_counter() - t0
            os.unlink(path)
            if tuple(ref) != tuple(answers[i]):
                mism.append([i, list(ref), list(answers[i])])
    return {"graphs": len(indices), "graphs_per_s": len(indices) / total, "cores": threads, "kind": "reference",
            "sample": f"kc_cpu -f on {len(indices)} seeded mix graphs of at most 4M draws, one at a time, "
                      "whole-process wall time",
            "answers_equal": not mism, "mismatches": mism,
            "multithreaded_failures": failed,
            "failure_note": "graphs on which kc_cpu on all host threads crashed or gave no answer within 30 s; "
                            "their answers (and times) are from kc_cpu on one thread"}


TUNE_FIRST = 2_000_000  # mix graphs of the autotuner's sample (away from the measured ones)
SERVE_FIRST = 1_000_000  # mix graphs of the serving workload (away from the batched ones)


def rank_index_ranges(rank: int, mix_graphs: int, tune_graphs: int, serve_requests: int, calib_graphs: int) -> dict:
    """Mix-graph index ranges [first, end) a replica uses.  Replicas solve
    independent graphs (no data-path collective): every rank takes its own
    slice of the batched mix, of the tuner's sample, and of the serving
    workload's calibration batch and requests, and no two ranges overlap."""
    serve = SERVE_FIRST + rank * (serve_requests + calib_graphs)
    return {
        "mix": (rank * mix_graphs, (rank + 1) * mix_graphs),
        "tune": (TUNE_FIRST + rank * tune_graphs, TUNE_FIRST + (rank + 1) * tune_graphs),
        "calib": (serve, serve + calib_graphs),
        "serve": (serve + calib_graphs, serve + calib_graphs + serve_requests),
    }


def ranges_for(args, rank: int) -> dict:
    return rank_index_ranges(rank, args.mix_graphs, args.tune_graphs, args.serve_requests, args.calib_graphs)


def autotune(ctx, args, rank):
    """Tunes the context's kernel thresholds on `tune_graphs` mix graphs from
    TUNE_FIRST on (kt_autotune); returns its report, or None when off."""
    if not args.tune_graphs:
        return None
    first = ranges_for(args, rank)["tune"][0]
    b = ctx.batch()
    b.add_mix(first, args.tune_graphs)
    t0 = time.perf_counter()
    tune = b.autotune(passes=1)
    b.free()
    tune["wall_s"] = round(time.perf_counter() - t0, 1)
    tune["sample_graphs"] = args.tune_graphs
    tune["sample_first"] = first
    return tune


def mix_sizes(first: int, count: int):
    """(index, edge keys) of mix graphs first..first+count-1: the generated
    draws plus the planted clique's edges."""
    from kc_cuda_b200 import gen
    out = []
    for i in range(first, first + count):
        s = gen.mix_graph(i)
        c = s.cliques[0] if s.cliques else 0
        out.append((i, s.draws + c * (c - 1) // 2))
    return out


def batch_run(ctx, indices=None, first=0, count=0, stages=None):
    """One kt_batch_run over mix graphs (a list of indices, or a range);
    returns (device ms of the whole run, waves, answers); `stages` (a dict)
    receives the stage times summed over the lanes."""
    b = ctx.batch()
    if indices is None:
        b.add_mix(first, count)
    else:
        for i in indices:
            b.add_mix(i, 1)
    b.run()
    st = ctx.stats()
    k, c = b.results()
    b.free()
    if stages is not None:
        stages.update({x[3:]: round(st[x], 1) for x in ("ms_parse", "ms_csr", "ms_kcore", "ms_subgraph",
                                                         "ms_support", "ms_peel", "ms_support_kernel",
                                                         "ms_peel_kernel")})
    return st["ms_total"], st["batch_waves"], [(int(a), int(e)) for a, e in zip(k, c)]


def solve_alone(ctx, index: int):
    """Mix graph `index` through the one-graph-per-launch path: device time of
    its generation, CSR build and solve (ms), and its answer."""
    g = ctx.load_mix_graph(index)
    st = ctx.stats()
    ms = st["ms_parse"] + st["ms_csr"]
    ans = g.kmax_truss()
    ms += ctx.stats()["ms_total"]
    g.free()
    return ms, ans


def measure_mix(ctx, args, rank, pg, threads):
    """Batched path vs the one-graph-per-launch path over graphs first..first+G-1
    of the mix (n log-uniform over [1e3, 1e6], R-MAT or Erdos-Renyi, edge factor
    4..64, one clique of 5..60), generated on the device (generation included
    in both: device time from the first generated draw to the last answer).
    Every batched answer is compared with the graph solved alone."""
    import numpy as np
    G = args.mix_graphs
    first = ranges_for(args, rank)["mix"][0]
    idx = list(range(first, first + G))
    # One graph per launch sequence: kt_load_mix_graph + kt_solve.
    for i in idx[: min(3, G)]:
        solve_alone(ctx, i)
    lat, alone = {}, {}
    for i in idx:
        lat[i], alone[i] = solve_alone(ctx, i)
    per_graph_ms = max_over_ranks(pg, sum(lat.values()))
    # Batched: a warm-up batch, then the whole mix in one kt_batch_run per step.
    batch_run(ctx, first=first, count=min(G, 64))
    barrier(pg)
    times = []
    stages = {}
    for _ in range(args.mix_steps):
        ms, waves, got = batch_run(ctx, first=first, count=G, stages=stages)
        times.append(ms)
    mism = [i for i, a in zip(idx, got) if a != alone[i]]
    batched_ms = max_over_ranks(pg, sum(times) / len(times))
    total = sum_over_ranks(pg, float(G))
    # Where the ratio comes from: each size decile (by edge keys) as a batch
    # of its own, against the same graphs one at a time.
    deciles = []
    order = sorted(mix_sizes(first, G), key=lambda t: (t[1], t[0]))
    for d in range(10):
        part = order[d * G // 10:(d + 1) * G // 10]
        if not part:
            continue
        ids = [i for i, _ in part]
        bms, bw, dgot = batch_run(ctx, indices=ids)
        mism += [i for i, a in zip(ids, dgot) if a != alone[i]]
        pms = sum(lat[i] for i in ids)
        deciles.append({"decile": d + 1, "graphs": len(ids), "edge_keys": int(sum(s for _, s in part)),
                        "keys_min": int(part[0][1]), "keys_max": int(part[-1][1]), "waves": bw,
                        "per_graph_ms": round(pms, 2), "batched_ms": round(bms, 2), "ratio": round(pms / bms, 3)})
    lat_np = np.array([lat[i] for i in idx])
    out = {
        "workload": f"mix graphs {first}..{first + G - 1}", "graphs": G, "steps": args.mix_steps,
        "lanes": args.batch_lanes,
        "graphs_per_s": total / (batched_ms / 1000.0), "ms_per_step": batched_ms, "waves": waves,
        "stage_ms_summed_over_lanes": stages,
        "per_graph": {"graphs_per_s": total / (per_graph_ms / 1000.0), "ms_total": per_graph_ms, "graphs": G,
                      "p50_ms": float(np.percentile(lat_np, 50)), "p99_ms": float(np.percentile(lat_np, 99))},
        "ratio": per_graph_ms / batched_ms,
        "answers_equal_alone": not mism, "mismatches": sorted(set(mism))[:20], "deciles": deciles,
    }
    if rank == 0 and not args.no_cpu_baseline:
        from kc_cuda_b200 import gen
        rng = np.random.default_rng(7)
        small = [i for i in idx if gen.mix_graph(i).draws <= 4_000_000]
        sample = sorted(int(x) for x in rng.choice(small, size=min(16, len(small)), replace=False))
        try:
            cpu = cpu_mix_sample(sample, threads, alone)
        except Exception as e:  # the reference failed even on one thread
            cpu = {"error": f"{type(e).__name__}: {str(e)[:300]}", "sample": sample}
        if cpu is not None:
            out["cpu_baseline"] = cpu
    return out


def fifo_latencies(arrivals_s, service_ms):
    """Latencies (ms) of requests served one at a time in arrival order, each
    taking its measured service time: the per-graph path under the same
    arrivals."""
    done = 0.0
    out = []
    for a, s in zip(arrivals_s, service_ms):
        start = max(a * 1000.0, done)
        done = start + s
        out.append(done - a * 1000.0)
    return out


def measure_serve(ctx, args, rank, pg, batched_gps=None):
    """Serving loop: R requests, request i = mix graph (first + i), Poisson
    arrivals (fixed seed) at 0.8 x the batched graphs/s (measured on the mix,
    or on a calibration batch of other mix graphs).  Latency = submission ->
    result, measured by the library.  Every served answer is compared with the
    graph solved alone, whose device time also gives the per-graph path's
    latencies under the same arrivals."""
    import numpy as np

    from kc_cuda_b200 import serving
    R = args.serve_requests
    ranges = ranges_for(args, rank)
    calib_first, first = ranges["calib"][0], ranges["serve"][0]
    calib = None
    if batched_gps is None:
        batch_run(ctx, first=calib_first, count=min(64, args.calib_graphs))
        ms, _, _ = batch_run(ctx, first=calib_first, count=args.calib_graphs)
        batched_gps = args.calib_graphs / (ms / 1000.0)
        calib = {"graphs": args.calib_graphs, "first": calib_first}
    rate = args.serve_rate if args.serve_rate > 0 else 0.8 * batched_gps
    arrivals = serving.poisson_arrivals(R, rate, seed=55 + rank)
    barrier(pg)
    srv = ctx.server()
    submitted = serving.drive(arrivals, lambda i: srv.submit_mix(first + i))
    results = [srv.wait(rid) for rid, _ in submitted]
    sst = srv.stats()
    srv.close()
    if not all(r["status"] == 0 for r in results):
        raise RuntimeError("serving: a request failed")
    summ = serving.summarize(submitted, results)
    service, mism = [], []
    for j in range(R):
        ms, ans = solve_alone(ctx, first + j)
        service.append(ms)
        if ans != (results[j]["kmax"], results[j]["edges"]):
            mism.append(first + j)
    pg_lat = fifo_latencies(arrivals, service)
    span = max_over_ranks(pg, summ["span_s"])
    total = sum_over_ranks(pg, float(R))
    return {
        "workload": f"{R} Poisson requests, mix graphs {first}..{first + R - 1}", "requests": R,
        "lanes": args.serve_lanes,
        "arrival_rate_per_s": rate, "arrival_seed": 55 + rank, "rate_basis_graphs_per_s": batched_gps,
        "calibration": calib, "graphs_per_s": total / span, "span_s": span,
        "p50_ms": summ["p50_ms"], "p99_ms": max_over_ranks(pg, summ["p99_ms"]), "mean_ms": summ["mean_ms"],
        "max_ms": summ["max_ms"], "wait_p50_ms": summ["wait_p50_ms"],
        "waves": sst["waves"], "mean_wave_graphs": summ["mean_wave_graphs"],
        "max_wave_graphs": sst["max_wave_graphs"], "device_bytes_peak": sst["device_bytes_peak"],
        "per_lane": summ["per_lane"],
        "per_graph_same_arrivals": {
            "p50_ms": float(np.percentile(pg_lat, 50)), "p99_ms": float(np.percentile(pg_lat, 99)),
            "service_p50_ms": float(np.percentile(service, 50)),
            "method": "one request at a time in arrival order, each taking its measured per-graph device time"},
        "answers_equal_alone": not mism, "mismatches": mism[:20],
    }


def lane_options(ctx, args):
    """Options of the batched and serving contexts: a memory pool grown once
    to the budget (graphs of new sizes then map no memory mid-solve), and the
    waves in flight at once."""
    ctx.set_option("pool_reserve_mb", 1 << 30)
    ctx.set_option("batch_lanes", args.batch_lanes)
    ctx.set_option("serve_lanes", args.serve_lanes)
    for o in args.option:
        name, value = o.split("=", 1)
        ctx.set_option(name, int(value))


def progress(name: str, obj) -> None:
    """A finished part of the run, on stderr, so a later failure keeps it."""
    print(json.dumps({name: obj}), file=sys.stderr, flush=True)


def line_base(metric, value, unit, world, steps, warmup, ms, config):
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": steps, "warmup": warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": config}


def run_mix(args, world, rank, local, pg):
    """--workload mix4096: the batched figures as the line itself."""
    import kc_cuda_b200 as K
    ctx = K.Context(local)
    lane_options(ctx, args)
    tune = autotune(ctx, args, rank)
    ctx.reset_stats()
    with ClockSampler(local) as clk:
        mix = measure_mix(ctx, args, rank, pg, os.cpu_count() or 1)
    launches = ctx.stats()["kernel_launches"]
    if rank == 0:
        line = line_base("batched kmax-truss graphs/s (mix of graphs 0..G-1)", mix["graphs_per_s"], "graphs/s",
                         world, args.mix_steps, 1, mix["ms_per_step"],
                         {"workload": f"mix{args.mix_graphs}", "graphs": args.mix_graphs, "waves": mix["waves"]})
        line.update({"batched": mix, "autotune": tune, "gpu_launches": launches, "clocks": clk.summary()})
        print(json.dumps(line))
    ctx.close()
    if not mix["answers_equal_alone"]:
        raise SystemExit("batched answers differ from the graphs solved alone")


def run_serve(args, world, rank, local, pg):
    """--workload serve: the serving figures as the line itself."""
    import kc_cuda_b200 as K
    ctx = K.Context(local)
    lane_options(ctx, args)
    tune = autotune(ctx, args, rank)
    ctx.reset_stats()
    with ClockSampler(local) as clk:
        srv = measure_serve(ctx, args, rank, pg)
    launches = ctx.stats()["kernel_launches"]
    if rank == 0:
        line = line_base("served kmax-truss graphs/s with p50/p99 latency (Poisson arrivals of mix graphs)",
                         srv["graphs_per_s"], "graphs/s", world, 1, 1, srv["span_s"] * 1000.0,
                         {"workload": f"serve{args.serve_requests}", "requests": args.serve_requests})
        line.update({"serving": srv, "autotune": tune, "gpu_launches": launches, "clocks": clk.summary()})
        print(json.dumps(line))
    ctx.close()
    if not srv["answers_equal_alone"]:
        raise SystemExit("served answers differ from the graphs solved alone")


def run_reference(args, rank, threads):
    if rank != 0:
        return
    metric = "kmax-truss solve edges/s per graph"
    v, desc, times = cpu_baseline_run(args.steps, args.warmup, threads)
    if v is None:
        print(json.dumps({"impl": "reference", "unavailable": desc}))
        return
    line = line_base(metric, v, "edges/s", args.gpus, args.steps, args.warmup, 1000 * statistics.median(times),
                     {"workload": "rmat20_ef32_seed2_k80_120_200 (CPU sample of the rmat24 family: kc_cpu takes "
                                  "about 2 minutes on the full graph, too long for a bounded step)",
                      "threads": threads, "same_config": False})
    line.update({
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "edges/s", "cores": threads, "kind": "reference", "sample": desc},
        "e2e": {"value": v, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(line))


# DRAM traffic of the dense support kernel, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of a k_dense_support launch
# on the core55k-support case of cases.py: G(n=55455, 95M draws), whose core
# has the bench graph's search-core shape (92.1M edges, rows of 1736 words);
# the launch read 166.3G row words.  The bench graph's launches are too large
# to capture under the profiling size rule, so their traffic is scaled from
# this one by the row words each launch reads.
SUPPORT_CAPTURE = {"dram_bytes": 6_683_428_000 + 373_861_632, "row_words": 166_313_504_560}


def roofline(name, kbytes, kms, klaunch, steps, hbm, peak_kind, **extra):
    achieved = (kbytes / (kms / 1000.0)) / 1e9 if kms > 0 else 0.0
    r = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
         "frac": achieved / hbm if hbm else None, "traffic": None, "peak_kind": peak_kind,
         "bytes_per_step": kbytes / steps, "kernel_ms_per_step": kms / steps, "launches_per_step": klaunch / steps}
    r.update(extra)
    return r


def run_single(args, world, rank, local, pg, threads):
    import kc_cuda_b200 as K
    metric = "kmax-truss solve edges/s per graph"
    config_name, spec = workload_spec(args.workload)
    g, tsv = make_tsv(spec, pinned=True)
    n_edges, n_vertices = g.num_edges, g.num_vertices
    del g
    ctx = K.Context(local)
    # The memory pool grown once up front (as a long-running process would
    # hold it): a step then never maps new device memory mid-solve.
    ctx.set_option("pool_reserve_mb", 1 << 30)
    staged = ctx.stage_tsv(tsv)

    # Warm-up (device-resident and end-to-end paths).
    answer = None
    for _ in range(args.warmup):
        answer = staged.solve()
    ctx.solve_tsv(tsv)

    # Timed: device-resident solves.
    barrier(pg)
    ctx.reset_stats()
    dev_ms = []
    stats_last = None
    acc = {k: 0.0 for k in ("ms_support_kernel", "ms_peel_kernel", "support_bytes", "support_kernel_bytes",
                            "support_row_words", "peel_bytes", "peel_recount_bytes")}
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            got = staged.solve()
            st = ctx.stats()
            if got != answer:
                raise SystemExit(f"answer changed between steps: {got} vs {answer}")
            dev_ms.append(st["ms_total"])
            for k in acc:
                acc[k] += st[k]
            stats_last = st
    launches = ctx.stats()["kernel_launches"]
    # Launch counters run from reset_stats: they cover the timed steps.
    sup_launch = stats_last["support_launches"]
    peel_launch = stats_last["peel_launches"]
    barrier(pg)
    step_ms = max_over_ranks(pg, sum(dev_ms) / len(dev_ms))
    total_edges = sum_over_ranks(pg, float(n_edges))
    value = total_edges / (step_ms / 1000.0)

    # Timed: end to end through the public API from pinned host memory.
    barrier(pg)
    ctx.reset_stats()
    e2e_s = []
    e2e_copy_parse_ms = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        got = ctx.solve_tsv(tsv)
        e2e_s.append(time.perf_counter() - t0)
        if got != answer:
            raise SystemExit(f"end-to-end answer differs: {got} vs {answer}")
        # The pipelined load's parse stage spans the host-to-device copy.
        e2e_copy_parse_ms.append(ctx.stats()["ms_parse"])
    est = ctx.stats()
    barrier(pg)
    e2e_step = max_over_ranks(pg, sum(e2e_s) / len(e2e_s))
    e2e_value = total_edges / e2e_step

    hbm, peak_kind = load_peaks()
    S = args.steps
    sup_traffic = None
    if SUPPORT_CAPTURE and sup_launch:
        per_word = SUPPORT_CAPTURE["dram_bytes"] / SUPPORT_CAPTURE["row_words"]
        sup_traffic = per_word * acc["support_row_words"] / sup_launch
    roof_sup = roofline(
        "support: k_dense_support (edge support by bitset AND/popcount, all launches of a solve)",
        acc["support_kernel_bytes"], acc["ms_support_kernel"], sup_launch, S, hbm, peak_kind,
        bytes_model="row words the kernels read (row u loads, row v words ANDed) x 4 + 16 per edge",
        merge_model_bytes_per_step=acc["support_bytes"] / S, row_words_per_step=acc["support_row_words"] / S)
    roof_sup["traffic"] = sup_traffic
    if sup_traffic is not None:
        roof_sup["traffic_basis"] = ("DRAM bytes per row word of the core55k-support capture x the row words "
                                     "of an average launch here")
    roof_peel = roofline(
        "peel: k_cascade (one cooperative launch per truss level)", acc["peel_bytes"], acc["ms_peel_kernel"],
        peel_launch, S, hbm, peak_kind,
        bytes_model="8 per alive-degree unit of each deleted edge + 8 per support decrement + 4 per alive-list "
                    "entry scanned",
        recount_bytes_per_step=acc["peel_recount_bytes"] / S)
    dominant = roof_sup if acc["ms_support_kernel"] >= acc["ms_peel_kernel"] else roof_peel

    attributed = sum(stats_last[k] for k in ("ms_parse", "ms_csr", "ms_kcore", "ms_subgraph", "ms_support",
                                              "ms_peel"))
    progress("single_graph", {"value": value, "e2e": e2e_value, "answer": list(answer),
                              "ms_total": stats_last["ms_total"],
                              "ms_outside_stages": stats_last["ms_total"] - attributed,
                              "stage_ms": {k: round(stats_last[k], 3) for k in
                                           ("ms_parse", "ms_csr", "ms_kcore", "ms_subgraph", "ms_support",
                                            "ms_peel")},
                              "support_ms": acc["ms_support_kernel"] / S, "peel_ms": acc["ms_peel_kernel"] / S})
    ref = reference_answer(config_name)
    parity = None
    if ref is not None:
        parity = {"reference": ref[0], "ours": list(answer), "equal": list(answer) == ref[0],
                  "reference_solver": f"{ref[1].get('reference_binary', 'kc_cpu')} "
                                      f"({ref[1].get('reference_threads')} threads)"}

    mix = srv = None
    mix_tune = None
    if not args.no_batched or not args.no_serving:
        staged.free()
        staged = None
        ctx.close()
        ctx = K.Context(local)
        lane_options(ctx, args)
        mix_tune = autotune(ctx, args, rank)
        if not args.no_batched:
            mix = measure_mix(ctx, args, rank, pg, threads)
            mix["autotune"] = mix_tune
            progress("batched", mix)
        if not args.no_serving:
            srv = measure_serve(ctx, args, rank, pg, mix["graphs_per_s"] / world if mix else None)
            progress("serving", srv)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v, desc, _ = cpu_baseline_run(3, 1, threads)
        if v is not None:
            cpu = {"value": v, "unit": "edges/s", "cores": threads, "kind": "reference", "sample": desc}
    if rank == 0:
        line = line_base(metric, value, "edges/s", world, args.steps, args.warmup, step_ms, {
            "workload": config_name, "vertices": n_vertices, "edges": n_edges, "tsv_bytes": int(tsv.nbytes),
            "kmax": answer[0], "kmax_truss_edges": answer[1], "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (TSV bytes re-read every step)",
            "cmax": stats_last["cmax"], "core_vertices": stats_last["core_vertices"],
            "core_edges": stats_last["core_edges"], "predict_vertices": stats_last["predict_vertices"],
            "predict_edges": stats_last["predict_edges"], "levels": stats_last["levels"],
            "rounds": stats_last["rounds"], "peel_decrements": stats_last["peel_decrements"]})
        line.update({
            "parity": parity,
            "e2e": {"value": e2e_value, "unit": "edges/s", "h2d_bytes_per_step": est["h2d_bytes"] // args.steps,
                    "d2h_bytes_per_step": est["d2h_bytes"] // args.steps, "ms_per_step": 1000 * e2e_step,
                    "step_ms": [round(1000 * x, 1) for x in e2e_s],
                    "copy_parse_ms": [round(x, 1) for x in e2e_copy_parse_ms],
                    "copy_gbs": [round(tsv.nbytes / (x / 1000.0) / 1e9, 1) for x in e2e_copy_parse_ms if x > 0],
                    "copy_note": "copy_parse_ms: the host-to-device copy of the TSV bytes in chunks with each "
                                 "chunk's parse overlapped (copy-bound); copy_gbs: TSV bytes over it"},
            "gpu_launches": launches,
            "device_step_ms": [round(x, 1) for x in dev_ms],
            "roofline": dict(dominant, note=(
                "dense support rows are read mostly from L2 (tile order), so frac near 1 of the HBM copy "
                "bandwidth is L2-served work; traffic is the DRAM share")),
            "rooflines": {"support": roof_sup, "peel": roof_peel},
            "stage_ms": dict({k: round(stats_last[k], 3) for k in
                              ("ms_parse", "ms_csr", "ms_kcore", "ms_subgraph", "ms_support", "ms_peel")},
                             outside_stages=round(stats_last["ms_total"] - attributed, 3)),
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "batched": mix,
            "serving": srv,
        })
        print(json.dumps(line), flush=True)
    if staged is not None:
        staged.free()
    ctx.close()
    bad = []
    if parity is not None and not parity["equal"]:
        bad.append(f"answer {list(answer)} differs from the reference solver's {ref[0]}")
    if mix is not None and not mix["answers_equal_alone"]:
        bad.append("batched answers differ from the graphs solved alone")
    if mix is not None and mix.get("cpu_baseline") and not mix["cpu_baseline"]["answers_equal"]:
        bad.append("batched answers differ from the reference solver's")
    if srv is not None and not srv["answers_equal_alone"]:
        bad.append("served answers differ from the graphs solved alone")
    if bad:
        raise SystemExit("; ".join(bad))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat24", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="single-graph workloads: skip the batched figures")
    ap.add_argument("--no-serving", action="store_true", help="single-graph workloads: skip the serving figures")
    ap.add_argument("--mix-graphs", type=int, default=4096)
    ap.add_argument("--mix-steps", type=int, default=1, help="timed kt_batch_run passes over the whole mix")
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-rate", type=float, default=0.0, help="requests/s (0: 0.8 x batched graphs/s)")
    ap.add_argument("--calib-graphs", type=int, default=512)
    ap.add_argument("--batch-lanes", type=int, default=2, help="batched: waves in flight at once (1 or 2)")
    ap.add_argument("--serve-lanes", type=int, default=2, help="serving: waves in flight at once (1..4)")
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="batched and serving contexts: a solver option to set (repeatable)")
    ap.add_argument("--tune-graphs", type=int, default=128,
                    help="autotune the kernel thresholds on this many other mix graphs first (0: off)")
    args = ap.parse_args()
    world, rank, local, pg = dist_setup()
    threads = os.cpu_count() or 1
    try:
        if args.impl == "reference":
            run_reference(args, rank, threads)
        elif args.workload == "mix4096":
            run_mix(args, world, rank, local, pg)
        elif args.workload == "serve":
            run_serve(args, world, rank, local, pg)
        else:
            run_single(args, world, rank, local, pg, threads)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
