"""Full-size parity of the single-graph configurations against the
reference's own CPU solver (run by hand on the GPU host; too large for the
test suite):

    python tests/large_parity.py [--configs 1 2 3] [--dir /dev/shm] [--record] [--ours-only]
                                 [--gpu-reference]

For each configuration: the seeded graph is generated and written as the
reference's TSV; the drop-in CLI (kc_cuda_b200/kt_solve -f) and kc_cpu (all
host cores; kc_cpu_large, the build with raised input limits, when the input
is beyond kc_cpu's own) solve the same file; the answers must be equal.
--gpu-reference also runs the reference's own GPU build (oracle/_ref/kc_gpu,
built for sm_100a from the reference sources) on the same file, once, and
records its wall time and answer beside the others.
--record writes the answers and wall times to tests/golden/large_configs.json;
bench.py compares its answer on a workload with the kc_cpu answer recorded
there.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import kt_oracle as O  # noqa: E402
from kc_cuda_b200 import gen  # noqa: E402

CONFIGS = {
    1: ("rmat16_ef16_seed1_k30", gen.rmat_s16_k30),
    2: ("rmat24_ef32_seed2_k80_120_200", gen.rmat_s24_ef32_k80_120_200),
    3: ("chunglu_n50m_g2.1_wmax2m_seed3_block150", gen.chunglu_50m),
}
RECORD = os.path.join(ROOT, "tests", "golden", "large_configs.json")
CLI = os.path.join(ROOT, "kc_cuda_b200", "kt_solve")
RESULT_RE = re.compile(r"kmax = (\d+), Edges in kmax-truss = (\d+)\.")


def run_cli(path: str):
    t = time.perf_counter()
    p = subprocess.run([CLI, "-f", path], capture_output=True, text=True, timeout=3600)
    wall = time.perf_counter() - t
    if p.returncode != 0:
        raise RuntimeError(f"kt_solve failed ({p.returncode}): {p.stderr[-400:]}")
    m = RESULT_RE.search(p.stdout)
    return (int(m.group(1)), int(m.group(2))), wall


def run_kc_gpu(path: str, timeout: float):
    """The reference's GPU solver on a TSV file (a stand-in vmtouch first on
    PATH, as for kc_cpu): (answer or None, wall seconds, status text)."""
    binary = os.path.join(O.REF, "kc_gpu")
    if not os.access(binary, os.X_OK):
        return None, None, "oracle/_ref/kc_gpu missing"
    env = dict(os.environ)
    env["PATH"] = O.HERE + os.pathsep + env.get("PATH", "")
    t = time.perf_counter()
    try:
        p = subprocess.run([binary, "-f", path], capture_output=True, text=True, timeout=timeout, env=env)
    except subprocess.TimeoutExpired:
        return None, time.perf_counter() - t, f"no answer within {timeout:.0f} s"
    wall = time.perf_counter() - t
    m = RESULT_RE.search(p.stdout)
    if p.returncode != 0 or not m:
        return None, wall, f"exit {p.returncode}: {(p.stderr or p.stdout)[-300:]}"
    return (int(m.group(1)), int(m.group(2))), wall, "ok"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", type=int, nargs="+", default=[2, 3])
    ap.add_argument("--dir", default="/dev/shm")
    ap.add_argument("--record", action="store_true")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--reference-only", action="store_true", help="no GPU: record kc_cpu's answers only")
    ap.add_argument("--ours-only", action="store_true",
                    help="compare with the recorded kc_cpu answer (when there is one) instead of running kc_cpu")
    ap.add_argument("--gpu-reference", action="store_true", help="also run the reference's kc_gpu once")
    ap.add_argument("--gpu-reference-timeout", type=float, default=1200)
    a = ap.parse_args()
    rec = json.load(open(RECORD)) if os.path.exists(RECORD) else {}
    ok = True
    for cfg in a.configs:
        name, spec_fn = CONFIGS[cfg]
        t = time.perf_counter()
        g = gen.Graph(spec_fn(), threads=a.threads)
        path = os.path.join(a.dir, f"kt_cfg{cfg}.tsv")
        g.write_tsv(path, threads=a.threads)
        n, m, size = g.num_vertices, g.num_edges, os.path.getsize(path)
        del g
        t_gen = time.perf_counter() - t
        ours, wall_ours = (None, None) if a.reference_only else run_cli(path)
        lines = 2 * m
        large = lines > 1_700_000_000 or 2 * m >= (1 << 31) - (1 << 24)
        binary = os.path.join(O.REF, "kc_cpu_large" if large else "kc_cpu")
        prev = rec.get(name, {})
        if a.ours_only and "kmax" in prev:
            ref, wall_ref = (prev["kmax"], prev["kmax_truss_edges"]), prev["reference_wall_s"]
            binary, a_threads = prev["reference_binary"], prev["reference_threads"]
        else:
            subprocess.run(["cat", path], stdout=subprocess.DEVNULL, check=True)  # page cache, as vmtouch would
            t = time.perf_counter()
            ref = O.run_kc_cpu(path, threads=a.threads, timeout=7200, binary=binary)
            wall_ref = time.perf_counter() - t
            a_threads = a.threads
        gpu_ref = None
        if a.gpu_reference:
            ans, wall_g, status = run_kc_gpu(path, a.gpu_reference_timeout)
            gpu_ref = {"answer": list(ans) if ans else None, "wall_s": round(wall_g, 2) if wall_g else None,
                       "status": status, "equal": (tuple(ans) == tuple(ref)) if ans else None}
        os.unlink(path)
        if ours is None and prev.get("ours"):
            ours, wall_ours = tuple(prev["ours"]), prev.get("ours_cli_wall_s")
        same = ours == ref if ours is not None else None
        ok &= same is not False
        entry = {"config": cfg, "workload": name, "vertices": n, "edges": m, "tsv_bytes": size,
                 "kmax": ref[0], "kmax_truss_edges": ref[1], "ours": list(ours) if ours else None, "equal": same,
                 "reference_binary": os.path.basename(binary), "reference_threads": a_threads,
                 "reference_wall_s": round(wall_ref, 2),
                 "ours_cli_wall_s": round(wall_ours, 2) if wall_ours else None,
                 "generate_s": round(t_gen, 1)}
        if gpu_ref is not None:
            entry["reference_gpu"] = gpu_ref
        elif "reference_gpu" in prev:
            entry["reference_gpu"] = prev["reference_gpu"]
        print(json.dumps(entry), flush=True)
        rec[name] = entry
    if a.record:
        with open(RECORD, "w") as f:
            json.dump(rec, f, indent=1, sort_keys=True)
    sys.exit(0 if ok else 1)


if __name__ == "__main__":
    main()
