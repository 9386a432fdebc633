"""The synchronisation protocol of the one-launch core decomposition
(k_core_levels in kc_cuda_b200/csrc/kcore.cu), checked on the CPU.

The kernel's blocks share rotating device counters (frontier sizes by round,
alive-list / candidate / minimum-degree counters by pass) that are reset by
one thread while other blocks may still be reading the previous ones, and
they meet only at grid barriers.  This test runs a block-level transcription
of the kernel -- same counter slots, same resets, same barrier placement,
every shared-memory access a scheduling point -- under random, skewed
interleavings of 2 to 8 blocks, and checks that no block leaves while others
wait at a barrier and that the core numbers equal the oracle's.  (A version
of the kernel that reused the frontier slot after a level without vertices
fails here on the union-of-cliques graph.)
"""
import random

import numpy as np
import pytest

import kt_oracle as O
from kc_cuda_b200 import gen

ALIVE = 0xffffffff
BIG = 4     # rows longer than this go to the dealt-window phase (the kernel's big_row)
WIN = 2     # entries per dealt window (the kernel deals 32-entry windows)
MAXU = (1 << 64) - 1


def run(e, n, B, seed, window):
    """Core numbers by the emulated kernel (None and a reason on a protocol failure)."""
    rng = random.Random(seed)
    u = (e >> np.uint64(32)).astype(np.int64); v = (e & np.uint64(0xffffffff)).astype(np.int64)
    adjl = [[] for _ in range(n)]
    for a, b in zip(u, v): adjl[a].append(b); adjl[b].append(a)
    off = [0]
    for r in adjl: off.append(off[-1] + len(r))
    adj = [w for r in adjl for w in r]
    deg = [len(r) for r in adjl]
    rem = [ALIVE if d else 0 for d in deg]
    core = [0] * n
    lists = [[x for x in range(n) if deg[x]], [0] * n]
    cands = [[0] * n, [0] * n]
    front = [[0] * n, [0] * n]
    big = [0] * n
    cnt = [0] * 24
    for s in (8, 9, 10): cnt[s] = MAXU
    S = {'bar_count': 0, 'bar_gen': 0, 'err': 0}

    def push(lst, ci, x):
        p = cnt[ci]; cnt[ci] += 1
        if p >= n: S['err'] = 1; return
        lst[p] = x

    def barrier():
        gen0 = S['bar_gen']
        yield
        S['bar_count'] += 1
        if S['bar_count'] == B:
            S['bar_count'] = 0; S['bar_gen'] += 1
        else:
            while S['bar_gen'] == gen0:
                yield 'wait'

    def drop(b0, e0, k, top, nx, nci, cn, cci):
        for j in range(b0, e0):
            w = adj[j]
            yield
            if rem[w] == ALIVE:
                old = deg[w]; deg[w] -= 1
                if old == k + 1:
                    rem[w] = 0; core[w] = k; push(nx, nci, w)
                elif old == top + 1:
                    push(cn, cci, w)
            yield

    def block(bid):
        nl = len(lists[0]); nc = 0; k = 1; top = 0; full = True
        i = 0; ps = 0; li = 0; ci = 0
        while True:
            lc = 5 + ps % 3; mc = 8 + ps % 3; cc = 11 + ps % 3
            if bid == 0:
                cnt[5 + (ps + 1) % 3] = 0; cnt[8 + (ps + 1) % 3] = MAXU; cnt[11 + (ps + 1) % 3] = 0
                cnt[(i + 2) % 3] = 0; cnt[3 + ((i + 1) & 1)] = 0
            yield
            if full: top = k + window - 1
            src = (lists[1] if li else lists[0]) if full else (cands[1] if ci else cands[0])
            nsrc = nl if full else nc
            lnext = lists[0] if li else lists[1]
            cnext = cands[0] if ci else cands[1]
            fpush = front[0] if (i & 1) else front[1]
            for j in range(bid, nsrc, B):
                x = src[j]
                yield
                if rem[x] == ALIVE:
                    d = deg[x]
                    if d <= k:
                        rem[x] = 0; core[x] = k; push(fpush, (i + 1) % 3, x)
                    else:
                        if full: push(lnext, lc, x)
                        if d <= top: push(cnext, cc, x)
                        cnt[mc] = min(cnt[mc], d)
                yield
            yield from barrier()
            if full:
                nl = cnt[lc]; yield
                li ^= 1
            dmin = cnt[mc]; yield
            ps += 1; i += 1
            nfz = cnt[i % 3] == 0; yield
            if nfz:
                nc = cnt[cc]; yield
                ci ^= 1
                if full:
                    if nl == 0: break
                    k = dmin; full = k > top
                elif nc:
                    k = dmin
                else:
                    k = top + 1; full = True
                continue
            while True:
                nf = cnt[i % 3]; yield
                if nf == 0: break
                fr = front[1] if (i & 1) else front[0]
                nx = front[0] if (i & 1) else front[1]
                nci = (i + 1) % 3; bc = 3 + (i & 1)
                for f in range(bid, nf, B):
                    x = fr[f]
                    if off[x + 1] - off[x] > BIG:
                        p = cnt[bc]; cnt[bc] += 1; big[p] = x
                        yield
                        continue
                    yield from drop(off[x], off[x + 1], k, top, nx, nci, cnext, cc)
                if bid == 0:
                    cnt[(i + 2) % 3] = 0; cnt[3 + ((i + 1) & 1)] = 0
                yield
                yield from barrier()
                nbig = cnt[bc]; yield
                if nbig:
                    # Windows of the big rows dealt to every block.
                    woff = [0]
                    for bi in range(nbig):
                        x = big[bi]
                        woff.append(woff[-1] + (off[x + 1] - off[x] + WIN - 1) // WIN)
                    for wi in range(bid, woff[-1], B):
                        r = max(j for j in range(nbig) if woff[j] <= wi)
                        x = big[r]
                        b0 = off[x] + (wi - woff[r]) * WIN
                        yield from drop(b0, min(off[x + 1], b0 + WIN), k, top, nx, nci, cnext, cc)
                    yield from barrier()
                i += 1
            nc = cnt[cc]; yield
            ci ^= 1
            k += 1
            full = k > top

    gens = {b: block(b) for b in range(B)}
    wts = {b: rng.random() ** 4 + 1e-3 for b in gens}
    steps = 0
    while gens:
        if rng.random() < 0.001:
            wts = {b: rng.random() ** 4 + 1e-3 for b in gens}
        ks = list(gens)
        b = rng.choices(ks, weights=[wts[x] for x in ks])[0]
        try:
            next(gens[b])
        except StopIteration:
            del gens[b]
            if gens and S['bar_count']:
                return None, 'exited while others wait at a barrier'
        steps += 1
        if steps > 3_000_000: return None, 'too many steps'
    if S['err']: return None, 'capacity'
    return np.array(core, dtype=np.uint32), 'ok'

def union_graph():
    """Cliques K5, K8, K10, a K5,5 and a path: levels without vertices."""
    ed = []; base = 0
    for c in (5, 8, 10):
        for a in range(c):
            for b in range(a + 1, c): ed.append((base + a, base + b))
        base += c
    for a in range(5):
        for b in range(5): ed.append((base + a, base + 5 + b))
    base += 10
    for a in range(6): ed.append((base + a, base + a + 1))
    return np.array(sorted((min(a, b) << 32) | max(a, b) for a, b in ed), dtype=np.uint64)



GRAPHS = {
    "cliques_bipartite_path": union_graph,
    "rmat7_k8": lambda: gen.Graph(gen.rmat(7, 4, 5, [8])).edges(),
    "er300_k7": lambda: gen.Graph(gen.GraphSpec(kind=gen.KTG_ER, n=300, draws=1200, seed=4, cliques=[7])).edges(),
}


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_core_levels_protocol(name):
    e = GRAPHS[name]()
    n = int(max((e >> np.uint64(32)).max(), (e & np.uint64(0xffffffff)).max())) + 1
    want = O.core_numbers(e, n)
    for seed in range(6):
        window = [1, 2, 32][seed % 3]
        blocks = [2, 3, 5, 8][seed % 4]
        got, msg = run(e, n, B=blocks, seed=seed, window=window)
        assert got is not None, (name, seed, msg)
        assert np.array_equal(got, want), (name, seed, window, blocks)
