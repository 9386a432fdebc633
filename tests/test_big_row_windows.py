"""The dealing of long rows' 32-entry windows to every warp of the grid
(deal_big_windows in kc_cuda_b200/csrc/kcore.cu, also used by
k_compact_big_rows), transcribed and checked on the CPU: rows are taken
kBigBatch at a time, each block computes the rows' first window numbers with
the same exclusive scan (4 rows per thread of a 256-thread block), and global
warp w takes windows w, w + warps, ... and finds its row by a binary search
for the last row whose first window is <= the window. Every entry of every
row must be handed out exactly once, in windows of at most 32 entries."""
import random

K_BIG_BATCH = 1024
PER = K_BIG_BATCH // 256


def deal(lengths, warps):
    """Returns the (row, begin, end) windows in the order warps take them."""
    out = []
    for base in range(0, len(lengths), K_BIG_BATCH):
        cnt = min(len(lengths) - base, K_BIG_BATCH)
        # Per-thread sums, then the block's exclusive scan over threads.
        w = [(lengths[base + r] + 31) // 32 if r < cnt else 0 for r in range(K_BIG_BATCH)]
        woff = [0] * (cnt + 1)
        pre = 0
        for t in range(256):
            for j in range(PER):
                r = t * PER + j
                if r < cnt:
                    woff[r] = pre
                pre += w[r]
        woff[cnt] = pre
        total = pre
        for gwarp in range(warps):
            for x in range(gwarp, total, warps):
                lo, hi = 0, cnt
                while hi - lo > 1:
                    mid = (lo + hi) >> 1
                    if woff[mid] <= x:
                        lo = mid
                    else:
                        hi = mid
                b = (x - woff[lo]) * 32
                out.append((base + lo, b, min(lengths[base + lo], b + 32)))
    return out


def test_every_entry_once():
    rng = random.Random(11)
    for trial in range(40):
        nrows = rng.choice([1, 3, 255, 1023, 1024, 1025, 2100])
        lengths = [rng.choice([0, 1, 31, 32, 33, 513, 2049]) for _ in range(nrows)]
        if rng.random() < 0.3:
            lengths[rng.randrange(nrows)] = 70001  # one hub row
        got = deal(lengths, warps=rng.choice([1, 7, 32, 5920]))
        assert all(0 < e - b <= 32 for _, b, e in got), trial
        want = [(r, b, min(n, b + 32)) for r, n in enumerate(lengths) for b in range(0, n, 32)]
        assert sorted(got) == want, trial
