"""The dealing of long rows' windows to every warp of the grid
(deal_big_windows<kWin> in kc_cuda_b200/csrc/kcore.cu: 256-entry windows in
the probes, 32-entry ones in the full decomposition; the same arithmetic in
k_compact_big_rows with 256-entry chunks), transcribed and checked on the
CPU: rows are taken
kBigBatch at a time, each block computes the rows' first window numbers with
the same exclusive scan (4 rows per thread of a 256-thread block), and global
warp w takes windows w, w + warps, ... and finds its row by a binary search
for the last row whose first window is <= the window. Every entry of every
row must be handed out exactly once, in windows of at most kWin entries; in
a 256-entry window lane l takes entries b + l + 32 k (k = 0..7), each once."""
import random

K_BIG_BATCH = 1024
PER = K_BIG_BATCH // 256


def deal(lengths, warps, win=32):
    """Returns the (row, begin, end) windows in the order warps take them."""
    out = []
    for base in range(0, len(lengths), K_BIG_BATCH):
        cnt = min(len(lengths) - base, K_BIG_BATCH)
        # Per-thread sums, then the block's exclusive scan over threads.
        w = [(lengths[base + r] + win - 1) // win if r < cnt else 0 for r in range(K_BIG_BATCH)]
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
                b = (x - woff[lo]) * win
                out.append((base + lo, b, min(lengths[base + lo], b + win)))
    return out


def test_every_entry_once():
    rng = random.Random(11)
    for win in (32, 256):
        for trial in range(40):
            nrows = rng.choice([1, 3, 255, 1023, 1024, 1025, 2100])
            lengths = [rng.choice([0, 1, 31, 32, 33, 255, 256, 257, 513, 2049]) for _ in range(nrows)]
            if rng.random() < 0.3:
                lengths[rng.randrange(nrows)] = 70001  # one hub row
            got = deal(lengths, warps=rng.choice([1, 7, 32, 5920]), win=win)
            assert all(0 < e - b <= win for _, b, e in got), (win, trial)
            want = [(r, b, min(n, b + win)) for r, n in enumerate(lengths) for b in range(0, n, win)]
            assert sorted(got) == want, (win, trial)


def test_wide_window_lanes_cover_each_entry_once():
    """Lane l of a 256-entry window [b, e) loads entries b + l + 32 k for
    k = 0..7 that lie below e (drop_neighbours_wide, k_compact_big_rows)."""
    for b, e in [(0, 256), (512, 700), (7, 8), (1000, 1255)]:
        taken = [b + l + 32 * k for l in range(32) for k in range(8) if b + l + 32 * k < e]
        assert sorted(taken) == list(range(b, e))
