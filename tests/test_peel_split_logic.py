"""The task dealing of the peel's split rounds (peel_edge_chunk in
kc_cuda_b200/csrc/peel.cu), transcribed and checked on the CPU: the common
neighbours of a chunk of kSplitWords words are numbered by a warp scan of
the words' popcounts, each lane finds its task's word with a 3-step search
over the first kSplitWords lanes and its bit with a 5-step select, so every
set bit of the chunk is visited exactly once, in rounds of 32."""
import random

K_SPLIT_WORDS = 8


def select_bit(m: int, r: int) -> int:
    """select_bit: position of the r-th (from 0) set bit of the 32-bit m."""
    pos = 0
    s = 16
    while s >= 1:
        low = bin(m & ((1 << s) - 1)).count("1")
        if r >= low:
            r -= low
            m >>= s
            pos += s
        s >>= 1
    return pos


def deal(words):
    """(word, bit) visited by each task of one chunk, as the warp does it."""
    c = [bin(w).count("1") for w in words] + [0] * (32 - len(words))
    excl = [sum(c[:i]) for i in range(32)]
    total = sum(c)
    visits = []
    for base in range(0, total, 32):
        for lane in range(32):
            t = base + lane
            lo = 0
            st = K_SPLIT_WORDS // 2
            while st >= 1:
                cand = lo + st
                if cand < K_SPLIT_WORDS and excl[cand & 31] <= t:
                    lo = cand
                st >>= 1
            if t < total:
                visits.append((lo, select_bit(words[lo], t - excl[lo])))
    return visits


def test_select_bit():
    rng = random.Random(3)
    for _ in range(20000):
        m = rng.getrandbits(32) or 1
        bits = [i for i in range(32) if m >> i & 1]
        r = rng.randrange(len(bits))
        assert select_bit(m, r) == bits[r]


def test_every_common_neighbour_once():
    rng = random.Random(5)
    for trial in range(3000):
        density = rng.choice([0.0, 0.05, 0.5, 0.95, 1.0])
        n = rng.randint(1, K_SPLIT_WORDS)
        words = [sum(1 << b for b in range(32) if rng.random() < density) for _ in range(n)]
        want = sorted((w, b) for w in range(n) for b in range(32) if words[w] >> b & 1)
        got = deal(words)
        assert sorted(got) == want and len(got) == len(want), (trial, words)
