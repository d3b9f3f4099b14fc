"""The serving loop's admission allocator (ctb_arena_*), host bookkeeping only:
checked against a plain Python model of first fit with merging over random
alloc/free sequences, plus the boundary cases (exact fit, out of space,
double free, unknown offsets)."""
import random

import pytest

import qtctreconstruction_b200 as ctb

UNIT = 256


class Model:
    def __init__(self, cap):
        self.cap = cap // UNIT * UNIT
        self.free = [(0, self.cap)]  # sorted (offset, size)
        self.held = {}
        self.used = self.peak = 0

    def alloc(self, n):
        n = max(1, n)
        n = (n + UNIT - 1) // UNIT * UNIT
        for k, (o, s) in enumerate(self.free):
            if s >= n:
                self.free[k:k + 1] = [(o + n, s - n)] if s > n else []
                self.held[o] = n
                self.used += n
                self.peak = max(self.peak, self.used)
                return o
        return None

    def release(self, o):
        if o not in self.held:
            return False
        n = self.held.pop(o)
        self.used -= n
        self.free.append((o, n))
        self.free.sort()
        merged = []
        for fo, fs in self.free:
            if merged and merged[-1][0] + merged[-1][1] == fo:
                merged[-1] = (merged[-1][0], merged[-1][1] + fs)
            else:
                merged.append((fo, fs))
        self.free = merged
        return True

    def largest(self):
        return max((s for _, s in self.free), default=0)


def test_arena_basic():
    a = ctb.Arena(4096)
    assert a.alloc(4096) == 0
    assert a.alloc(1) is None          # full
    assert a.free(0)
    assert not a.free(0)               # double free
    assert not a.free(12345)           # unknown offset
    assert a.stats() == (0, 4096, 4096)
    x, y, z = a.alloc(1000), a.alloc(1000), a.alloc(1000)
    assert (x, y, z) == (0, 1024, 2048)
    assert a.free(y)
    assert a.alloc(1025) is None       # two 1024-byte holes, no 1280-byte range
    assert a.alloc(1024) == 1024       # first fit reuses the hole
    a.close()


def test_arena_rejects_tiny_capacity():
    with pytest.raises(ctb.CtbError):
        ctb.Arena(100)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_arena_matches_model(seed):
    rnd = random.Random(seed)
    cap = 1 << 24
    a, m = ctb.Arena(cap), Model(cap)
    live = []
    for _ in range(3000):
        if live and rnd.random() < 0.45:
            o = live.pop(rnd.randrange(len(live)))
            assert a.free(o) == m.release(o)
        else:
            n = rnd.choice([rnd.randint(1, 4096), rnd.randint(1, 1 << 20), rnd.randint(1, 1 << 22)])
            got, want = a.alloc(n), m.alloc(n)
            assert got == want
            if got is not None:
                live.append(got)
        assert a.stats() == (m.used, m.peak, m.largest())
    for o in live:
        assert a.free(o)
    assert a.stats()[0] == 0 and a.stats()[2] == cap
