"""CPU checks of the shared-memory layout facts the NTT kernels rely on
(vortexstark_b200/csrc/ntt.cu), over every tile shape they are instantiated for:

* chunk rounds move 16-byte chunks with 128-bit accesses that are bank-conflict free
  per quarter warp under the swz<0> swizzle;
* the warp-barrier rule (`warp_local_next`, `warp_local_word`): where it says a warp
  barrier suffices between two rounds, every warp reads exactly the chunks it wrote.

The address maps are restated from ntt.cu (`ins4`, `swz<0>`, the C = 0 word round of
32 consecutive words per thread)."""
import pytest

MAX_T = 13


def ins4(p0, r, o, k):
    q = p0 - 2
    return (((o >> q) << (q + r)) | (k << q) | (o & ((1 << q) - 1))) << 2


def swz0(a):  # word address -> physical word address (chunk index ^= word bits 5-7)
    h = ((a >> 5) & 1) | (((a >> 6) & 1) << 1) | (((a >> 7) & 1) << 2)
    return a ^ (h << 2)


class Tile4:
    def __init__(self, m, c, s0):
        self.T = m + c
        self.NT = 1 << (self.T - 5)
        self.MC = self.T - s0
        self.NR = (self.MC + 2) // 3
        self.s0 = s0

    def p0(self, r):
        return self.s0 + 3 * r

    def R(self, r):
        return 3 if 3 * (r + 1) <= self.MC else self.MC - 3 * r


def rule_next(t: Tile4, r):  # restates warp_local_next
    same = t.NT >= 32 and r + 1 < t.NR
    b = 5
    while same and (1 << b) < t.NT:
        fa = b if b < t.p0(r) - 2 else b + t.R(r)
        fb = b if b < t.p0(r + 1) - 2 else b + t.R(r + 1)
        same = fa == fb
        b += 1
    return same


def rule_word(m):  # restates warp_local_word (C = 0, S0 = 5)
    t = Tile4(m, 0, 5)
    return t.NT >= 32 and t.R(0) == 3


def chunks_by_warp(t: Tile4, r):
    R, k_n = t.R(r), 1 << t.R(r)
    out = {}
    for th in range(t.NT):
        for s in range(1 << (3 - R)):
            for k in range(k_n):
                out.setdefault(th >> 5, set()).add(ins4(t.p0(r), R, th + s * t.NT, k) >> 2)
    return out


def word_round_by_warp(t: Tile4):
    return {w: {c for th in range(32 * w, min(32 * (w + 1), t.NT)) for c in range(8 * th, 8 * th + 8)}
            for w in range((t.NT + 31) // 32)}


SHAPES = [(m, 13 - m, 13 - m) for m in range(1, 12) if 13 - m >= 2] + [(m, 0, 5) for m in range(6, MAX_T + 1)]


@pytest.mark.parametrize("m,c,s0", SHAPES)
def test_chunk_rounds_are_conflict_free(m, c, s0):
    t = Tile4(m, c, s0)
    for r in range(t.NR):
        R = t.R(r)
        for s in range(1 << (3 - R)):
            for k in range(1 << R):
                for q0 in range(0, t.NT, 8):  # quarter warps of 128-bit accesses
                    lanes = range(q0, min(q0 + 8, t.NT))
                    slots = {(swz0(ins4(t.p0(r), R, th + s * t.NT, k)) >> 2) & 7 for th in lanes}
                    assert len(slots) == len(lanes), (m, c, r, s, k, q0)


@pytest.mark.parametrize("m,c,s0", SHAPES)
def test_warp_barrier_rule(m, c, s0):
    t = Tile4(m, c, s0)
    for r in range(t.NR - 1):
        a, b = chunks_by_warp(t, r), chunks_by_warp(t, r + 1)
        exact = t.NT >= 32 and a == b
        assert rule_next(t, r) == exact, (m, c, r)
    if c == 0:
        exact = t.NT >= 32 and word_round_by_warp(t) == chunks_by_warp(t, 0)
        assert rule_word(m) == exact, m


def test_rule_allows_the_step_shapes():
    """The shapes of the step's LDE: the top pass (M = 11, C = 2) and the lower
    passes (M = 13, C = 0) each drop one CTA barrier per tile pass."""
    assert rule_next(Tile4(11, 2, 2), 0) and not rule_next(Tile4(11, 2, 2), 1)
    assert rule_word(13) and not rule_next(Tile4(13, 0, 5), 0)
