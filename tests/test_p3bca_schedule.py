"""The slot-pair schedule of the P3BCA triplet kernel (k_p3bca in csrc/tbmd_kernels.cu), restated on the
host and enumerated for every block shape: each unordered slot pair of an item is visited exactly once,
the partner targets of one warp step are distinct (so the kernel's shared-memory read-modify-writes need
no atomics), the partner copies of the short-block lane groups stay inside their 32 entries, and the
shuffle tree over lanes l, l + m_B, l + 2 m_B, ... adds every copy into its partner's lane exactly once.

The reference visits every triplet i < j < k once (Algorithm.cpp:88-139); the kernel's items are the
half lists of particle i, so its schedule must cover every pair (j, k) of a list once."""
from collections import Counter

import pytest

COPIES = 32


def diagonal_steps(A0, mA):
    """Pairs inside block A: circular diagonals (x, (x + d) mod m_A), d = 1 .. m_A / 2; on the half
    diagonal of an even m_A only x < d."""
    for d in range(1, mA // 2 + 1):
        step = []
        for lane in range(32):
            own = lane < mA
            act = own and (2 * d < mA or lane < d)
            if act:
                step.append((A0 + lane, A0 + (lane + d) % mA, ("slot", A0 + (lane + d) % mA)))
        yield step


def cross_steps(A0, mA, B0, mB):
    """Pairs A x B.  A full B: a rotation (x, (x + t) & 31).  A short B: lane j of group g meets
    (j + t) mod m_B at step t; group 0 adds to B's slots, group g >= 1 to copy (g - 1) m_B + y."""
    if mB == 32:
        for t in range(32):
            step = []
            for lane in range(mA):
                y = (lane + t) & 31
                if y < mB:
                    step.append((A0 + lane, B0 + y, ("slot", B0 + y)))
            yield step
    else:
        for t in range(mB):
            step = []
            for lane in range(mA):
                g, j = divmod(lane, mB)
                y = (j + t) % mB
                tgt = ("slot", B0 + y) if g == 0 else ("copy", (g - 1) * mB + y)
                step.append((A0 + lane, B0 + y, tgt))
            yield step


def item_pairs(mI, mJ):
    """Every warp step of an item: slots [0, mI) and, for a chunk pair, [mI, mI + mJ)."""
    Ms = mI + mJ
    steps = []
    for A0 in range(0, mI, 32):
        mA = min(32, mI - A0)
        if mJ == 0:
            steps += list(diagonal_steps(A0, mA))
        for B0 in range(A0 + 32 if mJ == 0 else mI, Ms, 32):
            steps += list(cross_steps(A0, mA, B0, min(32, Ms - B0)))
    return steps


def tree_merge(mB, written):
    """Lane l takes copy l; rounds off = m_B, 2 m_B, ... while off < 32 add lane l + off's value when that
    lane exists.  Returns, per lane l < m_B, the multiset of copies it summed."""
    val = [Counter({l: 1}) if l in written else Counter() for l in range(32)]
    off = mB
    while off < 32:
        val = [val[l] + (val[l + off] if l + off < 32 else Counter()) for l in range(32)]
        off *= 2
    return val[:mB]


@pytest.mark.parametrize("mI,mJ", [(m, 0) for m in range(2, 65)] + [(64, m) for m in range(1, 65, 3)])
def test_every_pair_once_and_distinct_targets(mI, mJ):
    seen = Counter()
    for step in item_pairs(mI, mJ):
        targets = [t for _, _, t in step]
        assert len(targets) == len(set(targets))
        for a, b, t in step:
            assert a != b
            seen[(min(a, b), max(a, b))] += 1
            if t[0] == "copy":
                assert 0 <= t[1] < COPIES
    if mJ == 0:
        want = {(a, b) for a in range(mI) for b in range(a + 1, mI)}
    else:
        want = {(a, b) for a in range(mI) for b in range(mI, mI + mJ)}
    assert set(seen) == want
    assert all(c == 1 for c in seen.values())


@pytest.mark.parametrize("mA", [1, 7, 19, 32])
@pytest.mark.parametrize("mB", list(range(1, 32)))
def test_copy_tree_sums_each_copy_into_its_partner(mA, mB):
    written = set()
    for step in cross_steps(0, mA, 32, mB):
        for _, _, t in step:
            if t[0] == "copy":
                written.add(t[1])
    merged = tree_merge(mB, written)
    got = Counter()
    for lane, c in enumerate(merged):
        for k, n in c.items():
            assert k % mB == lane  # copy (g - 1) m_B + y belongs to partner y
            got[k] += n
    assert set(got) == written and all(n == 1 for n in got.values())
