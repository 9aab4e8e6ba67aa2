"""The frontier bound of the warp descents over 4-wide trees.

A warp pops min(size, 32) frontier entries per step (4 lanes per node when at
most 8 wait, 2 when at most 16, else 1: every step pops them all while at most
32 wait) and pushes every internal child of the popped nodes.  The shared
frontier is sized wide_frontier(depth) = 32 * 3 * depth + 32 * 4 entries
(csrc/rtcd_internal.cuh) for a tree whose deepest internal node is at
`depth`; the kernels fail a call that would overflow it.  This simulates that
policy on random 4-wide trees with every child overlapping the query (the
worst case) and from a top cut of up to 64 records, and checks the bound."""
import numpy as np
import pytest

KWIDE = 4


def wide_frontier(depth):
    return 32 * (KWIDE - 1) * depth + 32 * KWIDE


def random_tree(rng, max_depth, p_internal):
    """children[i]: internal child ids of node i (leaves are not frontier entries); depth[i]."""
    children, depth = [[]], [0]
    stack = [0]
    while stack:
        i = stack.pop()
        if depth[i] >= max_depth:
            continue
        for _ in range(KWIDE):
            if rng.random() < p_internal:
                j = len(children)
                children.append([])
                depth.append(depth[i] + 1)
                children[i].append(j)
                stack.append(j)
    return children, depth


def max_frontier(children, start):
    fr = list(start)
    worst = len(fr)
    while fr:
        take = min(len(fr), 32)   # the policy pops everything up to 32
        popped = fr[len(fr) - take:]
        del fr[len(fr) - take:]
        for n in popped:
            fr.extend(children[n])
        worst = max(worst, len(fr))
    return worst


def top_cut(children, limit=64):
    """The root's children, opened level by level while they fit (internal ones only count)."""
    cut = list(children[0])
    while True:
        nxt = []
        for n in cut:
            nxt.extend(children[n] if children[n] else [])
        if not nxt or len(nxt) > limit:
            return cut
        cut = nxt


@pytest.mark.parametrize('seed', range(12))
def test_frontier_within_bound(seed):
    rng = np.random.default_rng(seed)
    max_depth = int(rng.integers(3, 9))
    children, depth = random_tree(rng, max_depth, p_internal=float(rng.uniform(0.55, 0.95)))
    d = max(depth)  # every node here is an internal node of the wide tree
    assert max_frontier(children, [0]) <= wide_frontier(d)
    cut = top_cut(children)
    if cut:
        assert max_frontier(children, cut) <= wide_frontier(d)


def test_bound_is_reached_by_a_full_tree():
    """A complete 4-wide tree with every child overlapping fills half the
    bound, so the bound (and the shared memory it sizes) is not loose by more
    than a small factor."""
    children, depth = random_tree(np.random.default_rng(0), 6, p_internal=1.0)
    worst = max_frontier(children, [0])
    assert wide_frontier(6) * 0.4 < worst <= wide_frontier(6)
