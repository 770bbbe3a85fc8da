"""The placement rule the GPU BVH build (pfx_b200/csrc/bvh_gpu.cu, k_place)
uses for the in-place partition of bvh.rs:232-249, checked against that
partition's loop on random side patterns: with front element i (position i)
and back element j (position n-1-j), cf = failing elements before front i,
ct = passing elements before back j, P = front indices of the failing
elements, Q = back indices of the passing ones, every element lands where the
loop puts it."""
import numpy as np


def partition_loop(t):
    """bvh.rs:232-249: the left pointer tests, a failing element is swapped
    with the last unexamined one.  Returns the final arrangement of indices."""
    a = list(range(len(t)))
    left, right = 0, len(a)
    while left < right:
        if t[a[left]]:
            left += 1
        else:
            right -= 1
            a[left], a[right] = a[right], a[left]
    return a


def partition_rule(t):
    t = np.asarray(t, bool)
    n = len(t)
    passing = int(t.sum())
    cf = np.concatenate([[0], np.cumsum(~t)])
    P = np.flatnonzero(~t)
    Q = np.flatnonzero(t[::-1])
    out = [None] * n
    for i in range(n):
        j = n - 1 - i
        c = int(cf[i])
        k = c + 1
        front, qb = True, 0
        if k > 1:
            front = k - 2 < passing and i + int(Q[k - 2]) + 1 < n
            qb = int(Q[k - 2]) + 1 if k - 2 < passing else 0
        if front:
            dest = (i - c) + (k - 1) if t[i] else n - 1 - (c + (qb - (k - 1)))
        else:
            ct = int(t[i + 1:].sum())
            kb = ct + 1
            pk = int(P[kb - 1])
            dest = (pk + 1 - kb) + ct if t[i] else n - 1 - (kb + (j - ct))
        assert 0 <= dest < n and out[dest] is None
        out[dest] = i
    return out


def test_the_placement_rule_is_the_swap_partition():
    rng = np.random.default_rng(0)
    for _ in range(3000):
        n = int(rng.integers(1, 48))
        t = rng.random(n) < rng.random()
        assert partition_rule(t) == partition_loop(t)
    for n in (1, 2, 7):  # all passing, all failing
        assert partition_rule([True] * n) == partition_loop([True] * n)
        assert partition_rule([False] * n) == partition_loop([False] * n)
