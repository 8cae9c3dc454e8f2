"""The closed form of back-to-front swap_remove that device fate uses
(k_fate_resolve, block 1), restated in Python and checked against the
sequential removal the reference performs (crates/marl-sim/src/lib.rs:256-267)
on random death sets, including every small case exhaustively.

With n cells and ascending deaths, n1 = n - |deaths| cells remain.  D(x) is
the number of deaths below x; b_0 = n1 and b_{k+1} = b_k + D(b_k) - D(b_{k-1})
until the increment is zero.  A death q in [b_{k-1}, b_k) is first refilled
from position b_k + D(q) - D(b_{k-1}); hole i (the i-th death below n1) takes
the cell reached by following that map from n1 + i through dead positions.
"""
import bisect
import itertools

import numpy as np


def sequential(n0, deaths):
    cells = list(range(n0))
    for i in reversed(deaths):
        cells[i] = cells[-1]
        cells.pop()
    return cells


def closed_form(n0, deaths):
    n1 = n0 - len(deaths)
    dead = set(deaths)

    def D(x):
        return bisect.bisect_left(deaths, x)

    levels, prev = [n1], [0]  # b_k and D(b_{k-1})
    while True:
        m = D(levels[-1]) - prev[-1]
        if m == 0:
            break
        prev.append(D(levels[-1]))
        levels.append(levels[-1] + m)
    out = list(range(n1))
    for i, h in enumerate(d for d in deaths if d < n1):
        q, steps = n1 + i, 0
        while q in dead:
            k = bisect.bisect_right(levels, q)  # levels[k-1] <= q < levels[k]
            assert 0 < k < len(levels)
            q = levels[k] + D(q) - prev[k]
            steps += 1
            assert steps <= len(levels)
        out[h] = q
    return out, len(levels)


def test_exhaustive_small():
    for n0 in range(0, 11):
        for r in range(0, n0 + 1):
            for deaths in itertools.combinations(range(n0), r):
                deaths = list(deaths)
                assert closed_form(n0, deaths)[0] == sequential(n0, deaths), (n0, deaths)


def test_random_sets():
    rng = np.random.default_rng(12)
    deepest = 0
    for _ in range(5000):
        n0 = int(rng.integers(1, 400))
        k = int(rng.integers(0, n0 + 1))
        deaths = sorted(rng.choice(n0, size=k, replace=False).tolist())
        got, levels = closed_form(n0, deaths)
        assert got == sequential(n0, deaths)
        deepest = max(deepest, levels)
    assert deepest > 3  # the random sets reach several levels
