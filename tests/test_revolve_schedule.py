"""The binomial (revolve) checkpointing schedule on the host (no GPU): the
library's count of re-run forward steps equals the optimum of the recursion
it states, the schedule passes its own check (every slot holds the step it is
used for, steps reversed last to first), and the counts follow the known
limits (one slot: n (n + 1) / 2; a slot per step: n)."""
import functools
import sys

import pytest

from apollo_b200 import ApolloError, NodalDG2d

sys.setrecursionlimit(10000)


@functools.lru_cache(None)
def F(n, c):
    """Forward steps to reverse n steps from a stored state with c free slots."""
    if n == 1:
        return 1
    if c == 0:
        return n * (n + 1) // 2
    return min(m + F(n - m, c - 1) + F(m, c) for m in range(1, n))


@functools.lru_cache(None)
def G(n, c):
    """The same when the forward pass stored the first descent's states."""
    if n == 1:
        return 1
    if c == 0:
        return n * (n + 1) // 2
    return min(G(n - m, c - 1) + F(m, c) for m in range(1, n))


@pytest.mark.parametrize("n, S", [(1, 1), (2, 1), (10, 1), (10, 2), (37, 2), (60, 4), (100, 3), (150, 6), (120, 12)])
def test_schedule_is_optimal(n, S):
    steps, stored = NodalDG2d.revolve_schedule(n, S)
    assert steps == G(n, S - 1)
    assert 1 <= stored <= S


def test_schedule_limits():
    assert NodalDG2d.revolve_schedule(400, 1) == (400 * 401 // 2, 1)
    assert NodalDG2d.revolve_schedule(400, 400)[0] == 400
    # 400 steps: 20 slots re-run fewer than 2.5 n steps, 5 slots fewer than 5 n
    a20 = NodalDG2d.revolve_schedule(400, 20)[0]
    a5 = NodalDG2d.revolve_schedule(400, 5)[0]
    assert a20 < 2.5 * 400 and a5 < 5 * 400 and a20 < a5
    # beyond the dynamic-programming range the binomial rule still passes its check
    big, stored = NodalDG2d.revolve_schedule(6000, 20)
    assert stored == 20 and big < 6 * 6000
    # one free slot over a long trajectory: a deep schedule that the sweep
    # walks without deep recursion
    deep, stored = NodalDG2d.revolve_schedule(20000, 2)
    assert stored == 2 and deep > 20000


def test_schedule_arguments():
    for n, S in ((0, 5), (5, 0)):
        with pytest.raises(ApolloError):
            NodalDG2d.revolve_schedule(n, S)
