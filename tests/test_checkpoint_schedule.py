"""The binomial checkpoint schedule of dugks_adjoint_run (Griewank's revolve),
counted on the host through dugks_checkpoint_forward_steps: every step is
reversed once, in order, and the forward steps are the fewest possible,
T(N, s) = r N - C(s + r, s + 1) with r the least number of recomputations
with C(s + r, s) >= N for s snapshots (the start state's included)."""
import math

import pytest

from dugks_b200 import lib as dl


def _r_min(n, s):
    r = 0
    while math.comb(s + r, s) < n:
        r += 1
    return r


def _optimal(n, s):
    if n <= 1:
        return 0
    r = _r_min(n, s)
    return r * n - (math.comb(s + r, s + 1) if r >= 1 else 0)


def _optimal_by_search(n, k, memo={}):
    """The fewest forward steps by exhaustive search over the first split
    (k free slots besides the start's)."""
    if n == 1:
        return 0
    if k == 0:
        return n * (n - 1) // 2
    key = (n, k)
    if key not in memo:
        memo[key] = min(m + _optimal_by_search(n - m, k - 1) + _optimal_by_search(m, k) for m in range(1, n))
    return memo[key]


def test_closed_form_is_the_searched_optimum():
    for k in range(0, 5):
        for n in range(1, 80):
            assert _optimal(n, k + 1) == _optimal_by_search(n, k), (n, k)


@pytest.mark.parametrize("s", [1, 2, 3, 4, 8, 64])
def test_forward_steps_within_the_binomial_bound(s):
    lib = dl.load()
    for n in list(range(1, 120)) + [500, 1000, 4000]:
        f = lib.dugks_checkpoint_forward_steps(n, s)
        assert f >= n - 1, (n, s, f)
        if s >= n:
            assert f == n - 1, (n, s, f)     # every state kept: each step is run once
        assert f == _optimal(n, s), (n, s, f, _optimal(n, s))


def test_one_snapshot_recomputes_from_the_start():
    lib = dl.load()
    for n in (1, 2, 5, 17):
        assert lib.dugks_checkpoint_forward_steps(n, 1) == n * (n - 1) // 2


def test_named_configuration_and_bad_arguments():
    lib = dl.load()
    # 4000 steps in 64 snapshots: r = 3 (C(67, 64) = 47905 >= 4000) and
    # T = 3 * 4000 - C(67, 65) = 9789
    assert lib.dugks_checkpoint_forward_steps(4000, 64) == _optimal(4000, 64) == 9789
    assert lib.dugks_checkpoint_forward_steps(0, 4) == -1
    assert lib.dugks_checkpoint_forward_steps(4, 0) == -1
