"""The mixed solve's preconditioner-rebuild policy (host logic, no GPU)."""

from pyvl_b200.engine import RefreshPolicy


def run(policy, counts, idle=True, since0=5):
    """Feed one count per step; return the steps at which a rebuild was due (and taken)."""
    fired, since = [], since0
    for step, k in enumerate(counts):
        policy.observe([k])
        if policy.due(since, idle):
            fired.append(step)
            policy.rebuilt()
            since = 0
        since += 1
    return fired


def test_steady_counts_never_rebuild():
    assert run(RefreshPolicy(5, 128), [2] * 500) == []


def test_a_jump_well_above_the_best_rebuilds_at_once():
    p = RefreshPolicy(5, 128)
    assert run(p, [2, 2, 2, 6, 2, 2]) == [3]


def test_a_slow_count_near_the_best_is_left_to_the_excess_rule():
    # 5 iterations is slow, but the best since the rebuild is 4: not 3 above it
    p = RefreshPolicy(5, 128)
    assert run(p, [4] + [5] * 50) == []
    assert p.excess == 50


def test_excess_accumulates_to_a_rebuild_and_resets():
    p = RefreshPolicy(5, 10)
    fired = run(p, [2] + [3] * 30)
    assert fired == [10]  # one extra column per step above the best (2) adds up to 10
    assert (p.best, p.excess) == (3, 0)  # after the rebuild the best is the new count


def test_no_rebuild_while_one_is_in_flight_or_just_after_one():
    p = RefreshPolicy(5, 128)
    assert run(p, [2, 9, 9, 9], idle=False) == []
    p = RefreshPolicy(5, 128)
    p.observe([2, 9])
    assert not p.due(1, True)  # fewer than two steps since the last rebuild
    assert p.due(2, True)


def test_period_rebuilds_regardless():
    p = RefreshPolicy(5, 128, period=25)
    assert run(p, [2] * 60, idle=False, since0=0) == [25, 50]
