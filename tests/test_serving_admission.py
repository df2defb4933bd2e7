"""The serving loop's admission rule by device memory (host logic, no GPU):
the oldest requests, in arrival order, while the launch's work areas fit in
the room the launches in flight leave; the first one that does not fit
stops the launch (no younger request overtakes it); a request larger than
the whole budget runs alone once nothing else is in flight."""

from ttnumpy_b200.persistent_serving import admit


def test_no_budget_takes_everything():
    assert admit([5, 7, 9], None, idle=False) == [0, 1, 2]
    assert admit([], None, idle=True) == []


def test_oldest_first_while_they_fit():
    assert admit([3, 4, 5], 8, idle=False) == [0, 1]
    # a large request that does not fit yet holds back the younger ones
    # behind it, so it cannot be overtaken indefinitely
    assert admit([3, 6, 2], 6, idle=False) == [0]
    assert admit([6, 2], 6, idle=False) == [0]
    assert admit([2, 2, 2, 2], 8, idle=True) == [0, 1, 2, 3]


def test_nothing_fits():
    assert admit([9, 10], 8, idle=False) == []  # wait for launches in flight
    assert admit([9, 10], 8, idle=True) == [0]  # alone: larger than the budget
    assert admit([5], 0, idle=True) == [0]
    assert admit([], 8, idle=True) == []
