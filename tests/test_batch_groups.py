"""Record groups of the batched step (batch.record_groups): contiguous,
non-decreasing, each within the size unless one view alone exceeds it."""

from powerfoam_b200.batch import record_groups


def test_record_groups_pack_views_in_order():
    groups, sums = record_groups([5, 4, 3, 9, 1, 1], 10)
    assert groups == [0, 0, 1, 2, 2, 3]
    assert sums == [9, 3, 10, 1]
    assert all(s <= 10 for s in sums)


def test_record_groups_one_group_when_everything_fits():
    groups, sums = record_groups([3, 2, 1], 100)
    assert groups == [0, 0, 0] and sums == [6]


def test_record_groups_oversized_view_gets_its_own_group():
    groups, sums = record_groups([2, 50, 2, 2], 10)
    assert groups == [0, 1, 2, 2] and sums == [2, 50, 4]
    assert groups == sorted(groups)
