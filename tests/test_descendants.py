"""Descendant counts of exploration rows (refine.descendants), the labels of
the learned placement's training: whole subtrees and generation-limited
counts on a hand-made parent tree."""
import numpy as np
import pytest

from gpu_cdt_refine_b200 import refine

# rows: 0 root with children 1, 2; 3 child of 1; 4 child of 3 (lost its
# conflict: not inserted); 5 a second root.  Midpoints: 1 below row 0, 2 below
# row 2, 1 below row 3.
PARENT = np.array([-1, 0, 0, 1, 3, -1])
INSERTED = np.array([1, 1, 1, 1, 0, 1])
MIDS = np.array([1, 0, 2, 1, 0, 0])


def test_whole_subtrees():
    d = refine.descendants(PARENT, INSERTED, MIDS)
    # row 3: its midpoint; row 1: row 3 and its midpoint; row 2: two midpoints;
    # row 0: its midpoint + rows 1, 2 + their subtrees
    assert d.tolist() == [1 + 2 + 2 + 2, 2, 2, 1, 0, 0]


@pytest.mark.parametrize("depth,want", [(1, [3, 1, 2, 1, 0, 0]), (2, [6, 2, 2, 1, 0, 0]), (3, [7, 2, 2, 1, 0, 0])])
def test_generation_limited(depth, want):
    assert refine.descendants(PARENT, INSERTED, MIDS, depth).tolist() == want


def test_roots_account_for_everything():
    d = refine.descendants(PARENT, INSERTED, MIDS)
    roots = (PARENT < 0) & (INSERTED == 1)
    assert d[roots].sum() + roots.sum() == INSERTED.sum() + MIDS.sum()


def test_parent_after_child_is_rejected():
    with pytest.raises(ValueError):
        refine.descendants(np.array([1, -1]), np.array([1, 1]), np.array([0, 0]))
