"""The ordering rule of the reverse re-prune (csrc/prune_rev.cu, step 2), restated on
the CPU and checked against a plain sort.

Candidates are the reverse sources A (indices 0 .. nA-1) then the node's list B
(indices nA ..).  Their order is by (distance, index).  When B is in nondecreasing
distance order, the kernel places B_j at j + #{i : d(A_i) <= d(B_j)} and A_i at
#{j : d(B_j) < d(A_i)} + #{k : (d(A_k), k) < (d(A_i), i)}, with no sort.  Integer-valued
distances make ties frequent, which is where the index rule matters.
"""
import numpy as np
import pytest


def merged_positions(da, db):
    na, nb = len(da), len(db)
    pos = np.empty(na + nb, np.int64)
    for j in range(nb):
        pos[na + j] = j + int(np.sum(da <= db[j]))
    for i in range(na):
        pos[i] = int(np.sum(db < da[i])) + sum(1 for k in range(na) if da[k] < da[i] or (da[k] == da[i] and k < i))
    return pos


@pytest.mark.parametrize("seed", range(40))
def test_rule_equals_sort_by_distance_then_index(seed):
    rng = np.random.default_rng(seed)
    na = int(rng.integers(0, 9))
    nb = int(rng.integers(0, 121))
    span = int(rng.choice([4, 20, 1000]))  # few distinct values: many ties
    da = rng.integers(0, span, na).astype(np.float32)
    db = np.sort(rng.integers(0, span, nb)).astype(np.float32)
    d = np.concatenate([da, db])
    order = np.lexsort((np.arange(na + nb), d))  # by distance, then index
    expect = np.empty(na + nb, np.int64)
    expect[order] = np.arange(na + nb)
    assert np.array_equal(merged_positions(da, db), expect)


def test_out_of_order_list_is_detected():
    """The kernel takes the rule only when d(B_j) <= d(B_j+1) for every j; a list out of
    order would get wrong positions, so it is sorted instead."""
    db = np.array([1.0, 3.0, 2.0], np.float32)
    assert not np.all(db[:-1] <= db[1:])
    da = np.array([2.5], np.float32)
    d = np.concatenate([da, db])
    order = np.lexsort((np.arange(4), d))
    expect = np.empty(4, np.int64)
    expect[order] = np.arange(4)
    assert not np.array_equal(merged_positions(da, db), expect)
