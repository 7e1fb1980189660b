"""The oracle's octree and lists have the semantics of d3tstrcr (src/d3tstrcr.f:24-1069).

These are the properties the GPU tree is built on: list 1 = childless boxes
touching a childless box (any level); list 3 = boxes on finer levels that do
not touch it but whose parents do; list 4 = dual of list 3; list 2 = children
of the parent's colleagues that do not touch; boxes of a level are ordered by
(parent, child octant z-y-x).
"""
import numpy as np
import pytest

import oracle as O


def touch(b1, b2):
    l1, l2 = b1[0], b2[0]
    if l1 > l2:
        b1, b2, l1, l2 = b2, b1, l2, l1
    s = 1 << (l2 - l1)
    for d in range(3):
        i1, i2 = b1[1 + d] - 1, b2[1 + d] - 1
        if i1 * s > i2 + 1 or i2 > (i1 + 1) * s:
            return False
    return True


@pytest.fixture(scope="module", params=["sphere", "plummer"])
def tree(request):
    rng = np.random.default_rng(4)
    n = 6000
    if request.param == "sphere":
        v = rng.normal(size=(n, 3))
        src = v / np.linalg.norm(v, axis=1)[:, None]
    else:
        u = rng.random(n)
        r = 0.1 / np.sqrt(u ** (-2 / 3) - 1)
        v = rng.normal(size=(n, 3))
        src = r[:, None] * v / np.linalg.norm(v, axis=1)[:, None]
        src = src[r < 1]
    trg = rng.random((500, 3)) * 2 - 1
    return O.Tree(src, trg, 40), src.shape[0], trg.shape[0]


def test_boxes_partition_points(tree):
    T, n, m = tree
    leaves = [b for b in range(T.nboxes) if T.box[b, 5] < 0]
    assert sum(T.box[b, 14] for b in leaves) == n
    assert sum(T.box[b, 16] for b in leaves) == m
    assert sorted(T.iz) == list(range(n))
    for b in range(T.nboxes):
        if T.box[b, 5] < 0:
            continue
        assert T.box[b, 14] > 40 or T.box[b, 16] > 40       # split only when over nbox
        kids = [k for k in T.box[b, 5:13] if k >= 0]
        assert sum(T.box[k, 14] for k in kids) == T.box[b, 14]
        octs = [(T.box[k, 1] - 1) % 2 + 2 * ((T.box[k, 2] - 1) % 2) + 4 * ((T.box[k, 3] - 1) % 2) for k in kids]
        assert octs == sorted(octs)


def test_list1_is_touching_leaves(tree):
    T, _, _ = tree
    leaves = [b for b in range(1, T.nboxes) if T.box[b, 5] < 0]
    lv = set(leaves)
    for b in leaves[::7]:
        want = {c for c in lv if c != b and touch(T.box[b, :4], T.box[c, :4])}
        assert set(T.list_of(1, b)) == want


def test_list3_and_list4(tree):
    T, _, _ = tree
    for b in range(1, T.nboxes):
        l3 = set(T.list_of(3, b))
        if T.box[b, 5] >= 0:
            assert not l3
            continue
        for c in l3:
            assert T.box[c, 0] > T.box[b, 0]
            assert not touch(T.box[b, :4], T.box[c, :4])
            assert touch(T.box[b, :4], T.box[T.box[c, 4], :4])
            assert b in set(T.list_of(4, c))


def test_list2_and_list5(tree):
    T, _, _ = tree
    for b in range(1, T.nboxes, 5):
        par = T.box[b, 4]
        cands = [par] + list(T.list_of(5, par))
        kids = {k for c in cands for k in T.box[c, 5:13] if k >= 0 and k != b}
        l5 = set(T.list_of(5, b))
        l2 = set(T.list_of(2, b))
        assert l5 | l2 == kids and not (l5 & l2)
        assert all(touch(T.box[b, :4], T.box[c, :4]) for c in l5)
        assert not any(touch(T.box[b, :4], T.box[c, :4]) for c in l2)
