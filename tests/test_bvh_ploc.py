"""The PLOC builder's host specification (bvh_build.cpp): a valid binary
tree over the boxes, leaves in Morton order, node boxes the unions of their
children, and a surface-area cost close to the binned-SAH builder's."""
import numpy as np
import pytest

from atrc_b200 import bvh_cluster_tree


def _spread21(v):
    x = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    for shift, mask in ((32, 0x1F00000000FFFF), (16, 0x1F0000FF0000FF), (8, 0x100F00F00F00F00F),
                        (4, 0x10C30C30C30C30C3), (2, 0x1249249249249249)):
        x = (x | (x << np.uint64(shift))) & np.uint64(mask)
    return x


def _morton(boxes):
    c = np.float32(0.5) * (boxes[:, :3] + boxes[:, 3:])
    lo, hi = c.min(0), c.max(0)
    inv = np.where(hi > lo, np.float32(1) / np.where(hi > lo, hi - lo, 1), 0).astype(np.float32)
    t = np.clip(np.nan_to_num((c - lo) * inv), 0, 1).astype(np.float32)
    q = (t * np.float32(2097151.0)).astype(np.uint32)
    return _spread21(q[:, 0]) | (_spread21(q[:, 1]) << np.uint64(1)) | (_spread21(q[:, 2]) << np.uint64(2))


def random_boxes(n, seed, surface=False):
    rng = np.random.default_rng(seed)
    if surface:
        th, z = rng.uniform(0, 2 * np.pi, n), rng.uniform(-1, 1, n)
        r = np.sqrt(1 - z * z)
        c = 50 + 40 * np.stack([r * np.cos(th), r * np.sin(th), z], 1)
    else:
        c = rng.uniform(0, 100, (n, 3))
    e = rng.uniform(0, 0.3, (n, 3))
    return np.concatenate([c - e, c + e], 1).astype(np.float32)


def check_tree(boxes, t):
    n = len(boxes)
    order, left, right, nb = t["order"], t["left"], t["right"], t["boxes"]
    assert sorted(order.tolist()) == list(range(n))
    keys = _morton(boxes)[order]
    assert np.all(keys[1:] >= keys[:-1])                      # sorted by Morton code
    same = keys[1:] == keys[:-1]
    assert np.all(order[1:][same] > order[:-1][same])         # stable for equal keys
    if n == 1:
        assert t["root"] == 0
        return
    assert t["root"] == 2 * n - 2
    kids = np.concatenate([left, right])
    assert sorted(kids.tolist()) == list(range(2 * n - 2))    # every node but the root has one parent
    k = np.arange(n - 1) + n
    assert np.all(left < k) and np.all(right < k)             # children before parents
    allb = np.concatenate([boxes[order], nb])
    un = np.concatenate([np.minimum(allb[left, :3], allb[right, :3]), np.maximum(allb[left, 3:], allb[right, 3:])], 1)
    np.testing.assert_array_equal(nb, un)


@pytest.mark.parametrize("n,surface", [(1, False), (2, False), (3, True), (1000, False), (20000, True)])
def test_host_cluster_tree_is_valid(n, surface):
    boxes = random_boxes(n, 5 + n, surface)
    t = bvh_cluster_tree(boxes, device=-1)
    check_tree(boxes, t)
    assert n < 3 or t["rounds"] < 80


def test_identical_boxes_still_merge():
    # every key ties: the pair order breaks the ties, so each round merges
    boxes = np.tile(np.float32([0, 0, 0, 1, 1, 1]), (257, 1))
    t = bvh_cluster_tree(boxes, device=-1)
    check_tree(boxes, t)
    np.testing.assert_array_equal(t["order"], np.arange(257))


@pytest.mark.parametrize("surface", [False, True])
def test_host_ploc_tree_cost_close_to_sah(surface):
    from atrc_b200 import bvh_build
    boxes = random_boxes(50_000, 3, surface)
    s = bvh_build(boxes, "sah", device=-1)
    p = bvh_build(boxes, "ploc", device=-1)
    assert p["rounds"] == 0 and p["nodes"] > 0 and p["max_depth"] > 0
    assert p["sah_cost"] < 1.25 * s["sah_cost"], (p, s)
