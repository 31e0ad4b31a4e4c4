"""The BVH8 structural check (prt_bvh8_check) and the array traversal (prt_bvh8_trace), on CPU.

The check is what the device-build tests rely on, so it is tested here on host-built trees: a
valid tree passes, and each planted mistake -- made on the CPU in a copy of the arrays -- is
reported. The array traversal over a host-built tree returns what prt_bvh8_count returns.
"""
import numpy as np
import pytest

import prt_cuda
import prt_scenes


def host_tree(scene):
    tv = prt_scenes.tri_verts(scene)
    nodes, tris, top = prt_cuda.bvh8_build_host(tv)
    return tv, nodes, tris, top


def random_rays(tv, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = tv.reshape(-1, 3).min(0), tv.reshape(-1, 3).max(0)
    o = rng.uniform(lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo), (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3], r[:, 4:7], r[:, 3], r[:, 7] = o, d, 0.0, 1e30
    return r


@pytest.mark.parametrize("scene", [
    prt_scenes.cornell(seed=0, width=16, height=16),
    prt_scenes.triangle_soup(seed=1, n=3000),
    prt_scenes.triangle_soup(seed=2, n=1),
    prt_scenes.triangle_soup(seed=3, n=3),
    prt_scenes.triangle_soup(seed=4, n=9),
], ids=["cornell", "soup3000", "soup1", "soup3", "soup9"])
def test_host_tree_passes(scene):
    tv, nodes, tris, top = host_tree(scene)
    depth, msg = prt_cuda.bvh8_check(nodes, tris, tv, top)
    assert msg == "" and depth >= 1


@pytest.fixture(scope="module")
def tree():
    return host_tree(prt_scenes.cornell(seed=0, width=16, height=16))


def test_planted_box_shrink_is_caught(tree):
    tv, nodes, tris, top = tree
    bad = nodes.copy()
    # The upper bounds of the first used slot of node 3 lowered to its lower bounds (bytes 32..55
    # hold qlo x/y/z, 56..79 qhi x/y/z): the box shrinks to a point and no longer holds the subtree.
    used = (bad[3, 24:32] != 0) | (((bad[3, 15] >> np.arange(8)) & 1) != 0)
    slot = int(np.nonzero(used)[0][0])
    for axis in range(3):
        bad[3, 56 + 8 * axis + slot] = bad[3, 32 + 8 * axis + slot]
    assert "does not contain" in prt_cuda.bvh8_check(bad, tris, tv, top)[1]


def test_planted_vertex_change_is_caught(tree):
    tv, nodes, tris, top = tree
    bad = tris.copy()
    v = bad.view(np.float32).reshape(-1, 12)
    v[7, 4] += 1e-3  # e1.x of record 7
    assert "vertex data" in prt_cuda.bvh8_check(nodes, bad, tv, top)[1]


def test_planted_duplicate_reference_is_caught(tree):
    tv, nodes, tris, top = tree
    bad = nodes.copy()
    # A second inner node pointing its children at the first's: nodes reached twice.
    inner = [i for i in range(1, bad.shape[0]) if bad[i, 15] != 0]
    a, b = inner[0], inner[1]
    bad[b, 16:20] = bad[a, 16:20]
    bad[b, 15] = bad[a, 15]
    msg = prt_cuda.bvh8_check(bad, tris, tv, top)[1]
    assert msg != ""


def test_planted_top_count_is_caught(tree):
    tv, nodes, tris, top = tree
    assert prt_cuda.bvh8_check(nodes, tris, tv, top - 1)[1] != ""
    assert prt_cuda.bvh8_check(nodes, tris, tv, 0)[1] != ""


def test_planted_missing_triangle_is_caught(tree):
    tv, nodes, tris, top = tree
    extra = np.concatenate([tv, tv[:1] + 5.0])
    assert "never referenced" in prt_cuda.bvh8_check(nodes, np.concatenate([tris, tris[:1]]), extra, top)[1]


def test_array_trace_matches_the_counting_build():
    s = prt_scenes.triangle_soup(seed=5, n=4000)
    tv, nodes, tris, top = host_tree(s)
    rays = random_rays(tv, 4000, 6)
    a = prt_cuda.bvh8_trace(nodes, tris, rays)
    b = prt_cuda.bvh8_count(tv, rays)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
    assert a[2] == b[2] and a[3] == b[3]
    assert (a[0] >= 0).mean() > 0.2
