"""Device BVH8 build (PRT_BVH_DEVICE) against the host build (PRT_BVH_HOST).

The two builders make different trees in one format, and a ray's closest hit does not depend on
the tree (same triangle records, conservative boxes, ties to the smaller triangle index), so:
  * the device tree passes the structural check (every triangle stored once with the exact
    vertex data, every 8-bit child box holding its subtree, top levels first, depth within the
    traversal stack) -- including 1..9 triangles, the in-block clustering tail boundary, and
    soups with duplicate and degenerate triangles;
  * the host counting traversal over the device tree returns the same triangle and the same t,
    bit for bit, as over the host tree; so does the device trace kernel;
  * rendered images are bit-identical with either tree in the frame form, and equal to float
    rounding in a batch (whose accumulation order is that of its atomics);
  * the build is deterministic: the same scene gives the same bytes;
  * tree quality: node visits per ray at most 1.3x the host SAH tree's.
"""
import numpy as np
import pytest

import prt_cuda
import prt_scenes
import prt_types as T

pytestmark = pytest.mark.gpu


def with_builder(scene, builder):
    scene.bvh_build = builder
    return scene


def device_tree(dev, scene):
    with_builder(scene, T.PRT_BVH_DEVICE)
    dev.init_scene(scene)
    nodes, tris = dev.scene_bvh()
    return nodes, tris, dev.scene_stats()


def random_rays(tv, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = tv.reshape(-1, 3).min(0), tv.reshape(-1, 3).max(0)
    o = rng.uniform(lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo), (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3], r[:, 4:7], r[:, 3], r[:, 7] = o, d, 0.0, 1e30
    return r


SCENES = {
    "cornell": lambda: prt_scenes.cornell(seed=0, width=64, height=64, spp=4),
    "lobes": lambda: prt_scenes.cornell_lobes(seed=0, width=64, height=64, spp=4),
    "terrain": lambda: prt_scenes.terrain(seed=3, grid=256, n_spheres=40, width=128, height=64, spp=4),
    "soup5000": lambda: prt_scenes.triangle_soup(seed=1, n=5000),
    "soup4096": lambda: prt_scenes.triangle_soup(seed=2, n=4096),
    "soup4097": lambda: prt_scenes.triangle_soup(seed=3, n=4097),
    "soup70000": lambda: prt_scenes.triangle_soup(seed=4, n=70000),
}
TINY = [1, 2, 3, 4, 5, 9]


@pytest.mark.parametrize("name", list(SCENES) + [f"soup{n}" for n in TINY])
def test_device_tree_passes_the_check(device, name):
    s = SCENES[name]() if name in SCENES else prt_scenes.triangle_soup(seed=7, n=int(name[4:]))
    nodes, tris, st = device_tree(device, s)
    tv = prt_scenes.tri_verts(s)
    depth, msg = prt_cuda.bvh8_check(nodes, tris, tv, st["top_count"])
    assert msg == ""
    assert st["builder"] == T.PRT_BVH_DEVICE and st["depth"] == depth
    assert st["tri_count"] == tv.shape[0] and st["node_count"] == nodes.shape[0]


@pytest.mark.parametrize("name", ["cornell", "terrain", "soup5000", "soup70000"])
def test_hits_match_the_host_tree(device, name):
    s = SCENES[name]()
    tv = prt_scenes.tri_verts(s)
    nodes, tris, _ = device_tree(device, s)
    hn, ht, _ = prt_cuda.bvh8_build_host(tv)
    rays = random_rays(tv, 20000, 11)
    a = prt_cuda.bvh8_trace(nodes, tris, rays)
    b = prt_cuda.bvh8_trace(hn, ht, rays)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
    assert (a[0] >= 0).mean() > 0.05
    # The device trace kernel: the same answers over either tree.
    hit_dev = device.trace(rays)
    device.init_scene(with_builder(s, T.PRT_BVH_HOST))
    hit_host = device.trace(rays)
    for x, y in zip(hit_dev[:3], hit_host[:3]):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.parametrize("name", ["cornell", "lobes", "terrain"])
def test_images_match_the_host_tree(device, name):
    out = []
    for builder in (T.PRT_BVH_HOST, T.PRT_BVH_DEVICE):
        s = with_builder(SCENES[name](), builder)
        device.setup(s, seed=3)
        st = device.render(s.spp)
        out.append((device.blit_frame(), st["rays"]))
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


def test_batch_images_match_the_host_tree(device):
    frames = []
    for builder in (T.PRT_BVH_HOST, T.PRT_BVH_DEVICE):
        scenes = [with_builder(SCENES[n](), builder) for n in ("cornell", "terrain")]
        batch = prt_cuda.Batch(device, [(s, 5 + k, 0) for k, s in enumerate(scenes)])
        batch.render()
        frames.append([batch.blit(k) for k in range(len(scenes))])
        batch.close()
    # The batch adds samples with float atomics, so images agree to rounding, not bit for bit.
    for a, b in zip(*frames):
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


def test_build_is_deterministic(device):
    s = SCENES["terrain"]()
    a = device_tree(device, s)
    b = device_tree(device, s)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[2]["iterations"] > 0


@pytest.mark.parametrize("name", ["cornell", "terrain"])
def test_tree_quality(device, name):
    s = SCENES[name]()
    tv = prt_scenes.tri_verts(s)
    nodes, tris, _ = device_tree(device, s)
    hn, ht, _ = prt_cuda.bvh8_build_host(tv)
    rays = random_rays(tv, 20000, 12)
    dev_nodes = prt_cuda.bvh8_trace(nodes, tris, rays)[2]
    host_nodes = prt_cuda.bvh8_trace(hn, ht, rays)[2]
    assert dev_nodes <= 1.3 * host_nodes, (dev_nodes, host_nodes)
