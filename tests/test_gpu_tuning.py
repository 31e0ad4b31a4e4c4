"""Launch tuning (prt_cuda_set_tuning / prt_cuda_autotune) changes speed, never the image.

Every tuning axis -- path-pool size (samples per wave), traversal and shading blocks per SM,
staging of the top BVH levels in shared memory, grouping each bounce's extended rays by
direction octant (which reorders the traversal queue), the traversal stack's size -- leaves each path's samples and shading
unchanged and the accumulation adds each pixel's samples in sample order, so images are
bit-identical across tunings.
"""
import numpy as np
import pytest

import prt_cuda
import prt_scenes
import prt_types as T

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    d = prt_cuda.DeviceCuda(0)
    s = prt_scenes.terrain(seed=3, grid=128, n_spheres=40, width=256, height=128, spp=8)
    d.setup(s, seed=5)
    d.test_scene = s
    yield d
    d.close()


def render(dev, spp):
    dev.init_sampler(5)
    dev.clear_frame()
    st = dev.render(spp)
    return dev.blit_frame(), st["rays"]


@pytest.mark.parametrize("tuning", [
    dict(top_stage=1),
    dict(top_stage=2, trace_blocks=4, shade_blocks=2),
    dict(wave_paths=256 * 128 * 3),          # 3 samples per wave: waves of 3, 3, 2 samples
    dict(trace_blocks=12, shade_blocks=16, top_stage=1),
    dict(ray_bins=2),                        # queue in shading order instead of octant groups
    dict(ray_bins=1, top_stage=1, wave_paths=256 * 128 * 3),
    dict(trace_stack=48),                    # the 48-entry local-memory stack instead of shared memory
    dict(trace_stack=48, top_stage=1),
    dict(trace_stack=24),                    # the 24-entry local-memory stack
])
def test_tuning_keeps_the_image(dev, tuning):
    default = dev.get_tuning()
    ref, rays = render(dev, 8)
    try:
        dev.set_tuning(**tuning)
        img, rays2 = render(dev, 8)
    finally:
        dev.set_tuning(**default)
    assert rays2 == rays
    assert np.array_equal(img, ref)


def test_autotune_returns_a_valid_tuning(dev):
    default = dev.get_tuning()
    ref, _ = render(dev, 4)
    try:
        chosen, mrays = dev.autotune(2)
        assert mrays > 0
        assert chosen["top_stage"] in (1, 2) and 1 <= chosen["trace_blocks"] <= 32
        assert chosen["ray_bins"] in (1, 2) and chosen["trace_stack"] in (12, 24, 48)
        assert dev.get_tuning() == chosen
        img, _ = render(dev, 4)
        assert np.array_equal(img, ref)
    finally:
        dev.set_tuning(**default)


def test_tuning_rejects_out_of_range(dev):
    with pytest.raises(ValueError):
        dev.set_tuning(trace_blocks=64)
    with pytest.raises(ValueError):
        dev.set_tuning(top_stage=3)
    with pytest.raises(ValueError):
        dev.set_tuning(ray_bins=3)
    with pytest.raises(ValueError):
        dev.set_tuning(trace_stack=32)


def test_default_stack_is_the_shared_one(dev):
    """The terrain's tree has at most 12 wide levels, so the default tuning runs the traversal
    kernels with their 12-entry stack in shared memory."""
    assert dev.get_tuning()["trace_stack"] == 12
    assert dev.scene_stats()["depth"] <= 12


def chain_scene(n=150, ratio=1.7):
    """Small triangles at x = ratio^k along the x axis: each binned-SAH split peels off the farthest
    few, so the tree is a chain -- 19 wide levels for the defaults, deeper than the 12-entry
    shared-memory stack and within the 24-entry one. The camera looks along the chain, so its rays
    walk the whole depth."""
    s = prt_scenes.Scene()
    m = s.add_material(T.material(base_color=(0.7, 0.7, 0.7), specular_weight=0.0))
    x = ratio ** np.arange(n, dtype=np.float64)
    v = np.zeros((n, 3, 3), np.float32)
    v[:, :, 0] = x[:, None]
    v[:, 1, 1] = 0.5
    v[:, 2, 2] = 0.5
    s.add_mesh(v.reshape(-1, 3), np.arange(3 * n, dtype=np.int32).reshape(-1, 3), m)
    s.env.distant_color[:] = (0.0, 0.0, 0.0)
    s.env.ambient_color[:] = (1.0, 1.0, 1.0)
    s.camera = prt_scenes.look_at((-3.0, 2.0, 3.0), (4.0, 0.2, 0.2), fov_deg=50.0)
    s.width, s.height, s.spp, s.max_depth, s.rr_depth = 64, 64, 4, 3, 8
    return s


def test_deep_tree_takes_a_stack_that_fits():
    """A tree deeper than 12 wide levels: the default (12, shared memory) falls back to the
    24-entry stack, and every stack setting renders the same image with the same rays."""
    d = prt_cuda.DeviceCuda(0)
    try:
        d.setup(chain_scene(), seed=1)
        depth = d.scene_stats()["depth"]
        assert 12 < depth <= 24, depth
        out = {}
        for stack in (12, 24, 48):
            d.set_tuning(trace_stack=stack)
            d.init_sampler(1)
            d.clear_frame()
            st = d.render(4)
            out[stack] = (d.blit_frame(), st["rays"])
        for stack in (12, 24):
            assert np.array_equal(out[stack][0], out[48][0]), stack
            assert out[stack][1] == out[48][1], stack
        assert np.isfinite(out[48][0]).all()
    finally:
        d.close()
