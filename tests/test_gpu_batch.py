"""Batch rendering (prt_cuda_batch_*) against the frame form of the same GPU code.

A batch renders many frames in one persistent wavefront with path regeneration. Every path
of a frame is the path the frame form traces for it (same Sobol samples, same shading), so:
  * the ray counts match the per-frame renders exactly;
  * finished paths store their results per pixel-sample and each pixel's samples are summed in
    sample order, as the frame form sums them: a batch renders identically every time, its
    albedo1 and normal1 images equal the per-frame renders bit for bit, and its beauty image is
    within 8 ulps of theirs per channel (measured: at most 3, in ~15% of the pixels; with equal
    ray counts and bit-identical AOVs, this is FP32 rounding inside the two instantiations of the
    shading kernels rather than different paths).
"""
import numpy as np
import pytest

import prt_cuda
import prt_scenes
import prt_types as T

pytestmark = pytest.mark.gpu


def max_ulps(a, b):
    """Largest distance in units in the last place between two arrays of non-negative floats."""
    ia = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    ib = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    return int(np.abs(ia - ib).max(initial=0))


def small_batch(count, seed):
    return prt_scenes.batch_frames(count=count, seed=seed, tri_range=(1e3, 3e4), sizes=(64, 96, 128),
                                   spps=(2, 4, 8), depth_range=(3, 6))


@pytest.fixture(scope="module")
def dev():
    d = prt_cuda.DeviceCuda(0)
    yield d
    d.close()


def plain_render(dev, scene, seed, aov):
    dev.init_scene(scene)
    dev.init_frame(scene.width, scene.height, aov)
    dev.init_camera(scene.camera)
    dev.init_renderer(scene.max_depth, scene.rr_depth)
    dev.init_sampler(seed)
    dev.clear_frame()
    st = dev.render(scene.spp)
    out = [dev.blit_frame(T.PRT_BLIT_HDR)]
    if aov:
        out += [dev.blit_frame(T.PRT_BLIT_ALBEDO1), dev.blit_frame(T.PRT_BLIT_NORMAL1)]
    return out, st


def test_batch_matches_per_frame_renders(dev):
    frames = small_batch(6, seed=5)
    batch = prt_cuda.Batch(dev, frames)
    st = batch.render()
    rays = 0
    for k, (scene, seed, aov) in enumerate(frames):
        ref, rst = plain_render(dev, scene, seed, aov)
        rays += rst["rays"]
        got = [batch.blit(k, T.PRT_BLIT_HDR), batch.blit(k, T.PRT_BLIT_ALBEDO1), batch.blit(k, T.PRT_BLIT_NORMAL1)]
        assert np.isfinite(got[0]).all() and got[0].mean() > 0
        assert max_ulps(got[0], ref[0]) <= 8, (k, max_ulps(got[0], ref[0]))
        for g, r in zip(got[1:], ref[1:]):
            assert np.array_equal(g.view(np.uint32), r.view(np.uint32)), k
    assert st["rays"] == rays
    batch.close()


def test_batch_renders_twice_identically(dev):
    frames = small_batch(4, seed=9)
    batch = prt_cuda.Batch(dev, frames)
    st1 = batch.render()
    first = [batch.blit(k) for k in range(len(frames))]
    st2 = batch.render()
    assert st1["rays"] == st2["rays"]
    for k in range(len(frames)):
        assert np.array_equal(batch.blit(k).view(np.uint32), first[k].view(np.uint32)), k
    batch.close()


def test_batch_small_pool_regenerates_paths(dev):
    """A path pool far smaller than the work forces many regeneration rounds."""
    frames = small_batch(3, seed=2)
    dev.set_tuning(wave_paths=4096)
    try:
        batch = prt_cuda.Batch(dev, frames)
        st = batch.render()
    finally:
        dev.set_tuning(wave_paths=32 << 20)
    rays = 0
    for k, (scene, seed, aov) in enumerate(frames):
        ref, rst = plain_render(dev, scene, seed, aov)
        rays += rst["rays"]
        assert max_ulps(batch.blit(k), ref[0]) <= 8, k
    assert st["rays"] == rays
    batch.close()


def test_batch_destroy_returns_its_memory(dev):
    """A batch owns every buffer its items' uploads made -- scene, environment lights, path pool --
    so creating, rendering and destroying one leaves the device's free memory where it was."""
    import torch

    frames = small_batch(16, 5)
    b = prt_cuda.Batch(dev, frames)
    b.render()
    b.close()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        b = prt_cuda.Batch(dev, frames)
        b.render()
        b.close()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    assert free0 - free1 < (4 << 20), free0 - free1


def test_batch_rejects_bad_items(dev):
    scene = prt_scenes.cornell(seed=0)
    scene.width, scene.height = 100, 64   # width not a multiple of 32
    with pytest.raises(prt_cuda.LogicError):
        prt_cuda.Batch(dev, [(scene, 0, 0)])


def test_batch_with_a_deep_tree_matches_per_frame_renders(dev):
    """The batch takes the stack its deepest tree fits (a 19-level chain beside a terrain: the
    24-entry stack for both), and each frame still matches its per-frame render."""
    from test_gpu_tuning import chain_scene

    terrain = prt_scenes.terrain(seed=4, grid=64, n_spheres=8, width=64, height=64, spp=4, extent=10.0,
                                 relief=2.0, max_depth=4)
    frames = [(chain_scene(), 1, 0), (terrain, 2, 0)]
    batch = prt_cuda.Batch(dev, frames)
    st = batch.render()
    rays = 0
    for k, (scene, seed, aov) in enumerate(frames):
        ref, rst = plain_render(dev, scene, seed, aov)
        rays += rst["rays"]
        assert max_ulps(batch.blit(k), ref[0]) <= 8, k
    assert st["rays"] == rays
    batch.close()
