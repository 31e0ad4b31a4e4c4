"""prt_cuda_render_static: rendering for callers that cannot allocate device memory.

Some hosts own all of their device memory (a pool or a fixed budget that a library must not
grow behind their back), and some cannot take the device-wide synchronisation a cudaMalloc or
cudaFree may cause while their own work is in flight. prt_cuda_render_static serves them: it
renders from a scratch area compiled into the library and writes into an output buffer that the
caller allocated. These tests call it through the C ABI and check it against prt_cuda_render +
prt_cuda_blit, the entry points that allocate their path state on demand.

Tolerance: per-pixel relative difference <= 1e-6. Both paths add each pixel's samples in
sample order, so the images are expected to agree bit for bit; the bound only allows for that
expectation being too strict on some future build.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import prt_cuda
import prt_scenes
import prt_types as T

pytestmark = pytest.mark.gpu

W, H, SPP = 128, 128, 8   # 16,384 pixels: four samples per wave in the 65,536-path scratch area
STATIC_LIMIT = 1 << 16    # pixels


def bind(lib):
    lib.prt_cuda_render_static.argtypes = [C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p]
    lib.prt_cuda_render_static.restype = C.c_int
    return lib.prt_cuda_render_static


def rel_diff(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.max(np.abs(x - ref) / np.maximum(np.abs(ref), 1e-6)))


@pytest.fixture(scope="module")
def ctx():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    dev = prt_cuda.DeviceCuda(0)
    scene = prt_scenes.cornell(seed=0)
    scene.width, scene.height, scene.spp = W, H, SPP
    dev.setup(scene, seed=3)
    yield dev, bind(dev.lib), torch
    dev.close()


def render_static(dev, fn, torch, first_sample, spp):
    out = torch.full((H, W, 3), float("nan"), dtype=torch.float32, device="cuda")
    rc = fn(dev.h, first_sample, spp, C.c_void_p(out.data_ptr()))
    assert rc == T.PRT_OK, dev.lib.prt_cuda_last_error(dev.h)
    return out.cpu().numpy()


def test_static_render_matches_allocating_render_on_two_calls(ctx):
    dev, fn, torch = ctx
    # Allocating path: samples 0..7, then samples 8..15 into a cleared frame.
    dev.clear_frame()
    dev.render(SPP)
    first = dev.blit_frame()
    dev.clear_frame()
    dev.render(SPP)
    second = dev.blit_frame()
    assert np.isfinite(first).all() and first.mean() > 0

    # Two calls in a row of the static entry point, the second one reusing the scratch area.
    a = render_static(dev, fn, torch, 0, SPP)
    b = render_static(dev, fn, torch, SPP, SPP)
    assert np.isfinite(a).all() and np.isfinite(b).all()
    assert rel_diff(a, first) <= 1e-6
    assert rel_diff(b, second) <= 1e-6

    # The sums start from zero on every call: repeating call one gives call one's image.
    again = render_static(dev, fn, torch, 0, SPP)
    assert rel_diff(again, a) <= 1e-6

    # The context's own frame is untouched by the static calls.
    assert np.array_equal(dev.blit_frame(), second)


def test_static_render_allocates_nothing_on_a_fresh_context():
    """A context that has never rendered through the allocating path: after one warm-up call
    (which loads the library's kernels and looks up the scratch area's address), further calls
    leave the device's free memory exactly as it was, and give the allocating path's images."""
    torch = pytest.importorskip("torch")
    dev = prt_cuda.DeviceCuda(0)
    try:
        scene = prt_scenes.cornell(seed=0)
        scene.width, scene.height, scene.spp = W, H, SPP
        dev.setup(scene, seed=5)
        fn = bind(dev.lib)
        outs = [torch.full((H, W, 3), float("nan"), dtype=torch.float32, device="cuda") for _ in range(3)]
        torch.cuda.synchronize()

        def call(k, first):
            rc = fn(dev.h, first, SPP, C.c_void_p(outs[k].data_ptr()))
            assert rc == T.PRT_OK, dev.lib.prt_cuda_last_error(dev.h)

        call(0, 0)  # warm-up
        free_before, _ = torch.cuda.mem_get_info()
        call(1, 0)
        call(2, SPP)
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before, (free_before, free_after)

        warm, a, b = (o.cpu().numpy() for o in outs)
        assert np.isfinite(a).all() and a.mean() > 0
        assert rel_diff(warm, a) <= 1e-6
        # The allocating path on the same context afterwards: samples 0..7, then 8..15.
        dev.clear_frame()
        dev.render(SPP)
        assert rel_diff(a, dev.blit_frame()) <= 1e-6
        dev.clear_frame()
        dev.render(SPP)
        assert rel_diff(b, dev.blit_frame()) <= 1e-6
    finally:
        dev.close()


def test_static_render_rejects_another_devices_memory():
    """The output must live on the context's own device."""
    torch = pytest.importorskip("torch")
    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second GPU to hold the output")
    dev = prt_cuda.DeviceCuda(0)
    try:
        scene = prt_scenes.cornell(seed=0)
        scene.width, scene.height, scene.spp = W, H, SPP
        dev.setup(scene, seed=0)
        fn = bind(dev.lib)
        other = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda:1")
        rc = fn(dev.h, 0, 1, C.c_void_p(other.data_ptr()))
        assert rc == T.PRT_ERR_INVALID_ARG
        assert b"device 1" in dev.lib.prt_cuda_last_error(dev.h)
    finally:
        dev.close()


def test_static_render_rejects_frames_beyond_the_scratch_limit(ctx):
    dev, fn, torch = ctx
    big = prt_scenes.cornell(seed=0)
    big.width, big.height = 512, 256   # 131,072 pixels
    assert big.width * big.height > STATIC_LIMIT
    dev.init_frame(big.width, big.height)
    dev.init_camera(big.camera)
    out = torch.zeros((big.height, big.width, 3), dtype=torch.float32, device="cuda")
    rc = fn(dev.h, 0, 1, C.c_void_p(out.data_ptr()))
    assert rc == T.PRT_ERR_INVALID_ARG
    assert b"65536" in dev.lib.prt_cuda_last_error(dev.h)
    # Host memory is not accepted as the output (copying through the device would need an allocation).
    dev.init_frame(W, H)
    dev.init_camera(big.camera)
    host = np.zeros((H, W, 3), np.float32)
    rc = fn(dev.h, 0, 1, host.ctypes.data_as(C.c_void_p))
    assert rc == T.PRT_ERR_INVALID_ARG
