"""The device through the reference's own interface: prt::DeviceCuda
(oidn-protoray_b200/host/reference/device_cuda.h, compiled against the reference's headers into
oracle/_ref/libprt_adapter.so) driven as the reference's application drives a prt::Device --
initScene(path, props) on an rkscene file written by the reference's rkscene::save, the sun-sky
light given by its Props keys (sunSkyLightDir, sunSkyLightTurbidity, sunSkyLightAlbedo),
initFrame, initCamera, initRenderer, initSampler, one render() per sample, blitFrame.

The image is compared with the reference's own render of the same file and light (same seed):
relMSE < 0.5 x the reference's seed-to-seed relMSE, ray count within 2%.
"""
import ctypes as C

import numpy as np
import pytest

import prt_scenes
import prt_types as T
import ref
from conftest import rel_mse
from test_cpu_sunsky_adapter import ADAPTER, lib

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ADAPTER.exists(), reason="oracle/_ref/libprt_adapter.so is not built")]


def light_props(params):
    d = params[0:3]
    return (f"sunSkyLightDir v3 {float(d[0])!r} {float(d[1])!r} {float(d[2])!r}\n"
            f"sunSkyLightTurbidity f {float(params[3])!r}\nsunSkyLightAlbedo f {float(params[4])!r}").encode()


def adapter_render(path, scene, props, seed, spp, aov_mask=0):
    L = lib()
    P = C.POINTER(C.c_float)
    L.adapter_render.argtypes = [C.c_char_p, C.c_char_p, P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                 C.c_uint32, C.c_int, P, P, P, C.POINTER(C.c_double)]
    c = scene.camera
    cam = np.array(list(c.position) + list(c.basis_u) + list(c.basis_v) + list(c.basis_n) + [c.fov, c.near_clip],
                   np.float32)
    r = (C.c_int * 2)(scene.max_depth, scene.rr_depth)
    hdr = np.zeros((scene.height, scene.width, 3), np.float32)
    alb = np.zeros_like(hdr)
    nrm = np.zeros_like(hdr)
    st = (C.c_double * 4)()
    rc = L.adapter_render(str(path).encode(), props, T.fptr(cam), scene.width, scene.height, aov_mask, r, seed, spp,
                          T.fptr(hdr), T.fptr(alb), T.fptr(nrm), st)
    assert rc == 0, L.adapter_last_error().decode()
    return hdr, alb, nrm, st


def test_second_sun_through_the_reference_device_interface(golden, tmp_path):
    z = golden("terrain_e60_img.npz")
    s = prt_scenes.terrain(seed=1, grid=96, n_spheres=24, width=128, height=64, spp=16, extent=12.0, relief=3.0,
                           sun_elevation_deg=60.0, turbidity=5.0)
    path = ref.write_rkscene(s, tmp_path)
    img, _, _, st = adapter_render(path, s, light_props(s.sunsky), seed=0, spp=16)
    assert np.isfinite(img).all()
    same = rel_mse(img, z["spp16_seed0"])
    other = rel_mse(z["spp16_seed1"], z["spp16_seed0"])
    assert same < 0.5 * other, (same, other)
    assert abs(st[0] / float(z["spp16_seed0_rays"]) - 1.0) < 0.02


def test_first_hit_aovs_through_the_reference_device_interface(golden, tmp_path):
    """The small terrain under the workload's sun, with albedo1 and normal1 requested through
    initFrame's aovAlbedo1 / aovNormal1 keys and read through blitFrame(FrameAovs&)."""
    z = golden("aov_img.npz")
    s = prt_scenes.terrain(seed=1, grid=96, n_spheres=24, width=128, height=64, spp=16, extent=12.0, relief=3.0)
    path = ref.write_rkscene(s, tmp_path)
    img, alb, nrm, _ = adapter_render(path, s, light_props(s.sunsky), seed=0, spp=16,
                                      aov_mask=T.PRT_AOV_ALBEDO1 | T.PRT_AOV_NORMAL1)
    assert rel_mse(img, z["terrain_seed0_hdr"]) < 0.5 * rel_mse(z["terrain_seed1_hdr"], z["terrain_seed0_hdr"])
    for got, key in ((alb, "albedo1"), (nrm, "normal1")):
        diff = np.abs(got.astype(np.float64) - z[f"terrain_seed0_{key}"])
        assert diff.mean() < 1e-4 and np.mean(diff > 1e-3) < 0.002, (key, diff.mean())


def test_adapter_runs_on_the_reference_tables():
    """prt::DeviceCuda uploads the energy-compensation tables the reference computes on the host
    (precomputeAlbedoTables, as DeviceCpu's constructor does): its context holds them bit for
    bit. With hostTables = false it keeps the tables the context built on the GPU, which differ
    from them in the last digits."""
    L = lib()
    P = C.POINTER(C.c_float)
    L.adapter_tables.argtypes = [C.c_int, P, C.c_int64, C.POINTER(C.c_int64)]
    want = ref.albedo_tables()
    got = {}
    for host in (1, 0):
        out = np.zeros(want.size, np.float32)
        n = C.c_int64(0)
        rc = L.adapter_tables(host, T.fptr(out), out.size, C.byref(n))
        assert rc == 0, L.adapter_last_error().decode()
        assert n.value == want.size
        got[host] = out
    assert np.array_equal(got[1].view(np.uint32), want.view(np.uint32))
    assert not np.array_equal(got[0], want)
    assert np.abs(got[0] - want).max() < 2e-3
