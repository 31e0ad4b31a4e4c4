"""The reference-side adapter prt::DeviceCuda (oidn-protoray_b200/host/reference/device_cuda.h),
compiled against the reference's headers with the integration's light accessors
(oracle/_ref/libprt_adapter.so, built by oracle/Makefile), forwards the reference's lights to the
device's environment description exactly: for a sun-sky light, the sun as the distant light and
the sky as the image light that the reference's own SunSkyLight computes
(light/sun_sky_light.cpp:17-193, keyed as Scene::initLights, render/scene.cpp:365-450).

The comparison target is the oracle's direct export of the same products (ref.sunsky, which reads
the reference's light objects). The products the tests and the benchmark hand to the scene
generators (tests/golden/sunsky_*.npz) are checked against the adapter too.
"""
import ctypes as C
import math
import pathlib

import numpy as np
import pytest

import prt_scenes
import ref

ROOT = pathlib.Path(__file__).resolve().parent.parent
ADAPTER = ROOT / "oracle" / "_ref" / "libprt_adapter.so"
GOLDEN = ROOT / "tests" / "golden"

pytestmark = pytest.mark.skipif(not ADAPTER.exists(), reason="oracle/_ref/libprt_adapter.so is not built")

_lib = None


def lib():
    global _lib
    if _lib is None:
        ref._lib()  # libstdc++ and the reference library first, in the global scope
        import prt_cuda

        prt_cuda.load_library()
        _lib = C.CDLL(str(ADAPTER))
        _lib.adapter_last_error.restype = C.c_char_p
        _lib.adapter_env.argtypes = [C.c_char_p, C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_float)]
    return _lib


def props(**kv):
    lines = []
    for k, v in kv.items():
        if isinstance(v, str):
            lines.append(f"{k} s {v}")
        elif isinstance(v, int):
            lines.append(f"{k} i {v}")
        elif np.ndim(v) == 0:
            lines.append(f"{k} f {float(v)!r}")
        else:
            lines.append(f"{k} v3 " + " ".join(repr(float(x)) for x in v))
    return "\n".join(lines).encode()


def adapter_env(spec):
    f = (C.c_float * 10)()
    i = (C.c_int32 * 4)()
    rc = lib().adapter_env(spec, f, i, None)
    if rc != 0:
        return rc, lib().adapter_last_error().decode(), None
    img = None
    if i[0] > 0:
        img = np.zeros((i[1], i[0], 3), np.float32)
        assert lib().adapter_env(spec, f, i, img.ctypes.data_as(C.POINTER(C.c_float))) == 0
    env = {"distant_color": np.array(f[0:3], np.float32), "distant_dir": np.array(f[3:6], np.float32),
           "distant_angle": np.float32(f[6]), "ambient_color": np.array(f[7:10], np.float32),
           "image_size": (i[0], i[1]), "lut": i[2], "flags": i[3]}
    return 0, env, img


def f32_normalize(d):
    d = np.asarray(d, np.float32)
    return d / np.float32(math.sqrt(float(np.dot(d.astype(np.float64), d))))


SUNS = [(30.0, 3.0), (60.0, 5.0), (12.0, 2.0), (75.0, 8.0)]


@pytest.mark.parametrize("elevation,turbidity", SUNS)
def test_sun_sky_forwarded_as_the_reference_computes_it(elevation, turbidity):
    d = prt_scenes.sun_direction(elevation, 45.0)
    rc, env, sky = adapter_env(props(sunSkyLightDir=d, sunSkyLightTurbidity=turbidity, sunSkyLightAlbedo=0.2))
    assert rc == 0, env
    sun, angle, ref_sky = ref.sunsky(d, turbidity, 0.2)
    assert np.array_equal(env["distant_color"], sun)
    assert env["distant_angle"] == np.float32(angle)
    assert np.allclose(env["distant_dir"], f32_normalize(d), rtol=0, atol=2e-7)
    assert sky is not None and np.array_equal(sky, ref_sky)
    assert env["image_size"] == (512, 256) and env["lut"] == 128 and env["flags"] == 0
    assert not env["ambient_color"].any()


def test_registered_products_equal_the_adapters():
    """The products the harness registers with the scene generators are the adapter's."""
    for path in sorted(GOLDEN.glob("sunsky_*.npz")):
        z = np.load(path)
        p = z["params"]
        rc, env, sky = adapter_env(props(sunSkyLightDir=p[0:3], sunSkyLightTurbidity=float(p[3]),
                                         sunSkyLightAlbedo=float(p[4])))
        assert rc == 0, env
        assert np.array_equal(env["distant_color"], z["sun_color"]), path.name
        assert env["distant_angle"] == z["sun_angle"], path.name
        assert np.array_equal(sky, z["sky"]), path.name


def test_sun_sky_scales_and_ambient_order():
    d = prt_scenes.sun_direction(40.0, 10.0)
    _, base, base_sky = adapter_env(props(sunSkyLightDir=d))
    _, env, sky = adapter_env(props(sunSkyLightDir=d, sunSkyLightSunScale=2.0, sunSkyLightSkyScale=0.5,
                                    ambientLight=(0.1, 0.2, 0.3)))
    assert np.allclose(env["distant_color"], 2.0 * base["distant_color"], rtol=1e-6)
    assert np.allclose(sky, 0.5 * base_sky, rtol=1e-6)
    # Scene::initLights lists the ambient light before the sun and the sky.
    assert env["flags"] == 1 and np.allclose(env["ambient_color"], (0.1, 0.2, 0.3))
    # Turbidity and ground albedo default to the reference's 3 and 0.2.
    _, explicit, explicit_sky = adapter_env(props(sunSkyLightDir=d, sunSkyLightTurbidity=3.0, sunSkyLightAlbedo=0.2))
    assert np.array_equal(explicit["distant_color"], base["distant_color"]) and np.array_equal(explicit_sky, base_sky)


def test_distant_and_ambient_lights():
    rc, env, sky = adapter_env(props(distantLight=(3.0, 2.0, 1.0), distantLightDir=(1.0, 2.0, 0.5),
                                     distantLightAngle=0.25, ambientLight=(0.5, 0.5, 0.5)))
    assert rc == 0 and sky is None
    assert np.array_equal(env["distant_color"], np.float32([3, 2, 1]))
    assert np.allclose(env["distant_dir"], f32_normalize((1.0, 2.0, 0.5)), rtol=0, atol=2e-7)
    assert env["distant_angle"] == np.float32(0.25) and env["flags"] == 0
    # DistantLight's defaults: direction (0.3, 1, 0.1), angular diameter 9.35e-3 (light/distant_light.h:24-29).
    _, env, _ = adapter_env(props(distantLight=(1.0, 1.0, 1.0)))
    assert np.allclose(env["distant_dir"], f32_normalize((0.3, 1.0, 0.1)), rtol=0, atol=2e-7)
    assert env["distant_angle"] == np.float32(9.35e-3)


def test_image_light_file(tmp_path):
    rng = np.random.default_rng(3)
    img = rng.uniform(0.0, 2.0, (32, 64, 3)).astype(np.float32)
    path = tmp_path / "env.pfm"
    prt_scenes.write_pfm(path, img)
    rc, env, out = adapter_env(props(imageLight=str(path), imageLightLutSize=16))
    assert rc == 0, env
    assert env["image_size"] == (64, 32) and env["lut"] == 16
    assert np.array_equal(out, img)


@pytest.mark.parametrize("extra", [dict(distantLight=(1.0, 1.0, 1.0)), dict(imageLight="unused.pfm")])
def test_two_lights_of_a_kind_are_rejected(extra):
    rc, msg, _ = adapter_env(props(sunSkyLightDir=(0.0, 1.0, 0.0), **extra))
    assert rc == 1 and "one distant and one image light" in msg, msg
