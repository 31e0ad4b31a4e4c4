"""Scene files on the device (prt_cuda_scene_load, Device::initScene(path) + initLights).

A scene written as an rkscene file and loaded from it renders bit-identically to the same scene
uploaded from its in-memory description (same meshes in the same order, same materials and
textures), with either BVH builder; the loader itself is pinned against files written by the
reference's rkscene::save in test_cpu_rkscene.py.
"""
import numpy as np
import pytest

import prt_scenes
import prt_types as T

pytestmark = pytest.mark.gpu

SCENES = {
    "cornell": lambda: prt_scenes.cornell(seed=0, width=64, height=64, spp=4),
    "textured": lambda: prt_scenes.cornell_inverse(seed=0, width=64, height=64, spp=4, tex_size=64)[0],
    "lobes": lambda: prt_scenes.cornell_lobes(seed=0, width=64, height=64, spp=4),
    "terrain": lambda: prt_scenes.terrain(seed=3, grid=128, n_spheres=20, width=96, height=64, spp=4),
}


def render_loaded(dev, scene, path, builder, seed=7):
    desc = scene.desc()
    dev.load_scene(path, env=desc.env, bvh_build=builder)
    dev.init_frame(scene.width, scene.height)
    dev.init_camera(scene.camera)
    dev.init_renderer(scene.max_depth, scene.rr_depth)
    dev.init_sampler(seed)
    st = dev.render(scene.spp)
    return dev.blit_frame(), st["rays"]


@pytest.mark.parametrize("builder", [T.PRT_BVH_HOST, T.PRT_BVH_DEVICE], ids=["host_bvh", "device_bvh"])
@pytest.mark.parametrize("name", list(SCENES))
def test_file_renders_like_the_description(device, tmp_path, name, builder):
    s = SCENES[name]()
    path = prt_scenes.write_rkscene(s, tmp_path / f"{name}.rkscene")
    img_file, rays_file = render_loaded(device, s, path, builder)
    s.bvh_build = builder
    device.setup(s, seed=7)
    st = device.render(s.spp)
    img = device.blit_frame()
    assert rays_file == st["rays"]
    assert np.array_equal(img_file, img)
    assert device.scene_stats()["builder"] == builder


def test_load_errors_leave_a_usable_device(device, tmp_path):
    bad = tmp_path / "bad.rkscene"
    bad.write_text("{")
    with pytest.raises(ValueError):
        device.load_scene(bad)
    s = SCENES["cornell"]()
    device.setup(s, seed=0)
    assert device.render(1)["rays"] > 0


def test_mesh_file_tracks_the_reference(device, golden, tmp_path):
    """The textured room written as a .mesh file, loaded by the device and (for the fixture) by
    the reference's Scene::loadMesh: the same-seed image follows the reference's far closer than
    two seeds do, with the same ray count within 1% (material 0 renders as a miss in both)."""
    z = golden("mesh_img.npz")
    s = prt_scenes.cornell_inverse(seed=0, width=128, height=128, spp=16, tex_size=64)[0]
    path = prt_scenes.write_mesh(s, tmp_path / "room.mesh")
    img, rays = render_loaded(device, s, path, T.PRT_BVH_HOST, seed=0)
    rel = lambda a, b: float(np.mean((a.astype(np.float64) - b) ** 2 / (b.astype(np.float64) ** 2 + 1e-2)))
    same = rel(img, z["spp16_seed0"])
    other = rel(z["spp16_seed1"], z["spp16_seed0"])
    assert same < 0.2 * other, (same, other)
    assert abs(rays / float(z["spp16_seed0_rays"]) - 1.0) < 0.01
