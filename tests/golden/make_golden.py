"""Generates the golden fixtures in tests/golden/ from the oracle.

The reference has no tests and no golden data (its repository ships none), so the fixtures
are produced by the reference's own code compiled here (oracle/_ref/libprt_ref.so, built
by `make -C oracle` from the reference sources): its SIMD Sobol-Burley sampler, its
PinholeCamera ray generation, its pathStream renderer, with the oracle BVH in place of
Embree for the hit queries. Run from the repository root:

    python tests/golden/make_golden.py

Fixtures (small, seeded, committed):
  sobol.npz        Sobol-Burley 1D/2D/3D draws: (seed, sampleIndex, pixelId, dimSet) grids
  cornell_rays.npz primary rays of the small scene at 64x64 (sample indices 0 and 1) with their
                   closest hits, plus random interior rays with closest hits and occlusion
  cornell_img.npz  small-scene renders at 128x128: 16 spp with seeds 0 and 1, 1024 spp with
                   seeds 0 and 1
  terrain_img.npz  small terrain renders (96^2 heightfield, 24 spheres of all four material
                   kinds, sun-sky) at 128x64: 16 spp and 256 spp, seeds 0 and 1
  lobes_img.npz    the small scene with Oren-Nayar, sheen and layered spheres, 16 spp, seeds 0, 1
  mesh_img.npz     the textured room written as a .mesh file and loaded by the reference's
                   Scene::loadMesh (material 0 renders as a miss there), 16 spp, seeds 0, 1
  translucent_img.npz  the small scene with thin glass, opacity, subsurface, transparent and backlit
                   surfaces (shadow rays through transparent surfaces), 16 spp, seeds 0, 1
  siblings_img.npz primaryStream, aoStream, diffuseStream, diffuse2Stream and their ...Fast variants
                   rendered on the small scene
  film.npz         sample variance, tone-mapped LDR images and frame errors of the small scene
  bsdf.npz         the reference's Standard-material BSDF (eval, sample) on 512 seeded tuples
                   for each case of tests/bsdf_cases.py
  sh_img.npz       the SH AOV (four coefficient images) and the irradiance mode's image of the
                   small scene and the small terrain, 16 spp, seeds 0 and 1
  aov_img.npz      first-hit albedo1 and normal1 AOVs with the HDR image: the small scene and the
                   small terrain, 16 spp, seeds 0 and 1
  sunsky_t3_e30.npz, sunsky_t5_e60.npz  the reference's sun-sky products (sun radiance and angle,
                   512x256 sky) for the terrain scene's sun (elevation 30 deg, turbidity 3, ground
                   albedo 0.2) and for a second sun (elevation 60 deg, turbidity 5)
  terrain_e60_img.npz the small terrain under the second sun, 16 spp, seeds 0 and 1
"""
import pathlib
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oidn-protoray_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
import prt_scenes  # noqa: E402
import prt_types as T  # noqa: E402
import ref  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent


def make_sobol():
    rng = np.random.default_rng(12345)
    out = {}
    n = 1024
    si = rng.integers(0, 4096, n).astype(np.uint32)
    x = rng.integers(0, 4096, n)
    y = rng.integers(0, 4096, n)
    pid = (x | (y << 16)).astype(np.uint32)
    ds = rng.integers(0, 80, n).astype(np.uint32)
    out.update(sample_index=si, pixel_id=pid, dim_set=ds)
    for seed in (0, 1, 0xDEADBEEF):
        for dims in (1, 2, 3):
            simd, scalar = ref.sobol(seed, si, pid, ds, dims)
            out[f"s{seed}_d{dims}_simd"] = simd
            out[f"s{seed}_d{dims}_scalar"] = scalar
    np.savez_compressed(OUT / "sobol.npz", **out)


def small_scene(width, height, spp):
    s = prt_scenes.cornell(seed=0)
    s.width, s.height, s.spp = width, height, spp
    return s


def make_rays():
    s = small_scene(64, 64, 1)
    dev = ref.RefDevice(s, seed=0)
    out = {}
    for si in range(2):
        rays, g, p, t = dev.query_primary(si)
        out[f"primary{si}_rays"] = rays
        out[f"primary{si}_geom"] = g
        out[f"primary{si}_prim"] = p
        out[f"primary{si}_t"] = t
    rng = np.random.default_rng(7)
    n = 4096
    org = np.stack([rng.uniform(-0.95, 0.95, n), rng.uniform(0.05, 1.95, n), rng.uniform(-0.95, 0.95, n)], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    far = np.where(rng.uniform(size=n) < 0.5, 3.4028234663852886e38, rng.uniform(0.05, 2.0, n))
    rays = np.concatenate([org, np.full((n, 1), 1e-4), d, far[:, None]], 1).astype(np.float32)
    g, p, t, u, v = dev.trace(rays)
    occ = dev.occluded(rays)
    out.update(random_rays=rays, random_geom=g, random_prim=p, random_t=t, random_u=u, random_v=v, random_occ=occ)
    np.savez_compressed(OUT / "cornell_rays.npz", **out)
    dev.close()


def make_images():
    out = {}
    for spp in (16, 1024):
        for seed in (0, 1):
            s = small_scene(128, 128, spp)
            dev = ref.RefDevice(s, seed=seed)
            t0 = time.time()
            st = dev.render(spp)
            out[f"spp{spp}_seed{seed}"] = dev.blit()
            out[f"spp{spp}_seed{seed}_rays"] = np.float64(st["rays"])
            print(f"spp {spp} seed {seed}: {time.time() - t0:.1f} s, {st['rays'] / 1e6 / st['seconds']:.1f} Mrays/s")
            dev.close()
    np.savez_compressed(OUT / "cornell_img.npz", **out)


def make_lobe_images():
    """The small scene with Oren-Nayar, sheen and layered spheres at 16 spp, seeds 0 and 1."""
    out = {}
    for seed in (0, 1):
        s = prt_scenes.cornell_lobes(seed=0)
        dev = ref.RefDevice(s, seed=seed)
        st = dev.render(16)
        out[f"spp16_seed{seed}"] = dev.blit()
        out[f"spp16_seed{seed}_rays"] = np.float64(st["rays"])
        dev.close()
    np.savez_compressed(OUT / "lobes_img.npz", **out)


def make_translucent_images():
    """The small scene with thin glass, opacity, subsurface, transparent and backlit surfaces at
    16 spp, seeds 0 and 1 (shadow rays through the reference's transparent-shadow filter)."""
    out = {}
    for seed in (0, 1):
        s = prt_scenes.cornell_translucent(seed=0)
        dev = ref.RefDevice(s, seed=seed)
        st = dev.render(16)
        out[f"spp16_seed{seed}"] = dev.blit()
        out[f"spp16_seed{seed}_rays"] = np.float64(st["rays"])
        dev.close()
    np.savez_compressed(OUT / "translucent_img.npz", **out)


def mesh_scene():
    return prt_scenes.cornell_inverse(seed=0, width=128, height=128, spp=16, tex_size=64)[0]


def make_mesh_images():
    """The textured room written as a .mesh file (prt_scenes.write_mesh) and loaded by the
    reference's own Scene::loadMesh, 16 spp, seeds 0 and 1."""
    import tempfile

    out = {}
    with tempfile.TemporaryDirectory() as d:
        s = mesh_scene()
        path = prt_scenes.write_mesh(s, pathlib.Path(d) / "room.mesh")
        for seed in (0, 1):
            dev = ref.RefDevice(s, seed=seed, scene_path=path)
            st = dev.render(16)
            out[f"spp16_seed{seed}"] = dev.blit()
            out[f"spp16_seed{seed}_rays"] = np.float64(st["rays"])
            dev.close()
    np.savez_compressed(OUT / "mesh_img.npz", **out)


def sibling_scene(kind):
    s = prt_scenes.cornell(seed=0, width=64, height=64, spp=4)
    s.renderer_type = kind
    s.ao_samples = 8
    return s


def make_sibling_images():
    """primaryStream, aoStream (8 rays), diffuseStream, diffuse2Stream and their ...Fast
    variants on the small scene, 64x64, 4 spp, seed 0."""
    out = {}
    for kind in (1, 2, 3, 4, 5, 6, 7, 8):
        dev = ref.RefDevice(sibling_scene(kind), seed=0)
        st = dev.render(4)
        out[f"type{kind}"] = dev.blit()
        out[f"type{kind}_rays"] = np.float64(st["rays"])
        dev.close()
    np.savez_compressed(OUT / "siblings_img.npz", **out)


TONES = [(0, 1.0, 0.0), (1, 1.5, 0.0), (2, 1.0, 0.3), (3, 1.2, 0.0), (4, 0.8, 0.0), (5, 2.0, 0.0)]


def make_film():
    """Film post-step of the small scene (64x64, 5 one-sample renders, variance on): the HDR
    image and its sample variance, and per tone mapper the 8-bit and float LDR images and the
    frame error against the checkpoint."""
    s = prt_scenes.cornell(seed=0, width=64, height=64, spp=1)
    dev = ref.RefDevice(s, seed=0, aov_mask=T.PRT_AOV_HDR_VAR)
    for _ in range(5):
        dev.render(1)
    out = {"hdr": dev.blit(T.PRT_BLIT_HDR), "var": dev.blit(T.PRT_BLIT_HDR_VAR)}
    for kind, exposure, burn in TONES:
        dev.tone_mapper(kind, exposure, burn)
        out[f"ldr{kind}"] = dev.blit(T.PRT_BLIT_LDR)
        out[f"ldrrgb{kind}"] = dev.blit(T.PRT_BLIT_LDR_RGB)
        out[f"error{kind}"] = np.float64(dev.frame_error())
    dev.close()
    np.savez_compressed(OUT / "film.npz", **out)


def make_bsdf():
    sys.path.insert(0, str(ROOT / "tests"))
    import bsdf_cases

    tup = bsdf_cases.tuples(512, 1)
    out = {name: ref.bsdf_query(m, tup, med) for name, m, med in bsdf_cases.cases()}
    np.savez_compressed(OUT / "bsdf.npz", **out)


def small_terrain(spp):
    return prt_scenes.terrain(seed=1, grid=96, n_spheres=24, width=128, height=64, spp=spp, extent=12.0, relief=3.0)


def make_terrain_images():
    out = {}
    for spp in (16, 256):
        for seed in (0, 1):
            dev = ref.RefDevice(small_terrain(spp), seed=seed)
            st = dev.render(spp)
            out[f"spp{spp}_seed{seed}"] = dev.blit()
            out[f"spp{spp}_seed{seed}_rays"] = np.float64(st["rays"])
            dev.close()
    np.savez_compressed(OUT / "terrain_img.npz", **out)


def make_aovs():
    """First-hit AOVs (albedo1, normal1) as DeviceCpu::blitFrame writes them, with the HDR image,
    for the small scene (128x128) and the small terrain (128x64, sun-sky), 16 spp, seeds 0 and 1."""
    out = {}
    mask = T.PRT_AOV_ALBEDO1 | T.PRT_AOV_NORMAL1
    for name, scene in (("cornell", small_scene(128, 128, 16)), ("terrain", small_terrain(16))):
        for seed in (0, 1):
            dev = ref.RefDevice(scene, seed=seed, aov_mask=mask)
            st = dev.render(16)
            out[f"{name}_seed{seed}_hdr"] = dev.blit(T.PRT_BLIT_HDR)
            out[f"{name}_seed{seed}_albedo1"] = dev.blit(T.PRT_BLIT_ALBEDO1)
            out[f"{name}_seed{seed}_normal1"] = dev.blit(T.PRT_BLIT_NORMAL1)
            out[f"{name}_seed{seed}_rays"] = np.float64(st["rays"])
            dev.close()
    np.savez_compressed(OUT / "aov_img.npz", **out)


# (sun elevation in degrees, turbidity) of the sun-sky fixtures: the terrain workload's, and a
# second sun for the boundary tests.
SUNSKY_SETS = [(30.0, 3.0), (60.0, 5.0)]


def make_sh_images():
    """The SH AOV (aovSh: four coefficient images) with the HDR image, and the irradiance mode's
    HDR image, of the small scene (128x128) and the small terrain (128x64, sun-sky), 16 spp,
    seeds 0 and 1."""
    out = {}
    for name, make in (("cornell", lambda: small_scene(128, 128, 16)), ("terrain", lambda: small_terrain(16))):
        for seed in (0, 1):
            dev = ref.RefDevice(make(), seed=seed, aov_mask=T.PRT_AOV_SH)
            st = dev.render(16)
            out[f"{name}_seed{seed}_hdr"] = dev.blit(T.PRT_BLIT_HDR)
            for k in range(4):
                out[f"{name}_seed{seed}_sh{k}"] = dev.blit(T.PRT_BLIT_SH0 + k)
            out[f"{name}_seed{seed}_rays"] = np.float64(st["rays"])
            dev.close()
            s = make()
            s.renderer_flags = T.PRT_RENDERER_IRRADIANCE
            dev = ref.RefDevice(s, seed=seed)
            st = dev.render(16)
            out[f"{name}_seed{seed}_irradiance"] = dev.blit(T.PRT_BLIT_HDR)
            out[f"{name}_seed{seed}_irradiance_rays"] = np.float64(st["rays"])
            dev.close()
    np.savez_compressed(OUT / "sh_img.npz", **out)


def make_sunsky():
    for elevation, turbidity in SUNSKY_SETS:
        params = prt_scenes.sunsky_params(elevation, turbidity=turbidity)
        sun, angle, sky = ref.sunsky(params[0:3], float(params[3]), float(params[4]))
        np.savez_compressed(OUT / f"sunsky_t{turbidity:g}_e{elevation:g}.npz", params=params, sun_color=sun,
                            sun_angle=np.float32(angle), sky=sky, direction=params[0:3])


def make_terrain_e60_images():
    """The small terrain under the second sun (elevation 60 degrees, turbidity 5), 16 spp, seeds 0
    and 1: the reference builds its SunSkyLight from the parameters itself."""
    out = {}
    for seed in (0, 1):
        s = prt_scenes.terrain(seed=1, grid=96, n_spheres=24, width=128, height=64, spp=16, extent=12.0, relief=3.0,
                               sun_elevation_deg=60.0, turbidity=5.0)
        dev = ref.RefDevice(s, seed=seed)
        st = dev.render(16)
        out[f"spp16_seed{seed}"] = dev.blit()
        out[f"spp16_seed{seed}_rays"] = np.float64(st["rays"])
        dev.close()
    np.savez_compressed(OUT / "terrain_e60_img.npz", **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["sobol", "rays", "images", "sunsky", "bsdf", "terrain", "lobes", "translucent", "siblings",
                             "film", "mesh", "aovs", "terrain_e60", "sh"]
    if "sh" in which:
        make_sh_images()
    if "terrain_e60" in which:
        make_terrain_e60_images()
    if "aovs" in which:
        make_aovs()
    if "terrain" in which:
        make_terrain_images()
    if "bsdf" in which:
        make_bsdf()
    if "lobes" in which:
        make_lobe_images()
    if "translucent" in which:
        make_translucent_images()
    if "mesh" in which:
        make_mesh_images()
    if "siblings" in which:
        make_sibling_images()
    if "film" in which:
        make_film()
    if "sunsky" in which:
        make_sunsky()
    if "sobol" in which:
        make_sobol()
    if "rays" in which:
        make_rays()
    if "images" in which:
        make_images()
