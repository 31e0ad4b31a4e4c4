"""Seeded synthetic scenes for the path-tracing workloads.

The reference publishes no scenes for its path tracer, so the workloads are generated here,
deterministically from a seed, with the shapes and value distributions of each workload:

* cornell():  the small plain-render scene: a Cornell-style room (5 axis-aligned quads,
  10 triangles) with a ceiling area light (2 triangles, emission 15) and 32 icospheres of
  subdivision 2 (320 triangles each), about 10.3k triangles, 256x256, 16 spp, depth 5.
* terrain():  the large plain-render scene: a 1024x1024 fBm heightfield (8 octaves,
  lacunarity 2, gain 0.5) plus 400 icospheres of subdivision 3 (1280 triangles each), about
  2.6M triangles, four material kinds and a sun-sky light, 1920x1080, 64 spp, depth 8,
  Russian roulette from depth 3.

A sun-sky light is described by the reference's parameters (Scene.sunsky: direction,
turbidity, ground albedo). The device takes its two products, the sun as a distant light and the
sky as an image light (what the reference's SunSkyLight computes from the parameters); the
caller supplies them with Scene.set_sunsky_products, or once per parameter set with
register_sunsky_products, after which every generated scene with those parameters gets them.

A Scene keeps every numpy array alive for as long as its ctypes descriptor is in use.
"""
import ctypes as C
import math
import pathlib

import numpy as np

import prt_types as T


class Scene:
    """Triangle meshes + Standard materials + environment lights, ready for the C ABI."""

    def __init__(self):
        self.meshes = []      # dicts: positions, normals, texcoords, indices, material
        self.materials = []   # prt_types.Material
        self.textures = []    # (h, w, 3) float32, row 0 at the top
        self.env = T.EnvDesc()
        self.env_image = None
        self.sunsky = None    # (dir xyz, turbidity, albedo) for the reference's SunSkyLight
        self.sunsky_applied = False
        self.camera = None
        self.width = 0
        self.height = 0
        self.spp = 1
        self.max_depth = 5
        self.rr_depth = 8
        self.renderer_type = T.PRT_RENDERER_PATH
        self.ao_samples = 16
        self.renderer_flags = 0   # PRT_RENDERER_IRRADIANCE
        self._keep = []

    # -- construction ---------------------------------------------------------------------
    def add_material(self, m):
        self.materials.append(m)
        return len(self.materials) - 1

    def add_mesh(self, positions, indices, material, normals=None, texcoords=None):
        self.meshes.append(dict(
            positions=np.ascontiguousarray(positions, np.float32).reshape(-1, 3),
            indices=np.ascontiguousarray(indices, np.int32).reshape(-1, 3),
            normals=None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3),
            texcoords=None if texcoords is None else np.ascontiguousarray(texcoords, np.float32).reshape(-1, 2),
            material=int(material)))

    def add_texture(self, rgb):
        self.textures.append(np.ascontiguousarray(rgb, np.float32))
        return len(self.textures) - 1

    def set_env_image(self, rgb, lut_size=0):
        self.env_image = np.ascontiguousarray(rgb, np.float32)
        self.env.image_width = self.env_image.shape[1]
        self.env.image_height = self.env_image.shape[0]
        self.env.image_lut_size = lut_size

    def set_sunsky_products(self, sun_color, sun_angle, sky):
        """The sun-sky light's products as environment lights: the sun (radiance, angular
        diameter) as the distant light toward sunsky[0:3], the sky (equirectangular RGB, top row
        first) as the image light with the reference's 128-entry LUT."""
        d = self.sunsky[0:3]
        self.env.distant_color[:] = tuple(float(c) for c in sun_color)
        self.env.distant_dir[:] = tuple(float(c) for c in d)
        self.env.distant_angle = float(sun_angle)
        self.set_env_image(sky, lut_size=128)
        self.sunsky_applied = True

    @property
    def tri_count(self):
        return sum(m["indices"].shape[0] for m in self.meshes)

    # -- C ABI ----------------------------------------------------------------------------
    def desc(self, oracle=False):
        """The C-ABI scene descriptor. With oracle=True and a sun-sky light, the sun/sky
        products are left out: the reference builds them itself from `sunsky`."""
        meshes = (T.Mesh * len(self.meshes))()
        for i, m in enumerate(self.meshes):
            meshes[i].positions = T.fptr(m["positions"])
            meshes[i].normals = T.fptr(m["normals"])
            meshes[i].texcoords = T.fptr(m["texcoords"])
            meshes[i].indices = T.iptr(m["indices"])
            meshes[i].vertex_count = m["positions"].shape[0]
            meshes[i].tri_count = m["indices"].shape[0]
            meshes[i].material = m["material"]
        mats = (T.Material * len(self.materials))(*self.materials)
        texs = (T.Texture * max(len(self.textures), 1))()
        for i, t in enumerate(self.textures):
            texs[i].rgb = T.fptr(t)
            texs[i].height, texs[i].width = t.shape[0], t.shape[1]
        d = T.SceneDesc()
        d.meshes = meshes
        d.mesh_count = len(self.meshes)
        d.materials = mats
        d.material_count = len(self.materials)
        d.textures = texs
        d.texture_count = len(self.textures)
        d.bvh_build = getattr(self, "bvh_build", T.PRT_BVH_HOST)
        d.env = self.env
        d.env.image_rgb = T.fptr(self.env_image)
        if self.sunsky is not None:
            if oracle:
                d.env.distant_color[:] = (0.0, 0.0, 0.0)
                d.env.image_rgb = None
            elif not self.sunsky_applied:
                raise ValueError("the scene has a sun-sky light but no sun-sky products: call set_sunsky_products "
                                 "or register_sunsky_products for its parameters")
        self._keep = [meshes, mats, texs]
        return d

    def renderer_desc(self, max_radiance=3.4028234663852886e38, min_weight=1e-4):
        r = T.RendererDesc()
        r.max_depth = self.max_depth
        r.rr_depth = self.rr_depth
        r.min_weight = min_weight
        r.type = self.renderer_type
        r.samples = self.ao_samples
        r.flags = self.renderer_flags
        r.max_radiance = max_radiance
        return r


def look_at(position, target, up=(0.0, 1.0, 0.0), fov_deg=40.0, near_clip=1e-3):
    """Pinhole camera descriptor; basis (U right, V up, N back) as camera/pinhole_camera.h expects."""
    p = np.asarray(position, np.float64)
    f = np.asarray(target, np.float64) - p
    f /= np.linalg.norm(f)
    n = -f
    u = np.cross(np.asarray(up, np.float64), n)
    u /= np.linalg.norm(u)
    v = np.cross(n, u)
    c = T.CameraDesc()
    c.position[:] = tuple(p.astype(np.float32))
    c.basis_u[:] = tuple(u.astype(np.float32))
    c.basis_v[:] = tuple(v.astype(np.float32))
    c.basis_n[:] = tuple(n.astype(np.float32))
    c.fov = float(np.float32(math.radians(fov_deg)))
    c.near_clip = near_clip
    return c


def icosphere(subdiv):
    """Unit icosphere: 20 * 4**subdiv triangles (midpoint subdivision, vertices projected)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
             (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    for _ in range(subdiv):
        cache = {}
        new_faces = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new_faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new_faces
    return np.array(verts, np.float64), np.array(faces, np.int32)


def _quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3); normal = cross(p1-p0, p2-p0)."""
    return np.array([p0, p1, p2, p3], np.float32), np.array([[0, 1, 2], [0, 2, 3]], np.int32)


def cornell(seed=0, width=256, height=256, spp=16, max_depth=5, n_spheres=32, sphere_subdiv=2):
    """The small plain-render scene (about 10.3k triangles)."""
    rng = np.random.default_rng(seed)
    s = Scene()
    white = s.add_material(T.material(base_color=(0.8, 0.8, 0.8), specular_weight=0.0))
    red = s.add_material(T.material(base_color=(0.6, 0.0, 0.0), specular_weight=0.0))
    green = s.add_material(T.material(base_color=(0.0, 0.6, 0.0), specular_weight=0.0))
    light = s.add_material(T.material(emission_luminance=15.0, emission_color=(1.0, 1.0, 1.0),
                                      specular_weight=0.0))
    # Room [-1,1] x [0,2] x [-1,1], open towards +z. Quads face into the room.
    for quad, mat in [
        (_quad((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1)), white),      # floor, normal +y
        (_quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)), white),      # ceiling, normal -y
        (_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)), white),    # back wall, normal +z
        (_quad((-1, 0, 1), (-1, 0, -1), (-1, 2, -1), (-1, 2, 1)), red),      # left wall, normal +x
        (_quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)), green),        # right wall, normal -x
    ]:
        s.add_mesh(quad[0], quad[1], mat)
    # Ceiling light just below the ceiling, facing down (emits where dot(dir, normal) < 0).
    y = 1.99
    lp, li = _quad((-0.25, y, -0.25), (0.25, y, -0.25), (0.25, y, 0.25), (-0.25, y, 0.25))
    s.add_mesh(lp, li, light)
    sv, sf = icosphere(sphere_subdiv)
    for _ in range(n_spheres):
        r = rng.uniform(0.05, 0.15)
        c = np.array([rng.uniform(-1 + r, 1 - r), rng.uniform(r, 2 - r), rng.uniform(-1 + r, 1 - r)])
        albedo = rng.uniform(0.1, 0.9, 3)
        m = s.add_material(T.material(base_color=albedo, specular_weight=0.0))
        s.add_mesh(sv * r + c, sf, m, normals=sv)
    s.camera = look_at((0.0, 1.0, 3.4), (0.0, 1.0, 0.0), fov_deg=40.0)
    s.width, s.height, s.spp, s.max_depth, s.rr_depth = width, height, spp, max_depth, 8
    return s


def tri_verts(scene):
    """The scene's triangles as (N, 9) float32 (v0, v1, v2), meshes concatenated in scene order:
    row i is global triangle i, the index the BVH8 stores."""
    rows = [m["positions"][m["indices"]].reshape(-1, 9) for m in scene.meshes]
    return np.concatenate(rows).astype(np.float32) if rows else np.zeros((0, 9), np.float32)


def triangle_soup(seed=0, n=5000, dup_frac=0.1, degenerate_frac=0.05, width=64, height=64, spp=1):
    """Random triangles in [-1, 1]^3 with exact duplicates and degenerate (zero-area or
    collapsed) triangles mixed in, for BVH builds: a worst case for both builders."""
    rng = np.random.default_rng(seed)
    s = Scene()
    m = s.add_material(T.material(base_color=(0.7, 0.7, 0.7), specular_weight=0.0))
    c = rng.uniform(-1.0, 1.0, (n, 1, 3))
    v = (c + rng.normal(0.0, 0.05, (n, 3, 3))).astype(np.float32)
    if n >= 4:
        k = int(n * dup_frac)
        src = rng.integers(0, n, k)
        dst = rng.integers(0, n, k)
        v[dst] = v[src]
        k = int(n * degenerate_frac)
        d = rng.integers(0, n, k)
        v[d[: k // 2], 1] = v[d[: k // 2], 0]                     # two equal vertices
        v[d[k // 2:], :] = v[d[k // 2:], :1]                       # a point
    s.add_mesh(v.reshape(-1, 3), np.arange(3 * n, dtype=np.int32).reshape(-1, 3), m)
    s.env.distant_color[:] = (0.0, 0.0, 0.0)
    s.env.ambient_color[:] = (1.0, 1.0, 1.0)
    s.camera = look_at((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), fov_deg=40.0)
    s.width, s.height, s.spp, s.max_depth, s.rr_depth = width, height, spp, 3, 8
    return s


def cornell_lobes(seed=0, width=128, height=128, spp=16, max_depth=5):
    """The small scene with its spheres cycling through the Oren-Nayar, sheen and layered
    lobes (rough diffuse, rough-diffuse plastic, sheen over Lambert, sheen over coated plastic)."""
    s = cornell(seed=seed, width=width, height=height, spp=spp, max_depth=max_depth)
    rng = np.random.default_rng(seed + 77)
    first = 4  # the room's white, red, green and light materials come first
    for k in range(first, len(s.materials)):
        c = tuple(float(x) for x in s.materials[k].base_color)
        kind = (k - first) % 4
        if kind == 0:
            m = T.material(base_color=c, specular_weight=0.0, diffuse_roughness=float(rng.uniform(0.3, 1.0)))
        elif kind == 1:
            m = T.material(base_color=c, diffuse_roughness=0.6, specular_roughness=float(rng.uniform(0.1, 0.5)))
        elif kind == 2:
            m = T.material(base_color=c, specular_weight=0.0, sheen_weight=1.0, sheen_color=(1.0, 0.9, 0.8),
                           sheen_roughness=float(rng.uniform(0.2, 0.6)))
        else:
            m = T.material(base_color=c, specular_roughness=0.3, coat_weight=0.5, coat_roughness=0.1,
                           sheen_weight=0.6, sheen_roughness=0.3)
        s.materials[k] = m
    return s


def cornell_translucent(seed=0, width=128, height=128, spp=16, max_depth=6):
    """The small scene with the see-through lobes: spheres cycling through thin smooth glass,
    thin rough tinted glass, half-opaque Lambert, Standard subsurface, half transmission at the
    ambient IOR and a thin-walled Oren-Nayar subsurface that transmits most of its light (the
    structure of a Principled backlight); plus a thin glass pane under the ceiling light and a
    half-opaque panel, so that shadow rays cross transparent surfaces. Standard materials only:
    the reference renders scenes from rkscene files, which hold Standard materials."""
    s = cornell(seed=seed, width=width, height=height, spp=spp, max_depth=max_depth)
    rng = np.random.default_rng(seed + 91)
    first = 4
    for k in range(first, len(s.materials)):
        c = tuple(float(x) for x in s.materials[k].base_color)
        kind = (k - first) % 6
        if kind == 0:
            m = T.material(transmission_weight=1.0, thin_walled=1, specular_roughness=0.0,
                           transmission_color=(0.9, 0.95, 0.8))
        elif kind == 1:
            m = T.material(transmission_weight=1.0, thin_walled=1, specular_roughness=float(rng.uniform(0.1, 0.3)),
                           transmission_color=c, transmission_depth=0.5)
        elif kind == 2:
            m = T.material(base_color=c, specular_weight=0.0, opacity=0.5)
        elif kind == 3:
            m = T.material(base_color=c, specular_roughness=0.3, subsurface_weight=0.6,
                           subsurface_color=(0.9, 0.6, 0.4), subsurface_anisotropy=float(rng.uniform(-0.5, 0.5)))
        elif kind == 4:
            m = T.material(base_color=c, transmission_weight=0.5, specular_ior=1.0)
        else:
            m = T.material(base_color=c, specular_roughness=0.4, diffuse_roughness=0.4, thin_walled=1,
                           subsurface_weight=1.0, subsurface_color=c, subsurface_anisotropy=0.5)
        s.materials[k] = m
    pane = s.add_material(T.material(transmission_weight=1.0, thin_walled=1, specular_roughness=0.05,
                                     transmission_color=(0.8, 0.9, 1.0)))
    p, i = _quad((-0.6, 1.6, -0.6), (0.3, 1.6, -0.6), (0.3, 1.6, 0.4), (-0.6, 1.6, 0.4))
    s.add_mesh(p, i, pane)
    panel = s.add_material(T.material(base_color=(0.9, 0.8, 0.3), specular_weight=0.0, opacity=0.4))
    p, i = _quad((0.2, 0.0, -0.8), (0.9, 0.0, -0.2), (0.9, 1.2, -0.2), (0.2, 1.2, -0.8))
    s.add_mesh(p, i, panel)
    return s


def smooth_noise_texture(size, seed, lo=0.1, hi=0.9):
    """(size, size, 3) smooth value noise in [lo, hi], one seeded noise per channel."""
    u = (np.arange(size) + 0.5) / size
    U, V = np.meshgrid(u, u, indexing="xy")
    out = np.empty((size, size, 3), np.float32)
    for c in range(3):
        n = value_noise_fbm(U, V, seed * 3 + c, octaves=4, base_freq=3.0)
        n = (n - n.min()) / max(n.max() - n.min(), 1e-9)
        out[..., c] = lo + (hi - lo) * n
    return out


def cornell_inverse(seed=0, target=False, tex_size=256, width=256, height=256, spp=16, max_depth=5, n_spheres=32,
                    albedo_init=0.5, roughness_init=0.3):
    """The inverse-rendering scene: the small scene with the floor and the back wall textured by
    tex_size^2 RGB albedo textures and every sphere given a specular layer whose roughness is a
    parameter. target=False: textures at albedo_init, roughness roughness_init. target=True:
    textures from seeded smooth noise in [0.1, 0.9], roughness uniform in [0.05, 0.6].
    Returns (scene, params) with params = {"textures": [ids], "roughness": [material ids]}."""
    rng = np.random.default_rng(seed)
    trng = np.random.default_rng(seed + 1000)
    s = Scene()
    if target:
        floor_tex = s.add_texture(smooth_noise_texture(tex_size, seed + 1))
        back_tex = s.add_texture(smooth_noise_texture(tex_size, seed + 2))
    else:
        floor_tex = s.add_texture(np.full((tex_size, tex_size, 3), albedo_init, np.float32))
        back_tex = s.add_texture(np.full((tex_size, tex_size, 3), albedo_init, np.float32))
    floor_m = s.add_material(T.material(base_color=(1.0, 1.0, 1.0), base_color_texture=floor_tex, specular_weight=0.0))
    back_m = s.add_material(T.material(base_color=(1.0, 1.0, 1.0), base_color_texture=back_tex, specular_weight=0.0))
    white = s.add_material(T.material(base_color=(0.8, 0.8, 0.8), specular_weight=0.0))
    red = s.add_material(T.material(base_color=(0.6, 0.0, 0.0), specular_weight=0.0))
    green = s.add_material(T.material(base_color=(0.0, 0.6, 0.0), specular_weight=0.0))
    light = s.add_material(T.material(emission_luminance=15.0, emission_color=(1.0, 1.0, 1.0), specular_weight=0.0))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    for quad, mat, tex in [
        (_quad((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1)), floor_m, True),
        (_quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)), white, False),
        (_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)), back_m, True),
        (_quad((-1, 0, 1), (-1, 0, -1), (-1, 2, -1), (-1, 2, 1)), red, False),
        (_quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)), green, False),
    ]:
        s.add_mesh(quad[0], quad[1], mat, texcoords=uv if tex else None)
    y = 1.99
    lp, li = _quad((-0.25, y, -0.25), (0.25, y, -0.25), (0.25, y, 0.25), (-0.25, y, 0.25))
    s.add_mesh(lp, li, light)
    sv, sf = icosphere(2)
    rough_ids = []
    for _ in range(n_spheres):
        r = rng.uniform(0.05, 0.15)
        c = np.array([rng.uniform(-1 + r, 1 - r), rng.uniform(r, 2 - r), rng.uniform(-1 + r, 1 - r)])
        albedo = rng.uniform(0.1, 0.9, 3)
        rough = float(trng.uniform(0.05, 0.6)) if target else roughness_init
        m = s.add_material(T.material(base_color=albedo, specular_weight=1.0, specular_roughness=rough,
                                      specular_ior=1.5))
        rough_ids.append(m)
        s.add_mesh(sv * r + c, sf, m, normals=sv)
    s.camera = look_at((0.0, 1.0, 3.4), (0.0, 1.0, 0.0), fov_deg=40.0)
    s.width, s.height, s.spp, s.max_depth, s.rr_depth = width, height, spp, max_depth, 8
    return s, {"textures": [floor_tex, back_tex], "roughness": rough_ids}


def lit_plane(albedo=(0.5, 0.5, 0.5), width=128, height=128, spp=64, sun_elevation_deg=50.0, sun_angle=0.1,
              sun_color=250.0):
    """A single Lambertian plane (y = 0, albedo from a 1x1 texture) under a distant light, seen
    from above so that it fills the frame; max depth 1. Each pixel's expected value is
    albedo * sun_color * sin^2(sun_angle / 2) * cos(zenith angle of the sun)."""
    s = Scene()
    tex = s.add_texture(np.array(albedo, np.float32).reshape(1, 1, 3))
    m = s.add_material(T.material(base_color=(1.0, 1.0, 1.0), base_color_texture=tex, specular_weight=0.0))
    q = _quad((-4, 0, 4), (4, 0, 4), (4, 0, -4), (-4, 0, -4))
    s.add_mesh(q[0], q[1], m, texcoords=np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32))
    d = sun_direction(sun_elevation_deg, 30.0)
    s.env.distant_color[:] = (sun_color, sun_color, sun_color)
    s.env.distant_dir[:] = tuple(float(c) for c in d)
    s.env.distant_angle = sun_angle
    s.camera = look_at((0.0, 2.0, 0.0), (0.0, 0.0, 0.0), up=(0.0, 0.0, -1.0), fov_deg=60.0)
    s.width, s.height, s.spp, s.max_depth, s.rr_depth = width, height, spp, 1, 8
    k = sun_color * math.sin(sun_angle / 2) ** 2 * math.sin(math.radians(sun_elevation_deg))
    return s, k


# ---- large plain-render scene: fBm terrain + icospheres under a sun-sky ----------------------

SUN_ELEVATION_DEG = 30.0
SUN_AZIMUTH_DEG = 45.0
SUN_TURBIDITY = 3.0
SUN_GROUND_ALBEDO = 0.2


def sun_direction(elevation_deg=SUN_ELEVATION_DEG, azimuth_deg=SUN_AZIMUTH_DEG):
    """Unit vector toward the sun; y is up (light/sun_sky_light.cpp:34-36 uses acos(dir.y))."""
    el, az = math.radians(elevation_deg), math.radians(azimuth_deg)
    return np.array([math.cos(el) * math.sin(az), math.sin(el), -math.cos(el) * math.cos(az)], np.float32)


def value_noise_fbm(x, z, rng_seed, octaves=8, lacunarity=2.0, gain=0.5, base_freq=4.0, lattice=256):
    """Seeded value-noise fBm in [-1, 1]-ish, vectorised over arrays x, z in [0, 1]."""
    rng = np.random.default_rng(rng_seed)
    table = rng.uniform(-1.0, 1.0, (lattice, lattice)).astype(np.float64)
    total = np.zeros_like(x, dtype=np.float64)
    amp, freq = 1.0, base_freq
    for o in range(octaves):
        px = x * freq + o * 17.31
        pz = z * freq + o * 9.73
        ix, iz = np.floor(px).astype(np.int64), np.floor(pz).astype(np.int64)
        fx, fz = px - ix, pz - iz
        sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
        a = table[ix % lattice, iz % lattice]
        b = table[(ix + 1) % lattice, iz % lattice]
        c = table[ix % lattice, (iz + 1) % lattice]
        d = table[(ix + 1) % lattice, (iz + 1) % lattice]
        total += amp * ((a * (1 - sx) + b * sx) * (1 - sz) + (c * (1 - sx) + d * sx) * sz)
        amp *= gain
        freq *= lacunarity
    return total


_SUNSKY_PRODUCTS = {}


def _sunsky_key(params):
    return tuple(np.asarray(params, np.float32).tolist())


def register_sunsky_products(params, sun_color, sun_angle, sky):
    """Products of the reference's SunSkyLight for `params` = (direction xyz, turbidity, ground
    albedo): every scene generated afterwards with those parameters gets them."""
    _SUNSKY_PRODUCTS[_sunsky_key(params)] = (np.asarray(sun_color, np.float32), float(sun_angle),
                                             np.ascontiguousarray(sky, np.float32))


def sunsky_params(elevation_deg=SUN_ELEVATION_DEG, azimuth_deg=SUN_AZIMUTH_DEG, turbidity=SUN_TURBIDITY,
                  albedo=SUN_GROUND_ALBEDO):
    d = sun_direction(elevation_deg, azimuth_deg)
    return np.array([d[0], d[1], d[2], turbidity, albedo], np.float32)


def terrain(seed=0, grid=1024, n_spheres=400, sphere_subdiv=3, width=1920, height=1080, spp=64, max_depth=8,
            rr_depth=3, extent=50.0, relief=10.0, sun_elevation_deg=SUN_ELEVATION_DEG, turbidity=SUN_TURBIDITY):
    """The large plain-render scene: grid^2 fBm heightfield (2 (grid-1)^2 triangles) plus
    n_spheres icospheres; spheres get one of four materials uniformly at random. Lit by a sun-sky
    light (sun at sun_elevation_deg, azimuth 45 degrees, ground albedo 0.2) whose products are
    applied when they were registered for those parameters."""
    rng = np.random.default_rng(seed)
    s = Scene()
    # Heightfield over [-extent, extent]^2 in xz, UVs = grid coordinates in [0, 1].
    u = np.linspace(0.0, 1.0, grid)
    U, V = np.meshgrid(u, u, indexing="xy")
    H = value_noise_fbm(U, V, seed) * relief
    X = (U * 2.0 - 1.0) * extent
    Z = (V * 2.0 - 1.0) * extent
    pos = np.stack([X, H, Z], -1).reshape(-1, 3).astype(np.float32)
    # Smooth vertex normals from central differences of the height.
    dx = 2.0 * extent / (grid - 1)
    gx = np.gradient(H, dx, axis=1)
    gz = np.gradient(H, dx, axis=0)
    nrm = np.stack([-gx, np.ones_like(H), -gz], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    i = np.arange(grid - 1)
    I, J = np.meshgrid(i, i, indexing="xy")
    v00 = (J * grid + I).ravel()
    v10 = v00 + 1
    v01 = v00 + grid
    v11 = v01 + 1
    # Counter-clockwise seen from +y.
    tris = np.concatenate([np.stack([v00, v01, v10], 1), np.stack([v10, v01, v11], 1)]).astype(np.int32)
    ground = s.add_material(T.material(base_color=(0.45, 0.42, 0.36), specular_weight=0.0))
    uvs = np.stack([U, V], -1).reshape(-1, 2).astype(np.float32)
    s.add_mesh(pos, tris, ground, normals=nrm.reshape(-1, 3).astype(np.float32), texcoords=uvs)
    # Spheres resting on the terrain.
    sv, sf = icosphere(sphere_subdiv)
    # Gold-like conductor through the Standard material's artistic Fresnel: reflectivity (F0)
    # of gold and a white edge tint. The edge tint stays (1, 1, 1) because the reference's
    # scene format does not store a metal's specular colour (rkscene/rkscene.h:626-627), so a
    # metal loaded by the reference always has that tint.
    gold_r = (1.0, 0.766, 0.336)
    gold_g = (1.0, 1.0, 1.0)
    for _ in range(n_spheres):
        r = rng.uniform(0.3, 1.5)
        cx, cz = rng.uniform(-0.9 * extent, 0.9 * extent, 2)
        hy = float(value_noise_fbm(np.array([(cx / extent + 1) / 2]), np.array([(cz / extent + 1) / 2]), seed)[0] * relief)
        kind = int(rng.integers(0, 4))
        if kind == 0:
            m = T.material(base_color=rng.uniform(0.1, 0.9, 3), specular_weight=0.0)
        elif kind == 1:
            m = T.material(metalness=1.0, base_color=gold_r, specular_color=gold_g,
                           specular_roughness=rng.uniform(0.05, 0.5))
        elif kind == 2:
            m = T.material(transmission_weight=1.0, specular_ior=1.5, specular_roughness=rng.uniform(0.0, 0.3))
        else:
            m = T.material(base_color=rng.uniform(0.1, 0.9, 3), specular_weight=0.0, coat_weight=1.0,
                           coat_roughness=rng.uniform(0.05, 0.5))
        mid = s.add_material(m)
        s.add_mesh(sv * r + np.array([cx, hy + r * 0.9, cz]), sf, mid, normals=sv)
    # Sun-sky light: the reference computes it from (direction, turbidity, albedo); the device
    # takes its two products, the sun as a distant light and the sky as an image light.
    s.sunsky = sunsky_params(sun_elevation_deg, SUN_AZIMUTH_DEG, turbidity, SUN_GROUND_ALBEDO)
    products = _SUNSKY_PRODUCTS.get(_sunsky_key(s.sunsky))
    if products is not None:
        s.set_sunsky_products(*products)
    s.camera = look_at((0.0, 0.56 * extent, 1.24 * extent), (0.0, 0.0, -0.1 * extent), fov_deg=45.0)
    s.width, s.height, s.spp, s.max_depth, s.rr_depth = width, height, spp, max_depth, rr_depth
    return s


BATCH_SIZES = (64, 96, 128, 192, 256, 384, 512)   # square frames, all multiples of 32
BATCH_SPPS = (4, 8, 16, 32, 64)


def batch_frames(count=64, seed=0, tri_range=(1e3, 5e5), sizes=BATCH_SIZES, spps=BATCH_SPPS, depth_range=(3, 10),
                 aov_mask=T.PRT_AOV_ALBEDO1 | T.PRT_AOV_NORMAL1):
    """The batched workload: `count` independent terrain scenes whose triangle count is
    log-uniform in tri_range (about 80% heightfield, 20% icospheres), each with a square
    frame from `sizes`, spp from `spps`, max depth uniform in depth_range and its own scene and
    sampler seed. Returns a list of (Scene, sampler seed, aov_mask)."""
    rng = np.random.default_rng(seed)
    frames = []
    for k in range(count):
        tris = float(np.exp(rng.uniform(np.log(tri_range[0]), np.log(tri_range[1]))))
        n_spheres = int(0.2 * tris / 1280)
        grid = max(8, int(np.sqrt(max(tris - 1280 * n_spheres, 128) / 2.0)) + 1)
        size = int(rng.choice(sizes))
        spp = int(rng.choice(spps))
        depth = int(rng.integers(depth_range[0], depth_range[1] + 1))
        scene_seed = int(rng.integers(0, 2**31 - 1))
        s = terrain(seed=scene_seed, grid=grid, n_spheres=n_spheres, width=size, height=size, spp=spp,
                    max_depth=depth, rr_depth=3)
        frames.append((s, int(rng.integers(0, 2**31 - 1)), aov_mask))
    return frames


def terrain_inverse(seed=0, target=False, tris=2e5, size=512, spp=16, max_depth=6, tex_size=512,
                    albedo_init=0.5, roughness_init=0.3):
    """One inverse-rendering problem of the batched differentiable workload: a terrain from the
    large-scene generator with `tris` triangles (about 80% heightfield, 20% icospheres), its
    ground textured by a tex_size^2 RGB albedo texture and every sphere a Lambertian base under
    a specular layer whose roughness is a parameter; sun-sky light. target=False: texture at
    albedo_init, roughness roughness_init; target=True: texture from seeded smooth noise in
    [0.1, 0.9], roughness uniform in [0.05, 0.6]. Returns (scene, params)."""
    n_spheres = int(0.2 * tris / 1280)
    grid = max(8, int(math.sqrt(max(tris - 1280 * n_spheres, 128) / 2.0)) + 1)
    s = terrain(seed=seed, grid=grid, n_spheres=n_spheres, width=size, height=size, spp=spp, max_depth=max_depth,
                rr_depth=3)
    rng = np.random.default_rng(seed + 4242)
    tex = smooth_noise_texture(tex_size, seed + 7) if target else np.full((tex_size, tex_size, 3), albedo_init,
                                                                           np.float32)
    t = s.add_texture(tex)
    s.materials[0] = T.material(base_color=(1.0, 1.0, 1.0), base_color_texture=t, specular_weight=0.0)
    rough_ids = []
    for k in range(1, len(s.materials)):
        c = tuple(float(x) for x in rng.uniform(0.1, 0.9, 3))
        r = float(rng.uniform(0.05, 0.6)) if target else roughness_init
        s.materials[k] = T.material(base_color=c, specular_weight=1.0, specular_roughness=r, specular_ior=1.5)
        rough_ids.append(k)
    return s, {"textures": [t], "roughness": rough_ids}


def batch_inverse_frames(count=16, seed=0, tri_range=(1e5, 1e6), size=512, spp=16, max_depth=6, tex_size=512,
                         target=False):
    """The batched differentiable workload: `count` inverse problems with triangle counts
    log-uniform in tri_range. Returns a list of (scene, params, sampler seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        tris = float(np.exp(rng.uniform(np.log(tri_range[0]), np.log(tri_range[1]))))
        scene_seed = int(rng.integers(0, 2**31 - 1))
        sampler_seed = int(rng.integers(0, 2**31 - 1))
        s, params = terrain_inverse(seed=scene_seed, target=target, tris=tris, size=size, spp=spp,
                                    max_depth=max_depth, tex_size=tex_size)
        out.append((s, params, sampler_seed))
    return out



# -- rkscene files ---------------------------------------------------------------------------------
_RK_SCALARS = [("baseWeight", "base_weight"), ("metalness", "metalness"), ("diffuseRoughness", "diffuse_roughness"),
               ("specularWeight", "specular_weight"), ("specularRoughness", "specular_roughness"),
               ("specularIOR", "specular_ior"), ("transmissionWeight", "transmission_weight"),
               ("transmissionDepth", "transmission_depth"), ("subsurfaceWeight", "subsurface_weight"),
               ("subsurfaceAnisotropy", "subsurface_anisotropy"), ("coatWeight", "coat_weight"),
               ("coatRoughness", "coat_roughness"), ("coatIOR", "coat_ior"), ("sheenWeight", "sheen_weight"),
               ("sheenRoughness", "sheen_roughness"), ("emissionLuminance", "emission_luminance"),
               ("opacity", "opacity")]
_RK_COLORS = [("specularColor", "specular_color"), ("transmissionColor", "transmission_color"),
              ("subsurfaceColor", "subsurface_color"), ("coatColor", "coat_color"), ("sheenColor", "sheen_color"),
              ("emissionColor", "emission_color")]


def write_pfm(path, rgb):
    """Little-endian colour PFM of an (h, w, 3) image given top row first."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    with open(path, "wb") as f:
        f.write(f"PF\n{rgb.shape[1]} {rgb.shape[0]}\n-1.0\n".encode())
        f.write(rgb[::-1].astype("<f4").tobytes())


def write_rkscene(scene, path, objects=None):
    """Writes `scene` as an rkscene file (JSON + .rkbin buffer + PFM textures), the layout of
    rkscene::save (rkscene/rkscene.h:907-941). One geometry per mesh; `objects` is a list of
    (geometry indices, transforms or None) with transforms (k, 3, 4) arrays whose columns are
    U V N P -- by default one object per geometry, without instances. Only Standard materials
    are representable."""
    import json

    path = pathlib.Path(path)
    bin_path = path.with_suffix(".rkbin")
    blob = bytearray()

    def buf(arr, kind):
        nonlocal blob
        a = np.ascontiguousarray(arr)
        view = {"type": kind, "count": int(a.shape[0]), "byteOffset": len(blob)}
        blob += a.tobytes()
        return view

    mats = []
    for i, m in enumerate(scene.materials):
        if m.model != T.PRT_MATERIAL_STANDARD:
            raise ValueError("rkscene materials are Standard materials")
        j = {"name": f"mat{i}"}
        for key, field in _RK_SCALARS:
            j[key] = float(getattr(m, field))
        base = [float(x) for x in m.base_color]
        if m.base_color_texture >= 0:
            j["baseColor"] = {"image": f"{path.stem}_tex{m.base_color_texture}.pfm", "factor": base}
        else:
            j["baseColor"] = base
        for key, field in _RK_COLORS:
            j[key] = [float(x) for x in getattr(m, field)]
        j["thinWalled"] = bool(m.thin_walled)
        mats.append(j)
    for k, t in enumerate(scene.textures):
        write_pfm(path.parent / f"{path.stem}_tex{k}.pfm", t)
    geoms = []
    for g, mesh in enumerate(scene.meshes):
        j = {"name": f"mesh{g}", "type": "triangle", "positions": buf(mesh["positions"].astype("<f4"), "float3")}
        if mesh["normals"] is not None:
            j["normals"] = buf(mesh["normals"].astype("<f4"), "float3")
        if mesh["texcoords"] is not None:
            j["texcoords"] = buf(mesh["texcoords"].astype("<f4"), "float2")
        j["indices"] = buf(mesh["indices"].astype("<u4").reshape(-1), "uint")
        j["material"] = int(mesh["material"])
        geoms.append(j)
    if objects is None:
        objects = [([g], None) for g in range(len(scene.meshes))]
    objs = []
    for k, (ids, xfs) in enumerate(objects):
        j = {"name": f"object{k}", "geometries": [int(i) for i in ids]}
        if xfs is not None:
            xf = np.asarray(xfs, np.float32).reshape(-1, 3, 4)
            j["instances"] = buf(np.ascontiguousarray(xf.transpose(0, 2, 1)).astype("<f4").reshape(-1, 12), "float3x4")
        objs.append(j)
    doc = {"name": path.stem, "materials": mats, "geometries": geoms, "objects": objs, "lights": [],
           "buffers": [{"uri": bin_path.name, "byteLength": len(blob)}]}
    bin_path.write_bytes(bytes(blob))
    path.write_text(json.dumps(doc, indent=2))
    return path


_MESH_BLOB_ID = 0x04df8666  # TriangleMesh::blobId (geometry/triangle_mesh.h:21)


def write_mesh(scene, path):
    """Writes `scene`'s meshes as one TriangleMesh blob (.mesh: blob id, bounds, counts, indices,
    per-triangle material ids, interleaved position / normal / UV attributes, material names;
    geometry/triangle_mesh.cpp:362-378) with its material library (.mtl of Standard materials,
    "type Standard") and PFM textures beside it. Meshes are concatenated; normals and UVs are
    written when every mesh has them. Materials are reordered so that the emissive ones take ids
    1..k, the order Scene::Scene requires of a mesh file (render/scene.cpp:119-130)."""
    import struct

    path = pathlib.Path(path)
    n = len(scene.materials)
    emissive = [i for i in range(n) if scene.materials[i].emission_luminance > 0.0]
    others = [i for i in range(n) if i not in emissive]
    order = others[:1] + emissive + others[1:]
    new_id = {old: k for k, old in enumerate(order)}
    materials = [scene.materials[i] for i in order]
    pos, nrm, uv, idx, mid = [], [], [], [], []
    base = 0
    has_n = all(m["normals"] is not None for m in scene.meshes)
    has_t = all(m["texcoords"] is not None for m in scene.meshes)
    for m in scene.meshes:
        pos.append(m["positions"])
        if has_n:
            nrm.append(m["normals"])
        if has_t:
            uv.append(m["texcoords"])
        idx.append(m["indices"] + base)
        mid.append(np.full(m["indices"].shape[0], new_id[m["material"]], np.int32))
        base += m["positions"].shape[0]
    P = np.concatenate(pos).astype(np.float32)
    cols = [P] + ([np.concatenate(nrm).astype(np.float32)] if has_n else []) + \
           ([np.concatenate(uv).astype(np.float32)] if has_t else [])
    attribs = np.concatenate(cols, 1)
    I = np.concatenate(idx).astype(np.int32)
    M = np.concatenate(mid).astype(np.int32)
    names = [f"mat{i}" for i in range(len(materials))]
    with open(path, "wb") as f:
        f.write(struct.pack("<i", _MESH_BLOB_ID))
        f.write(np.concatenate([P.min(0), P.max(0)]).astype("<f4").tobytes())
        f.write(struct.pack("<iiBb", I.shape[0], P.shape[0], 1 if has_n else 0, 1 if has_t else 0))
        f.write(I.astype("<i4").tobytes())
        f.write(M.astype("<i4").tobytes())
        f.write(attribs.astype("<f4").tobytes())
        f.write(struct.pack("<i", len(names)))
        for n in names:
            f.write(struct.pack("<i", len(n)) + n.encode())
    lines = []
    for i, m in enumerate(materials):
        if m.model != T.PRT_MATERIAL_STANDARD:
            raise ValueError("the material library is written with Standard materials")
        lines.append(f"newmtl {names[i]}")
        lines.append("type Standard")
        for key, field in _RK_SCALARS:
            lines.append(f"{key} {float(getattr(m, field))!r}")
        lines.append("baseColor " + " ".join(repr(float(x)) for x in m.base_color))
        for key, field in _RK_COLORS:
            lines.append(f"{key} " + " ".join(repr(float(x)) for x in getattr(m, field)))
        if m.base_color_texture >= 0:
            lines.append(f"baseColorMap {path.stem}_tex{m.base_color_texture}.pfm")
        lines.append(f"thinWalled {int(m.thin_walled)}")
    path.with_suffix(".mtl").write_text("\n".join(lines) + "\n")
    for k, t in enumerate(scene.textures):
        write_pfm(path.parent / f"{path.stem}_tex{k}.pfm", t)
    return path
