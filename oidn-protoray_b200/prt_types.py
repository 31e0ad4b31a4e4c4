"""ctypes mirror of the structs declared in include/prt_cuda.h.

These are the C-ABI scene/camera/renderer descriptors of the B200 render device. They
flatten what the reference's Scene::loadScene builds from an rkscene file
(render/scene.cpp:174-330) and the Props keys of the Device API (render/device.h:56-114).
"""
import ctypes as C

import numpy as np

PRT_OK = 0
PRT_ERR_INVALID_ARG = -1
PRT_ERR_LOGIC = -2
PRT_ERR_OUT_OF_MEMORY = -3
PRT_ERR_CUDA = -4
PRT_ERR_DEVICE_ABORT = -5
PRT_ERR_STATE = -6

PRT_AOV_ALBEDO1 = 1 << 0
PRT_AOV_NORMAL1 = 1 << 1
PRT_AOV_HDR_VAR = 1 << 2
PRT_AOV_SH = 1 << 3
PRT_RENDERER_IRRADIANCE = 1
PRT_ENV_AMBIENT_FIRST = 1
PRT_MICROFACET_BECKMANN = 1
PRT_MICROFACET_GGX_VISIBLE = 2

PRT_BLIT_HDR = 0
PRT_BLIT_ALBEDO1 = 1
PRT_BLIT_NORMAL1 = 2
PRT_BLIT_HDR_VAR = 3
PRT_BLIT_LDR = 4
PRT_BLIT_LDR_RGB = 5
PRT_BLIT_SH0 = 6
PRT_BLIT_SH1 = 7
PRT_BLIT_SH2 = 8
PRT_BLIT_SH3 = 9
PRT_TONE_NONE = 0
PRT_TONE_LINEAR = 1
PRT_TONE_REINHARD = 2
PRT_TONE_ACES = 3
PRT_TONE_FILMIC = 4
PRT_TONE_LOG = 5

F3 = C.c_float * 3


class Mesh(C.Structure):
    _fields_ = [
        ("positions", C.POINTER(C.c_float)),
        ("normals", C.POINTER(C.c_float)),
        ("texcoords", C.POINTER(C.c_float)),
        ("indices", C.POINTER(C.c_int32)),
        ("vertex_count", C.c_int32),
        ("tri_count", C.c_int32),
        ("material", C.c_int32),
        ("reserved", C.c_int32),
    ]


class Material(C.Structure):
    """Standard material parameters (material/standard.cpp:21-76)."""
    _fields_ = [
        ("base_weight", C.c_float),
        ("base_color", F3),
        ("metalness", C.c_float),
        ("diffuse_roughness", C.c_float),
        ("specular_weight", C.c_float),
        ("specular_color", F3),
        ("specular_roughness", C.c_float),
        ("specular_ior", C.c_float),
        ("transmission_weight", C.c_float),
        ("transmission_color", F3),
        ("transmission_depth", C.c_float),
        ("subsurface_weight", C.c_float),
        ("subsurface_color", F3),
        ("subsurface_anisotropy", C.c_float),
        ("coat_weight", C.c_float),
        ("coat_color", F3),
        ("coat_roughness", C.c_float),
        ("coat_ior", C.c_float),
        ("sheen_weight", C.c_float),
        ("sheen_color", F3),
        ("sheen_roughness", C.c_float),
        ("emission_luminance", C.c_float),
        ("emission_color", F3),
        ("opacity", C.c_float),
        ("thin_walled", C.c_int32),
        ("base_color_texture", C.c_int32),
        ("model", C.c_int32),
        ("ambient_ior", C.c_float),
        ("coat_thickness", C.c_float),
        ("sheen_tint", C.c_float),
        ("backlight", C.c_float),
        ("thickness", C.c_float),
        ("reserved", C.c_int32 * 2),
    ]


def material(**kw):
    """A Material with the rkscene defaults (rkscene/rkscene.h:161-207), overridden by kw."""
    m = Material()
    m.base_weight = 1.0
    m.base_color[:] = (0.8, 0.8, 0.8)
    m.metalness = 0.0
    m.diffuse_roughness = 0.0
    m.specular_weight = 1.0
    m.specular_color[:] = (1.0, 1.0, 1.0)
    m.specular_roughness = 0.3
    m.specular_ior = 1.5
    m.transmission_weight = 0.0
    m.transmission_color[:] = (1.0, 1.0, 1.0)
    m.transmission_depth = 1.0
    m.subsurface_weight = 0.0
    m.subsurface_color[:] = (0.8, 0.8, 0.8)
    m.subsurface_anisotropy = 0.0
    m.coat_weight = 0.0
    m.coat_color[:] = (1.0, 1.0, 1.0)
    m.coat_roughness = 0.0
    m.coat_ior = 1.6
    m.sheen_weight = 0.0
    m.sheen_color[:] = (1.0, 1.0, 1.0)
    m.sheen_roughness = 0.3
    m.emission_luminance = 0.0
    m.emission_color[:] = (1.0, 1.0, 1.0)
    m.opacity = 1.0
    m.thin_walled = 0
    m.base_color_texture = -1
    m.model = PRT_MATERIAL_STANDARD
    m.ambient_ior = 1.0
    m.coat_thickness = 1.0
    m.thickness = 1.0
    for k, v in kw.items():
        if isinstance(v, (tuple, list, np.ndarray)):
            getattr(m, k)[:] = tuple(float(x) for x in v)
        else:
            setattr(m, k, v)
    return m


PRT_MATERIAL_STANDARD = 0
PRT_MATERIAL_PRINCIPLED = 1
PRT_MATERIAL_MISS = 2


def principled(**kw):
    """A Material of the Principled model with PrincipledMaterial's defaults
    (material/principled.cpp:21-60), overridden by kw (field names of the shared record:
    base_color = baseColor, specular_color = edgeColor, metalness = metallic, base_weight =
    diffuse, specular_weight = specular, specular_ior = ior, specular_roughness = roughness, ...)."""
    m = material(specular_color=(1.0, 1.0, 1.0), specular_roughness=0.0, specular_ior=1.0, coat_ior=1.5,
                 sheen_roughness=0.2)
    m.model = PRT_MATERIAL_PRINCIPLED
    for k, v in kw.items():
        if isinstance(v, (tuple, list, np.ndarray)):
            getattr(m, k)[:] = tuple(float(x) for x in v)
        else:
            setattr(m, k, v)
    return m


class Texture(C.Structure):
    _fields_ = [("rgb", C.POINTER(C.c_float)), ("width", C.c_int32), ("height", C.c_int32)]


class EnvDesc(C.Structure):
    _fields_ = [
        ("distant_color", F3),
        ("distant_dir", F3),
        ("distant_angle", C.c_float),
        ("ambient_color", F3),
        ("image_rgb", C.POINTER(C.c_float)),
        ("image_width", C.c_int32),
        ("image_height", C.c_int32),
        ("image_lut_size", C.c_int32),
        ("flags", C.c_int32),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("meshes", C.POINTER(Mesh)),
        ("mesh_count", C.c_int32),
        ("material_count", C.c_int32),
        ("materials", C.POINTER(Material)),
        ("textures", C.POINTER(Texture)),
        ("texture_count", C.c_int32),
        ("bvh_build", C.c_int32),
        ("env", EnvDesc),
    ]


PRT_BVH_HOST = 0
PRT_BVH_DEVICE = 1


class SceneStats(C.Structure):
    _fields_ = [
        ("build_ms", C.c_double),
        ("node_count", C.c_int64),
        ("tri_count", C.c_int64),
        ("builder", C.c_int32),
        ("depth", C.c_int32),
        ("top_count", C.c_int32),
        ("iterations", C.c_int32),
        ("bounds_lo", F3),
        ("bounds_hi", F3),
    ]


class CameraDesc(C.Structure):
    _fields_ = [
        ("position", F3),
        ("basis_u", F3),
        ("basis_v", F3),
        ("basis_n", F3),
        ("fov", C.c_float),
        ("near_clip", C.c_float),
    ]


class RendererDesc(C.Structure):
    _fields_ = [
        ("max_depth", C.c_int32),
        ("rr_depth", C.c_int32),
        ("min_weight", C.c_float),
        ("max_radiance", C.c_float),
        ("type", C.c_int32),
        ("samples", C.c_int32),
        ("flags", C.c_int32),
    ]


PRT_RENDERER_PATH = 0
PRT_RENDERER_PRIMARY = 1
PRT_RENDERER_AO = 2
PRT_RENDERER_DIFFUSE = 3
PRT_RENDERER_DIFFUSE2 = 4
PRT_RENDERER_PRIMARY_FAST = 5
PRT_RENDERER_AO_FAST = 6
PRT_RENDERER_DIFFUSE_FAST = 7
PRT_RENDERER_DIFFUSE2_FAST = 8


class RenderStats(C.Structure):
    _fields_ = [
        ("mray", C.c_double),
        ("rays", C.c_int64),
        ("spp", C.c_int64),
        ("render_ms", C.c_double),
        ("closest_rays", C.c_int64),
        ("shadow_rays", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("trace_ms", C.c_double),
        ("shadow_ms", C.c_double),
        ("shade_ms", C.c_double),
        ("closest_nodes", C.c_int64),
        ("closest_tris", C.c_int64),
        ("shadow_nodes", C.c_int64),
        ("shadow_tris", C.c_int64),
        ("trace_launches", C.c_int64),
    ]


class BatchItem(C.Structure):
    _fields_ = [
        ("scene", C.POINTER(SceneDesc)),
        ("camera", CameraDesc),
        ("renderer", RendererDesc),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("spp", C.c_int32),
        ("aov_mask", C.c_int32),
        ("seed", C.c_uint32),
        ("reserved", C.c_int32),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("trace_blocks", C.c_int32),
        ("shade_blocks", C.c_int32),
        ("wave_paths", C.c_int32),
        ("top_stage", C.c_int32),
        ("ray_bins", C.c_int32),
        ("trace_stack", C.c_int32),
    ]


PRT_PROFILE_KERNELS = 1 << 0
PRT_PROFILE_COUNTS = 1 << 1


def fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None


def uptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32)) if a is not None else None
