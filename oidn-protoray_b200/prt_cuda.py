"""Python handle on libprt_cuda.so, the B200 render device, through its C ABI.

DeviceCuda mirrors the reference's Device API (render/device.h:56-114): initScene,
initRenderer, initSampler, initCamera, initFrame, clearFrame, render, blitFrame, plus the
ray queries. Errors come back as the exception types the reference throws
(std::invalid_argument -> ValueError, std::logic_error -> LogicError, others -> RuntimeError).

The library is built in place (make -C oidn-protoray_b200); there is no CPU fallback:
loading fails loudly when the library or a CUDA device is missing.
"""
import ctypes as C
import os
import weakref
import pathlib

import numpy as np

import prt_types as T

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libprt_cuda.so"

_lib = None


class LogicError(RuntimeError):
    """Counterpart of std::logic_error."""


class DeviceAbort(RuntimeError):
    """A device loop hit its iteration cap or a bounds check."""


def load_library():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} is not built (make -C oidn-protoray_b200)")
    # libstdc++ must be global before a C++ library loads (see oracle/ref.py).
    C.CDLL("libstdc++.so.6", mode=os.RTLD_GLOBAL)
    lib = C.CDLL(str(LIB_PATH))
    P = C.POINTER
    vp = C.c_void_p
    lib.prt_cuda_create.argtypes = [C.c_int, P(vp)]
    lib.prt_cuda_destroy.argtypes = [vp]
    lib.prt_cuda_last_error.argtypes = [vp]
    lib.prt_cuda_last_error.restype = C.c_char_p
    lib.prt_cuda_material_defaults.argtypes = [P(T.Material)]
    lib.prt_cuda_material_defaults.restype = None
    lib.prt_cuda_scene_upload.argtypes = [vp, P(T.SceneDesc)]
    lib.prt_cuda_renderer.argtypes = [vp, P(T.RendererDesc)]
    lib.prt_cuda_init_sampler.argtypes = [vp, C.c_uint32]
    lib.prt_cuda_camera.argtypes = [vp, P(T.CameraDesc)]
    lib.prt_cuda_frame.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32]
    lib.prt_cuda_clear.argtypes = [vp]
    lib.prt_cuda_render.argtypes = [vp, C.c_int32, P(T.RenderStats)]
    lib.prt_cuda_set_profiling.argtypes = [vp, C.c_int32]
    lib.prt_cuda_tone_mapper.argtypes = [vp, C.c_int32, C.c_float, C.c_float]
    lib.prt_cuda_frame_error.argtypes = [vp, P(C.c_float)]
    lib.prt_cuda_set_tuning.argtypes = [vp, P(T.Tuning)]
    lib.prt_cuda_adjoint.argtypes = [vp, C.c_uint32, C.c_int32, vp, vp, C.c_int64, vp, C.c_int32, P(T.RenderStats)]
    lib.prt_cuda_update_texture.argtypes = [vp, C.c_int32, vp]
    lib.prt_cuda_update_material.argtypes = [vp, C.c_int32, P(T.Material)]
    lib.prt_cuda_batch_create.argtypes = [vp, P(T.BatchItem), C.c_int32, P(vp)]
    lib.prt_cuda_batch_render.argtypes = [vp, P(T.RenderStats)]
    lib.prt_cuda_batch_blit.argtypes = [vp, C.c_int32, C.c_int32, P(C.c_float)]
    lib.prt_cuda_batch_destroy.argtypes = [vp]
    lib.prt_cuda_batch_enable_adjoint.argtypes = [vp]
    lib.prt_cuda_batch_adjoint.argtypes = [vp, P(vp), P(vp), P(vp), P(T.RenderStats)]
    lib.prt_cuda_batch_update_texture.argtypes = [vp, C.c_int32, C.c_int32, vp]
    lib.prt_cuda_batch_update_material.argtypes = [vp, C.c_int32, C.c_int32, P(T.Material)]
    lib.prt_cuda_batch_update_materials.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, P(T.Material)]
    lib.prt_cuda_update_materials.argtypes = [vp, C.c_int32, C.c_int32, P(T.Material)]
    lib.prt_cuda_get_tuning.argtypes = [vp, P(T.Tuning)]
    lib.prt_cuda_autotune.argtypes = [vp, C.c_int32, P(T.Tuning), P(C.c_double)]
    lib.prt_cuda_blit.argtypes = [vp, C.c_int32, P(C.c_float)]
    lib.prt_cuda_sobol.argtypes = [vp, C.c_int64, P(C.c_uint32), P(C.c_uint32), P(C.c_uint32), C.c_int32,
                                   P(C.c_float)]
    lib.prt_cuda_trace.argtypes = [vp, C.c_int64, P(C.c_float), P(C.c_int32), P(C.c_int32), P(C.c_float),
                                   P(C.c_float), P(C.c_float)]
    lib.prt_cuda_occluded.argtypes = [vp, C.c_int64, P(C.c_float), P(C.c_int32)]
    lib.prt_cuda_query_primary.argtypes = [vp, C.c_uint32, P(C.c_float), P(C.c_int32), P(C.c_int32), P(C.c_float)]
    lib.prt_cuda_bsdf_query.argtypes = [vp, P(T.Material), C.c_int32, C.c_int64, P(C.c_float), P(C.c_float)]
    lib.prt_cuda_albedo_tables.argtypes = [vp, P(C.c_float), C.c_int64, P(C.c_int64)]
    lib.prt_bvh8_count.argtypes = [P(C.c_float), C.c_int64, C.c_int64, P(C.c_float), P(C.c_int32), P(C.c_float),
                                   P(C.c_int64), P(C.c_int64), P(C.c_int64)]
    lib.prt_cuda_scene_stats.argtypes = [vp, P(T.SceneStats)]
    lib.prt_cuda_scene_bvh.argtypes = [vp, vp, C.c_int64, vp, C.c_int64, P(C.c_int64), P(C.c_int64)]
    lib.prt_bvh8_check.argtypes = [vp, C.c_int64, vp, C.c_int64, P(C.c_float), C.c_int32, P(C.c_int32),
                                   C.c_char_p, C.c_int32]
    lib.prt_bvh8_trace.argtypes = [vp, C.c_int64, vp, C.c_int64, C.c_int64, P(C.c_float), P(C.c_int32),
                                   P(C.c_float), P(C.c_int64), P(C.c_int64)]
    lib.prt_bvh8_build_host.argtypes = [P(C.c_float), C.c_int64, vp, C.c_int64, vp, C.c_int64, P(C.c_int64),
                                        P(C.c_int32)]
    lib.prt_scene_file_load.argtypes = [C.c_char_p, P(vp), C.c_char_p, C.c_int32]
    lib.prt_scene_file_desc.argtypes = [vp, P(T.SceneDesc)]
    lib.prt_scene_file_free.argtypes = [vp]
    lib.prt_cuda_scene_load.argtypes = [vp, C.c_char_p, P(T.EnvDesc), C.c_int32]
    lib.prt_cuda_scene_lights.argtypes = [vp, P(T.EnvDesc)]
    lib.prt_cuda_microfacet_query.argtypes = [vp, C.c_int32, C.c_int64, P(C.c_float), P(C.c_float)]
    lib.prt_cuda_set_albedo_tables.argtypes = [vp, P(C.c_float), C.c_int64]
    _lib = lib
    return lib


def bvh8_count(tri_verts, rays):
    """Host-only BVH8 build + counting traversal (no GPU): (tri ids, t, nodes/ray, tris/ray, node count)."""
    lib = load_library()
    tv = np.ascontiguousarray(tri_verts, np.float32).reshape(-1, 9)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    tri = np.zeros(r.shape[0], np.int32)
    t = np.zeros(r.shape[0], np.float32)
    nv, tt, nc = C.c_int64(0), C.c_int64(0), C.c_int64(0)
    rc = lib.prt_bvh8_count(T.fptr(tv), tv.shape[0], r.shape[0], T.fptr(r), T.iptr(tri), T.fptr(t), C.byref(nv),
                            C.byref(tt), C.byref(nc))
    if rc != T.PRT_OK:
        raise ValueError(f"prt_bvh8_count failed ({rc})")
    n = max(r.shape[0], 1)
    return tri, t, nv.value / n, tt.value / n, nc.value


BVH8_NODE_BYTES = 80
BVH8_TRI_BYTES = 48


class SceneFile:
    """A scene file (.rkscene or .mesh) loaded on the host (prt_scene_file_load): the flat scene
    description the device uploads, readable as numpy arrays. Raises ValueError for malformed or
    unsupported content and OSError for files that cannot be read."""

    def __init__(self, path):
        self.lib = load_library()
        self.h = None
        h = C.c_void_p()
        msg = C.create_string_buffer(512)
        rc = self.lib.prt_scene_file_load(str(path).encode(), C.byref(h), msg, 512)
        if rc == T.PRT_ERR_INVALID_ARG:
            raise ValueError(msg.value.decode())
        if rc != T.PRT_OK:
            raise OSError(msg.value.decode())
        self.h = h
        self.d = T.SceneDesc()
        self.lib.prt_scene_file_desc(self.h, C.byref(self.d))

    def close(self):
        if getattr(self, "h", None):
            self.lib.prt_scene_file_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def meshes(self):
        out = []
        for i in range(self.d.mesh_count):
            m = self.d.meshes[i]
            nv, nt = m.vertex_count, m.tri_count
            arr = lambda p, n: np.ctypeslib.as_array(p, (n,)).copy()
            out.append(dict(positions=arr(m.positions, 3 * nv).reshape(-1, 3) if nv else np.zeros((0, 3), np.float32),
                            normals=arr(m.normals, 3 * nv).reshape(-1, 3) if m.normals else None,
                            texcoords=arr(m.texcoords, 2 * nv).reshape(-1, 2) if m.texcoords else None,
                            indices=arr(m.indices, 3 * nt).reshape(-1, 3) if nt else np.zeros((0, 3), np.int32),
                            material=m.material))
        return out

    def materials(self):
        return [T.Material.from_buffer_copy(self.d.materials[i]) for i in range(self.d.material_count)]

    def textures(self):
        out = []
        for i in range(self.d.texture_count):
            t = self.d.textures[i]
            out.append(np.ctypeslib.as_array(t.rgb, (t.height * t.width * 3,)).reshape(t.height, t.width, 3).copy())
        return out


def bvh8_build_host(tri_verts):
    """Host-only PRT_BVH_HOST build into arrays: (nodes uint8[N, 80], tris uint8[M, 48], top count)."""
    lib = load_library()
    tv = np.ascontiguousarray(tri_verts, np.float32).reshape(-1, 9)
    n = tv.shape[0]
    nodes = np.zeros((max(n, 1), BVH8_NODE_BYTES), np.uint8)
    tris = np.zeros((n, BVH8_TRI_BYTES), np.uint8)
    nc, top = C.c_int64(0), C.c_int32(0)
    rc = lib.prt_bvh8_build_host(T.fptr(tv), n, nodes.ctypes.data, nodes.shape[0], tris.ctypes.data if n else None,
                                 n, C.byref(nc), C.byref(top))
    if rc != T.PRT_OK:
        raise ValueError(f"prt_bvh8_build_host failed ({rc})")
    return nodes[: nc.value].copy(), tris, top.value


def bvh8_check(nodes, tris, tri_verts, top_count):
    """Host-only structural check of a BVH8 given as byte arrays (prt_bvh8_check): returns
    (depth, "") for a valid tree, (depth, first violation) otherwise."""
    lib = load_library()
    nb = np.ascontiguousarray(nodes, np.uint8).reshape(-1, BVH8_NODE_BYTES)
    tb = np.ascontiguousarray(tris, np.uint8).reshape(-1, BVH8_TRI_BYTES)
    tv = np.ascontiguousarray(tri_verts, np.float32).reshape(-1, 9)
    depth = C.c_int32(0)
    msg = C.create_string_buffer(256)
    rc = lib.prt_bvh8_check(nb.ctypes.data, nb.shape[0], tb.ctypes.data if tb.size else None, tb.shape[0],
                            T.fptr(tv), int(top_count), C.byref(depth), msg, 256)
    if rc not in (T.PRT_OK, T.PRT_ERR_INVALID_ARG):
        raise RuntimeError(f"prt_bvh8_check failed ({rc})")
    return depth.value, msg.value.decode()


def bvh8_trace(nodes, tris, rays):
    """Host-only counting traversal over a BVH8 given as byte arrays: (tri ids, t, nodes/ray, tris/ray)."""
    lib = load_library()
    nb = np.ascontiguousarray(nodes, np.uint8).reshape(-1, BVH8_NODE_BYTES)
    tb = np.ascontiguousarray(tris, np.uint8).reshape(-1, BVH8_TRI_BYTES)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    tri = np.zeros(r.shape[0], np.int32)
    t = np.zeros(r.shape[0], np.float32)
    nv, tt = C.c_int64(0), C.c_int64(0)
    rc = lib.prt_bvh8_trace(nb.ctypes.data, nb.shape[0], tb.ctypes.data if tb.size else None, tb.shape[0],
                            r.shape[0], T.fptr(r), T.iptr(tri), T.fptr(t), C.byref(nv), C.byref(tt))
    if rc != T.PRT_OK:
        raise ValueError(f"prt_bvh8_trace failed ({rc})")
    n = max(r.shape[0], 1)
    return tri, t, nv.value / n, tt.value / n


class DeviceCuda:
    """The CUDA render device; one per host thread."""

    def __init__(self, device_ordinal=0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.prt_cuda_create(device_ordinal, C.byref(h))
        if rc != T.PRT_OK:
            raise RuntimeError(f"prt_cuda_create failed ({rc}): no usable CUDA device")
        self.h = h
        self.scene = None
        self.width = self.height = 0
        self._keep = None

    def close(self):
        for b in list(getattr(self, "_batches", [])):
            b.close()
        if getattr(self, "h", None):
            self.lib.prt_cuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc == T.PRT_OK:
            return
        msg = self.lib.prt_cuda_last_error(self.h).decode()
        if rc == T.PRT_ERR_INVALID_ARG:
            raise ValueError(msg)
        if rc == T.PRT_ERR_LOGIC:
            raise LogicError(msg)
        if rc == T.PRT_ERR_DEVICE_ABORT:
            raise DeviceAbort(msg)
        if rc == T.PRT_ERR_OUT_OF_MEMORY:
            raise MemoryError(msg)
        raise RuntimeError(f"prt_cuda error {rc}: {msg}")

    # -- Device API --------------------------------------------------------------------------
    def init_scene(self, scene):
        desc = scene.desc()
        self._keep = desc
        self._check(self.lib.prt_cuda_scene_upload(self.h, C.byref(desc)))
        self.scene = scene

    def load_scene(self, path, env=None, bvh_build=T.PRT_BVH_HOST):
        """Device::initScene(path) + initLights: uploads a .rkscene or .mesh file (prt_cuda_scene_load);
        `env` is a prt_types.EnvDesc or None (no environment light)."""
        self._check(self.lib.prt_cuda_scene_load(self.h, str(path).encode(), C.byref(env) if env is not None else None,
                                                 int(bvh_build)))

    def scene_stats(self):
        """BVH statistics of the uploaded scene (prt_scene_stats) as a dict."""
        st = T.SceneStats()
        self._check(self.lib.prt_cuda_scene_stats(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in T.SceneStats._fields_}

    def scene_bvh(self):
        """The uploaded scene's BVH8 copied back: (nodes uint8[N, 80], tris uint8[M, 48])."""
        nc, tc = C.c_int64(0), C.c_int64(0)
        self._check(self.lib.prt_cuda_scene_bvh(self.h, None, 0, None, 0, C.byref(nc), C.byref(tc)))
        nodes = np.zeros((nc.value, BVH8_NODE_BYTES), np.uint8)
        tris = np.zeros((tc.value, BVH8_TRI_BYTES), np.uint8)
        self._check(self.lib.prt_cuda_scene_bvh(self.h, nodes.ctypes.data, nc.value, tris.ctypes.data if tc.value else None,
                                            tc.value, C.byref(nc), C.byref(tc)))
        return nodes, tris

    def init_renderer(self, max_depth=100, rr_depth=8, min_weight=1e-4, max_radiance=3.4028234663852886e38,
                      type=T.PRT_RENDERER_PATH, samples=16, flags=0):
        r = T.RendererDesc(max_depth, rr_depth, min_weight, max_radiance, type, samples, flags)
        self._check(self.lib.prt_cuda_renderer(self.h, C.byref(r)))

    def init_sampler(self, seed):
        self._check(self.lib.prt_cuda_init_sampler(self.h, seed))

    def init_frame(self, width, height, aov_mask=0):
        self._check(self.lib.prt_cuda_frame(self.h, width, height, aov_mask))
        self.width, self.height = width, height

    def init_camera(self, camera):
        self._check(self.lib.prt_cuda_camera(self.h, C.byref(camera)))

    def clear_frame(self):
        self._check(self.lib.prt_cuda_clear(self.h))

    def render(self, spp=1):
        st = T.RenderStats()
        self._check(self.lib.prt_cuda_render(self.h, spp, C.byref(st)))
        return {name: getattr(st, name) for name, _ in T.RenderStats._fields_}

    def set_tuning(self, trace_blocks=0, shade_blocks=0, wave_paths=0, top_stage=0, ray_bins=0, trace_stack=0):
        t = T.Tuning(trace_blocks, shade_blocks, wave_paths, top_stage, ray_bins, trace_stack)
        self._check(self.lib.prt_cuda_set_tuning(self.h, C.byref(t)))

    def get_tuning(self):
        t = T.Tuning()
        self._check(self.lib.prt_cuda_get_tuning(self.h, C.byref(t)))
        return {name: getattr(t, name) for name, _ in T.Tuning._fields_}

    def autotune(self, spp=4):
        """Picks the fastest launch tuning for the current scene/frame; clears the frame."""
        t = T.Tuning()
        m = C.c_double()
        self._check(self.lib.prt_cuda_autotune(self.h, spp, C.byref(t), C.byref(m)))
        return {name: getattr(t, name) for name, _ in T.Tuning._fields_}, m.value

    # -- differentiation -------------------------------------------------------------------
    @staticmethod
    def _ptr(a):
        if a is None:
            return None
        if hasattr(a, "data_ptr"):
            return C.c_void_p(a.data_ptr())
        return a.ctypes.data_as(C.c_void_p)

    def adjoint(self, d_loss_d_image, spp, first_sample=0, grad_textures=None, grad_roughness=None):
        """Path-replay adjoint: accumulates dLoss/d(texel) into grad_textures (all scene textures
        concatenated, each (h, w, 3), row 0 at the top) and dLoss/d(specular roughness) into
        grad_roughness (one per material). Arrays may be numpy or CUDA torch tensors (float32);
        numpy outputs are created when None. Returns (grad_textures, grad_roughness, stats)."""
        sc = self.scene
        tex_floats = sum(int(t.size) for t in sc.textures)
        if grad_textures is None:
            grad_textures = np.zeros(max(tex_floats, 1), np.float32)
        if grad_roughness is None:
            grad_roughness = np.zeros(len(sc.materials), np.float32)
        if not hasattr(d_loss_d_image, "data_ptr"):
            d_loss_d_image = np.ascontiguousarray(d_loss_d_image, np.float32)
        st = T.RenderStats()
        self._check(self.lib.prt_cuda_adjoint(self.h, first_sample, spp, self._ptr(d_loss_d_image),
                                              self._ptr(grad_textures), tex_floats, self._ptr(grad_roughness),
                                              len(sc.materials), C.byref(st)))
        return grad_textures, grad_roughness, {name: getattr(st, name) for name, _ in T.RenderStats._fields_}

    def update_texture(self, index, rgb):
        if not hasattr(rgb, "data_ptr"):
            rgb = np.ascontiguousarray(rgb, np.float32)
        self._check(self.lib.prt_cuda_update_texture(self.h, index, self._ptr(rgb)))

    def update_material(self, index, material):
        self._check(self.lib.prt_cuda_update_material(self.h, index, C.byref(material)))

    def update_materials(self, first, materials):
        arr = (T.Material * len(materials))(*materials)
        self._check(self.lib.prt_cuda_update_materials(self.h, first, len(materials), arr))

    def set_profiling(self, flags):
        self._check(self.lib.prt_cuda_set_profiling(self.h, flags))

    def tone_mapper(self, kind, exposure=1.0, burn=0.0):
        self._check(self.lib.prt_cuda_tone_mapper(self.h, kind, exposure, burn))

    def frame_error(self):
        e = C.c_float()
        self._check(self.lib.prt_cuda_frame_error(self.h, C.byref(e)))
        return e.value

    def blit_frame(self, aov=T.PRT_BLIT_HDR, out=None):
        """Returns (height, width, 3) float32 ((height, width) uint32 for PRT_BLIT_LDR); `out` may
        be a CUDA torch tensor (zero copy)."""
        if aov == T.PRT_BLIT_LDR and out is None:
            ldr = np.zeros((self.height, self.width), np.uint32)
            self._check(self.lib.prt_cuda_blit(self.h, aov, ldr.ctypes.data_as(C.POINTER(C.c_float))))
            return ldr
        if out is not None and hasattr(out, "data_ptr"):
            self._check(self.lib.prt_cuda_blit(self.h, aov, C.cast(C.c_void_p(out.data_ptr()), C.POINTER(C.c_float))))
            return out
        img = np.zeros((self.height, self.width, 3), np.float32)
        self._check(self.lib.prt_cuda_blit(self.h, aov, T.fptr(img)))
        return img

    def setup(self, scene, seed=0, aov_mask=0):
        """initScene + initFrame + initCamera + initRenderer + initSampler for a Scene."""
        self.init_scene(scene)
        self.init_frame(scene.width, scene.height, aov_mask)
        self.init_camera(scene.camera)
        self.init_renderer(scene.max_depth, scene.rr_depth, type=scene.renderer_type, samples=scene.ao_samples,
                           flags=scene.renderer_flags)
        self.init_sampler(seed)

    # -- queries --------------------------------------------------------------------------------
    def sobol(self, sample_index, pixel_id, dim_set, dims):
        n = len(sample_index)
        si = np.ascontiguousarray(sample_index, np.uint32)
        pi = np.ascontiguousarray(pixel_id, np.uint32)
        ds = np.ascontiguousarray(dim_set, np.uint32)
        out = np.zeros(n * dims, np.float32)
        self._check(self.lib.prt_cuda_sobol(self.h, n, T.uptr(si), T.uptr(pi), T.uptr(ds), dims, T.fptr(out)))
        return out.reshape(n, dims)

    def trace(self, rays):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        g = np.zeros(n, np.int32)
        p = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        self._check(self.lib.prt_cuda_trace(self.h, n, T.fptr(rays), T.iptr(g), T.iptr(p), T.fptr(t), T.fptr(u),
                                            T.fptr(v)))
        return g, p, t, u, v

    def bsdf_query(self, material, tuples, medium_id=0):
        """(n, 13) float32: eval value, eval pdf, sample weight, sampled wi, sample pdf, type, flags."""
        t = np.ascontiguousarray(tuples, np.float32).reshape(-1, 9)
        out = np.zeros((t.shape[0], 13), np.float32)
        self._check(self.lib.prt_cuda_bsdf_query(self.h, C.byref(material), medium_id, t.shape[0], T.fptr(t),
                                                 T.fptr(out)))
        return out

    def init_lights(self, env):
        """Device::initLights: replaces the uploaded scene's environment lights (an EnvDesc)."""
        self._check(self.lib.prt_cuda_scene_lights(self.h, C.byref(env)))

    def microfacet_query(self, distribution, tuples):
        """(n, 4) float32: sampled microfacet normal and pdf for (alpha, s.x, s.y, wo) tuples."""
        t = np.ascontiguousarray(tuples, np.float32).reshape(-1, 6)
        out = np.zeros((t.shape[0], 4), np.float32)
        self._check(self.lib.prt_cuda_microfacet_query(self.h, distribution, t.shape[0], T.fptr(t), T.fptr(out)))
        return out

    def set_albedo_tables(self, tables):
        """Replaces the context's energy-compensation tables (layout of albedo_tables())."""
        t = np.ascontiguousarray(tables, np.float32)
        self._check(self.lib.prt_cuda_set_albedo_tables(self.h, T.fptr(t), t.size))

    def albedo_tables(self):
        n = C.c_int64(0)
        self._check(self.lib.prt_cuda_albedo_tables(self.h, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        self._check(self.lib.prt_cuda_albedo_tables(self.h, T.fptr(out), n.value, C.byref(n)))
        return out

    def occluded(self, rays):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        occ = np.zeros(rays.shape[0], np.int32)
        self._check(self.lib.prt_cuda_occluded(self.h, rays.shape[0], T.fptr(rays), T.iptr(occ)))
        return occ

    def query_primary(self, sample_index):
        n = self.width * self.height
        rays = np.zeros((n, 8), np.float32)
        g = np.zeros(n, np.int32)
        p = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        self._check(self.lib.prt_cuda_query_primary(self.h, sample_index, T.fptr(rays), T.iptr(g), T.iptr(p),
                                                    T.fptr(t)))
        return rays, g, p, t


class Batch:
    """Many frames rendered in one persistent wavefront (prt_cuda_batch_*).

    `frames` is a list of (Scene, seed, aov_mask); each Scene carries its own width, height,
    spp, max_depth, rr_depth and camera.
    """

    def __init__(self, device, frames):
        self.dev = device
        self.frames = [(sc, seed, aov) for sc, seed, aov in frames]
        descs = [sc.desc() for sc, _, _ in self.frames]
        items = (T.BatchItem * len(descs))()
        for k, ((sc, seed, aov), d) in enumerate(zip(self.frames, descs)):
            it = items[k]
            it.scene = C.pointer(d)
            it.camera = sc.camera
            it.renderer = T.RendererDesc(sc.max_depth, sc.rr_depth, 1e-4, 3.4028234663852886e38, T.PRT_RENDERER_PATH, 16)
            it.width, it.height, it.spp, it.aov_mask, it.seed = sc.width, sc.height, sc.spp, aov, seed
        h = C.c_void_p()
        device._check(device.lib.prt_cuda_batch_create(device.h, items, len(descs), C.byref(h)))
        self.h = h
        if not hasattr(device, "_batches"):
            device._batches = weakref.WeakSet()
        device._batches.add(self)
        self.samples = sum(sc.width * sc.height * sc.spp for sc, _, _ in self.frames)

    def render(self):
        st = T.RenderStats()
        self.dev._check(self.dev.lib.prt_cuda_batch_render(self.h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in T.RenderStats._fields_}

    def blit(self, item, aov=T.PRT_BLIT_HDR, out=None):
        """(height, width, 3) float32 of one item; `out` may be a CUDA torch tensor (zero copy)."""
        if out is not None and hasattr(out, "data_ptr"):
            self.dev._check(self.dev.lib.prt_cuda_batch_blit(self.h, item, aov,
                                                             C.cast(C.c_void_p(out.data_ptr()), C.POINTER(C.c_float))))
            return out
        sc = self.frames[item][0]
        img = np.zeros((sc.height, sc.width, 3), np.float32)
        self.dev._check(self.dev.lib.prt_cuda_batch_blit(self.h, item, aov, T.fptr(img)))
        return img

    # -- differentiation ---------------------------------------------------------------------
    def enable_adjoint(self):
        """Later renders also keep each pixel-sample's radiance for adjoint()."""
        self.dev._check(self.dev.lib.prt_cuda_batch_enable_adjoint(self.h))

    def adjoint(self, d_loss_d_images, grad_textures, grad_roughness):
        """Path-replay adjoint of the last render for every item at once. Arguments are lists
        (one entry per item) of CUDA torch tensors: dLoss/dImage (h, w, 3), the concatenated
        texture gradients, the per-material roughness gradients (written)."""
        n = len(self.frames)
        ptr = DeviceCuda._ptr
        dl = (C.c_void_p * n)(*[ptr(x.contiguous()) for x in d_loss_d_images])
        gt = (C.c_void_p * n)(*[ptr(x) for x in grad_textures])
        gr = (C.c_void_p * n)(*[ptr(x) for x in grad_roughness])
        st = T.RenderStats()
        self.dev._check(self.dev.lib.prt_cuda_batch_adjoint(self.h, dl, gt, gr, C.byref(st)))
        return {name: getattr(st, name) for name, _ in T.RenderStats._fields_}

    def update_texture(self, item, texture, rgb):
        if not hasattr(rgb, "data_ptr"):
            rgb = np.ascontiguousarray(rgb, np.float32)
        self.dev._check(self.dev.lib.prt_cuda_batch_update_texture(self.h, item, texture, DeviceCuda._ptr(rgb)))

    def update_material(self, item, material, m):
        self.dev._check(self.dev.lib.prt_cuda_batch_update_material(self.h, item, material, C.byref(m)))

    def update_materials(self, item, first, materials):
        arr = (T.Material * len(materials))(*materials)
        self.dev._check(self.dev.lib.prt_cuda_batch_update_materials(self.h, item, first, len(materials), arr))

    def close(self):
        # A batch lives inside its device's context: destroy it first (DeviceCuda.close does).
        if getattr(self, "h", None) and getattr(self.dev, "h", None):
            self.dev.lib.prt_cuda_batch_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

