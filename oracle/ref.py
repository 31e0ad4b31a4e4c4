"""Test infrastructure: Python handle on the oracle libraries.

* RefDevice wraps oracle/_ref/libprt_ref.so, the reference's own C++ path tracer
  (DeviceCpu + PathRendererStream + SobolBurleySamplerSimd) compiled from its sources by
  oracle/Makefile, with the oracle BVH in place of Embree.
* restate() loads oracle/_ref/libprt_oracle.so, the plain-C restatement in oracle/restate.

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this module.
"""
import ctypes as C
import os
import pathlib
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oidn-protoray_b200"))
import prt_types as T  # noqa: E402

REF_LIB = ROOT / "oracle" / "_ref" / "libprt_ref.so"
RESTATE_LIB = ROOT / "oracle" / "_ref" / "libprt_oracle.so"

_ref = None


def ref_available():
    return REF_LIB.exists()


def _lib():
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} is not built (make -C oracle)")
        # libstdc++ must be in the global symbol scope before a C++ library is loaded;
        # when an RTLD_LOCAL extension (numpy) loaded it first, the library's own copies of
        # vague-linkage statics (std::locale::id) would shadow libstdc++'s and break iostreams.
        C.CDLL("libstdc++.so.6", mode=os.RTLD_GLOBAL)
        lib = C.CDLL(str(REF_LIB))
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_create.argtypes = [C.POINTER(T.SceneDesc), C.POINTER(T.CameraDesc), C.POINTER(T.RendererDesc),
                                   C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_char_p, C.POINTER(C.c_float),
                                   C.POINTER(C.c_void_p)]
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_init_sampler.argtypes = [C.c_void_p, C.c_uint32]
        lib.ref_clear.argtypes = [C.c_void_p]
        lib.ref_render.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        lib.ref_blit.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float)]
        lib.ref_sobol.argtypes = [C.c_uint32, C.c_int64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint32), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        lib.ref_trace.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_float)]
        lib.ref_occluded.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_int32)]
        lib.ref_query_primary.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32), C.POINTER(C.c_float)]
        _ref = lib
    return _ref


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + _lib().ref_last_error().decode())


def sunsky(direction, turbidity, albedo):
    """The reference's sun-sky products: (sun radiance, sun angular diameter, sky image)."""
    lib = _lib()
    P = C.POINTER(C.c_float)
    d = np.ascontiguousarray(direction, np.float32)
    sun = np.zeros(3, np.float32)
    ang = C.c_float()
    w, h = C.c_int(), C.c_int()
    lib.ref_sunsky.argtypes = [P, C.c_float, C.c_float, P, P, P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    _check(lib.ref_sunsky(T.fptr(d), turbidity, albedo, T.fptr(sun), C.byref(ang), None, C.byref(w), C.byref(h)))
    sky = np.zeros((h.value, w.value, 3), np.float32)
    _check(lib.ref_sunsky(T.fptr(d), turbidity, albedo, T.fptr(sun), C.byref(ang), T.fptr(sky), C.byref(w),
                          C.byref(h)))
    return sun, ang.value, sky


def bsdf_query(material, tuples, medium_id=0):
    """The reference's Standard material BSDF on (wo, wi, sample) tuples: (n, 13) float32."""
    lib = _lib()
    t = np.ascontiguousarray(tuples, np.float32).reshape(-1, 9)
    out = np.zeros((t.shape[0], 13), np.float32)
    lib.ref_bsdf_query.argtypes = [C.POINTER(T.Material), C.c_int, C.c_int64, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float)]
    if lib.ref_bsdf_query(C.byref(material), medium_id, t.shape[0], T.fptr(t), T.fptr(out)) != 0:
        raise RuntimeError("oracle BSDF query failed")
    return out


def bsdf_query_scalar(material, tuples, medium_id=0, frame=None):
    """The same query through the reference's scalar BSDF path (Bsdf rather than BsdfSimd).
    `frame`: the shading frame U, V, N and the geometric normal Ng (12 floats); default the
    canonical frame (x, y, z, z)."""
    lib = _lib()
    t = np.ascontiguousarray(tuples, np.float32).reshape(-1, 9)
    out = np.zeros((t.shape[0], 13), np.float32)
    if frame is None:
        frame = [1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 1]
    f = np.ascontiguousarray(frame, np.float32).reshape(12)
    lib.ref_bsdf_query_scalar_frame.argtypes = [C.POINTER(T.Material), C.c_int, C.POINTER(C.c_float), C.c_int64,
                                                C.POINTER(C.c_float), C.POINTER(C.c_float)]
    if lib.ref_bsdf_query_scalar_frame(C.byref(material), medium_id, T.fptr(f), t.shape[0], T.fptr(t),
                                       T.fptr(out)) != 0:
        raise RuntimeError("oracle scalar BSDF query failed")
    return out


def microfacet_query(distribution, tuples, simd=True):
    """The reference's BeckmannDistribution::sample / GGXDistribution::sampleVisible on
    (alpha, s.x, s.y, wo) tuples: (n, 4) float32 (m, pdf); SIMD or scalar instantiation."""
    lib = _lib()
    t = np.ascontiguousarray(tuples, np.float32).reshape(-1, 6)
    out = np.zeros((t.shape[0], 4), np.float32)
    lib.ref_microfacet_query.argtypes = [C.c_int, C.c_int, C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    _check(lib.ref_microfacet_query(distribution, 1 if simd else 0, t.shape[0], T.fptr(t), T.fptr(out)))
    return out


def albedo_tables():
    lib = _lib()
    lib.ref_albedo_tables.restype = C.c_int64
    lib.ref_albedo_tables.argtypes = [C.POINTER(C.c_float)]
    n = lib.ref_albedo_tables(None)
    out = np.zeros(n, np.float32)
    lib.ref_albedo_tables(T.fptr(out))
    return out


def hardware_threads():
    return _lib().ref_hardware_threads()


def sobol(seed, sample_index, pixel_id, dim_set, dims):
    """Sobol-Burley draws through the reference's SIMD sampler and its scalar functions."""
    n = len(sample_index)
    si = np.ascontiguousarray(sample_index, np.uint32)
    pi = np.ascontiguousarray(pixel_id, np.uint32)
    ds = np.ascontiguousarray(dim_set, np.uint32)
    out_simd = np.zeros(n * dims, np.float32)
    out_scalar = np.zeros(n * dims, np.float32)
    _check(_lib().ref_sobol(seed, n, T.uptr(si), T.uptr(pi), T.uptr(ds), dims,
                            T.fptr(out_simd), T.fptr(out_scalar)))
    return out_simd.reshape(n, dims), out_scalar.reshape(n, dims)


def write_rkscene(scene, directory):
    """Writes `scene` with the reference's own rkscene::save (textures as PFM beside it) and
    returns the .rkscene path."""
    lib = _lib()
    lib.ref_write_rkscene.argtypes = [C.POINTER(T.SceneDesc), C.c_char_p, C.c_char_p, C.c_int]
    desc = scene.desc(oracle=True)
    out = C.create_string_buffer(4096)
    _check(lib.ref_write_rkscene(C.byref(desc), str(directory).encode(), out, 4096))
    return out.value.decode()


class RefDevice:
    """The reference's DeviceCpu running pathStream/sobolBurley on a Scene."""

    def __init__(self, scene, seed=0, aov_mask=0, sunsky=None, scene_path=None):
        """`scene_path` (a .rkscene or .mesh file) makes the reference load that file itself;
        the camera, frame, renderer and lights still come from `scene`."""
        self.scene = scene
        self.desc = scene.desc(oracle=True)
        self.rdesc = scene.renderer_desc()
        self.tmp = tempfile.TemporaryDirectory(prefix="prt_oracle_")
        ss = None
        if scene.sunsky is not None or sunsky is not None:
            ss_arr = np.asarray(sunsky if sunsky is not None else scene.sunsky, np.float32)
            self._ss = ss_arr
            ss = T.fptr(ss_arr)
        h = C.c_void_p()
        lib = _lib()
        lib.ref_create_file.argtypes = [C.c_char_p] + list(lib.ref_create.argtypes)
        _check(lib.ref_create_file(None if scene_path is None else str(scene_path).encode(), C.byref(self.desc),
                                   C.byref(scene.camera), C.byref(self.rdesc), scene.width, scene.height, aov_mask,
                                   seed, self.tmp.name.encode(), ss, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            _lib().ref_destroy(self.h)
            self.h = None
            self.tmp.cleanup()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_sampler(self, seed):
        _check(_lib().ref_init_sampler(self.h, seed))

    def clear(self):
        _check(_lib().ref_clear(self.h))

    def render(self, spp):
        st = (C.c_double * 2)()
        _check(_lib().ref_render(self.h, spp, st))
        return dict(rays=st[0], seconds=st[1])

    def blit(self, aov=T.PRT_BLIT_HDR):
        if aov == T.PRT_BLIT_LDR:
            out = np.zeros((self.scene.height, self.scene.width), np.uint32)
            _check(_lib().ref_blit(self.h, aov, out.ctypes.data_as(C.POINTER(C.c_float))))
            return out
        out = np.zeros((self.scene.height, self.scene.width, 3), np.float32)
        _check(_lib().ref_blit(self.h, aov, T.fptr(out)))
        return out

    def tone_mapper(self, kind, exposure=1.0, burn=0.0):
        _lib().ref_tone_mapper.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_float]
        _check(_lib().ref_tone_mapper(self.h, kind, exposure, burn))

    def frame_error(self):
        e = C.c_float()
        _lib().ref_frame_error.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
        _check(_lib().ref_frame_error(self.h, C.byref(e)))
        return e.value

    def trace(self, rays):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        g = np.zeros(n, np.int32)
        p = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        _check(_lib().ref_trace(self.h, n, T.fptr(rays), T.iptr(g), T.iptr(p), T.fptr(t), T.fptr(u), T.fptr(v)))
        return g, p, t, u, v

    def occluded(self, rays):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        occ = np.zeros(rays.shape[0], np.int32)
        _check(_lib().ref_occluded(self.h, rays.shape[0], T.fptr(rays), T.iptr(occ)))
        return occ

    def query_primary(self, sample_index):
        n = self.scene.width * self.scene.height
        rays = np.zeros((n, 8), np.float32)
        g = np.zeros(n, np.int32)
        p = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        _check(_lib().ref_query_primary(self.h, sample_index, T.fptr(rays), T.iptr(g), T.iptr(p), T.fptr(t)))
        return rays, g, p, t
