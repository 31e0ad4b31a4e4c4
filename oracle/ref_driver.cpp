// Test infrastructure: the oracle driver. It is compiled together with the reference's
// own sources (oracle/Makefile) into oracle/_ref/libprt_ref.so and is loaded only by the
// tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the
// product.
//
// It turns the flat scene description of include/prt_cuda.h into an rkscene file
// (rkscene/rkscene.h:161-261), loads it through the reference's DeviceCpu
// (render/device_cpu.cpp:96) exactly as the reference application does, and drives the
// reference's "pathStream" renderer with the "sobolBurley" sampler
// (render/renderer_factory_stream.cpp:17-76). Every entry point returns 0 on success or a
// negative code, with the message in ref_last_error().
#define RKSCENE_FLOAT2   prt::Vec2f
#define RKSCENE_FLOAT3   prt::Vec3f
#define RKSCENE_FLOAT4   prt::Vec4f
#define RKSCENE_FLOAT3X4 prt::Affine3f

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <memory>
#include <string>
#include <vector>

#include "math/vec2.h"
#include "math/vec3.h"
#include "math/vec4.h"
#include "math/affine3.h"
#include "render/device_cpu.h"
#include "render/scene.h"
#include "camera/pinhole_camera.h"
#include "sampling/sobol_burley.h"
#include "sampling/sobol_burley_sampler_simd.h"
#include "image/image_io.h"
#include "image/morton.h"
#include "image/surface.h"
#include "bsdf/albedo_tables.h"
#include "accel/embree_intersector_stream.h"
#include "render/integrator.h"
#include "rkscene/rkscene.h"

#include "../include/prt_cuda.h"

using namespace prt;

namespace {

thread_local std::string g_lastError;

int fail(const std::string& msg, int code = -1)
{
  g_lastError = msg;
  return code;
}

struct RefHandle
{
  DeviceCpu device;
  Vec2i size;
  std::string dir;
  std::string scenePath;
  Props sceneProps;
  std::shared_ptr<Scene> queryScene;                // loaded on first ray query
  std::shared_ptr<OracleIntersectorBase> tracer;    // for ray queries outside the renderer
  std::shared_ptr<PinholeCamera> camera;
  uint32_t seed = 0;
};

void writePfm(const std::string& path, const float* rgb, int w, int h)
{
  ImageIo::Desc desc;
  desc.size = Vec2i(w, h);
  desc.format = PixelFormat::Rgb32f;
  if (!ImageIo::save(path, desc, rgb))
    throw std::runtime_error("cannot write " + path);
}

Vec3f v3(const float* p) { return Vec3f(p[0], p[1], p[2]); }

Props cameraProps(const prt_camera_desc* cam, int w, int h)
{
  Props p;
  p.set("type", "pinhole");
  p.set("position", v3(cam->position));
  p.set("basis", Basis3f(v3(cam->basis_u), v3(cam->basis_v), v3(cam->basis_n)));
  p.set("fov", cam->fov);
  p.set("nearClip", cam->near_clip);
  p.set("width", w);
  p.set("height", h);
  return p;
}

// Writes the rkscene (and PFM textures) describing `s` into `dir`; returns the scene path.
std::string writeScene(const prt_scene_desc* s, const std::string& dir)
{
  rkscene::Scene scene;
  scene.name = "oracle";
  for (int i = 0; i < s->texture_count; ++i)
    writePfm(dir + "/tex" + std::to_string(i) + ".pfm", s->textures[i].rgb, s->textures[i].width, s->textures[i].height);
  for (int i = 0; i < s->material_count; ++i)
  {
    const prt_material& m = s->materials[i];
    auto mat = std::make_shared<rkscene::Material>();
    mat->name = "mat" + std::to_string(i);
    mat->baseWeight = m.base_weight;
    mat->baseColor = rkscene::Texture3f(v3(m.base_color));
    if (m.base_color_texture >= 0)
      mat->baseColor.image = "tex" + std::to_string(m.base_color_texture) + ".pfm";
    mat->metalness = m.metalness;
    mat->diffuseRoughness = m.diffuse_roughness;
    mat->specularWeight = m.specular_weight;
    mat->specularColor = rkscene::Texture3f(v3(m.specular_color));
    mat->specularRoughness = m.specular_roughness;
    mat->specularIor = m.specular_ior;
    mat->transmissionWeight = m.transmission_weight;
    mat->transmissionColor = rkscene::Texture3f(v3(m.transmission_color));
    mat->transmissionDepth = m.transmission_depth;
    mat->subsurfaceWeight = m.subsurface_weight;
    mat->subsurfaceColor = rkscene::Texture3f(v3(m.subsurface_color));
    mat->subsurfaceAnisotropy = m.subsurface_anisotropy;
    mat->coatWeight = m.coat_weight;
    mat->coatColor = rkscene::Texture3f(v3(m.coat_color));
    mat->coatRoughness = m.coat_roughness;
    mat->coatIor = m.coat_ior;
    mat->sheenWeight = m.sheen_weight;
    mat->sheenColor = rkscene::Texture3f(v3(m.sheen_color));
    mat->sheenRoughness = m.sheen_roughness;
    mat->emissionLuminance = m.emission_luminance;
    mat->emissionColor = rkscene::Texture3f(v3(m.emission_color));
    mat->thinWalled = m.thin_walled != 0;
    mat->opacity = m.opacity;
    scene.materials.push_back(mat);
  }
  for (int g = 0; g < s->mesh_count; ++g)
  {
    const prt_mesh& mesh = s->meshes[g];
    auto geom = std::make_shared<rkscene::Geometry>();
    geom->name = "mesh" + std::to_string(g);
    geom->material = mesh.material;
    geom->indices.resize((size_t)mesh.tri_count * 3);
    for (size_t i = 0; i < geom->indices.size(); ++i)
      geom->indices[i] = (uint32_t)mesh.indices[i];
    geom->positions.resize(mesh.vertex_count);
    for (int i = 0; i < mesh.vertex_count; ++i)
      geom->positions[i] = v3(mesh.positions + 3 * (size_t)i);
    if (mesh.normals)
    {
      geom->normals.resize(mesh.vertex_count);
      for (int i = 0; i < mesh.vertex_count; ++i)
        geom->normals[i] = v3(mesh.normals + 3 * (size_t)i);
    }
    if (mesh.texcoords)
    {
      geom->texcoords.resize(1);
      geom->texcoords[0].resize(mesh.vertex_count);
      for (int i = 0; i < mesh.vertex_count; ++i)
        geom->texcoords[0][i] = Vec2f(mesh.texcoords[2 * (size_t)i], mesh.texcoords[2 * (size_t)i + 1]);
    }
    scene.geometries.push_back(geom);
    auto obj = std::make_shared<rkscene::Object>();
    obj->name = geom->name;
    obj->geometries.push_back(g);
    scene.objects.push_back(obj);
  }
  const std::string path = dir + "/scene.rkscene";
  rkscene::save(scene, path);
  return path;
}

Props lightProps(const prt_scene_desc* s, const std::string& dir, const float* sunsky /* dir xyz, turbidity, albedo or null */)
{
  Props p;
  const prt_env_desc& e = s->env;
  if (e.distant_color[0] > 0.f || e.distant_color[1] > 0.f || e.distant_color[2] > 0.f)
  {
    p.set("distantLight", v3(e.distant_color));
    p.set("distantLightDir", v3(e.distant_dir));
    p.set("distantLightAngle", e.distant_angle);
  }
  if (e.ambient_color[0] > 0.f || e.ambient_color[1] > 0.f || e.ambient_color[2] > 0.f)
    p.set("ambientLight", v3(e.ambient_color));
  if (e.image_rgb)
  {
    const std::string path = dir + "/envmap.pfm";
    writePfm(path, e.image_rgb, e.image_width, e.image_height);
    p.set("imageLight", path);
    if (e.image_lut_size > 0)
      p.set("imageLightLutSize", e.image_lut_size);
  }
  if (sunsky)
  {
    p.set("sunSkyLightDir", Vec3f(sunsky[0], sunsky[1], sunsky[2]));
    p.set("sunSkyLightTurbidity", sunsky[3]);
    p.set("sunSkyLightAlbedo", sunsky[4]);
  }
  return p;
}

} // namespace

extern "C" {

const char* ref_last_error() { return g_lastError.c_str(); }

int ref_hardware_threads() { return tbb::this_task_arena::max_concurrency(); }

// Creates a DeviceCpu with the scene, camera, frame and pathStream renderer loaded.
// sunsky: NULL, or 5 floats (direction xyz, turbidity, ground albedo) for the reference's
// sun-sky light (render/scene.cpp:412-431) in addition to the env lights of the scene.
int ref_create_file(const char* scene_path, const prt_scene_desc* scene, const prt_camera_desc* cam,
                    const prt_renderer_desc* rd, int width, int height, int aov_mask, uint32_t seed,
                    const char* workdir, const float* sunsky, void** out);

int ref_create(const prt_scene_desc* scene, const prt_camera_desc* cam, const prt_renderer_desc* rd,
               int width, int height, int aov_mask, uint32_t seed, const char* workdir,
               const float* sunsky, void** out)
{
  return ref_create_file(nullptr, scene, cam, rd, width, height, aov_mask, seed, workdir, sunsky, out);
}

// The reference's DeviceCpu on a given scene file (scene_path: .rkscene or .mesh, loaded by the
// reference's own Scene::Scene), or, with scene_path null, on `scene` written as an rkscene; the
// lights always come from `scene`'s environment description.
int ref_create_file(const char* scene_path, const prt_scene_desc* scene, const prt_camera_desc* cam,
                    const prt_renderer_desc* rd, int width, int height, int aov_mask, uint32_t seed,
                    const char* workdir, const float* sunsky, void** out)
{
  try
  {
    auto h = std::make_unique<RefHandle>();
    h->dir = workdir;
    std::filesystem::create_directories(h->dir);
    const std::string path = scene_path ? std::string(scene_path) : writeScene(scene, h->dir);
    h->scenePath = path;
    h->sceneProps = lightProps(scene, h->dir, sunsky);
    h->device.initScene(path, h->sceneProps);
    h->device.initCamera(cameraProps(cam, width, height));
    h->camera = std::make_shared<PinholeCamera>(cameraProps(cam, width, height));
    Props frameProps;
    if (aov_mask & PRT_AOV_ALBEDO1) frameProps.set("aovAlbedo1");
    if (aov_mask & PRT_AOV_NORMAL1) frameProps.set("aovNormal1");
    if (aov_mask & PRT_AOV_HDR_VAR) frameProps.set("aovHdrVar");
    if (aov_mask & PRT_AOV_SH) frameProps.set("aovSh");
    h->size = Vec2i(width, height);
    h->device.initFrame(h->size, frameProps);
    Props rprops;
    static const char* kTypes[] = {"pathStream",        "primaryStream",     "aoStream",
                                   "diffuseStream",     "diffuse2Stream",    "primaryStreamFast",
                                   "aoStreamFast",      "diffuseStreamFast", "diffuse2StreamFast"};
    rprops.set("type", kTypes[(rd->type >= 0 && rd->type <= 8) ? rd->type : 0]);
    rprops.set("samples", rd->samples > 0 ? rd->samples : 16);
    rprops.set("sampler", "sobolBurley");
    rprops.set("maxDepth", rd->max_depth);
    rprops.set("rrDepth", rd->rr_depth);
    rprops.set("minWeight", rd->min_weight);
    rprops.set("maxRadiance", rd->max_radiance);
    rprops.set("imageSize", Vec2i(width, height));
    if (rd->flags & PRT_RENDERER_IRRADIANCE) rprops.set("irradiance");
    Props stats;
    h->device.initRenderer(rprops, stats);
    h->device.initSampler(seed);
    h->seed = seed;
    h->device.clearFrame();
    *out = h.release();
    return 0;
  }
  catch (const std::exception& e)
  {
    return fail(e.what());
  }
}

// The scene written by the reference's own rkscene::save (rkscene/rkscene.h:907-941) into
// `dir`; the path of the .rkscene file goes to path_out (capacity bytes).
int ref_write_rkscene(const prt_scene_desc* scene, const char* dir, char* path_out, int capacity)
{
  try
  {
    const std::string path = writeScene(scene, dir);
    if (!path_out || capacity <= (int)path.size()) return -1;
    std::memcpy(path_out, path.c_str(), path.size() + 1);
    return 0;
  }
  catch (const std::exception&)
  {
    return -1;
  }
}

int ref_destroy(void* handle)
{
  delete (RefHandle*)handle;
  return 0;
}

int ref_init_sampler(void* handle, uint32_t seed)
{
  auto h = (RefHandle*)handle;
  h->device.initSampler(seed);
  h->seed = seed;
  return 0;
}

int ref_clear(void* handle)
{
  ((RefHandle*)handle)->device.clearFrame();
  return 0;
}

// Runs spp frames (one Device::render call per sample, render/device_cpu.cpp:53-59).
// stats (optional): [rays, seconds] summed over the calls.
int ref_render(void* handle, int spp, double* stats)
{
  try
  {
    auto h = (RefHandle*)handle;
    double rays = 0.0, seconds = 0.0;
    for (int i = 0; i < spp; ++i)
    {
      Props st;
      auto t0 = std::chrono::steady_clock::now();
      h->device.render(st);
      auto t1 = std::chrono::steady_clock::now();
      seconds += std::chrono::duration<double>(t1 - t0).count();
      rays += (double)st.get<int64_t>("ray");
    }
    if (stats)
    {
      stats[0] = rays;
      stats[1] = seconds;
    }
    return 0;
  }
  catch (const std::exception& e)
  {
    return fail(e.what());
  }
}

// Device::blitFrame for one AOV (PRT_BLIT_*), width*height*3 floats.
int ref_blit(void* handle, int aov, float* dst)
{
  try
  {
    auto h = (RefHandle*)handle;
    FrameAovs aovs;
    std::vector<Vec3f> hdr((size_t)h->size.x * h->size.y);
    if (aov == PRT_BLIT_LDR)
    {
      // blitLdr stores whole SIMD vectors: give it a 64-byte aligned surface.
      const size_t bytes = (size_t)h->size.x * h->size.y * sizeof(int);
      void* aligned = std::aligned_alloc(64, (bytes + 63) / 64 * 64);
      Surface surface{aligned, h->size.x, h->size.y, (int)(h->size.x * sizeof(int))};
      h->device.blitFrame(surface);
      std::memcpy(dst, aligned, bytes);
      std::free(aligned);
      return 0;
    }
    if (aov == PRT_BLIT_HDR) aovs.hdr = (Vec3f*)dst;
    else if (aov == PRT_BLIT_ALBEDO1) aovs.albedo1 = (Vec3f*)dst;
    else if (aov == PRT_BLIT_NORMAL1) aovs.normal1 = (Vec3f*)dst;
    else if (aov == PRT_BLIT_HDR_VAR)
    {
      aovs.hdr = hdr.data();
      aovs.hdrVar = (Vec3f*)dst;
    }
    else if (aov == PRT_BLIT_LDR_RGB) aovs.ldr = (Vec3f*)dst;
    else if (aov >= PRT_BLIT_SH0 && aov <= PRT_BLIT_SH3)
    {
      // sh[1..3] are written relative to sh[0], so all four are blitted together.
      std::vector<Vec3f> sh[4];
      for (int k = 0; k < 4; ++k)
      {
        sh[k].resize((size_t)h->size.x * h->size.y);
        aovs.sh[k] = sh[k].data();
      }
      h->device.blitFrame(aovs);
      std::memcpy(dst, sh[aov - PRT_BLIT_SH0].data(), sizeof(Vec3f) * sh[0].size());
      return 0;
    }
    else return fail("invalid aov");
    h->device.blitFrame(aovs);
    return 0;
  }
  catch (const std::exception& e)
  {
    return fail(e.what());
  }
}

// Sobol-Burley samples through both the SIMD sampler the stream renderer uses
// (sampling/sobol_burley_sampler_simd.h) and the scalar functions (sampling/sobol_burley.h).
int ref_sobol(uint32_t seed, int64_t n, const uint32_t* sampleIndex, const uint32_t* pixelId,
              const uint32_t* dimSet, int dims, float* outSimd, float* outScalar)
{
  if (dims < 1 || dims > 3) return fail("dims must be 1, 2 or 3");
  SobolBurleySamplerSimd<false> sampler;
  sampler.init(0, 0, seed);
  for (int64_t base = 0; base < n; base += simdSize)
  {
    // One SIMD batch per simdSize queries: lanes share the dimension set of lane 0
    // only if equal, so evaluate lane by lane with a full active mask.
    for (int64_t i = base; i < std::min<int64_t>(n, base + simdSize); ++i)
    {
      SobolBurleySamplerSimd<false>::State st;
      sampler.setSample(vbool(one), st, vuint(sampleIndex[i]), vuint(pixelId[i]));
      if (dims == 1)
      {
        vfloat r = sampler.get1D(vbool(one), st, dimSet[i]);
        outSimd[i] = r[0];
      }
      else if (dims == 2)
      {
        Vec2vf r = sampler.get2D(vbool(one), st, dimSet[i]);
        outSimd[2 * i] = r.x[0];
        outSimd[2 * i + 1] = r.y[0];
      }
      else
      {
        Vec3vf r = sampler.get3D(vbool(one), st, dimSet[i]);
        outSimd[3 * i] = r.x[0];
        outSimd[3 * i + 1] = r.y[0];
        outSimd[3 * i + 2] = r.z[0];
      }
      if (outScalar)
      {
        uint32_t scramble = murmurHash3Finalize(murmurHash3Mix(seed, pixelId[i]));
        if (dims == 1)
          outScalar[i] = sobolBurleySample1D(sampleIndex[i], dimSet[i], scramble, 0xffffffffu);
        else if (dims == 2)
        {
          Vec2f r = sobolBurleySample2D(sampleIndex[i], dimSet[i], scramble, 0xffffffffu);
          outScalar[2 * i] = r.x;
          outScalar[2 * i + 1] = r.y;
        }
        else
        {
          Vec3f r = sobolBurleySample3D(sampleIndex[i], dimSet[i], scramble, 0xffffffffu);
          outScalar[3 * i] = r.x;
          outScalar[3 * i + 1] = r.y;
          outScalar[3 * i + 2] = r.z;
        }
      }
    }
  }
  return 0;
}

namespace {
OracleIntersectorBase* tracerOf(RefHandle* h)
{
  if (!h->tracer)
  {
    Props st;
    h->queryScene = std::make_shared<Scene>(h->scenePath, h->sceneProps);
    h->tracer = std::make_shared<OracleIntersectorBase>(h->queryScene->geometry, false, Props(), st);
  }
  return h->tracer.get();
}
} // namespace

// Closest hits of n rays (8 floats each: org, near, dir, far) with the oracle BVH.
int ref_trace(void* handle, int64_t n, const float* rays, int32_t* geomId, int32_t* primId, float* t, float* u, float* v)
{
  try
  {
    const oracle_bvh::Bvh& bvh = tracerOf((RefHandle*)handle)->getBvh();
    tbb::parallel_for(tbb::blocked_range<int64_t>(0, n), [&](const tbb::blocked_range<int64_t>& r) {
      for (int64_t i = r.begin(); i != r.end(); ++i)
      {
        const float* ray = rays + 8 * i;
        const float o[3] = {ray[0], ray[1], ray[2]};
        const float d[3] = {ray[4], ray[5], ray[6]};
        float tf = ray[7], uu = 0.f, vv = 0.f;
        int ti = bvh.intersect(o, d, ray[3], tf, uu, vv);
        geomId[i] = ti >= 0 ? bvh.tris[ti].geomId : -1;
        primId[i] = ti >= 0 ? bvh.tris[ti].primId : -1;
        t[i] = tf;
        if (u) u[i] = uu;
        if (v) v[i] = vv;
      }
    });
    return 0;
  }
  catch (const std::exception& e)
  {
    return fail(e.what());
  }
}

int ref_occluded(void* handle, int64_t n, const float* rays, int32_t* occluded)
{
  try
  {
    const oracle_bvh::Bvh& bvh = tracerOf((RefHandle*)handle)->getBvh();
    tbb::parallel_for(tbb::blocked_range<int64_t>(0, n), [&](const tbb::blocked_range<int64_t>& r) {
      for (int64_t i = r.begin(); i != r.end(); ++i)
      {
        const float* ray = rays + 8 * i;
        const float o[3] = {ray[0], ray[1], ray[2]};
        const float d[3] = {ray[4], ray[5], ray[6]};
        occluded[i] = bvh.occluded(o, d, ray[3], ray[7]) ? 1 : 0;
      }
    });
    return 0;
  }
  catch (const std::exception& e)
  {
    return fail(e.what());
  }
}

// Primary rays of one sample for every pixel, generated with the stream renderer's own
// sequence (render/path_renderer_stream.h:218-256: Morton 8x8 order inside 32-wide tiles,
// pixelId = x | y << 16, setSample, pixel sample from dimension set 0, lens from set 2,
// PinholeCamera::getRay SIMD form), then traced with the oracle BVH.
// rays_out: width*height*8 floats in row-major pixel order.
int ref_query_primary(void* handle, uint32_t sampleIndex, float* raysOut, int32_t* geomId, int32_t* primId, float* t)
{
  try
  {
    auto h = (RefHandle*)handle;
    const int W = h->size.x, H = h->size.y;
    SobolBurleySamplerSimd<false> sampler;
    sampler.init(0, 0, h->seed);
    const Vec2f invSize = rcp(toFloat(h->size));
    for (int y = 0; y < H; ++y)
    {
      for (int x0 = 0; x0 < W; x0 += simdSize)
      {
        Vec2vi pixel(vint(step) + x0, vint(y));
        vint pixelId = pixel.x | (pixel.y << 16);
        SobolBurleySamplerSimd<false>::State st;
        sampler.setSample(vbool(one), st, vuint(sampleIndex), vuint(pixelId));
        Vec2vf pixelSample = sampler.get2D(vbool(one), st, IntegratorBase::sampleDimPixel);
        CameraSampleSimd cs;
        cs.image = (toFloat(pixel) + pixelSample) * Vec2vf(invSize);
        cs.lens = sampler.get2D(vbool(one), st, IntegratorBase::sampleDimLens);
        RaySimd ray;
        h->camera->getRay(ray, cs);
        for (int k = 0; k < simdSize && x0 + k < W; ++k)
        {
          float* r = raysOut + 8 * ((int64_t)y * W + x0 + k);
          r[0] = ray.org.x[k]; r[1] = ray.org.y[k]; r[2] = ray.org.z[k]; r[3] = ray.near[k];
          r[4] = ray.dir.x[k]; r[5] = ray.dir.y[k]; r[6] = ray.dir.z[k]; r[7] = ray.far[k];
        }
      }
    }
    return ref_trace(handle, (int64_t)W * H, raysOut, geomId, primId, t, nullptr, nullptr);
  }
  catch (const std::exception& e)
  {
    return fail(e.what());
  }
}

int ref_tone_mapper(void* handle, int type, float exposure, float burn)
{
  auto* h = static_cast<RefHandle*>(handle);
  try
  {
    static const char* kTypes[] = {"none", "linear", "reinhard", "aces", "filmic", "log"};
    Props p;
    p.set("type", std::string(kTypes[(type >= 0 && type <= 5) ? type : 0]));
    p.set("exposure", exposure);
    p.set("burn", burn);
    h->device.initToneMapper(p);
    return 0;
  }
  catch (const std::exception& e)
  {
    return fail(e.what());
  }
}

int ref_frame_error(void* handle, float* error)
{
  auto* h = static_cast<RefHandle*>(handle);
  try
  {
    *error = h->device.getFrameError();
    return 0;
  }
  catch (const std::exception& e)
  {
    return fail(e.what());
  }
}

} // extern "C"
