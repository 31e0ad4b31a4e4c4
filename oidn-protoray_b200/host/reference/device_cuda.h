// The B200 render device as a device of the reference renderer: prt::DeviceCuda derives the
// reference's prt::Device (render/device.h:56-114) beside prt::DeviceCpu
// (render/device_cpu.cpp:20-366) and forwards every call to the C ABI in prt_cuda.h.
//
// This file belongs in the reference's tree as render/device_cuda.h, compiled with the rest of
// render/ and linked with libprt_cuda.so; main/render/render.cpp then selects it for
// `-dev cuda` (see the device selection at main/render/render.cpp:233-241). It reads the
// parameters of the reference's own light objects through four accessors that the integration
// adds to light/distant_light.h and light/image_light.h (reference_light_accessors/*.inc, one
// block each, inserted at the start of the classes' public section).
//
// Behaviour that differs from DeviceCpu, each reported with the reference's exception types:
// * renderer types: pathStream (with its irradiance option), primaryStream, aoStream,
//   diffuseStream, diffuse2Stream and their ...Fast variants (render/renderer_factory_stream.cpp:
//   54-71); the sampler is sobolBurley; other types and samplers, and the static option, are
//   std::invalid_argument;
// * frame AOVs: hdr, hdrVar, ldr, albedo1, normal1, sh; requesting another AOV in initFrame is
//   std::invalid_argument; pixel filters other than box are std::invalid_argument;
// * lights: at most one distant light and one image light reach the device, so a
//   distantLight together with a sunSkyLight (two distant lights), or an imageLight together
//   with a sunSkyLight (two image lights), is std::invalid_argument;
// * queryPixel, the host-side blitFrameLdr/blitFrameHdr conversions and jitter are not part of
//   the device: std::logic_error (jitter: none);
// * motion cameras (initCamera with previous and next props) render with the current camera.
#pragma once

#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "render/device.h"
#include "bsdf/albedo_tables.h"
#include "camera/pinhole_camera.h"
#include "image/image_texture.h"
#include "light/distant_light.h"
#include "light/image_light.h"
#include "light/sun_sky_light.h"
#include "prt_cuda.h"

namespace prt {

// The environment lights of Scene::initLights (render/scene.cpp:365-450) as the device takes
// them: built by the reference's own light classes from the same Props keys, then read back.
// `image` owns the image light's pixels (top row first); env.image_rgb points into it.
struct CudaEnvLights
{
  prt_env_desc env;
  std::vector<float> image;

  CudaEnvLights() { std::memset(&env, 0, sizeof(env)); }
  CudaEnvLights(const CudaEnvLights&) = delete;
  CudaEnvLights& operator=(const CudaEnvLights&) = delete;
};

inline void cudaSetDistantLight(prt_env_desc& e, const DistantLight& light)
{
  const Vec3f c = light.getColor(), d = light.getDirection();
  const float color[3] = {c.x, c.y, c.z}, dir[3] = {d.x, d.y, d.z};
  std::copy(color, color + 3, e.distant_color);
  std::copy(dir, dir + 3, e.distant_dir);
  e.distant_angle = light.getAngle();
}

// The image light's texture, which the reference stores bottom row first, as an image whose
// row 0 is the top; the LUT size that reproduces the light's sampling distribution.
inline void cudaSetImageLight(CudaEnvLights& out, const ImageLight& light)
{
  const std::shared_ptr<ImageTexture>& tex = light.getTexture();
  const Vec2i size = tex->getSize();
  out.image.assign((size_t)size.x * size.y * 3, 0.f);
  for (int y = 0; y < size.y; ++y)
    for (int x = 0; x < size.x; ++x)
    {
      const Vec3f c = tex->get3f(Vec2i(x, size.y - 1 - y));
      float* o = &out.image[3 * ((size_t)y * size.x + x)];
      o[0] = c.x;
      o[1] = c.y;
      o[2] = c.z;
    }
  const Vec2i lut = light.getLutSize();
  out.env.image_rgb = out.image.data();
  out.env.image_width = size.x;
  out.env.image_height = size.y;
  out.env.image_lut_size = std::max(lut.x, lut.y);
}

// Scene::initLights's keys: distantLight (+Dir, +Angle), ambientLight, imageLight
// (+LutSize), sunSkyLightDir (+Turbidity, +Albedo, +Horizon, +RadiusScale, +SunScale, +SkyScale,
// +SunSaturation, +SkySaturation, +SunHue, +SkyHue). The device computes the lights' powers (the
// light-selection weights) from its own scene bounds, so the lights are built here with a unit
// scene radius, which their parameters do not depend on.
inline void cudaEnvLightsFromProps(const Props& props, CudaEnvLights& out)
{
  std::memset(&out.env, 0, sizeof(out.env));
  out.image.clear();
  prt_env_desc& e = out.env;
  const float radius = 1.f;
  const Vec3f distantLightColor = props.get("distantLight", Vec3f(zero));
  const std::string imageLightFilename = props.get("imageLight", "");
  const Vec3f sunSkyLightDir = props.get("sunSkyLightDir", Vec3f(zero));
  if (sunSkyLightDir != Vec3f(zero) && (reduceMax(distantLightColor) > 0.0f || !imageLightFilename.empty()))
    throw std::invalid_argument("the CUDA device takes one distant and one image light: sunSkyLight cannot be "
                                "combined with distantLight or imageLight");

  if (reduceMax(distantLightColor) > 0.0f)
  {
    Props lightProps;
    lightProps.set("Ke", distantLightColor);
    if (props.exists("distantLightDir")) lightProps.set("direction", props.get<Vec3f>("distantLightDir"));
    if (props.exists("distantLightAngle")) lightProps.set("angle", props.get<float>("distantLightAngle"));
    cudaSetDistantLight(e, DistantLight(lightProps, radius));
  }

  const Vec3f ambientLightColor = props.get("ambientLight", Vec3f(zero));
  const bool ambient = reduceMax(ambientLightColor) > 0.0f;
  if (ambient)
  {
    e.ambient_color[0] = ambientLightColor.x;
    e.ambient_color[1] = ambientLightColor.y;
    e.ambient_color[2] = ambientLightColor.z;
  }

  if (!imageLightFilename.empty())
  {
    std::shared_ptr<ImageTextureBuffer> texture = loadImageTexture(imageLightFilename);
    Props lightProps;
    if (props.exists("imageLightLutSize")) lightProps.set("lutSize", props.get<int>("imageLightLutSize"));
    cudaSetImageLight(out, ImageLight(texture, lightProps, radius));
  }

  if (sunSkyLightDir != Vec3f(zero))
  {
    Props lightProps;
    lightProps.set("direction", sunSkyLightDir);
    static const char* kKeys[][2] = {
      {"sunSkyLightTurbidity", "turbidity"},         {"sunSkyLightAlbedo", "albedo"},
      {"sunSkyLightHorizon", "horizon"},             {"sunSkyLightRadiusScale", "radiusScale"},
      {"sunSkyLightSunScale", "sunScale"},           {"sunSkyLightSkyScale", "skyScale"},
      {"sunSkyLightSunSaturation", "sunSaturation"}, {"sunSkyLightSkySaturation", "skySaturation"},
      {"sunSkyLightSunHue", "sunHue"},               {"sunSkyLightSkyHue", "skyHue"}};
    for (const auto& k : kKeys)
      if (props.exists(k[0])) lightProps.set(k[1], props.get<float>(k[0]));
    const SunSkyLight sunSky(lightProps, radius);
    const auto sun = std::dynamic_pointer_cast<DistantLight>(sunSky.getSunLight());
    const auto sky = std::dynamic_pointer_cast<ImageLight>(sunSky.getSkyLight());
    if (!sun || !sky) throw std::logic_error("unexpected sun-sky light types");
    cudaSetDistantLight(e, *sun);
    cudaSetImageLight(out, *sky);
    // The reference lists an ambient light before the sun and the sky.
    if (ambient) e.flags |= PRT_ENV_AMBIENT_FIRST;
  }
}

class DeviceCuda : public Device
{
public:
  // hostTables: run on the energy-compensation tables that the reference computes on the host,
  // as DeviceCpu's constructor does (render/device_cpu.cpp:20-23), so that the compensation
  // terms -- which amplify a table's last digits by 1 / (1 - E_avg) -- match the CPU device's.
  // false keeps the tables the device builds on the GPU at creation (within ~2e-6 of these)
  // and skips the ~3 s of host integration.
  explicit DeviceCuda(int deviceOrdinal = 0, bool hostTables = true)
  {
    if (prt_cuda_create(deviceOrdinal, &ctx) != PRT_OK) throw std::runtime_error("no usable CUDA device");
    if (hostTables)
    {
      try
      {
        uploadHostTables();
      }
      catch (...)
      {
        prt_cuda_destroy(ctx);
        throw;
      }
    }
  }

  ~DeviceCuda() override
  {
    if (ctx) prt_cuda_destroy(ctx);
  }

  DeviceCuda(const DeviceCuda&) = delete;
  DeviceCuda& operator=(const DeviceCuda&) = delete;

  std::string getInfo() override { return "NVIDIA B200 (sm_100a) wavefront path tracer"; }

  // Scene: Scene::Scene reads the file and calls initLights (render/scene.cpp:65-140).
  void initScene(const std::string& path, const Props& props) override
  {
    CudaEnvLights lights;
    cudaEnvLightsFromProps(props, lights);
    const int builder = props.get("cudaBvh", std::string("host")) == "device" ? PRT_BVH_DEVICE : PRT_BVH_HOST;
    check(prt_cuda_scene_load(ctx, path.c_str(), &lights.env, builder));
  }

  Box3f getSceneBounds() override
  {
    prt_scene_stats st{};
    check(prt_cuda_scene_stats(ctx, &st));
    return Box3f(Vec3f(st.bounds_lo[0], st.bounds_lo[1], st.bounds_lo[2]),
                 Vec3f(st.bounds_hi[0], st.bounds_hi[1], st.bounds_hi[2]));
  }

  void initLights(const Props& props) override
  {
    CudaEnvLights lights;
    cudaEnvLightsFromProps(props, lights);
    check(prt_cuda_scene_lights(ctx, &lights.env));
  }

  // Renderer (DeviceCpu::initRenderer, render/device_cpu.cpp:32-46).
  void initRenderer(const Props& props, Props& stats) override
  {
    static const std::pair<const char*, int> kTypes[] = {
      {"pathStream", PRT_RENDERER_PATH},
      {"primaryStream", PRT_RENDERER_PRIMARY},           {"aoStream", PRT_RENDERER_AO},
      {"diffuseStream", PRT_RENDERER_DIFFUSE},           {"diffuse2Stream", PRT_RENDERER_DIFFUSE2},
      {"primaryStreamFast", PRT_RENDERER_PRIMARY_FAST},  {"aoStreamFast", PRT_RENDERER_AO_FAST},
      {"diffuseStreamFast", PRT_RENDERER_DIFFUSE_FAST},  {"diffuse2StreamFast", PRT_RENDERER_DIFFUSE2_FAST}};
    const std::string type = props.get("type");
    int t = -1;
    for (const auto& k : kTypes)
      if (type == k.first) t = k.second;
    if (t < 0) throw std::invalid_argument("renderer type not supported by the CUDA device: " + type);
    const std::string sampler = props.get("sampler", "sobolBurley");
    if (sampler != "sobolBurley") throw std::invalid_argument("sampler not supported by the CUDA device: " + sampler);
    if (props.exists("static")) throw std::invalid_argument("the CUDA device advances the sample index every render");
    const int flags = props.exists("irradiance") ? PRT_RENDERER_IRRADIANCE : 0;
    const prt_renderer_desc r{props.get("maxDepth", 100),          props.get("rrDepth", 8),
                              props.get("minWeight", 1e-4f),       props.get("maxRadiance", float(posMax)),
                              t,                                   props.get("samples", 16),
                              flags};
    check(prt_cuda_renderer(ctx, &r));
    samplerType = sampler;
    stats.set("device", getInfo());
  }

  void initSampler(unsigned int seed) override { check(prt_cuda_init_sampler(ctx, seed)); }

  // One sample per pixel per call and the statistics PathRendererStream::render reports
  // (render/path_renderer_stream.h:175-178).
  void render(Props& stats) override
  {
    prt_render_stats st{};
    check(prt_cuda_render(ctx, 1, &st));
    stats.set("mray", st.mray);
    stats.set("ray", (int64_t)st.rays);
    stats.set("spp", 1);
  }

  Props queryPixel(const Vec2f&) override { throw std::logic_error("queryPixel is not supported by the CUDA device"); }
  void queryPixel(const Vec2f&, Array<Props>&) override
  {
    throw std::logic_error("queryPixel is not supported by the CUDA device");
  }
  Props queryPixel(int, int) override { throw std::logic_error("queryPixel is not supported by the CUDA device"); }
  void queryPixel(int, int, Array<Props>&) override
  {
    throw std::logic_error("queryPixel is not supported by the CUDA device");
  }

  // The closest hit of one ray (RendererStream::queryRay, render/renderer_stream.h:16-60): the
  // geometric part of its answer -- hit point, distance, primitive and geometry, barycentrics.
  Props queryRay(const Ray& ray) override
  {
    const float r[8] = {ray.org.x, ray.org.y, ray.org.z, ray.near, ray.dir.x, ray.dir.y, ray.dir.z, ray.far};
    int32_t geom = -1, prim = -1;
    float t = 0.f, u = 0.f, v = 0.f;
    check(prt_cuda_trace(ctx, 1, r, &geom, &prim, &t, &u, &v));
    Props result;
    if (geom < 0) return result;
    result.set("p", ray.org + ray.dir * t);
    result.set("dist", t);
    result.set("primId", prim);
    result.set("geomId", geom);
    result.set("uv", Vec2f(u, v));
    return result;
  }

  bool queryOcclusionRay(const Ray& ray) override
  {
    const float r[8] = {ray.org.x, ray.org.y, ray.org.z, ray.near, ray.dir.x, ray.dir.y, ray.dir.z, ray.far};
    int32_t occ = 0;
    check(prt_cuda_occluded(ctx, 1, r, &occ));
    return occ != 0;
  }

  // Camera (DeviceCpu::initCamera, render/device_cpu.cpp:110-125): the pinhole camera; its
  // matrices come from the reference's own PinholeCamera.
  void initCamera(const Props& props) override
  {
    const std::string type = props.get("type", "pinhole");
    if (type != "pinhole" && props.get("lensRadius", 0.f) != 0.f)
      throw std::invalid_argument("the CUDA device renders pinhole cameras");
    camera = std::make_shared<PinholeCamera>(props);
    const Basis3f b = props.get<Basis3f>("basis");
    const Vec3f p = props.get<Vec3f>("position");
    cameraDesc = prt_camera_desc{{p.x, p.y, p.z},       {b.U.x, b.U.y, b.U.z}, {b.V.x, b.V.y, b.V.z},
                                 {b.N.x, b.N.y, b.N.z}, props.get<float>("fov"), props.get<float>("nearClip")};
    // The reference's camera carries its own raster size, so initCamera may come before
    // initFrame; the device's camera takes the frame's aspect, so it is set once a frame exists.
    if (size.x > 0) check(prt_cuda_camera(ctx, &cameraDesc));
  }

  void initCamera(const Props& props, const Props&, const Props&) override { initCamera(props); }

  Mat4f getWorldToViewD3D() override { return requireCamera().worldToViewD3D; }
  Mat4f getViewToClipD3D() override { return requireCamera().viewToClipD3D; }
  Mat4f getWorldToRaster() override { return requireCamera().worldToRaster; }

  bool hasJitter() override { return false; }
  Vec2f getJitter() override { return Vec2f(0.f); }
  void setJitter(const Vec2f&) override { throw std::logic_error("the CUDA device renders without jitter"); }
  void disableJitter() override {}

  // Framebuffer (DeviceCpu::initFrame, render/device_cpu.cpp:178-232).
  void initFrame(const Vec2i& s, const Props& props) override
  {
    static const char* kUnsupported[] = {"aovHdrUnclamp", "aovAlbedo", "aovDiffuseAlbedo", "aovDiffuseAlbedo1",
                                         "aovSpecularAlbedo", "aovSpecularAlbedo1", "aovNormal", "aovDepth",
                                         "aovHWDepth", "aovRoughness", "aovRoughness1", "aovAlpha",
                                         "aovMotionBack", "aovMotionFore"};
    for (const char* k : kUnsupported)
      if (props.exists(k)) throw std::invalid_argument(std::string("AOV not supported by the CUDA device: ") + k);
    const int aov = (props.exists("aovAlbedo1") ? PRT_AOV_ALBEDO1 : 0) |
                    (props.exists("aovNormal1") ? PRT_AOV_NORMAL1 : 0) |
                    (props.exists("aovHdrVar") ? PRT_AOV_HDR_VAR : 0) | (props.exists("aovSh") ? PRT_AOV_SH : 0);
    check(prt_cuda_frame(ctx, s.x, s.y, aov));
    size = s;
    aovMask = aov;
    if (camera) check(prt_cuda_camera(ctx, &cameraDesc));
  }

  void initFilter(const Props& props) override
  {
    filterType = props.get("filter");
    if (filterType != "box") throw std::invalid_argument("pixel filter not supported by the CUDA device: " + filterType);
  }

  void initToneMapper(const Props& props) override
  {
    static const std::pair<const char*, int> kTypes[] = {{"none", PRT_TONE_NONE},         {"linear", PRT_TONE_LINEAR},
                                                         {"reinhard", PRT_TONE_REINHARD}, {"aces", PRT_TONE_ACES},
                                                         {"filmic", PRT_TONE_FILMIC},     {"log", PRT_TONE_LOG}};
    const std::string type = props.get("type");
    int t = -1;
    for (const auto& k : kTypes)
      if (type == k.first) t = k.second;
    if (t < 0) throw std::invalid_argument("invalid tone mapper type");
    check(prt_cuda_tone_mapper(ctx, t, props.get("exposure", 1.f), props.get("burn", 0.f)));
  }

  void clearFrame() override { check(prt_cuda_clear(ctx)); }

  // The tone-mapped 8-bit image (AccumBuffer3f::blitLdr) into the surface's rows.
  void blitFrame(Surface& dest) override
  {
    std::vector<uint32_t> ldr((size_t)size.x * size.y);
    check(prt_cuda_blit(ctx, PRT_BLIT_LDR, reinterpret_cast<float*>(ldr.data())));
    for (int y = 0; y < std::min(size.y, dest.height); ++y)
      std::memcpy(dest.getRow(y), &ldr[(size_t)y * size.x], sizeof(uint32_t) * std::min(size.x, dest.width));
  }

  void blitFrame(FrameAovs& dest) override
  {
    if (dest.hdr) check(prt_cuda_blit(ctx, PRT_BLIT_HDR, &dest.hdr->x));
    if (dest.hdrVar)
    {
      if (!(aovMask & PRT_AOV_HDR_VAR)) throw std::invalid_argument("hdrVar needs aovHdrVar in initFrame");
      check(prt_cuda_blit(ctx, PRT_BLIT_HDR_VAR, &dest.hdrVar->x));
    }
    if (dest.ldr) check(prt_cuda_blit(ctx, PRT_BLIT_LDR_RGB, &dest.ldr->x));
    if (dest.albedo1) check(prt_cuda_blit(ctx, PRT_BLIT_ALBEDO1, &dest.albedo1->x));
    if (dest.normal1) check(prt_cuda_blit(ctx, PRT_BLIT_NORMAL1, &dest.normal1->x));
    for (int k = 0; k < 4; ++k)
      if (dest.sh[k])
      {
        if (!(aovMask & PRT_AOV_SH)) throw std::invalid_argument("sh needs aovSh in initFrame");
        check(prt_cuda_blit(ctx, PRT_BLIT_SH0 + k, &dest.sh[k]->x));
      }
  }

  void blitFrameLdr(Surface&, const float*, float, float) override
  {
    throw std::logic_error("blitFrameLdr is a host-side conversion; not provided by the CUDA device");
  }
  void blitFrameLdr(Surface&, const Vec3f*, float, float) override
  {
    throw std::logic_error("blitFrameLdr is a host-side conversion; not provided by the CUDA device");
  }
  void blitFrameHdr(Surface&, const Vec3f*) override
  {
    throw std::logic_error("blitFrameHdr is a host-side conversion; not provided by the CUDA device");
  }

  float getFrameError() override
  {
    float e = 0.f;
    check(prt_cuda_frame_error(ctx, &e));
    return e;
  }

  float getFilterWidth() const override { return 1.f; }

  prt_context* handle() const { return ctx; }

private:
  void check(int rc) const
  {
    if (rc == PRT_OK) return;
    const std::string msg = prt_cuda_last_error(ctx);
    if (rc == PRT_ERR_INVALID_ARG) throw std::invalid_argument(msg);
    if (rc == PRT_ERR_LOGIC) throw std::logic_error(msg);
    throw std::runtime_error("prt_cuda error " + std::to_string(rc) + ": " + msg);
  }

  const PinholeCamera& requireCamera() const
  {
    if (!camera) throw std::logic_error("no camera");
    return *camera;
  }

  // The reference's tables (bsdf/albedo_tables.cpp:173-188) in prt_cuda_albedo_tables' layout.
  void uploadHostTables()
  {
    precomputeAlbedoTables();
    std::vector<float> t;
    auto put = [&](const float* src, int n) { t.insert(t.end(), src, src + n); };
    put(MicrofacetAlbedoTable::dir, 32 * 32);
    put(MicrofacetAlbedoTable::avg, 32);
    put(MicrofacetDielectricAlbedoTable::etaDir, 16 * 16 * 16);
    put(MicrofacetDielectricAlbedoTable::etaAvg, 16 * 16);
    put(MicrofacetDielectricAlbedoTable::rcpEtaDir, 16 * 16 * 16);
    put(MicrofacetDielectricAlbedoTable::rcpEtaAvg, 16 * 16);
    put(MicrofacetDielectricReflectionAlbedoTable::etaDir, 16 * 16 * 16);
    put(MicrofacetDielectricReflectionAlbedoTable::etaAvg, 16 * 16);
    put(MicrofacetSheenAlbedoTable::dir, 16 * 16);
    check(prt_cuda_set_albedo_tables(ctx, t.data(), (int64_t)t.size()));
  }

  prt_context* ctx = nullptr;
  Vec2i size = Vec2i(0);
  int aovMask = 0;
  std::shared_ptr<PinholeCamera> camera;
  prt_camera_desc cameraDesc{};
};

} // namespace prt
