// C ABI of the B200 render device (include/prt_cuda.h) and its host runtime: context,
// scene upload (BVH8 build, materials, lights, media), camera, frame and render calls.
// This is the CUDA sibling of the reference's DeviceCpu (render/device_cpu.cpp).
#include "../../include/prt_cuda.h"
#include "runtime.h"
#include "bvh_build.h"
#include "host_rcp.h"
#include "scene_file.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

using namespace prt;

struct prt_context
{
  Context c;
};

struct prt_scene_file
{
  RkScene scene;
};

namespace {

struct ApiError
{
  int code;
  std::string msg;
};

void cuCheck(cudaError_t e, const char* what)
{
  if (e == cudaErrorMemoryAllocation)
    throw ApiError{PRT_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e)};
  if (e != cudaSuccess) throw ApiError{PRT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

template <class F>
int guarded(prt_context* ctx, F&& f)
{
  if (!ctx) return PRT_ERR_INVALID_ARG;
  ctx->c.stageNext = 0;  // staging slots are per call (a call that threw may not have released its own)
  try
  {
    f(ctx->c);
    return PRT_OK;
  }
  catch (const ApiError& e)
  {
    ctx->c.lastError = e.msg;
    return e.code;
  }
  catch (const std::bad_alloc&)
  {
    ctx->c.lastError = "host out of memory";
    return PRT_ERR_OUT_OF_MEMORY;
  }
  catch (const std::invalid_argument& e)
  {
    ctx->c.lastError = e.what();
    return PRT_ERR_INVALID_ARG;
  }
  catch (const std::logic_error& e)
  {
    ctx->c.lastError = e.what();
    return PRT_ERR_LOGIC;
  }
  catch (const std::exception& e)
  {
    ctx->c.lastError = e.what();
    return PRT_ERR_CUDA;
  }
}

void* devAlloc(Context& c, size_t bytes, std::vector<DevBuf>* owner)
{
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  cuCheck(cudaMalloc(&p, bytes), "cudaMalloc");
  if (owner) owner->push_back(DevBuf{p, bytes});
  return p;
}

template <class T>
T* upload(Context& c, const std::vector<T>& v, std::vector<DevBuf>* owner = nullptr)
{
  T* p = (T*)devAlloc(c, v.size() * sizeof(T), owner ? owner : &c.sceneBufs);
  if (!v.empty()) cuCheck(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c.stream), "upload");
  return p;
}

void freeScene(Context& c)
{
  cudaStreamSynchronize(c.stream);
  for (auto& b : c.sceneBufs) cudaFree(b.ptr);
  c.sceneBufs.clear();
  for (auto& b : c.envBufs) cudaFree(b.ptr);
  c.envBufs.clear();
  c.hasScene = false;
}

void freeFrame(Context& c)
{
  cudaStreamSynchronize(c.stream);
  auto f = [](auto*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
  };
  f(c.accum);
  f(c.accumA);
  f(c.accumN);
  f(c.accumC);
  f(c.accum2);
  f(c.accumSH);
  f(c.errPartials);
  PathState& s = c.ps;
  f(s.rayO); f(s.rayD); f(s.hit); f(s.thr); f(s.rad); f(s.info);
  f(s.shO); f(s.shD); f(s.shL); f(s.out); f(s.aovA); f(s.aovN);
  f(s.sphL); f(s.sphWi); f(s.sphDirL); f(s.sphDirWi); f(s.sphOut); f(s.sphDirScale);
  f(s.queue[0]); f(s.queue[1]); f(s.classQueues);
  s.capacity = 0;
}

// Bit-level host mirror of float operations used to build light tables.
float luminanceHost(const float c[3]) { return 0.212671f * c[0] + 0.715160f * c[1] + 0.072169f * c[2]; }

// Distribution1D::init (sampling/distribution1d.cpp:14-28).
void cdfInit(float* cdf, const float* f, int size)
{
  cdf[0] = 0.f;
  for (int i = 1; i < size + 1; ++i) cdf[i] = cdf[i - 1] + f[i - 1];
  const float norm = (cdf[size] == 0.f) ? 0.f : 1.f / cdf[size];
  for (int i = 1; i < size + 1; ++i) cdf[i] *= norm;
  cdf[size] = 1.f;
}

void makeFrameHost(const float N[3], float U[3], float V[3])
{
  const float U0[3] = {0.f, N[2], -N[1]};
  const float U1[3] = {-N[2], 0.f, N[0]};
  const float l0 = U0[0] * U0[0] + U0[1] * U0[1] + U0[2] * U0[2];
  const float l1 = U1[0] * U1[0] + U1[1] * U1[1] + U1[2] * U1[2];
  const float* u = l0 > l1 ? U0 : U1;
  const float il = 1.f / std::sqrt(l0 > l1 ? l0 : l1);
  for (int k = 0; k < 3; ++k) U[k] = u[k] * il;
  V[0] = N[1] * U[2] - N[2] * U[1];
  V[1] = N[2] * U[0] - N[0] * U[2];
  V[2] = N[0] * U[1] - N[1] * U[0];
  const float iv = 1.f / std::sqrt(V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
  for (int k = 0; k < 3; ++k) V[k] *= iv;
}

// Reads a Standard material as StandardMaterial's constructor does (material/standard.cpp:21-150).
DevMaterial resolveMaterial(const prt_material& m, std::vector<float>& media, int textureCount)
{
  DevMaterial d;
  std::memset(&d, 0, sizeof(d));
  auto ior = [](float x) {
    x = std::max(x, 0.f);
    return x < 1.f ? (x > 0.f ? hostRcp(x) : INFINITY) : x;
  };
  // Both sides of an interface between media of these indices (DevEta).
  auto sides = [](DevEta* out, float outsideIor, float insideIor) {
    const float etas[2] = {outsideIor * hostRcp(insideIor), insideIor * hostRcp(outsideIor)};
    for (int s = 0; s < 2; ++s)
    {
      const float e = std::min(std::max(etas[s], 1.f / 3.f), 3.f);
      out[s].eta = e;
      out[s].rcpEta = hostRcp(e);
      out[s].rcpEta2 = hostRcp(e * e);
      out[s].favg = hostFresnelDielectricAvg(e);
      out[s].favgRcp = hostFresnelDielectricAvg(out[s].rcpEta);
    }
  };
  d.ambientIor = ior(m.ambient_ior > 0.f ? m.ambient_ior : 1.f);
  d.principled = m.model == PRT_MATERIAL_PRINCIPLED ? 1 : 0;
  if (m.model == PRT_MATERIAL_MISS)
  {
    d.type = kMatMiss;
    d.shadeClass = 0;
    d.baseColorTex = -1;
    d.opacity = 1.f;
    return d;
  }
  if (m.model != PRT_MATERIAL_STANDARD && m.model != PRT_MATERIAL_PRINCIPLED)
    throw std::invalid_argument("unknown material model");
  d.baseWeight = m.base_weight;
  for (int k = 0; k < 3; ++k) d.baseColor[k] = m.base_color[k];
  d.baseColorTex = m.base_color_texture;
  if (d.baseColorTex >= textureCount) throw std::invalid_argument("material references a missing texture");
  d.metalness = m.metalness;
  d.diffuseRoughness = m.diffuse_roughness;
  d.hasDiffuseRoughness = m.diffuse_roughness != 0.f;
  d.specularWeight = m.specular_weight;
  for (int k = 0; k < 3; ++k) d.specularColor[k] = m.specular_color[k];
  d.specularRoughness = m.specular_roughness;
  d.hasSpecularRoughness = m.specular_roughness != 0.f;
  d.specularIor = ior(m.specular_ior);
  d.transmissionWeight = m.transmission_weight;
  for (int k = 0; k < 3; ++k) d.transmissionColor[k] = std::min(std::max(m.transmission_color[k], 0.f), 1.f);
  d.transmissionDepth = std::max(m.transmission_depth, 0.f);
  d.subsurfaceWeight = m.subsurface_weight;
  for (int k = 0; k < 3; ++k) d.subsurfaceColor[k] = m.subsurface_color[k];
  d.subsurfaceAnisotropy = m.subsurface_anisotropy;
  d.coatWeight = m.coat_weight;
  for (int k = 0; k < 3; ++k) d.coatColor[k] = m.coat_color[k];
  d.coatRoughness = m.coat_roughness;
  d.hasCoatRoughness = m.coat_roughness != 0.f;
  d.coatIor = ior(m.coat_ior);
  sides(d.spec, d.ambientIor, d.specularIor);
  sides(d.coat, d.ambientIor, d.coatIor);
  d.sheenWeight = m.sheen_weight;
  for (int k = 0; k < 3; ++k) d.sheenColor[k] = m.sheen_color[k];
  d.sheenRoughness = m.sheen_roughness;
  d.sheenTint = d.principled ? m.sheen_tint : 0.f;
  for (int k = 0; k < 3; ++k) d.emission[k] = m.emission_color[k] * m.emission_luminance;
  d.coatThickness = d.principled ? std::max(m.coat_thickness, 0.f) : 0.5f;
  if (d.principled)
  {
    // PrincipledMaterial: "roughness" also turns the diffuse lobe into Oren-Nayar, and the
    // material has no emission.
    d.diffuseRoughness = d.specularRoughness;
    d.hasDiffuseRoughness = d.hasSpecularRoughness;
    for (int k = 0; k < 3; ++k) d.emission[k] = 0.f;
  }
  d.thinWalled = m.thin_walled;
  d.opacity = m.opacity;
  // Thin-walled transmission: thickness / transmissionDepth, the thickness being 1 for Standard
  // (its "thickness" parameter has scale 1 and no prop) and "thickness" for Principled.
  d.thinThickness = (d.principled ? std::max(m.thickness, 0.f) : 1.f) / d.transmissionDepth;
  d.subsurfaceFromBase = 0;
  if (d.principled)
  {
    // PrincipledMaterial has no subsurface; a thin one has "backlight" (material/principled.cpp:
    // 334-360): Multi{diffuse BRDF x (1 - b/2), diffuse BTDF x b/2} in the diffuse colour, b in
    // [0, 2] -- the Standard subsurface blend with weight 1, anisotropy b - 1 and the diffuse
    // colour.
    d.subsurfaceWeight = 0.f;
    const float backlight = m.thin_walled ? std::min(std::max(m.backlight, 0.f), 2.f) : 0.f;
    if (backlight > 0.f)
    {
      d.subsurfaceWeight = 1.f;
      d.subsurfaceAnisotropy = backlight - 1.f;
      d.subsurfaceFromBase = 1;
    }
  }
  d.type = 0;
  if (m.emission_luminance > 0.f && m.model == PRT_MATERIAL_STANDARD) d.type |= kMatEmissive;
  d.mediumInt = d.mediumExt = 0;
  if (m.opacity != 1.f) d.type |= kMatTransparent;
  if (m.transmission_weight != 0.f)
  {
    d.type |= kMatTransmissive;
    if (m.thin_walled)
      d.type |= kMatTransparent;
    else
    {
      d.type |= kMatMediaInterface;
      // MaterialFactory::makeMedium (material/material_factory.cpp:159-175): media are
      // deduplicated by (colour, ior); medium 0 is the default (1, 1).
      auto medium = [&](const float c[3], float n) {
        const int count = (int)media.size() / 4;
        for (int i = 0; i < count; ++i)
          if (media[4 * i] == c[0] && media[4 * i + 1] == c[1] && media[4 * i + 2] == c[2] && media[4 * i + 3] == n)
            return i;
        media.insert(media.end(), {c[0], c[1], c[2], n});
        return count;
      };
      float col[3];
      for (int k = 0; k < 3; ++k) col[k] = std::pow(d.transmissionColor[k], d.transmissionDepth);
      d.mediumInt = medium(col, d.specularIor);
      const float one[3] = {1.f, 1.f, 1.f};
      d.mediumExt = medium(one, d.ambientIor);
    }
  }
  // Static lobe features (StandardMaterial::getBsdfLobes branch conditions with the
  // material's constant parameters; only the base colour can be textured).
  auto c01 = [](float x) { return std::min(std::max(x, 0.f), 1.f); };
  const float eps = 1e-4f;
  const float metal = c01(d.metalness), spec = c01(d.specularWeight), trans = c01(d.transmissionWeight);
  const float diel = 1.f - metal;
  d.features = 0;
  if (diel > eps && diel * (1.f - trans) > eps)
  {
    d.features |= kFeatOpaque;
    if (d.hasDiffuseRoughness) d.features |= kFeatRoughDiffuse;
    if (std::fabs(d.specularIor - d.ambientIor) > eps && spec > eps) d.features |= kFeatSpecular;
    if (c01(d.subsurfaceWeight) > eps) d.features |= kFeatSubsurface;
  }
  if (diel > eps && diel * trans * spec > eps)
  {
    if (std::fabs(d.specularIor - d.ambientIor) <= eps) d.features |= kFeatTransparent;
    else d.features |= d.thinWalled ? kFeatThin : kFeatDielectric;
  }
  if (1.f - c01(d.opacity) > eps) d.features |= kFeatTransparent;
  if (metal * spec > eps) d.features |= kFeatConductor;
  if (c01(d.coatWeight) > eps && std::fabs(d.coatIor - d.ambientIor) > eps) d.features |= kFeatCoat;
  if (c01(d.sheenWeight) > eps) d.features |= kFeatSheen;
  d.shadeClass = kShadeClasses - 1;
  for (int k = 1; k < kShadeClasses; ++k)
    if (kShadeClassFeatures[k] == d.features)
    {
      d.shadeClass = k;
      break;
    }
  if (d.type & kMatEmissive) d.shadeClass = 0;
  return d;
}

// Environment lights in Scene::initLights order (render/scene.cpp:372-440) -- distant,
// ambient, image, or ambient first with PRT_ENV_AMBIENT_FIRST -- and the light-selection CDF
// over the area lights (their powers in c.areaLightPowerHost) followed by them. The buffers go
// to c.envBufs, which a later call (prt_cuda_scene_lights) frees and replaces.
void buildEnvLights(Context& c, DevScene& sc, const prt_env_desc& e)
{
  if (e.flags & ~PRT_ENV_AMBIENT_FIRST) throw std::invalid_argument("unknown environment flags");
  cudaStreamSynchronize(c.stream);
  for (auto& buf : c.envBufs) cudaFree(buf.ptr);
  c.envBufs.clear();
  sc.image = DevImageLight{};
  std::vector<float> lightPower = c.areaLightPowerHost;
  const float sceneRadius = c.sceneRadius;
  const float pi = 3.14159265358979323846f;
  auto pos3 = [](const float* v) { return v[0] > 0.f || v[1] > 0.f || v[2] > 0.f; };
  int ne = 0;
  auto addAmbient = [&]() {
    if (!pos3(e.ambient_color)) return;
    DevEnvLight& L = sc.env[ne++];
    L.kind = kEnvAmbient;
    for (int k = 0; k < 3; ++k) L.color[k] = e.ambient_color[k];
    lightPower.push_back(4.f * pi * pi * sceneRadius * sceneRadius * luminanceHost(L.color));
  };
  if (e.flags & PRT_ENV_AMBIENT_FIRST) addAmbient();
  if (pos3(e.distant_color))
  {
    DevEnvLight& L = sc.env[ne++];
    L.kind = kEnvDistant;
    for (int k = 0; k < 3; ++k) L.color[k] = e.distant_color[k];
    float d[3] = {e.distant_dir[0], e.distant_dir[1], e.distant_dir[2]};
    const float il = 1.f / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int k = 0; k < 3; ++k) L.dir[k] = d[k] * il;
    makeFrameHost(L.dir, L.frameU, L.frameV);
    L.halfAngle = e.distant_angle * 0.5f;
    L.cosAngle = std::cos(L.halfAngle);
    const float sh = std::sin(0.5f * L.halfAngle);
    L.conePdf = 1.f / (4.f * pi * sh * sh);
    lightPower.push_back(4.f * pi * pi * sh * sh * sceneRadius * sceneRadius * luminanceHost(L.color));
  }
  if (!(e.flags & PRT_ENV_AMBIENT_FIRST)) addAmbient();
  if (e.image_rgb)
  {
    if (e.image_width <= 0 || e.image_height <= 0) throw std::invalid_argument("invalid image light");
    DevEnvLight& L = sc.env[ne++];
    L.kind = kEnvImage;
    const int W = e.image_width, H = e.image_height;
    // Texture-row order (bottom row first), as ImageTextureBuffer stores it.
    std::vector<float> tex((size_t)W * H * 3);
    for (int y = 0; y < H; ++y)
      std::memcpy(&tex[(size_t)y * W * 3], e.image_rgb + (size_t)(H - 1 - y) * W * 3, sizeof(float) * 3 * W);
    // ImageLight LUT (light/image_light.h:19-62).
    int lw = W, lh = H, bucket = 1;
    if (e.image_lut_size > 0)
      while (std::max(lw, lh) > e.image_lut_size && lw % 2 == 0 && lh % 2 == 0)
      {
        lw /= 2;
        lh /= 2;
        bucket *= 2;
      }
    std::vector<float> weights((size_t)lw * lh);
    for (int y = 0; y < lh; ++y)
      for (int x = 0; x < lw; ++x)
      {
        float sum = 0.f;
        for (int y2 = 0; y2 < bucket; ++y2)
          for (int x2 = 0; x2 < bucket; ++x2)
            sum += luminanceHost(&tex[3 * ((size_t)(y * bucket + y2) * W + (x * bucket + x2))]);
        weights[(size_t)y * lw + x] = sum * std::sin((y + 0.5f) / lh * pi);
      }
    // Distribution2D::init (sampling/distribution2d.cpp:13-30).
    std::vector<float> xCdfs((size_t)lh * (lw + 1)), fy(lh), yCdf(lh + 1);
    for (int y = 0; y < lh; ++y)
    {
      fy[y] = 0.f;
      for (int x = 0; x < lw; ++x) fy[y] += weights[(size_t)y * lw + x];
      cdfInit(&xCdfs[(size_t)y * (lw + 1)], &weights[(size_t)y * lw], lw);
    }
    cdfInit(yCdf.data(), fy.data(), lh);
    sc.image.rgb = upload(c, tex, &c.envBufs);
    sc.image.width = W;
    sc.image.height = H;
    sc.image.lutW = lw;
    sc.image.lutH = lh;
    sc.image.yCdf = upload(c, yCdf, &c.envBufs);
    sc.image.xCdfs = upload(c, xCdfs, &c.envBufs);
    float sumL = 0.f;
    for (int i = 0; i < W * H; ++i) sumL += luminanceHost(&tex[3 * (size_t)i]);
    lightPower.push_back(4.f * pi * pi * sceneRadius * sceneRadius * (sumL / float(W * H)));
  }
  if (sc.areaLightCount == 0 && ne == 0)
  {
    // Default ambient light (render/scene.cpp:435-440).
    DevEnvLight& L = sc.env[ne++];
    L.kind = kEnvAmbient;
    L.color[0] = L.color[1] = L.color[2] = 1.f;
    lightPower.push_back(4.f * pi * pi * sceneRadius * sceneRadius * luminanceHost(L.color));
  }
  sc.envCount = ne;
  sc.lightCount = sc.areaLightCount + ne;
  sc.distantLight = -1;
  for (int k = 0; k < ne; ++k)
    if (sc.env[k].kind == kEnvDistant) sc.distantLight = sc.areaLightCount + k;
  std::vector<float> lightCdf(sc.lightCount + 1);
  cdfInit(lightCdf.data(), lightPower.data(), sc.lightCount);
  sc.lightCdf = upload(c, lightCdf, &c.envBufs);
}

void uploadScene(Context& c, const prt_scene_desc* s)
{
  if (!s || s->mesh_count < 0 || s->material_count <= 0 || !s->materials)
    throw std::invalid_argument("invalid scene description");
  if (s->bvh_build != PRT_BVH_HOST && s->bvh_build != PRT_BVH_DEVICE)
    throw std::invalid_argument("unknown BVH builder");
  const bool hostBuild = s->bvh_build == PRT_BVH_HOST;
  freeScene(c);
  DevScene sc;
  std::memset(&sc, 0, sizeof(sc));
  // Materials and media.
  std::vector<float> media = {1.f, 1.f, 1.f, 1.f};
  std::vector<DevMaterial> mats;
  for (int i = 0; i < s->material_count; ++i) mats.push_back(resolveMaterial(s->materials[i], media, s->texture_count));
  // Textures, stored in texture-row order (bottom row first).
  std::vector<DevTexture> texs;
  for (int i = 0; i < s->texture_count; ++i)
  {
    const prt_texture& t = s->textures[i];
    if (!t.rgb || t.width <= 0 || t.height <= 0) throw std::invalid_argument("invalid texture");
    std::vector<float> flipped((size_t)t.width * t.height * 3);
    for (int y = 0; y < t.height; ++y)
      std::memcpy(&flipped[(size_t)y * t.width * 3], t.rgb + (size_t)(t.height - 1 - y) * t.width * 3,
                  sizeof(float) * 3 * t.width);
    DevTexture dt;
    dt.rgb = upload(c, flipped);
    dt.width = t.width;
    dt.height = t.height;
    texs.push_back(dt);
  }
  // Geometry: concatenated vertices and triangles.
  int64_t totalTris = 0, totalVerts = 0;
  for (int g = 0; g < s->mesh_count; ++g)
  {
    const prt_mesh& m = s->meshes[g];
    if (m.tri_count < 0 || m.vertex_count < 0 || (m.tri_count > 0 && (!m.positions || !m.indices)))
      throw std::invalid_argument("invalid mesh");
    if (m.material < 0 || m.material >= s->material_count) throw std::invalid_argument("mesh material out of range");
    totalTris += m.tri_count;
    totalVerts += m.vertex_count;
  }
  if (totalTris > (int64_t)0x3fffffff || totalVerts > (int64_t)0x7fffffff)
    throw std::invalid_argument("scene too large");
  std::vector<float4> pos(totalVerts), nrm;
  std::vector<float2> uv;
  bool anyN = false, anyUV = false;
  for (int g = 0; g < s->mesh_count; ++g)
  {
    anyN |= s->meshes[g].normals != nullptr;
    anyUV |= s->meshes[g].texcoords != nullptr;
  }
  if (anyN) nrm.assign(totalVerts, make_float4(0.f, 0.f, 1.f, 0.f));
  if (anyUV) uv.assign(totalVerts, make_float2(0.f, 0.f));
  std::vector<int4> triVerts(totalTris);
  std::vector<float> triPos(hostBuild ? (size_t)totalTris * 9 : 0);
  std::vector<int> meshFlags(s->mesh_count), meshMat(s->mesh_count), meshOff(s->mesh_count), meshLight(s->mesh_count, -1);
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  int64_t vbase = 0, tbase = 0;
  for (int g = 0; g < s->mesh_count; ++g)
  {
    const prt_mesh& m = s->meshes[g];
    meshFlags[g] = (m.normals ? 1 : 0) | (m.texcoords ? 2 : 0);
    meshMat[g] = m.material;
    meshOff[g] = (int)tbase;
    for (int v = 0; v < m.vertex_count; ++v)
    {
      pos[vbase + v] = make_float4(m.positions[3 * v], m.positions[3 * v + 1], m.positions[3 * v + 2], 0.f);
      if (m.normals) nrm[vbase + v] = make_float4(m.normals[3 * v], m.normals[3 * v + 1], m.normals[3 * v + 2], 0.f);
      if (m.texcoords) uv[vbase + v] = make_float2(m.texcoords[2 * v], m.texcoords[2 * v + 1]);
    }
    for (int t = 0; t < m.tri_count; ++t)
    {
      int idx[3];
      for (int k = 0; k < 3; ++k)
      {
        idx[k] = m.indices[3 * t + k];
        if (idx[k] < 0 || idx[k] >= m.vertex_count) throw std::invalid_argument("triangle index out of range");
      }
      triVerts[tbase + t] = make_int4((int)(vbase + idx[0]), (int)(vbase + idx[1]), (int)(vbase + idx[2]), g);
      float* tp = hostBuild ? &triPos[(size_t)(tbase + t) * 9] : nullptr;
      for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a)
        {
          const float x = m.positions[3 * idx[k] + a];
          if (tp) tp[3 * k + a] = x;
          lo[a] = std::min(lo[a], x);
          hi[a] = std::max(hi[a], x);
        }
    }
    vbase += m.vertex_count;
    tbase += m.tri_count;
  }
  if (totalTris == 0)
    for (int a = 0; a < 3; ++a) lo[a] = hi[a] = 0.f;
  sc.triCount = totalTris;
  sc.triVerts = upload(c, triVerts);
  sc.pos = upload(c, pos);
  // BVH8, on the host or on the device from the vertex and index arrays just uploaded.
  c.bvh = Bvh8();
  c.bvhBuilder = s->bvh_build;
  if (hostBuild)
  {
    buildBvh8(triPos.data(), totalTris, c.bvh);
    sc.nodes = reinterpret_cast<const uint4*>(upload(c, c.bvh.nodes));
    sc.tris = reinterpret_cast<const float4*>(upload(c, c.bvh.tris));
    c.bvhBuildMs = c.bvh.buildMs;
    c.bvhNodes = (int64_t)c.bvh.nodes.size();
    c.bvhTris = (int64_t)c.bvh.tris.size();
    c.bvhDepth = c.bvh.maxDepth;
    c.bvhTop = std::min(c.bvh.topCount, kBvh8TopNodes);
    c.bvhIterations = 0;
  }
  else
  {
    DeviceBvh8 db;
    buildBvh8Device(sc.pos, sc.triVerts, totalTris, c.stream, db);
    c.sceneBufs.push_back(DevBuf{db.nodes, sizeof(Bvh8Node) * (size_t)db.nodeCount});
    c.sceneBufs.push_back(DevBuf{db.tris, sizeof(Bvh8Tri) * (size_t)std::max<int64_t>(db.triCount, 1)});
    sc.nodes = reinterpret_cast<const uint4*>(db.nodes);
    sc.tris = reinterpret_cast<const float4*>(db.tris);
    c.bvhBuildMs = db.buildMs;
    c.bvhNodes = db.nodeCount;
    c.bvhTris = db.triCount;
    c.bvhDepth = db.maxDepth;
    c.bvhTop = db.topCount;
    c.bvhIterations = db.plocIterations;
  }
  if (c.bvhDepth > kBvh8TraceStack) throw std::runtime_error("BVH8 deeper than the traversal stack");
  sc.topNodes = c.bvhTop;
  sc.hasTransparent = 0;
  for (const DevMaterial& m : mats) sc.hasTransparent |= (m.type & kMatTransparent) ? 1 : 0;
  sc.nrm = anyN ? upload(c, nrm) : nullptr;
  sc.uv = anyUV ? upload(c, uv) : nullptr;
  sc.meshFlags = upload(c, meshFlags);
  sc.meshMaterial = upload(c, meshMat);
  sc.meshTriOffset = upload(c, meshOff);
  sc.meshCount = s->mesh_count;
  sc.materials = upload(c, mats);
  sc.materialCount = (int)mats.size();
  sc.textures = upload(c, texs);
  c.meshTriOffsetHost = meshOff;
  // Scene radius (render/scene.cpp:367): half the diagonal of the bounds.
  const float ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const float sceneRadius = std::sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2]) * 0.5f;
  sc.sceneRadius = sceneRadius;
  // Area lights: one TriangleLight per emissive mesh (render/scene.cpp:79-116, light/triangle_light.h:29-60).
  std::vector<float> etris, areaCdf, lightPower;
  std::vector<int> areaOff, areaCnt, areaCdfOff;
  for (int g = 0; g < s->mesh_count; ++g)
  {
    const prt_mesh& m = s->meshes[g];
    const DevMaterial& mat = mats[m.material];
    if (!(mat.type & kMatEmissive) || m.tri_count == 0) continue;
    meshLight[g] = (int)areaOff.size();
    areaOff.push_back((int)(etris.size() / 16));
    areaCnt.push_back(m.tri_count);
    std::vector<float> w(m.tri_count);
    float sumL = 0.f;
    for (int t = 0; t < m.tri_count; ++t)
    {
      float tp[9];
      for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) tp[3 * k + a] = m.positions[3 * m.indices[3 * t + k] + a];
      const float e1[3] = {tp[3] - tp[0], tp[4] - tp[1], tp[5] - tp[2]};
      const float e2[3] = {tp[6] - tp[0], tp[7] - tp[1], tp[8] - tp[2]};
      const float n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      const float len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      w[t] = len * luminanceHost(mat.emission);
      sumL += len * luminanceHost(mat.emission);
      etris.insert(etris.end(), {tp[0], tp[1], tp[2], tp[3], tp[4], tp[5], tp[6], tp[7], tp[8], n[0], n[1], n[2],
                                 mat.emission[0], mat.emission[1], mat.emission[2], 0.f});
    }
    areaCdfOff.push_back((int)areaCdf.size());
    const size_t o = areaCdf.size();
    areaCdf.resize(o + m.tri_count + 1);
    cdfInit(&areaCdf[o], w.data(), m.tri_count);
    lightPower.push_back(3.14159265358979323846f * sumL);
  }
  sc.areaLightCount = (int)areaOff.size();
  sc.meshLight = upload(c, meshLight);
  std::vector<int> meshClass(s->mesh_count);
  for (int g = 0; g < s->mesh_count; ++g) meshClass[g] = mats[s->meshes[g].material].shadeClass;
  sc.meshClass = upload(c, meshClass);
  sc.areaTriOffset = upload(c, areaOff);
  sc.areaTriCount = upload(c, areaCnt);
  sc.areaCdfOffset = upload(c, areaCdfOff);
  sc.areaCdf = upload(c, areaCdf);
  sc.etris = upload(c, etris);
  c.areaLightPowerHost = lightPower;
  c.sceneRadius = sceneRadius;
  for (int k = 0; k < 3; ++k)
  {
    c.boundsLo[k] = lo[k];
    c.boundsHi[k] = hi[k];
  }
  buildEnvLights(c, sc, s->env);
  std::vector<float> mediaColor;
  for (size_t i = 0; i < media.size() / 4; ++i) mediaColor.insert(mediaColor.end(), {media[4 * i], media[4 * i + 1], media[4 * i + 2]});
  sc.mediaColor = upload(c, mediaColor);
  sc.mediaCount = (int)(media.size() / 4);
  cuCheck(cudaStreamSynchronize(c.stream), "scene upload");
  c.scene = sc;
  c.hasScene = true;
  c.materialsHost = mats;
  c.texturesHost = texs;
}

void allocFrame(Context& c, int width, int height, int aovMask)
{
  if (width <= 0 || height <= 0) throw std::invalid_argument("invalid frame size");
  if (width % 32 != 0 || height % 8 != 0)
    throw std::logic_error("image size is not divisible by the tile size");
  if (width > 4096 || height > 4096) throw std::logic_error("image size is too large");
  if (aovMask & ~(PRT_AOV_ALBEDO1 | PRT_AOV_NORMAL1 | PRT_AOV_HDR_VAR | PRT_AOV_SH))
    throw std::invalid_argument("unknown AOV bits");
  freeFrame(c);
  c.width = width;
  c.height = height;
  c.aovMask = aovMask & (PRT_AOV_ALBEDO1 | PRT_AOV_NORMAL1);  // per-path first-hit AOVs
  c.aovSh = (aovMask & PRT_AOV_SH) != 0;
  const size_t px = (size_t)width * height;
  c.accum = (float*)devAlloc(c, px * sizeof(float4), nullptr);
  c.accumC = (float*)devAlloc(c, px * sizeof(float4), nullptr);
  c.errPartials = (double*)devAlloc(c, sizeof(double) * (size_t)c.smCount * 16, nullptr);
  if (aovMask & PRT_AOV_HDR_VAR) c.accum2 = (float*)devAlloc(c, px * sizeof(float4), nullptr);
  if (c.aovSh) c.accumSH = (float*)devAlloc(c, 4 * px * sizeof(float4), nullptr);
  if (c.aovMask)
  {
    c.accumA = (float*)devAlloc(c, px * sizeof(float4), nullptr);
    c.accumN = (float*)devAlloc(c, px * sizeof(float4), nullptr);
  }
  cuCheck(launchClear(c), "clear");
  cuCheck(cudaStreamSynchronize(c.stream), "frame");
}

// Per-bounce counter blocks of 16 ints (see renderSamples), maxDepth + 2 of them.
// Path state for waves of `samples` whole-frame samples (at least one), capped at wavePaths
// paths (128M by default: one 64-spp 1080p frame, about 31 GB). Allocated on the first render
// and grown when a call needs more.
void ensurePathState(Context& c, int spp)
{
  const int64_t px = (int64_t)c.width * c.height;
  const int64_t target = c.wavePaths;
  const int maxWave = (int)std::max<int64_t>(1, target / px);
  const int want = std::max(1, std::min(spp, maxWave));
  if (c.ps.capacity >= want * px && c.ps.capacity <= std::max<int64_t>(target, px))
  {
    c.waveSamples = (int)(c.ps.capacity / px);
    return;
  }
  cudaStreamSynchronize(c.stream);
  PathState& s = c.ps;
  auto f = [](auto*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
  };
  f(s.rayO); f(s.rayD); f(s.hit); f(s.thr); f(s.rad); f(s.info);
  f(s.shO); f(s.shD); f(s.shL); f(s.out); f(s.aovA); f(s.aovN);
  f(s.sphL); f(s.sphWi); f(s.sphDirL); f(s.sphDirWi); f(s.sphOut); f(s.sphDirScale);
  f(s.queue[0]); f(s.queue[1]); f(s.classQueues);
  c.waveSamples = want;
  const int64_t cap = (int64_t)want * px;
  if (cap > (int64_t)kQueuePathMask) throw std::invalid_argument("path capacity above 2^29 - 1");
  s.capacity = cap;
  auto a4 = [&](size_t n) { return (float4*)devAlloc(c, n * sizeof(float4), nullptr); };
  s.rayO = a4(cap); s.rayD = a4(cap); s.hit = a4(cap); s.thr = a4(cap); s.rad = a4(cap);
  s.info = (uint4*)devAlloc(c, cap * sizeof(uint4), nullptr);
  s.shO = a4(cap); s.shD = a4(cap); s.shL = a4(cap); s.out = a4(cap);
  if (c.aovMask)
  {
    s.aovA = a4(cap);
    s.aovN = a4(cap);
  }
  if (c.aovSh)
  {
    s.sphL = a4(cap); s.sphWi = a4(cap); s.sphDirL = a4(cap); s.sphDirWi = a4(cap);
    s.sphOut = a4(3 * cap);
    s.sphDirScale = (float*)devAlloc(c, cap * sizeof(float), nullptr);
  }
  s.queue[0] = (int*)devAlloc(c, cap * sizeof(int), nullptr);
  s.queue[1] = (int*)devAlloc(c, cap * sizeof(int), nullptr);
  s.classQueues = (int*)devAlloc(c, (size_t)cap * kShadeClasses * sizeof(int), nullptr);
}

void ensureCounters(Context& c)
{
  const size_t blocks = 16 * (size_t)(c.renderer.maxDepth + 2);
  cudaStreamSynchronize(c.stream);
  if (c.ps.counters) cudaFree(c.ps.counters);
  c.ps.counters = (int*)devAlloc(c, sizeof(int) * (blocks + 16), nullptr);
  c.ps.octBins = c.ps.counters + blocks;
}

// Borrowed buffer: device memory is used in place; host memory (pinned or pageable) is staged
// through one of the context's staging slots. A call's k-th Staged takes slot k, which keeps its
// allocation for later calls, so repeated calls (a blit per frame) allocate nothing. Growing a
// slot frees its old buffer only after the stream has drained. Slots are taken and released in
// LIFO order (Staged objects are locals of one entry point).
struct Staged
{
  void* dev = nullptr;
  void* host = nullptr;
  size_t bytes = 0;
  bool owned = false;
  Context* c = nullptr;

  Staged(const Staged&) = delete;
  Staged& operator=(const Staged&) = delete;
  Staged(Context& ctx, const void* p, size_t n, bool copyIn) : bytes(n), c(&ctx)
  {
    cudaPointerAttributes attr;
    if (p && cudaPointerGetAttributes(&attr, p) == cudaSuccess &&
        (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged))
    {
      dev = const_cast<void*>(p);
      return;
    }
    cudaGetLastError();
    host = const_cast<void*>(p);
    const size_t slot = (size_t)ctx.stageNext;
    if (ctx.stage.size() <= slot) ctx.stage.resize(slot + 1);
    DevBuf& b = ctx.stage[slot];
    const size_t need = std::max<size_t>(n, 256);
    if (b.bytes < need)
    {
      cuCheck(cudaStreamSynchronize(ctx.stream), "staging sync");
      if (b.ptr) cudaFree(b.ptr);
      b = DevBuf{};
      cuCheck(cudaMalloc(&b.ptr, need), "cudaMalloc (staging)");
      b.bytes = need;
    }
    ++ctx.stageNext;
    owned = true;
    dev = b.ptr;
    if (copyIn && n) cuCheck(cudaMemcpyAsync(dev, p, n, cudaMemcpyHostToDevice, ctx.stream), "copy in");
  }
  void copyOut()
  {
    if (owned && host && bytes) cuCheck(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream), "copy out");
  }
  ~Staged()
  {
    if (owned)
    {
      // The call returns only after its copies of the caller's host memory are done (a pinned
      // buffer is read or written asynchronously otherwise).
      cudaStreamSynchronize(c->stream);
      --c->stageNext;
    }
  }
};

void freeStaging(Context& c)
{
  cudaStreamSynchronize(c.stream);
  for (auto& buf : c.stage)
    if (buf.ptr) cudaFree(buf.ptr);
  c.stage.clear();
  c.stageNext = 0;
}

void checkDeviceErrors(Context& c)
{
  uint32_t err = 0;
  cuCheck(cudaMemcpyAsync(&err, c.ps.err, sizeof(err), cudaMemcpyDeviceToHost, c.stream), "error flag");
  cuCheck(cudaStreamSynchronize(c.stream), "sync");
  if (err)
  {
    cudaMemsetAsync(c.ps.err, 0, sizeof(uint32_t), c.stream);
    throw ApiError{PRT_ERR_DEVICE_ABORT, "device traversal aborted (flags " + std::to_string(err) +
                                             "): stack overflow or iteration cap"};
  }
}

// PinholeCamera constructor (camera/pinhole_camera.h:20-36) for a width x height frame.
DevCamera makeCamera(const prt_camera_desc& cam, int width, int height)
{
  DevCamera d;
  const float aspect = float(width) / float(height);
  const float hh = std::tan(0.5f * cam.fov);
  const float hw = hh * aspect;
  auto basis = [&](float x, float y, float z, float* out) {
    for (int k = 0; k < 3; ++k) out[k] = x * cam.basis_u[k] + y * cam.basis_v[k] + z * cam.basis_n[k];
  };
  for (int k = 0; k < 3; ++k) d.org[k] = cam.position[k];
  basis(-hw, hh, -1.f, d.imageO);
  basis(2.f * hw, 0.f, 0.f, d.imageDx);
  basis(0.f, -2.f * hh, 0.f, d.imageDy);
  d.nearClip = cam.near_clip;
  return d;
}

void requireScene(Context& c)
{
  if (!c.hasScene) throw ApiError{PRT_ERR_STATE, "no scene uploaded"};
}

} // namespace

extern "C" {

int prt_cuda_create(int device_ordinal, prt_context** out_ctx)
{
  if (!out_ctx) return PRT_ERR_INVALID_ARG;
  *out_ctx = nullptr;
  auto* ctx = new (std::nothrow) prt_context();
  if (!ctx) return PRT_ERR_OUT_OF_MEMORY;
  Context& c = ctx->c;
  c.device = device_ordinal;
  cudaError_t e = cudaSetDevice(device_ordinal);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c.smCount, cudaDevAttrMultiProcessorCount, device_ordinal);
  if (e == cudaSuccess) e = cudaMalloc(&c.ps.err, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(c.ps.err, 0, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&c.ps.travCounts, 4 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaEventCreate(&c.ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c.ev1);
  if (e == cudaSuccess) e = buildAlbedoTables(c.tables, &c.tableStorage);
  if (e != cudaSuccess)
  {
    delete ctx;
    return e == cudaErrorMemoryAllocation ? PRT_ERR_OUT_OF_MEMORY : PRT_ERR_CUDA;
  }
  *out_ctx = ctx;
  return PRT_OK;
}

int prt_cuda_destroy(prt_context* ctx)
{
  if (!ctx) return PRT_ERR_INVALID_ARG;
  Context& c = ctx->c;
  cudaSetDevice(c.device);
  freeScene(c);
  freeFrame(c);
  freeStaging(c);
  if (c.ps.counters) cudaFree(c.ps.counters);
  if (c.ps.err) cudaFree(c.ps.err);
  if (c.ps.travCounts) cudaFree(c.ps.travCounts);
  if (c.tableStorage) cudaFree(c.tableStorage);
  if (c.whiteMaterialDev) cudaFree(c.whiteMaterialDev);
  if (c.ev0) cudaEventDestroy(c.ev0);
  if (c.ev1) cudaEventDestroy(c.ev1);
  if (c.stream) cudaStreamDestroy(c.stream);
  delete ctx;
  return PRT_OK;
}

const char* prt_cuda_last_error(const prt_context* ctx)
{
  return ctx ? ctx->c.lastError.c_str() : "null context";
}

void prt_cuda_material_defaults(prt_material* m)
{
  if (!m) return;
  std::memset(m, 0, sizeof(*m));
  m->base_weight = 1.f;
  m->base_color[0] = m->base_color[1] = m->base_color[2] = 0.8f;
  m->specular_weight = 1.f;
  m->specular_color[0] = m->specular_color[1] = m->specular_color[2] = 1.f;
  m->specular_roughness = 0.3f;
  m->specular_ior = 1.5f;
  m->transmission_color[0] = m->transmission_color[1] = m->transmission_color[2] = 1.f;
  m->transmission_depth = 1.f;
  m->subsurface_color[0] = m->subsurface_color[1] = m->subsurface_color[2] = 0.8f;
  m->coat_color[0] = m->coat_color[1] = m->coat_color[2] = 1.f;
  m->coat_ior = 1.6f;
  m->sheen_color[0] = m->sheen_color[1] = m->sheen_color[2] = 1.f;
  m->sheen_roughness = 0.3f;
  m->emission_color[0] = m->emission_color[1] = m->emission_color[2] = 1.f;
  m->opacity = 1.f;
  m->base_color_texture = -1;
  m->model = PRT_MATERIAL_STANDARD;
  m->ambient_ior = 1.f;
  m->coat_thickness = 1.f;
  m->thickness = 1.f;
}

void prt_cuda_principled_defaults(prt_material* m)
{
  if (!m) return;
  prt_cuda_material_defaults(m);
  m->model = PRT_MATERIAL_PRINCIPLED;
  m->specular_color[0] = m->specular_color[1] = m->specular_color[2] = 1.f;  // edgeColor
  m->specular_roughness = 0.f;                                               // roughness
  m->specular_ior = 1.f;                                                     // ior = outsideIor
  m->coat_ior = 1.5f;
  m->sheen_roughness = 0.2f;
  m->emission_luminance = 0.f;
}

int prt_cuda_scene_upload(prt_context* ctx, const prt_scene_desc* scene)
{
  return guarded(ctx, [&](Context& c) {
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    uploadScene(c, scene);
  });
}

int prt_cuda_renderer(prt_context* ctx, const prt_renderer_desc* r)
{
  return guarded(ctx, [&](Context& c) {
    if (!r || r->max_depth < 0 || r->max_depth > 1000) throw std::invalid_argument("invalid renderer settings");
    if (r->type < PRT_RENDERER_PATH || r->type > PRT_RENDERER_DIFFUSE2_FAST) throw std::invalid_argument("invalid renderer type");
    if (r->samples < 0 || r->samples > 4096) throw std::invalid_argument("invalid renderer samples");
    if (r->flags & ~PRT_RENDERER_IRRADIANCE) throw std::invalid_argument("unknown renderer flags");
    if (r->flags && r->type != PRT_RENDERER_PATH) throw std::invalid_argument("irradiance mode is a pathStream option");
    if (r->flags & PRT_RENDERER_IRRADIANCE)
    {
      // render/path_renderer_stream.h:131-139: a Principled material with base colour 1.
      prt_material white;
      prt_cuda_principled_defaults(&white);
      white.base_color[0] = white.base_color[1] = white.base_color[2] = 1.f;
      std::vector<float> media = {1.f, 1.f, 1.f, 1.f};
      c.whiteMaterial = resolveMaterial(white, media, 0);
      c.whiteClass = c.whiteMaterial.shadeClass;
      if (!c.whiteMaterialDev) c.whiteMaterialDev = (DevMaterial*)devAlloc(c, sizeof(DevMaterial), nullptr);
      cuCheck(cudaMemcpy(c.whiteMaterialDev, &c.whiteMaterial, sizeof(DevMaterial), cudaMemcpyHostToDevice),
              "white material");
    }
    c.renderer.flags = r->flags;
    c.renderer.type = r->type;
    c.renderer.aoSamples = r->samples ? r->samples : 16;
    c.renderer.maxDepth = r->max_depth;
    c.renderer.rrDepth = r->rr_depth;
    c.renderer.minWeight = r->min_weight;
    c.renderer.maxRadiance = r->max_radiance;
    c.hasRenderer = true;
    c.sampleIndex = 0;
    ensureCounters(c);
  });
}

int prt_cuda_init_sampler(prt_context* ctx, uint32_t seed)
{
  return guarded(ctx, [&](Context& c) {
    c.renderer.seed = seed;
    c.sampleIndex = 0;
  });
}

int prt_cuda_camera(prt_context* ctx, const prt_camera_desc* cam)
{
  return guarded(ctx, [&](Context& c) {
    if (!cam) throw std::invalid_argument("null camera");
    if (c.width <= 0) throw ApiError{PRT_ERR_STATE, "initialise the frame before the camera"};
    c.camera = makeCamera(*cam, c.width, c.height);
    c.hasCamera = true;
  });
}

int prt_cuda_frame(prt_context* ctx, int32_t width, int32_t height, int32_t aov_mask)
{
  return guarded(ctx, [&](Context& c) {
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    allocFrame(c, width, height, aov_mask);
  });
}

int prt_cuda_clear(prt_context* ctx)
{
  return guarded(ctx, [&](Context& c) {
    if (!c.accum) throw ApiError{PRT_ERR_STATE, "no frame"};
    cuCheck(launchClear(c), "clear");
  });
}

int prt_cuda_render(prt_context* ctx, int32_t spp, prt_render_stats* stats)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    if (!c.hasRenderer || !c.hasCamera || !c.accum) throw ApiError{PRT_ERR_STATE, "renderer, camera and frame are required"};
    if (spp < 0) throw std::invalid_argument("spp must be >= 0");
    if (c.aovSh && c.renderer.type != PRT_RENDERER_PATH) throw std::invalid_argument("the SH AOV is a pathStream AOV");
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    ensurePathState(c, spp);
    cuCheck(cudaEventRecord(c.ev0, c.stream), "event");
    RenderCounters rc;
    cuCheck(renderSamples(c, spp, rc), "render");
    const int64_t rays = rc.closestRays + rc.shadowRays;
    cuCheck(cudaEventRecord(c.ev1, c.stream), "event");
    cuCheck(cudaEventSynchronize(c.ev1), "render sync");
    checkDeviceErrors(c);
    float ms = 0.f;
    cuCheck(cudaEventElapsedTime(&ms, c.ev0, c.ev1), "event time");
    if (stats)
    {
      stats->rays = rays;
      stats->spp = spp;
      stats->render_ms = ms;
      stats->mray = ms > 0.f ? (double)rays / 1e6 / (ms * 1e-3) : 0.0;
      stats->closest_rays = rc.closestRays;
      stats->shadow_rays = rc.shadowRays;
      stats->kernel_launches = rc.launches;
      stats->trace_ms = rc.traceMs;
      stats->shadow_ms = rc.shadowMs;
      stats->shade_ms = rc.shadeMs;
      stats->closest_nodes = (int64_t)rc.trav[0];
      stats->closest_tris = (int64_t)rc.trav[1];
      stats->shadow_nodes = (int64_t)rc.trav[2];
      stats->shadow_tris = (int64_t)rc.trav[3];
      stats->trace_launches = rc.traceLaunches;
    }
  });
}

int prt_cuda_set_profiling(prt_context* ctx, int32_t flags)
{
  return guarded(ctx, [&](Context& c) {
    if (flags & ~3) throw std::invalid_argument("unknown profiling flags");
    c.profileFlags = flags;
  });
}

int prt_cuda_blit(prt_context* ctx, int32_t aov, float* dst)
{
  return guarded(ctx, [&](Context& c) {
    if (!c.accum || !dst) throw std::invalid_argument("no frame or null destination");
    if (aov < 0 || aov > PRT_BLIT_SH3 || ((aov == PRT_BLIT_ALBEDO1 || aov == PRT_BLIT_NORMAL1) && !c.accumA) ||
        (aov == PRT_BLIT_HDR_VAR && !c.accum2) || (aov >= PRT_BLIT_SH0 && !c.accumSH))
      throw std::invalid_argument("AOV not enabled");
    const size_t px = (size_t)c.width * c.height;
    Staged out(c, dst, aov == PRT_BLIT_LDR ? px * sizeof(uint32_t) : px * 3 * sizeof(float), false);
    if (aov == PRT_BLIT_HDR_VAR) cuCheck(launchBlitVariance(c, (float*)out.dev), "blit");
    else if (aov == PRT_BLIT_LDR) cuCheck(launchBlitLdr(c, (uint32_t*)out.dev), "blit");
    else if (aov == PRT_BLIT_LDR_RGB) cuCheck(launchBlitLdrRgb(c, (float*)out.dev), "blit");
    else cuCheck(launchBlit(c, aov, (float*)out.dev), "blit");
    out.copyOut();
    cuCheck(cudaStreamSynchronize(c.stream), "blit sync");
  });
}

int prt_cuda_tone_mapper(prt_context* ctx, int32_t type, float exposure, float burn)
{
  return guarded(ctx, [&](Context& c) {
    if (type < PRT_TONE_NONE || type > PRT_TONE_LOG) throw std::invalid_argument("invalid tone mapper type");
    if (type == PRT_TONE_REINHARD && (burn < 0.f || burn > 1.f)) throw std::invalid_argument("burn must be between 0 and 1");
    c.toneType = type;
    // FilmicToneMapper folds its 18% middle-grey bias into the exposure (image/filmic_tone_mapper.h).
    c.toneExposure = type == PRT_TONE_FILMIC ? exposure * 1.758141f : exposure;
    c.toneInvWhite2 = burn * burn;
  });
}

int prt_cuda_frame_error(prt_context* ctx, float* error)
{
  return guarded(ctx, [&](Context& c) {
    if (!error) throw std::invalid_argument("null output");
    if (!c.accum) throw ApiError{PRT_ERR_STATE, "no frame"};
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    double e = 0.0;
    cuCheck(frameError(c, e), "frame error");
    *error = (float)e;
  });
}

int prt_cuda_scene_load(prt_context* ctx, const char* path, const prt_env_desc* env, int32_t bvh_build)
{
  return guarded(ctx, [&](Context& c) {
    if (!path) throw std::invalid_argument("null path");
    RkScene scene;
    try
    {
      loadSceneFile(path, scene);
    }
    catch (const std::runtime_error& e)
    {
      throw std::invalid_argument(e.what());  // a path that cannot be read is a bad argument here
    }
    prt_scene_desc desc;
    scene.describe(desc);
    if (env) desc.env = *env;
    desc.bvh_build = bvh_build;
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    uploadScene(c, &desc);
  });
}

int prt_cuda_scene_stats(prt_context* ctx, prt_scene_stats* out)
{
  return guarded(ctx, [&](Context& c) {
    if (!out) throw std::invalid_argument("null output");
    if (!c.hasScene) throw ApiError{PRT_ERR_STATE, "no scene"};
    out->build_ms = c.bvhBuildMs;
    out->node_count = c.bvhNodes;
    out->tri_count = c.bvhTris;
    out->builder = c.bvhBuilder;
    out->depth = c.bvhDepth;
    out->top_count = c.bvhTop;
    out->iterations = c.bvhIterations;
    for (int k = 0; k < 3; ++k)
    {
      out->bounds_lo[k] = c.boundsLo[k];
      out->bounds_hi[k] = c.boundsHi[k];
    }
  });
}

int prt_cuda_scene_lights(prt_context* ctx, const prt_env_desc* env)
{
  return guarded(ctx, [&](Context& c) {
    if (!env) throw std::invalid_argument("null environment description");
    requireScene(c);
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    DevScene sc = c.scene;
    buildEnvLights(c, sc, *env);
    cuCheck(cudaStreamSynchronize(c.stream), "scene lights");
    c.scene = sc;
  });
}

int prt_cuda_scene_bvh(prt_context* ctx, void* nodes, int64_t node_capacity, void* tris, int64_t tri_capacity,
                       int64_t* node_count, int64_t* tri_count)
{
  return guarded(ctx, [&](Context& c) {
    if (node_capacity < 0 || tri_capacity < 0 || (node_capacity > 0 && !nodes) || (tri_capacity > 0 && !tris))
      throw std::invalid_argument("invalid output arrays");
    if (!c.hasScene) throw ApiError{PRT_ERR_STATE, "no scene"};
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    const int64_t nn = std::min(node_capacity, c.bvhNodes), nt = std::min(tri_capacity, c.bvhTris);
    if (nn > 0)
      cuCheck(cudaMemcpyAsync(nodes, c.scene.nodes, sizeof(Bvh8Node) * (size_t)nn, cudaMemcpyDeviceToHost, c.stream),
              "copy nodes");
    if (nt > 0)
      cuCheck(cudaMemcpyAsync(tris, c.scene.tris, sizeof(Bvh8Tri) * (size_t)nt, cudaMemcpyDeviceToHost, c.stream),
              "copy triangles");
    cuCheck(cudaStreamSynchronize(c.stream), "copy BVH");
    if (node_count) *node_count = c.bvhNodes;
    if (tri_count) *tri_count = c.bvhTris;
  });
}

int prt_cuda_sobol(prt_context* ctx, int64_t n, const uint32_t* sample_index, const uint32_t* pixel_id,
                   const uint32_t* dim_set, int32_t dims, float* out)
{
  return guarded(ctx, [&](Context& c) {
    if (n < 0 || dims < 1 || dims > 3 || (n > 0 && (!sample_index || !pixel_id || !dim_set || !out)))
      throw std::invalid_argument("invalid sobol query");
    if (n == 0) return;
    Staged si(c, sample_index, n * 4, true), pid(c, pixel_id, n * 4, true), ds(c, dim_set, n * 4, true);
    Staged o(c, out, (size_t)n * dims * 4, false);
    cuCheck(launchSobol(c, n, (const uint32_t*)si.dev, (const uint32_t*)pid.dev, (const uint32_t*)ds.dev, dims,
                        (float*)o.dev), "sobol");
    o.copyOut();
    cuCheck(cudaStreamSynchronize(c.stream), "sobol sync");
  });
}

int prt_cuda_trace(prt_context* ctx, int64_t n, const float* rays, int32_t* geom_id, int32_t* prim_id, float* t,
                   float* u, float* v)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    if (n < 0 || (n > 0 && (!rays || !geom_id || !prim_id || !t))) throw std::invalid_argument("invalid trace query");
    if (n == 0) return;
    Staged r(c, rays, (size_t)n * 32, true);
    Staged tri(c, nullptr, (size_t)n * 4, false);
    Staged to(c, t, (size_t)n * 4, false);
    Staged uo(c, u, u ? (size_t)n * 4 : 0, false), vo(c, v, v ? (size_t)n * 4 : 0, false);
    cuCheck(launchTrace(c, n, (const float*)r.dev, (int32_t*)tri.dev, (float*)to.dev, u ? (float*)uo.dev : nullptr,
                        v ? (float*)vo.dev : nullptr), "trace");
    std::vector<int32_t> triHost(n);
    cuCheck(cudaMemcpyAsync(triHost.data(), tri.dev, n * 4, cudaMemcpyDeviceToHost, c.stream), "copy");
    to.copyOut();
    if (u) uo.copyOut();
    if (v) vo.copyOut();
    checkDeviceErrors(c);
    // Global triangle index -> (mesh, triangle within mesh).
    const std::vector<int>& off = c.meshTriOffsetHost;
    for (int64_t i = 0; i < n; ++i)
    {
      const int id = triHost[i];
      if (id < 0)
      {
        geom_id[i] = prim_id[i] = -1;
        continue;
      }
      const int g = (int)(std::upper_bound(off.begin(), off.end(), id) - off.begin()) - 1;
      geom_id[i] = g;
      prim_id[i] = id - off[g];
    }
  });
}

int prt_cuda_occluded(prt_context* ctx, int64_t n, const float* rays, int32_t* occluded)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    if (n < 0 || (n > 0 && (!rays || !occluded))) throw std::invalid_argument("invalid occlusion query");
    if (n == 0) return;
    Staged r(c, rays, (size_t)n * 32, true);
    Staged o(c, occluded, (size_t)n * 4, false);
    cuCheck(launchOccluded(c, n, (const float*)r.dev, (int32_t*)o.dev), "occluded");
    o.copyOut();
    checkDeviceErrors(c);
  });
}

int prt_cuda_query_primary(prt_context* ctx, uint32_t sample_index, float* rays_out, int32_t* geom_id,
                           int32_t* prim_id, float* t)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    if (!c.hasCamera || c.width <= 0) throw ApiError{PRT_ERR_STATE, "camera and frame are required"};
    if (!rays_out || !geom_id || !prim_id || !t) throw std::invalid_argument("null output");
    const int64_t n = (int64_t)c.width * c.height;
    Staged r(c, rays_out, (size_t)n * 32, false);
    Staged tri(c, nullptr, (size_t)n * 4, false);
    Staged to(c, t, (size_t)n * 4, false);
    cuCheck(launchPrimary(c, sample_index, (float*)r.dev, (int32_t*)tri.dev, (float*)to.dev), "primary");
    r.copyOut();
    to.copyOut();
    std::vector<int32_t> triHost(n);
    cuCheck(cudaMemcpyAsync(triHost.data(), tri.dev, n * 4, cudaMemcpyDeviceToHost, c.stream), "copy");
    checkDeviceErrors(c);
    const std::vector<int>& off = c.meshTriOffsetHost;
    for (int64_t i = 0; i < n; ++i)
    {
      const int id = triHost[i];
      if (id < 0)
      {
        geom_id[i] = prim_id[i] = -1;
        continue;
      }
      const int g = (int)(std::upper_bound(off.begin(), off.end(), id) - off.begin()) - 1;
      geom_id[i] = g;
      prim_id[i] = id - off[g];
    }
  });
}

int prt_bvh8_count(const float* tri_verts, int64_t tri_count, int64_t n, const float* rays, int32_t* tri_out,
                   float* t_out, int64_t* node_visits, int64_t* tri_tests, int64_t* node_count)
{
  if (tri_count < 0 || n < 0 || (tri_count > 0 && !tri_verts) || (n > 0 && (!rays || !tri_out || !t_out)) ||
      !node_visits || !tri_tests || !node_count)
    return PRT_ERR_INVALID_ARG;
  try
  {
    Bvh8 bvh;
    buildBvh8(tri_verts, tri_count, bvh);
    *node_count = (int64_t)bvh.nodes.size();
    int64_t nv = 0, tt = 0;
    for (int64_t i = 0; i < n; ++i)
    {
      const float* r = rays + 8 * i;
      float tfar = r[7];
      tri_out[i] = bvh8TraceCount(bvh, r, r + 4, r[3], tfar, nv, tt);
      t_out[i] = tfar;
    }
    *node_visits += nv;
    *tri_tests += tt;
    return PRT_OK;
  }
  catch (const std::invalid_argument&)
  {
    return PRT_ERR_INVALID_ARG;
  }
  catch (...)
  {
    return PRT_ERR_LOGIC;
  }
}

int prt_bvh8_check(const void* nodes, int64_t node_count, const void* tris, int64_t tri_count,
                   const float* tri_verts, int32_t top_count, int32_t* depth, char* msg, int32_t msg_capacity)
{
  if (node_count < 1 || !nodes || tri_count < 0 || (tri_count > 0 && (!tris || !tri_verts)) || msg_capacity < 0 ||
      (msg_capacity > 0 && !msg))
    return PRT_ERR_INVALID_ARG;
  try
  {
    int d = 0;
    const std::string err = bvh8Check(static_cast<const Bvh8Node*>(nodes), node_count,
                                      static_cast<const Bvh8Tri*>(tris), tri_count, tri_verts, top_count, d);
    if (depth) *depth = d;
    if (msg_capacity > 0)
    {
      const size_t k = std::min(err.size(), (size_t)msg_capacity - 1);
      std::memcpy(msg, err.data(), k);
      msg[k] = 0;
    }
    return err.empty() ? PRT_OK : PRT_ERR_INVALID_ARG;
  }
  catch (...)
  {
    return PRT_ERR_LOGIC;
  }
}

int prt_scene_file_load(const char* path, prt_scene_file** out, char* msg, int32_t msg_capacity)
{
  auto report = [&](const char* what) {
    if (msg && msg_capacity > 0)
    {
      const size_t k = std::min(std::strlen(what), (size_t)msg_capacity - 1);
      std::memcpy(msg, what, k);
      msg[k] = 0;
    }
  };
  if (!path || !out || msg_capacity < 0 || (msg_capacity > 0 && !msg)) return PRT_ERR_INVALID_ARG;
  report("");
  *out = nullptr;
  try
  {
    std::unique_ptr<prt_scene_file> r(new prt_scene_file);
    loadSceneFile(path, r->scene);
    *out = r.release();
    return PRT_OK;
  }
  catch (const std::invalid_argument& e)
  {
    report(e.what());
    return PRT_ERR_INVALID_ARG;
  }
  catch (const std::exception& e)
  {
    report(e.what());
    return PRT_ERR_LOGIC;
  }
}

int prt_scene_file_desc(const prt_scene_file* scene, prt_scene_desc* desc)
{
  if (!scene || !desc) return PRT_ERR_INVALID_ARG;
  scene->scene.describe(*desc);
  return PRT_OK;
}

int prt_scene_file_free(prt_scene_file* scene)
{
  delete scene;
  return PRT_OK;
}

int prt_bvh8_build_host(const float* tri_verts, int64_t tri_count, void* nodes, int64_t node_capacity, void* tris,
                        int64_t tri_capacity, int64_t* node_count, int32_t* top_count)
{
  if (tri_count < 0 || (tri_count > 0 && !tri_verts) || !nodes || node_capacity < std::max<int64_t>(tri_count, 1) ||
      (tri_count > 0 && (!tris || tri_capacity < tri_count)) || !node_count || !top_count)
    return PRT_ERR_INVALID_ARG;
  try
  {
    Bvh8 bvh;
    buildBvh8(tri_verts, tri_count, bvh);
    if ((int64_t)bvh.nodes.size() > node_capacity) return PRT_ERR_LOGIC;
    std::memcpy(nodes, bvh.nodes.data(), sizeof(Bvh8Node) * bvh.nodes.size());
    if (!bvh.tris.empty()) std::memcpy(tris, bvh.tris.data(), sizeof(Bvh8Tri) * bvh.tris.size());
    *node_count = (int64_t)bvh.nodes.size();
    *top_count = std::min(bvh.topCount, kBvh8TopNodes);
    return PRT_OK;
  }
  catch (const std::invalid_argument&)
  {
    return PRT_ERR_INVALID_ARG;
  }
  catch (...)
  {
    return PRT_ERR_LOGIC;
  }
}

int prt_bvh8_trace(const void* nodes, int64_t node_count, const void* tris, int64_t tri_count, int64_t n,
                   const float* rays, int32_t* tri_out, float* t_out, int64_t* node_visits, int64_t* tri_tests)
{
  if (node_count < 1 || !nodes || tri_count < 0 || (tri_count > 0 && !tris) || n < 0 ||
      (n > 0 && (!rays || !tri_out || !t_out)) || !node_visits || !tri_tests)
    return PRT_ERR_INVALID_ARG;
  int64_t nv = 0, tt = 0;
  for (int64_t i = 0; i < n; ++i)
  {
    const float* r = rays + 8 * i;
    float tfar = r[7];
    tri_out[i] = bvh8TraceCount(static_cast<const Bvh8Node*>(nodes), static_cast<const Bvh8Tri*>(tris), r, r + 4,
                                r[3], tfar, nv, tt);
    t_out[i] = tfar;
  }
  *node_visits += nv;
  *tri_tests += tt;
  return PRT_OK;
}

int prt_cuda_bsdf_query(prt_context* ctx, const prt_material* material, int32_t medium_id, int64_t n,
                        const float* tuples, float* out)
{
  return guarded(ctx, [&](Context& c) {
    if (!material || n < 0 || (n > 0 && (!tuples || !out))) throw std::invalid_argument("invalid BSDF query");
    if (material->base_color_texture >= 0) throw std::invalid_argument("BSDF queries take untextured materials");
    std::vector<float> media = {1.f, 1.f, 1.f, 1.f};
    const DevMaterial m = resolveMaterial(*material, media, 0);
    if (n == 0) return;
    Staged in(c, tuples, (size_t)n * 9 * sizeof(float), true);
    Staged o(c, out, (size_t)n * 13 * sizeof(float), false);
    cuCheck(launchBsdfQuery(c, m, medium_id, n, (const float*)in.dev, (float*)o.dev), "bsdf query");
    o.copyOut();
    cuCheck(cudaStreamSynchronize(c.stream), "bsdf sync");
  });
}

int prt_cuda_microfacet_query(prt_context* ctx, int32_t distribution, int64_t n, const float* in, float* out)
{
  return guarded(ctx, [&](Context& c) {
    if (distribution != PRT_MICROFACET_BECKMANN && distribution != PRT_MICROFACET_GGX_VISIBLE)
      throw std::invalid_argument("unknown microfacet distribution");
    if (n < 0 || (n > 0 && (!in || !out))) throw std::invalid_argument("invalid microfacet query");
    if (n == 0) return;
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    Staged i(c, in, (size_t)n * 6 * sizeof(float), true);
    Staged o(c, out, (size_t)n * 4 * sizeof(float), false);
    cuCheck(launchMicrofacetQuery(c, distribution, n, (const float*)i.dev, (float*)o.dev), "microfacet query");
    o.copyOut();
    cuCheck(cudaStreamSynchronize(c.stream), "microfacet sync");
  });
}

int prt_cuda_albedo_tables(prt_context* ctx, float* out, int64_t capacity, int64_t* count)
{
  return guarded(ctx, [&](Context& c) {
    if (!count || capacity < 0 || (capacity > 0 && !out)) throw std::invalid_argument("invalid table query");
    const int64_t head = 32 * 32 + 32 + 3 * (16 * 16 * 16 + 16 * 16);
    const int64_t total = head + 16 * 16;
    *count = total;
    if (capacity == 0) return;
    // GGX, dielectric and reflection tables were allocated back to back in this order
    // (albedo.cu); the sheen table follows them.
    cuCheck(cudaMemcpy(out, c.tableStorage, sizeof(float) * std::min(capacity, head), cudaMemcpyDeviceToHost),
            "table copy");
    if (capacity > head)
      cuCheck(cudaMemcpy(out + head, c.tables.sheenDir, sizeof(float) * std::min<int64_t>(capacity - head, 16 * 16),
                         cudaMemcpyDeviceToHost), "table copy");
  });
}

int prt_cuda_set_albedo_tables(prt_context* ctx, const float* tables, int64_t count)
{
  return guarded(ctx, [&](Context& c) {
    const int64_t head = 32 * 32 + 32 + 3 * (16 * 16 * 16 + 16 * 16);
    if (!tables || count != head + 16 * 16) throw std::invalid_argument("expected the tables of prt_cuda_albedo_tables");
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    cuCheck(cudaStreamSynchronize(c.stream), "sync");
    cuCheck(cudaMemcpy(c.tableStorage, tables, sizeof(float) * head, cudaMemcpyHostToDevice), "table copy");
    cuCheck(cudaMemcpy(const_cast<float*>(c.tables.sheenDir), tables + head, sizeof(float) * 16 * 16,
                       cudaMemcpyHostToDevice), "table copy");
  });
}

int prt_cuda_set_tuning(prt_context* ctx, const prt_tuning* t)
{
  return guarded(ctx, [&](Context& c) {
    if (!t) throw std::invalid_argument("null tuning");
    if (t->trace_blocks < 0 || t->trace_blocks > 32 || t->shade_blocks < 0 || t->shade_blocks > 32 || t->wave_paths < 0 ||
        t->top_stage < 0 || t->top_stage > 2 || t->ray_bins < 0 || t->ray_bins > 2 ||
        (t->trace_stack != 0 && t->trace_stack != 12 && t->trace_stack != 24 && t->trace_stack != 48))
      throw std::invalid_argument("tuning out of range");
    if (t->trace_stack) c.traceStack = t->trace_stack;
    if (t->top_stage) c.topStage = t->top_stage == 1 ? 1 : 0;
    if (t->ray_bins) c.rayBins = t->ray_bins == 1 ? 1 : 0;
    if (t->trace_blocks) c.traceBlocks = t->trace_blocks;
    if (t->shade_blocks) c.shadeBlocks = t->shade_blocks;
    if (t->wave_paths) c.wavePaths = t->wave_paths;
  });
}

int prt_cuda_get_tuning(prt_context* ctx, prt_tuning* t)
{
  return guarded(ctx, [&](Context& c) {
    if (!t) throw std::invalid_argument("null tuning");
    t->trace_blocks = c.traceBlocks;
    t->shade_blocks = c.shadeBlocks;
    t->wave_paths = (int32_t)std::min<int64_t>(c.wavePaths, 0x7fffffff);
    t->top_stage = c.topStage ? 1 : 2;
    t->ray_bins = c.rayBins ? 1 : 2;
    t->trace_stack = c.traceStack;
  });
}

int prt_cuda_autotune(prt_context* ctx, int32_t spp, prt_tuning* chosen, double* mrays)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    if (!c.hasRenderer || !c.hasCamera || !c.accum) throw ApiError{PRT_ERR_STATE, "renderer, camera and frame are required"};
    if (spp <= 0) throw std::invalid_argument("spp must be > 0");
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    auto timeOne = [&](int tb, int sb, int64_t wave, int top, int bins, int stack) {
      c.traceStack = stack;
      c.traceBlocks = tb;
      c.shadeBlocks = sb;
      c.wavePaths = wave;
      c.topStage = top;
      c.rayBins = bins;
      ensurePathState(c, spp);
      RenderCounters rc;
      cuCheck(cudaEventRecord(c.ev0, c.stream), "event");
      cuCheck(renderSamples(c, spp, rc), "autotune render");
      cuCheck(cudaEventRecord(c.ev1, c.stream), "event");
      cuCheck(cudaEventSynchronize(c.ev1), "autotune sync");
      float ms = 0.f;
      cuCheck(cudaEventElapsedTime(&ms, c.ev0, c.ev1), "event time");
      return (double)(rc.closestRays + rc.shadowRays) / 1e6 / (ms * 1e-3);
    };
    const int profile = c.profileFlags;
    c.profileFlags = 0;
    int bT = c.traceBlocks, bS = c.shadeBlocks, bTop = c.topStage, bBins = c.rayBins, bStack = c.traceStack;
    int64_t bW = c.wavePaths;
    timeOne(bT, bS, bW, bTop, bBins, bStack);  // warm-up
    double best = -1.0;
    // One axis at a time: wave size (paths in flight), traversal and shading grids, staging
    // of the top BVH levels in shared memory, octant binning of extended rays, stack depth.
    for (int64_t w : {8ll << 20, 16ll << 20, 32ll << 20, 64ll << 20, 128ll << 20})
    {
      const double v = timeOne(bT, bS, w, bTop, bBins, bStack);
      if (v > best) { best = v; bW = w; }
    }
    for (int tb : {4, 6, 8, 12})
    {
      const double v = timeOne(tb, bS, bW, bTop, bBins, bStack);
      if (v > best) { best = v; bT = tb; }
    }
    for (int sb : {2, 4, 8})
    {
      const double v = timeOne(bT, sb, bW, bTop, bBins, bStack);
      if (v > best) { best = v; bS = sb; }
    }
    for (int top : {0, 1})
    {
      const double v = timeOne(bT, bS, bW, top, bBins, bStack);
      if (v > best) { best = v; bTop = top; }
    }
    for (int bins : {0, 1})
    {
      const double v = timeOne(bT, bS, bW, bTop, bins, bStack);
      if (v > best) { best = v; bBins = bins; }
    }
    for (int stack : {12, 24, 48})
      if (c.bvhDepth <= stack && stack != bStack)
      {
        const double v = timeOne(bT, bS, bW, bTop, bBins, stack);
        if (v > best) { best = v; bStack = stack; }
      }
    c.traceStack = bStack;
    c.topStage = bTop;
    c.rayBins = bBins;
    c.traceBlocks = bT;
    c.shadeBlocks = bS;
    c.wavePaths = bW;
    c.profileFlags = profile;
    checkDeviceErrors(c);
    cuCheck(launchClear(c), "clear");
    c.sampleIndex = 0;
    cuCheck(cudaStreamSynchronize(c.stream), "sync");
    if (chosen)
    {
      chosen->trace_blocks = bT;
      chosen->ray_bins = bBins ? 1 : 2;
      chosen->shade_blocks = bS;
      chosen->wave_paths = (int32_t)bW;
      chosen->top_stage = bTop ? 1 : 2;
      chosen->trace_stack = bStack;
    }
    if (mrays) *mrays = best;
  });
}

} // extern "C"

// ---- Rendering without device allocation ------------------------------------------------------
//
// prt_cuda_render_static renders from a fixed scratch area compiled into this library instead of
// the path state that prt_cuda_render allocates on demand. The area holds the path state of at
// most kStaticPaths paths, three accumulation planes of as many pixels, and the per-bounce
// counters for maxDepth <= kStaticMaxDepth: about 18 MB on every GPU that loads the library,
// held until the process exits.

namespace {

constexpr int64_t kStaticPaths = 1 << 16;  // paths in flight = largest frame, in pixels
constexpr int kStaticMaxDepth = 1000;      // the deepest renderer prt_cuda_renderer accepts
constexpr size_t kStaticAlign = 256;

constexpr size_t staticRound(size_t n) { return (n + kStaticAlign - 1) / kStaticAlign * kStaticAlign; }

// Byte offsets of the carved buffers.
constexpr size_t kStaticPlane = staticRound(sizeof(float4) * kStaticPaths);  // one float4 per path
constexpr size_t kStaticQueue = staticRound(sizeof(int) * kStaticPaths);
constexpr size_t kStaticPathPlanes = 12;  // rayO rayD hit thr rad info shO shD shL out aovA aovN
constexpr size_t kStaticOffQueues = kStaticPathPlanes * kStaticPlane;
constexpr size_t kStaticOffAccum = kStaticOffQueues + (2 + kShadeClasses) * kStaticQueue;
constexpr size_t kStaticOffCounters = kStaticOffAccum + 3 * kStaticPlane;
// Per-bounce counter blocks (16 ints each) followed by the 16 ints of the octant bins, the layout
// ensureCounters gives the allocating path.
constexpr size_t kStaticOffTrav = kStaticOffCounters + staticRound(sizeof(int) * (16 * (kStaticMaxDepth + 2) + 16));
constexpr size_t kStaticOffErr = kStaticOffTrav + staticRound(4 * sizeof(unsigned long long));
constexpr size_t kStaticBytes = kStaticOffErr + kStaticAlign;

// The scratch area itself. Host code must not pass `gStaticScratch` to a kernel: on the host the
// name denotes a host-side shadow, not the device address. staticScratchOf() looks the device
// address up once per device.
static __device__ __align__(256) unsigned char gStaticScratch[kStaticBytes];

constexpr int kStaticMaxDevices = 64;
std::mutex gStaticMutex;
unsigned char* gStaticAddr[kStaticMaxDevices] = {};

// Device address of the scratch area on device `dev`, which must be the current device.
unsigned char* staticScratchOf(int dev)
{
  if (dev < 0 || dev >= kStaticMaxDevices) throw ApiError{PRT_ERR_INVALID_ARG, "device ordinal out of range"};
  std::lock_guard<std::mutex> lock(gStaticMutex);
  if (!gStaticAddr[dev])
  {
    void* p = nullptr;
    cuCheck(cudaGetSymbolAddress(&p, gStaticScratch), "cudaGetSymbolAddress(static scratch)");
    gStaticAddr[dev] = static_cast<unsigned char*>(p);
  }
  return gStaticAddr[dev];
}

// Restores the context's own path state, frame and sample index when the static render returns
// or throws.
struct StaticSwap
{
  Context& c;
  PathState ps;
  float *accum, *accumA, *accumN, *accumC, *accum2;
  int64_t accumCount;
  int waveSamples, profileFlags;
  uint32_t sampleIndex;
  explicit StaticSwap(Context& ctx)
      : c(ctx), ps(ctx.ps), accum(ctx.accum), accumA(ctx.accumA), accumN(ctx.accumN), accumC(ctx.accumC),
        accum2(ctx.accum2), accumCount(ctx.accumCount), waveSamples(ctx.waveSamples), profileFlags(ctx.profileFlags),
        sampleIndex(ctx.sampleIndex)
  {
  }
  ~StaticSwap()
  {
    c.ps = ps;
    c.accumC = accumC;
    c.accum2 = accum2;
    c.accumCount = accumCount;
    c.accum = accum;
    c.accumA = accumA;
    c.accumN = accumN;
    c.waveSamples = waveSamples;
    c.profileFlags = profileFlags;
    c.sampleIndex = sampleIndex;
  }
};

} // namespace

extern "C" {

int prt_cuda_render_static(prt_context* ctx, uint32_t first_sample, int32_t spp, float* hdr_out)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    // Only the frame's size and AOV mask are used: the sums live in the scratch area, so the
    // frame planes prt_cuda_frame allocated are neither needed nor touched.
    if (!c.hasRenderer || !c.hasCamera || c.width <= 0 || c.height <= 0)
      throw ApiError{PRT_ERR_STATE, "renderer, camera and frame size are required"};
    if (spp <= 0) throw std::invalid_argument("spp must be > 0");
    if (!hdr_out) throw std::invalid_argument("null output");
    const int64_t px = (int64_t)c.width * c.height;
    if (px > kStaticPaths)
      throw std::invalid_argument("frame of " + std::to_string(c.width) + "x" + std::to_string(c.height) + " = " +
                                  std::to_string(px) + " pixels exceeds the static scratch limit of " +
                                  std::to_string(kStaticPaths) + " pixels");
    if (c.renderer.maxDepth > kStaticMaxDepth) throw std::invalid_argument("maxDepth exceeds the static scratch limit");
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, hdr_out) != cudaSuccess ||
        (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged))
    {
      cudaGetLastError();
      throw std::invalid_argument("hdr_out must be device or managed memory");
    }
    // Device memory of another GPU would be written across the interconnect (or fault without
    // peer access): only this context's device is accepted.
    if (attr.type == cudaMemoryTypeDevice && attr.device != c.device)
      throw std::invalid_argument("hdr_out is on device " + std::to_string(attr.device) +
                                  ", the context renders on device " + std::to_string(c.device));
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    unsigned char* base = staticScratchOf(c.device);

    StaticSwap keep(c);
    c.accumC = nullptr;  // the static render keeps no checkpoint or variance of its own
    c.accum2 = nullptr;
    c.accumCount = 0;
    PathState s;
    s.capacity = kStaticPaths;
    float4* planes[kStaticPathPlanes];
    for (size_t k = 0; k < kStaticPathPlanes; ++k) planes[k] = reinterpret_cast<float4*>(base + k * kStaticPlane);
    s.rayO = planes[0]; s.rayD = planes[1]; s.hit = planes[2]; s.thr = planes[3]; s.rad = planes[4];
    s.info = reinterpret_cast<uint4*>(planes[5]);
    s.shO = planes[6]; s.shD = planes[7]; s.shL = planes[8]; s.out = planes[9];
    s.aovA = planes[10]; s.aovN = planes[11];
    s.queue[0] = reinterpret_cast<int*>(base + kStaticOffQueues);
    s.queue[1] = reinterpret_cast<int*>(base + kStaticOffQueues + kStaticQueue);
    s.classQueues = reinterpret_cast<int*>(base + kStaticOffQueues + 2 * kStaticQueue);
    s.counters = reinterpret_cast<int*>(base + kStaticOffCounters);
    s.octBins = s.counters + 16 * (c.renderer.maxDepth + 2);
    s.travCounts = reinterpret_cast<unsigned long long*>(base + kStaticOffTrav);
    s.err = reinterpret_cast<uint32_t*>(base + kStaticOffErr);
    c.ps = s;
    c.accum = reinterpret_cast<float*>(base + kStaticOffAccum);
    c.accumA = c.aovMask ? reinterpret_cast<float*>(base + kStaticOffAccum + kStaticPlane) : nullptr;
    c.accumN = c.aovMask ? reinterpret_cast<float*>(base + kStaticOffAccum + 2 * kStaticPlane) : nullptr;
    c.waveSamples = (int)(kStaticPaths / px);
    c.sampleIndex = first_sample;
    c.profileFlags = 0;
    // The area keeps the previous call's contents: zero the sums and the error flag.
    cuCheck(cudaMemsetAsync(base + kStaticOffAccum, 0, 3 * kStaticPlane, c.stream), "clear static sums");
    cuCheck(cudaMemsetAsync(s.err, 0, sizeof(uint32_t), c.stream), "clear static error flag");
    RenderCounters rc;
    cuCheck(renderSamples(c, spp, rc), "static render");
    cuCheck(launchBlit(c, 0, hdr_out), "static blit");
    checkDeviceErrors(c);
  });
}

} // extern "C"

// ---- batch rendering ----------------------------------------------------------------------------

struct prt_batch
{
  prt_context* ctx;
  BatchState b;
};

namespace {

void freeBatch(BatchState& b)
{
  if (b.exec) cudaGraphExecDestroy(b.exec);
  b.exec = nullptr;
  if (b.execReplay) cudaGraphExecDestroy(b.execReplay);
  b.execReplay = nullptr;
  for (auto& x : b.bufs) cudaFree(x.ptr);
  b.bufs.clear();
}

} // namespace

extern "C" {

int prt_cuda_batch_create(prt_context* ctx, const prt_batch_item* items, int32_t count, prt_batch** out)
{
  if (out) *out = nullptr;
  return guarded(ctx, [&](Context& c) {
    if (!out || !items || count <= 0) throw std::invalid_argument("invalid batch description");
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    std::unique_ptr<prt_batch> bp(new prt_batch{ctx, BatchState()});
    BatchState& B = bp->b;
    try
    {
      for (int i = 0; i < count; ++i)
      {
        const prt_batch_item& it = items[i];
        if (!it.scene) throw std::invalid_argument("batch item without a scene");
        if (it.width <= 0 || it.height <= 0 || it.spp <= 0) throw std::invalid_argument("invalid batch item frame");
        if (it.width % 32 != 0 || it.height % 8 != 0)
          throw std::logic_error("image size is not divisible by the tile size");
        if (it.width > 4096 || it.height > 4096) throw std::logic_error("image size is too large");
        if (it.renderer.max_depth < 0 || it.renderer.max_depth > 1000) throw std::invalid_argument("invalid renderer settings");
        if (it.renderer.type != PRT_RENDERER_PATH) throw std::invalid_argument("batches render with the path tracer");
        if (it.renderer.flags) throw std::invalid_argument("batches render with the standard path tracer");
        if (it.aov_mask & ~(PRT_AOV_ALBEDO1 | PRT_AOV_NORMAL1)) throw std::invalid_argument("unknown AOV bits");
        // Scene upload through the frame form's path, into buffers the batch owns.
        Context tmp;
        tmp.device = c.device;
        tmp.stream = c.stream;
        tmp.smCount = c.smCount;
        // Frees what an upload that throws part-way has allocated; the buffers move to the batch below.
        struct TmpBufs
        {
          Context& t;
          ~TmpBufs()
          {
            for (const DevBuf& b : t.sceneBufs) cudaFree(b.ptr);
            for (const DevBuf& b : t.envBufs) cudaFree(b.ptr);
          }
        } tmpGuard{tmp};
        uploadScene(tmp, it.scene);
        B.bvhDepth = std::max(B.bvhDepth, tmp.bvhDepth);
        B.bufs.insert(B.bufs.end(), tmp.sceneBufs.begin(), tmp.sceneBufs.end());
        tmp.sceneBufs.clear();
        // The environment lights' buffers too. Each item keeps its own copy of its image light even
        // where the sky is the same: one copy shared by the items measured 3.5% slower on a 64-frame
        // batch under one sky.
        B.bufs.insert(B.bufs.end(), tmp.envBufs.begin(), tmp.envBufs.end());
        tmp.envBufs.clear();
        B.itemMaterials.push_back(tmp.materialsHost);
        B.itemTextures.push_back(tmp.texturesHost);
        BatchItem bi;
        std::memset(&bi, 0, sizeof(bi));
        bi.sc = tmp.scene;
        bi.cam = makeCamera(it.camera, it.width, it.height);
        bi.rd = DevRenderer{it.renderer.max_depth, it.renderer.rr_depth, it.renderer.min_weight, it.renderer.max_radiance,
                            it.seed, PRT_RENDERER_PATH, 16};
        bi.width = it.width;
        bi.height = it.height;
        bi.pixelCount = it.width * it.height;
        bi.aovMask = it.aov_mask;
        bi.workBase = B.workTotal;
        bi.workCount = (long long)bi.pixelCount * it.spp;
        B.workTotal += bi.workCount;
        const size_t plane = (size_t)bi.pixelCount * sizeof(float4);
        bi.accum = (float4*)devAlloc(c, plane, &B.bufs);
        if (it.aov_mask)
        {
          bi.accA = (float4*)devAlloc(c, plane, &B.bufs);
          bi.accN = (float4*)devAlloc(c, plane, &B.bufs);
          B.anyAov = true;
        }
        B.maxDepth = std::max(B.maxDepth, it.renderer.max_depth);
        B.items.push_back(bi);
      }
      // Per work item: radiance and, for items with AOVs, first-hit albedo and normal (kBatchAccumulate).
      const size_t workBytes = (size_t)B.workTotal * sizeof(float4);
      B.workOut = (float4*)devAlloc(c, workBytes, &B.bufs);
      if (B.anyAov)
      {
        B.workA = (float4*)devAlloc(c, workBytes, &B.bufs);
        B.workN = (float4*)devAlloc(c, workBytes, &B.bufs);
      }
      // Shared path pool: as many slots as the frame form's wave, at most the whole batch.
      const int64_t C = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(c.wavePaths, B.workTotal), (int64_t)kQueuePathMask));
      PathState& s = B.ps;
      s.capacity = C;
      auto a4 = [&](int64_t n) { return (float4*)devAlloc(c, (size_t)n * sizeof(float4), &B.bufs); };
      s.rayO = a4(C); s.rayD = a4(C); s.hit = a4(C); s.thr = a4(C); s.rad = a4(C);
      s.info = (uint4*)a4(C);
      s.shO = a4(C); s.shD = a4(C); s.shL = a4(C);
      if (B.anyAov)
      {
        s.aovA = a4(C);
        s.aovN = a4(C);
      }
      s.queue[0] = (int*)devAlloc(c, (size_t)C * sizeof(int), &B.bufs);
      s.queue[1] = (int*)devAlloc(c, (size_t)C * sizeof(int), &B.bufs);
      s.classQueues = (int*)devAlloc(c, (size_t)C * kShadeClasses * sizeof(int), &B.bufs);
      s.err = c.ps.err;
      s.travCounts = c.ps.travCounts;
      B.freeList[0] = (int*)devAlloc(c, (size_t)C * sizeof(int), &B.bufs);
      B.freeList[1] = (int*)devAlloc(c, (size_t)C * sizeof(int), &B.bufs);
      B.ctl = (BatchCtl*)devAlloc(c, sizeof(BatchCtl), &B.bufs);
      B.dItems = (BatchItem*)devAlloc(c, B.items.size() * sizeof(BatchItem), &B.bufs);
      cuCheck(cudaMemcpyAsync(B.dItems, B.items.data(), B.items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice,
                              c.stream), "batch items");
      cuCheck(cudaStreamSynchronize(c.stream), "batch upload");
    }
    catch (...)
    {
      freeBatch(B);
      throw;
    }
    *out = bp.release();
  });
}

int prt_cuda_batch_render(prt_batch* batch, prt_render_stats* stats)
{
  if (!batch) return PRT_ERR_INVALID_ARG;
  return guarded(batch->ctx, [&](Context& c) {
    BatchState& B = batch->b;
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    RenderCounters rc;
    cuCheck(cudaEventRecord(c.ev0, c.stream), "event");
    const cudaError_t e = renderBatch(c, B, rc);
    if (e == cudaErrorLaunchTimeout)
      throw ApiError{PRT_ERR_DEVICE_ABORT, "batch render did not finish within its iteration bound"};
    cuCheck(e, "batch render");
    cuCheck(cudaEventRecord(c.ev1, c.stream), "event");
    cuCheck(cudaEventSynchronize(c.ev1), "batch sync");
    checkDeviceErrors(c);
    float ms = 0.f;
    cuCheck(cudaEventElapsedTime(&ms, c.ev0, c.ev1), "event time");
    if (stats)
    {
      std::memset(stats, 0, sizeof(*stats));
      stats->rays = rc.closestRays + rc.shadowRays;
      stats->spp = 0;
      stats->render_ms = ms;
      stats->mray = ms > 0.f ? (double)stats->rays / 1e6 / (ms * 1e-3) : 0.0;
      stats->closest_rays = rc.closestRays;
      stats->shadow_rays = rc.shadowRays;
      stats->kernel_launches = rc.launches;
      stats->trace_launches = rc.traceLaunches;
    }
  });
}

int prt_cuda_batch_blit(prt_batch* batch, int32_t item, int32_t aov, float* dst)
{
  if (!batch) return PRT_ERR_INVALID_ARG;
  return guarded(batch->ctx, [&](Context& c) {
    BatchState& B = batch->b;
    if (item < 0 || item >= (int)B.items.size() || !dst) throw std::invalid_argument("invalid batch item or destination");
    const BatchItem& it = B.items[item];
    if (aov < 0 || aov > 2 || (aov > 0 && !it.accA)) throw std::invalid_argument("AOV not enabled");
    const float4* plane = aov == 0 ? it.accum : (aov == 1 ? it.accA : it.accN);
    Staged o(c, dst, (size_t)it.pixelCount * 3 * sizeof(float), false);
    cuCheck(launchBlitPlane(c, plane, it.pixelCount, (float*)o.dev), "batch blit");
    o.copyOut();
    cuCheck(cudaStreamSynchronize(c.stream), "batch blit sync");
  });
}

int prt_cuda_batch_destroy(prt_batch* batch)
{
  if (!batch) return PRT_ERR_INVALID_ARG;
  cudaSetDevice(batch->ctx->c.device);
  cudaStreamSynchronize(batch->ctx->c.stream);
  freeBatch(batch->b);
  delete batch;
  return PRT_OK;
}

} // extern "C"

// ---- differentiation ----------------------------------------------------------------------------

namespace {

// New contents of one texture (caller order, row 0 at the top; host or device memory).
void updateTexture(Context& c, const std::vector<DevTexture>& textures, int texture, const float* rgb)
{
  if (texture < 0 || texture >= (int)textures.size() || !rgb) throw std::invalid_argument("invalid texture update");
  cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
  const DevTexture& t = textures[texture];
  Staged src(c, rgb, 3ull * t.width * t.height * sizeof(float), true);
  cuCheck(launchTextureUpdate(c, t, (const float*)src.dev), "texture update");
  cuCheck(cudaStreamSynchronize(c.stream), "texture update sync");
}

// New parameters of materials [first, first + count); each keeps its lobe set, emission and
// medium. One copy to the device for the whole range.
void updateMaterials(Context& c, DevMaterial* devMaterials, std::vector<DevMaterial>& host, int textureCount, int first,
                     int count, const prt_material* ms)
{
  if (first < 0 || count < 0 || first + count > (int)host.size() || (count > 0 && !ms))
    throw std::invalid_argument("invalid material update");
  if (count == 0) return;
  std::vector<DevMaterial> ds(count);
  for (int i = 0; i < count; ++i)
  {
    std::vector<float> media = {1.f, 1.f, 1.f, 1.f};
    DevMaterial d = resolveMaterial(ms[i], media, textureCount);
    const DevMaterial& old = host[first + i];
    if (d.type != old.type || d.features != old.features || d.shadeClass != old.shadeClass)
      throw std::invalid_argument("a material update must keep the material's lobes (re-upload the scene instead)");
    if ((d.type & kMatMediaInterface) && (d.specularIor != old.specularIor || d.transmissionDepth != old.transmissionDepth ||
                                          std::memcmp(d.transmissionColor, old.transmissionColor, sizeof(float) * 3) != 0))
      throw std::invalid_argument("a material update must keep the medium of a transmissive material");
    if (std::memcmp(d.emission, old.emission, sizeof(float) * 3) != 0)
      throw std::invalid_argument("a material update must keep the emission (re-upload the scene instead)");
    d.mediumInt = old.mediumInt;
    d.mediumExt = old.mediumExt;
    ds[i] = d;
  }
  cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
  cuCheck(cudaMemcpyAsync(devMaterials + first, ds.data(), sizeof(DevMaterial) * count, cudaMemcpyHostToDevice, c.stream),
          "material update");
  cuCheck(cudaStreamSynchronize(c.stream), "material update sync");
  for (int i = 0; i < count; ++i) host[first + i] = ds[i];
}

void requireAdjointMaterials(const std::vector<DevMaterial>& materials)
{
  for (const DevMaterial& m : materials)
    if ((m.type & kMatTransparent) || (!(m.type & kMatEmissive) && (m.features & ~(kFeatOpaque | kFeatSpecular))))
      throw std::invalid_argument("the adjoint supports opaque Lambertian materials with an optional specular layer");
}

bool isDeviceMemory(const void* p)
{
  cudaPointerAttributes attr;
  if (!p || cudaPointerGetAttributes(&attr, p) != cudaSuccess)
  {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

} // namespace


extern "C" {

int prt_cuda_adjoint(prt_context* ctx, uint32_t first_sample, int32_t spp, const float* d_loss_d_image,
                     float* grad_textures, int64_t grad_texture_count, float* grad_roughness,
                     int32_t grad_roughness_count, prt_render_stats* stats)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    if (!c.hasRenderer || !c.hasCamera || !c.accum) throw ApiError{PRT_ERR_STATE, "renderer, camera and frame are required"};
    if (spp <= 0 || !d_loss_d_image) throw std::invalid_argument("invalid adjoint request");
    if (c.renderer.type != PRT_RENDERER_PATH) throw std::invalid_argument("the adjoint differentiates the path tracer");
    if (c.renderer.flags || c.aovSh)
      throw std::invalid_argument("the adjoint differentiates the standard path tracer without the SH AOV");
    requireAdjointMaterials(c.materialsHost);
    if (c.texturesHost.size() > 32) throw std::invalid_argument("the adjoint supports at most 32 textures");
    int64_t texFloats = 0;
    for (const DevTexture& t : c.texturesHost) texFloats += 3ll * t.width * t.height;
    const int64_t mats = (int64_t)c.materialsHost.size();
    if ((grad_textures && grad_texture_count < texFloats) || (grad_roughness && grad_roughness_count < mats))
      throw std::invalid_argument("gradient buffers are too small");
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    const size_t px = (size_t)c.width * c.height;
    Staged dl(c, d_loss_d_image, px * 3 * sizeof(float), true);
    // Gradients are always accumulated on the device; host outputs are copied at the end.
    Staged gt(c, grad_textures, (size_t)std::max<int64_t>(texFloats, 1) * sizeof(float), false);
    Staged gr(c, grad_roughness, (size_t)std::max<int64_t>(mats, 1) * sizeof(float), false);
    cuCheck(cudaMemsetAsync(gt.dev, 0, (size_t)std::max<int64_t>(texFloats, 1) * sizeof(float), c.stream), "clear");
    cuCheck(cudaMemsetAsync(gr.dev, 0, (size_t)std::max<int64_t>(mats, 1) * sizeof(float), c.stream), "clear");
    ensurePathState(c, spp);
    RenderCounters rc;
    cuCheck(cudaEventRecord(c.ev0, c.stream), "event");
    cuCheck(launchAdjoint(c, first_sample, spp, (const float*)dl.dev, (float*)gt.dev, (float*)gr.dev, 1e-3f, rc),
            "adjoint");
    cuCheck(cudaEventRecord(c.ev1, c.stream), "event");
    if (grad_textures) gt.copyOut();
    if (grad_roughness) gr.copyOut();
    cuCheck(cudaStreamSynchronize(c.stream), "adjoint sync");
    checkDeviceErrors(c);
    float ms = 0.f;
    cuCheck(cudaEventElapsedTime(&ms, c.ev0, c.ev1), "event time");
    if (stats)
    {
      std::memset(stats, 0, sizeof(*stats));
      stats->spp = spp;
      stats->render_ms = ms;
      stats->rays = rc.closestRays + rc.shadowRays;
      stats->closest_rays = rc.closestRays;
      stats->shadow_rays = rc.shadowRays;
      stats->kernel_launches = rc.launches;
      stats->trace_launches = rc.traceLaunches;
    }
  });
}

int prt_cuda_update_texture(prt_context* ctx, int32_t texture, const float* rgb)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    updateTexture(c, c.texturesHost, texture, rgb);
  });
}

int prt_cuda_update_material(prt_context* ctx, int32_t material, const prt_material* m)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    updateMaterials(c, const_cast<DevMaterial*>(c.scene.materials), c.materialsHost, (int)c.texturesHost.size(),
                    material, 1, m);
  });
}

int prt_cuda_update_materials(prt_context* ctx, int32_t first, int32_t count, const prt_material* ms)
{
  return guarded(ctx, [&](Context& c) {
    requireScene(c);
    updateMaterials(c, const_cast<DevMaterial*>(c.scene.materials), c.materialsHost, (int)c.texturesHost.size(),
                    first, count, ms);
  });
}

} // extern "C"

// ---- batched differentiation --------------------------------------------------------------------

extern "C" {

int prt_cuda_batch_enable_adjoint(prt_batch* batch)
{
  if (!batch) return PRT_ERR_INVALID_ARG;
  return guarded(batch->ctx, [&](Context& c) {
    BatchState& B = batch->b;
    for (const auto& mats : B.itemMaterials) requireAdjointMaterials(mats);
    for (const auto& texs : B.itemTextures)
      if (texs.size() > (size_t)kAdjointMaxTextures) throw std::invalid_argument("the adjoint supports at most 32 textures");
    if (B.pathL) return;
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    cuCheck(cudaStreamSynchronize(c.stream), "sync");
    B.pathL = (float4*)devAlloc(c, (size_t)B.workTotal * sizeof(float4), &B.bufs);
    // The replay keeps each path's radiance still to come in ps.out, which the forward batch
    // does not use (it accumulates finished paths directly).
    B.ps.out = (float4*)devAlloc(c, (size_t)B.ps.capacity * sizeof(float4), &B.bufs);
    // Graphs capture the launch parameters: capture both again with the new buffers.
    if (B.exec) cudaGraphExecDestroy(B.exec);
    B.exec = nullptr;
    if (B.execReplay) cudaGraphExecDestroy(B.execReplay);
    B.execReplay = nullptr;
  });
}

int prt_cuda_batch_adjoint(prt_batch* batch, const float* const* d_loss_d_images, float* const* grad_textures,
                           float* const* grad_roughness, prt_render_stats* stats)
{
  if (!batch) return PRT_ERR_INVALID_ARG;
  return guarded(batch->ctx, [&](Context& c) {
    BatchState& B = batch->b;
    if (!B.pathL) throw ApiError{PRT_ERR_STATE, "call prt_cuda_batch_enable_adjoint and render the batch first"};
    if (!d_loss_d_images || !grad_textures || !grad_roughness) throw std::invalid_argument("null gradient arrays");
    cuCheck(cudaSetDevice(c.device), "cudaSetDevice");
    std::vector<BatchItem> items = B.items;
    for (size_t k = 0; k < items.size(); ++k)
    {
      const float* dl = d_loss_d_images[k];
      float* gt = grad_textures[k];
      float* gr = grad_roughness[k];
      int64_t texFloats = 0;
      for (const DevTexture& t : B.itemTextures[k]) texFloats += 3ll * t.width * t.height;
      const int64_t mats = (int64_t)B.itemMaterials[k].size();
      if (!isDeviceMemory(dl) || !isDeviceMemory(gr) || (texFloats > 0 && !isDeviceMemory(gt)))
        throw std::invalid_argument("batch adjoint buffers must be device or managed memory");
      AdjointView& A = items[k].adj;
      std::memset(&A, 0, sizeof(A));
      A.dLdI = dl;
      A.gradTex = gt;
      A.gradRough = gr;
      long long off = 0;
      for (size_t i = 0; i < B.itemTextures[k].size(); ++i)
      {
        A.texOffset[i] = off;
        off += 3ll * B.itemTextures[k][i].width * B.itemTextures[k][i].height;
      }
      A.step = 1e-3f;
      A.invSpp = (float)((double)items[k].pixelCount / (double)items[k].workCount);
      if (texFloats > 0) cuCheck(cudaMemsetAsync(gt, 0, (size_t)texFloats * sizeof(float), c.stream), "clear");
      cuCheck(cudaMemsetAsync(gr, 0, (size_t)mats * sizeof(float), c.stream), "clear");
    }
    cuCheck(cudaMemcpyAsync(B.dItems, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, c.stream),
            "batch items");
    RenderCounters rc;
    cuCheck(cudaEventRecord(c.ev0, c.stream), "event");
    const cudaError_t e = replayBatch(c, B, rc);
    if (e == cudaErrorLaunchTimeout)
      throw ApiError{PRT_ERR_DEVICE_ABORT, "batch replay did not finish within its iteration bound"};
    cuCheck(e, "batch adjoint");
    cuCheck(cudaEventRecord(c.ev1, c.stream), "event");
    cuCheck(cudaEventSynchronize(c.ev1), "batch adjoint sync");
    checkDeviceErrors(c);
    float ms = 0.f;
    cuCheck(cudaEventElapsedTime(&ms, c.ev0, c.ev1), "event time");
    if (stats)
    {
      std::memset(stats, 0, sizeof(*stats));
      stats->render_ms = ms;
      stats->closest_rays = rc.closestRays;
      stats->rays = rc.closestRays;
      stats->kernel_launches = rc.launches;
      stats->trace_launches = rc.traceLaunches;
    }
  });
}

int prt_cuda_batch_update_texture(prt_batch* batch, int32_t item, int32_t texture, const float* rgb)
{
  if (!batch) return PRT_ERR_INVALID_ARG;
  return guarded(batch->ctx, [&](Context& c) {
    BatchState& B = batch->b;
    if (item < 0 || item >= (int)B.items.size()) throw std::invalid_argument("invalid batch item");
    updateTexture(c, B.itemTextures[item], texture, rgb);
  });
}

int prt_cuda_batch_update_material(prt_batch* batch, int32_t item, int32_t material, const prt_material* m)
{
  if (!batch) return PRT_ERR_INVALID_ARG;
  return guarded(batch->ctx, [&](Context& c) {
    BatchState& B = batch->b;
    if (item < 0 || item >= (int)B.items.size()) throw std::invalid_argument("invalid batch item");
    updateMaterials(c, const_cast<DevMaterial*>(B.items[item].sc.materials), B.itemMaterials[item],
                    (int)B.itemTextures[item].size(), material, 1, m);
  });
}

int prt_cuda_batch_update_materials(prt_batch* batch, int32_t item, int32_t first, int32_t count,
                                    const prt_material* ms)
{
  if (!batch) return PRT_ERR_INVALID_ARG;
  return guarded(batch->ctx, [&](Context& c) {
    BatchState& B = batch->b;
    if (item < 0 || item >= (int)B.items.size()) throw std::invalid_argument("invalid batch item");
    updateMaterials(c, const_cast<DevMaterial*>(B.items[item].sc.materials), B.itemMaterials[item],
                    (int)B.itemTextures[item].size(), first, count, ms);
  });
}

} // extern "C"
