// Test infrastructure (oracle only): batched BSDF queries through the reference's own
// Standard material (material/standard.cpp:410-620) and BsdfSimd classes.
//
// Each query is a (wo, wi, 3D sample) tuple in a canonical shading context: the shading
// frame is the identity (U = x, V = y, N = z), the geometric normal is z, UV = (0.5, 0.5),
// the hit is front-facing and the path is in medium `mediumId`. For each tuple the output is
//   eval value (3), eval pdf, sample weight (3), sampled wi (3), sample pdf, sample type,
//   BSDF flags                                                        -> 13 floats
// computed with Material::getBsdf (material/material.h:66-76) then BsdfSimd::eval / ::sample,
// eight lanes at a time exactly as the stream renderer calls them.
#define RKSCENE_FLOAT2   prt::Vec2f
#define RKSCENE_FLOAT3   prt::Vec3f
#define RKSCENE_FLOAT4   prt::Vec4f
#define RKSCENE_FLOAT3X4 prt::Affine3f

#include <cstring>
#include <memory>
#include <string>

#include "bsdf/albedo_tables.h"
#include "material/material_factory.h"
#include "material/material.h"
#include "core/shading_context.h"
#include "bsdf/bsdf.h"
#include "bsdf/beckmann_distribution.h"
#include "bsdf/ggx_distribution.h"

#include "../include/prt_cuda.h"

using namespace prt;

namespace {

Props standardProps(const prt_material& m)
{
  // The keys Scene::loadScene sets for an rkscene material (render/scene.cpp:180-212).
  Props p;
  auto v3 = [](const float* a) { return Vec3f(a[0], a[1], a[2]); };
  p.set("type", "Standard");
  p.set("ambientIOR", m.ambient_ior);
  p.set("baseWeight", m.base_weight);
  p.set("baseColor", v3(m.base_color));
  p.set("metalness", m.metalness);
  p.set("diffuseRoughness", m.diffuse_roughness);
  p.set("specularWeight", m.specular_weight);
  p.set("specularColor", v3(m.specular_color));
  p.set("specularRoughness", m.specular_roughness);
  p.set("specularIOR", m.specular_ior);
  p.set("transmissionWeight", m.transmission_weight);
  p.set("transmissionColor", v3(m.transmission_color));
  p.set("transmissionDepth", m.transmission_depth);
  p.set("subsurfaceWeight", m.subsurface_weight);
  p.set("subsurfaceColor", v3(m.subsurface_color));
  p.set("subsurfaceAnisotropy", m.subsurface_anisotropy);
  p.set("coatWeight", m.coat_weight);
  p.set("coatColor", v3(m.coat_color));
  p.set("coatRoughness", m.coat_roughness);
  p.set("coatIOR", m.coat_ior);
  p.set("sheenWeight", m.sheen_weight);
  p.set("sheenColor", v3(m.sheen_color));
  p.set("sheenRoughness", m.sheen_roughness);
  p.set("emissionLuminance", m.emission_luminance);
  p.set("emissionColor", v3(m.emission_color));
  p.set("thinWalled", m.thin_walled);
  p.set("opacity", m.opacity);
  return p;
}

// The keys PrincipledMaterial reads (material/principled.cpp:21-60), from the same record.
Props principledProps(const prt_material& m)
{
  Props p;
  auto v3 = [](const float* a) { return Vec3f(a[0], a[1], a[2]); };
  p.set("type", "Principled");
  p.set("baseColor", v3(m.base_color));
  p.set("edgeColor", v3(m.specular_color));
  p.set("metallic", m.metalness);
  p.set("diffuse", m.base_weight);
  p.set("specular", m.specular_weight);
  p.set("outsideIor", m.ambient_ior);
  p.set("ior", m.specular_ior);
  p.set("transmission", m.transmission_weight);
  p.set("transmissionColor", v3(m.transmission_color));
  p.set("transmissionDepth", m.transmission_depth);
  p.set("roughness", m.specular_roughness);
  p.set("coat", m.coat_weight);
  p.set("coatIor", m.coat_ior);
  p.set("coatColor", v3(m.coat_color));
  p.set("coatThickness", m.coat_thickness);
  p.set("coatRoughness", m.coat_roughness);
  p.set("sheen", m.sheen_weight);
  p.set("sheenColor", v3(m.sheen_color));
  p.set("sheenTint", m.sheen_tint);
  p.set("sheenRoughness", m.sheen_roughness);
  p.set("thin", m.thin_walled);
  p.set("backlight", m.backlight);
  p.set("thickness", m.thickness);
  p.set("opacity", m.opacity);
  return p;
}

} // namespace

extern "C" {

int ref_bsdf_query(const prt_material* mat, int mediumId, int64_t n, const float* tuples, float* out)
{
  try
  {
    precomputeAlbedoTables();
    MaterialFactory factory("", Props());
    std::shared_ptr<Material> material =
      factory.make(mat->model == PRT_MATERIAL_PRINCIPLED ? principledProps(*mat) : standardProps(*mat));
    for (int64_t base = 0; base < n; base += simdSize)
    {
      const int lanes = (int)std::min<int64_t>(simdSize, n - base);
      vbool m = vint(step) < lanes;
      Vec3vf wo, wi, s;
      for (int k = 0; k < simdSize; ++k)
      {
        const float* t = tuples + 9 * (base + std::min(k, lanes - 1));
        wo.x[k] = t[0]; wo.y[k] = t[1]; wo.z[k] = t[2];
        wi.x[k] = t[3]; wi.y[k] = t[4]; wi.z[k] = t[5];
        s.x[k] = t[6]; s.y[k] = t[7]; s.z[k] = t[8];
      }
      ShadingContextSimd ctx;
      ctx.p = Vec3vf(zero);
      ctx.f.U = Vec3vf(1.f, 0.f, 0.f);
      ctx.f.V = Vec3vf(0.f, 1.f, 0.f);
      ctx.f.N = Vec3vf(0.f, 0.f, 1.f);
      ctx.Ng = Vec3vf(0.f, 0.f, 1.f);
      for (int u = 0; u < maxNumUVs; ++u) ctx.uv[u] = Vec2vf(0.5f);
      ctx.backfacing = vbool(zero);
      ctx.eps = vfloat(1e-6f);
      const BsdfSimd* bsdf = material->getBsdf(m, ctx, wo, vint(mediumId));
      vfloat evalPdf;
      Vec3vf evalValue = bsdf->eval(m, ctx, wo, wi, evalPdf);
      Vec3vf sWi = zero;
      vfloat sPdf = zero;
      vint sType = zero;
      Vec3vf sWeight = bsdf->sample(m, ctx, wo, sWi, sPdf, sType, BsdfSampleSimd(s));
      vint flags = bsdf->getFlags();
      for (int k = 0; k < lanes; ++k)
      {
        float* o = out + 13 * (base + k);
        o[0] = evalValue.x[k]; o[1] = evalValue.y[k]; o[2] = evalValue.z[k]; o[3] = evalPdf[k];
        o[4] = sWeight.x[k]; o[5] = sWeight.y[k]; o[6] = sWeight.z[k];
        o[7] = sWi.x[k]; o[8] = sWi.y[k]; o[9] = sWi.z[k];
        o[10] = sPdf[k];
        int ty = sType[k];
        int fl = flags[k];
        std::memcpy(&o[11], &ty, 4);
        std::memcpy(&o[12], &fl, 4);
      }
    }
    return 0;
  }
  catch (const std::exception&)
  {
    return -1;
  }
}

// The same query through the reference's scalar BSDF path (Material::getBsdf(ShadingContext&)
// -> Bsdf::eval/sample, material/material.h:54-64, bsdf/bsdf.h:66-89), whose arithmetic is the
// scalar library's rather than the SIMD path's approximate reciprocals and polynomials, in the
// shading frame `frame` (U, V, N and the geometric normal Ng: 12 floats). A rotated frame with
// correspondingly rotated directions poses the same problem in other coordinates: the exact
// answer is unchanged, the reference's rounding is not.
int ref_bsdf_query_scalar_frame(const prt_material* mat, int mediumId, const float* frame, int64_t n,
                                const float* tuples, float* out)
{
  try
  {
    precomputeAlbedoTables();
    MaterialFactory factory("", Props());
    std::shared_ptr<Material> material =
      factory.make(mat->model == PRT_MATERIAL_PRINCIPLED ? principledProps(*mat) : standardProps(*mat));
    auto ctx = std::make_unique<ShadingContext>();
    for (int64_t i = 0; i < n; ++i)
    {
      const float* t = tuples + 9 * i;
      const Vec3f wo(t[0], t[1], t[2]), wi(t[3], t[4], t[5]), s(t[6], t[7], t[8]);
      ctx->p = Vec3f(zero);
      ctx->f.U = Vec3f(frame[0], frame[1], frame[2]);
      ctx->f.V = Vec3f(frame[3], frame[4], frame[5]);
      ctx->f.N = Vec3f(frame[6], frame[7], frame[8]);
      ctx->Ng = Vec3f(frame[9], frame[10], frame[11]);
      for (int u = 0; u < maxNumUVs; ++u) ctx->uv[u] = Vec2f(0.5f);
      ctx->backfacing = false;
      ctx->eps = 1e-6f;
      const Bsdf* bsdf = material->getBsdf(*ctx, wo, mediumId);
      float evalPdf = 0.f;
      const Vec3f evalValue = bsdf->eval(*ctx, wo, wi, evalPdf);
      Vec3f sWi = zero;
      float sPdf = 0.f;
      int sType = 0;
      const Vec3f sWeight = bsdf->sample(*ctx, wo, sWi, sPdf, sType, BsdfSample(s));
      const int flags = bsdf->getFlags();
      float* o = out + 13 * i;
      o[0] = evalValue.x; o[1] = evalValue.y; o[2] = evalValue.z; o[3] = evalPdf;
      o[4] = sWeight.x; o[5] = sWeight.y; o[6] = sWeight.z;
      o[7] = sWi.x; o[8] = sWi.y; o[9] = sWi.z;
      o[10] = sPdf;
      std::memcpy(&o[11], &sType, 4);
      std::memcpy(&o[12], &flags, 4);
    }
    return 0;
  }
  catch (const std::exception&)
  {
    return -1;
  }
}

int ref_bsdf_query_scalar(const prt_material* mat, int mediumId, int64_t n, const float* tuples, float* out)
{
  static const float canonical[12] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 1.f};
  return ref_bsdf_query_scalar_frame(mat, mediumId, canonical, n, tuples, out);
}

// Microfacet sampling with the reference's distributions, in the layout of
// prt_cuda_microfacet_query: per tuple (alpha, s.x, s.y, wo.x, wo.y, wo.z) -> (m.x, m.y, m.z,
// pdf). simd != 0 runs the vfloat instantiation (8 tuples per call), else the float one.
int ref_microfacet_query(int distribution, int simd, int64_t n, const float* in, float* out)
{
  if (distribution != PRT_MICROFACET_BECKMANN && distribution != PRT_MICROFACET_GGX_VISIBLE) return -1;
  if (!simd)
  {
    for (int64_t i = 0; i < n; ++i)
    {
      const float* t = in + 6 * i;
      float pdf = 0.f;
      Vec3f m;
      if (distribution == PRT_MICROFACET_BECKMANN)
        m = BeckmannDistribution<float>(t[0]).sample(pdf, Vec2f(t[1], t[2]));
      else
        m = GGXDistribution<float>(Vec2f(t[0])).sampleVisible(Vec3f(t[3], t[4], t[5]), pdf, Vec2f(t[1], t[2]));
      float* o = out + 4 * i;
      o[0] = m.x; o[1] = m.y; o[2] = m.z; o[3] = pdf;
    }
    return 0;
  }
  for (int64_t base = 0; base < n; base += simdSize)
  {
    const int lanes = (int)std::min<int64_t>(simdSize, n - base);
    vfloat alpha, sx, sy;
    Vec3vf wo;
    for (int k = 0; k < simdSize; ++k)
    {
      const float* t = in + 6 * (base + std::min(k, lanes - 1));
      alpha[k] = t[0]; sx[k] = t[1]; sy[k] = t[2];
      wo.x[k] = t[3]; wo.y[k] = t[4]; wo.z[k] = t[5];
    }
    vfloat pdf = zero;
    Vec3vf m;
    if (distribution == PRT_MICROFACET_BECKMANN)
      m = BeckmannDistribution<vfloat>(alpha).sample(pdf, Vec2vf(sx, sy));
    else
      m = GGXDistribution<vfloat>(Vec2vf(alpha)).sampleVisible(wo, pdf, Vec2vf(sx, sy));
    for (int k = 0; k < lanes; ++k)
    {
      float* o = out + 4 * (base + k);
      o[0] = m.x[k]; o[1] = m.y[k]; o[2] = m.z[k]; o[3] = pdf[k];
    }
  }
  return 0;
}

// The reference's energy-compensation tables in the order of prt_cuda_albedo_tables.
int64_t ref_albedo_tables(float* out)
{
  precomputeAlbedoTables();
  float* o = out;
  auto put = [&](const float* src, int n) {
    if (out) std::memcpy(o, src, sizeof(float) * n);
    o += n;
  };
  put(MicrofacetAlbedoTable::dir, 32 * 32);
  put(MicrofacetAlbedoTable::avg, 32);
  put(MicrofacetDielectricAlbedoTable::etaDir, 16 * 16 * 16);
  put(MicrofacetDielectricAlbedoTable::etaAvg, 16 * 16);
  put(MicrofacetDielectricAlbedoTable::rcpEtaDir, 16 * 16 * 16);
  put(MicrofacetDielectricAlbedoTable::rcpEtaAvg, 16 * 16);
  put(MicrofacetDielectricReflectionAlbedoTable::etaDir, 16 * 16 * 16);
  put(MicrofacetDielectricReflectionAlbedoTable::etaAvg, 16 * 16);
  put(MicrofacetSheenAlbedoTable::dir, 16 * 16);
  return (int64_t)(o - out);
}

} // extern "C"
