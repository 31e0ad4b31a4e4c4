// BSDFs of the reference's Standard material on the device.
//
// StandardMaterial::getBsdfLobes (material/standard.cpp:410-620) builds, per hit, a small
// tree: MultiBsdf{opaque base, translucent base, metal base}, optionally wrapped by a coat
// and a sheen layer. Here the tree is a fixed struct: the per-hit parameters are resolved
// once (resolveStandard) and eval/sample walk the same composition with the same
// arithmetic as the reference classes, without virtual calls or an arena.
#pragma once

#include "shading.cuh"

namespace prt {

// BsdfType bits (bsdf/bsdf.h:15-44).
enum : int
{
  kDiffuseReflection = 1 << 0,
  kGlossyReflection = 1 << 1,
  kSpecularReflection = 1 << 2,
  kDiffuseTransmission = 1 << 3,
  kGlossyTransmission = 1 << 4,
  kSpecularTransmission = 1 << 5,
  kUnbentTransmission = 1 << 6,
  kTransparency = 1 << 7,
  kBsdfDiffuse = kDiffuseReflection | kDiffuseTransmission,
  kBsdfGlossy = kGlossyReflection | kGlossyTransmission,
  kBsdfSpecular = kSpecularReflection | kSpecularTransmission,
  kBsdfContinuation = kUnbentTransmission | kTransparency,
  kBsdfSmooth = kBsdfDiffuse | kBsdfGlossy,
  kBsdfDelta = kBsdfSpecular | kBsdfContinuation,
};

// ---- DiffuseBrdf (bsdf/diffuse.h:45-82) ------------------------------------------------------
struct DiffuseLobe
{
  f3 color;

  PRT_D float importance() const { return reduceMax(color); }

  PRT_D f3 eval(const Frame& fr, f3 wi, float& pdf) const
  {
    const float cosThetaI = fmaxf(dot(wi, fr.N), 0.f);
    pdf = cosThetaI * kInvPi;
    return color * kInvPi * cosThetaI;
  }

  PRT_D f3 sample(const Frame& fr, f3 Ng, float sx, float sy, f3& wi, float& pdf, int& type) const
  {
    wi = toWorld(fr, cosineSampleHemisphere(pdf, sx, sy));
    type = kDiffuseReflection;
    return dot(wi, Ng) > 0.f ? color : mk(0.f);
  }
};

// Per-hit Standard-material BSDF. Lobe slots follow the MultiBsdf order the reference adds
// them in (opaque, translucent, metal).
struct StdBsdf
{
  Frame fr;
  f3 Ng;
  int flags;
  int nLobes;
  float scale[3];
  float imp[3];
  float impSum;
  int kind[3];       // lobe kind per slot
  DiffuseLobe diffuse;
  f3 albedo;

  PRT_D f3 evalLobe(int i, f3 wo, f3 wi, float& pdf) const
  {
    (void)wo;
    return diffuse.eval(fr, wi, pdf);
  }

  PRT_D f3 sampleLobe(int i, f3 wo, float sx, float sy, float sz, f3& wi, float& pdf, int& type) const
  {
    (void)wo;
    (void)sz;
    return diffuse.sample(fr, Ng, sx, sy, wi, pdf, type);
  }

  // MultiBsdfSimd::eval (bsdf/multi_bsdf.h:173-190).
  PRT_D f3 eval(f3 wo, f3 wi, float& pdf) const
  {
    f3 value = mk(0.f);
    pdf = 0.f;
    for (int i = 0; i < nLobes; ++i)
    {
      if (!(imp[i] > 0.f)) continue;
      float p;
      const f3 v = evalLobe(i, wo, wi, p);
      value += v * scale[i];
      pdf += p * imp[i];
    }
    pdf *= 1.f / impSum;
    return value;
  }

  // MultiBsdfSimd::sample (bsdf/multi_bsdf.h:192-270).
  PRT_D f3 sample(f3 wo, float sx, float sy, float sz, f3& wi, float& pdf, int& type) const
  {
    pdf = 0.f;
    type = 0;
    if (!(impSum > 0.f)) return mk(0.f);
    if (nLobes == 1)
    {
      const f3 w = sampleLobe(0, wo, sx, sy, sz, wi, pdf, type);
      return w * scale[0];
    }
    const float x = sz * impSum;
    int choice = 0;
    float prefix = imp[0], importance = imp[0], sc = scale[0];
    for (int i = 1; i < nLobes; ++i)
    {
      if (!(x > prefix)) break;
      choice = i;
      prefix += imp[i];
      importance = imp[i];
      sc = scale[i];
    }
    const float s1 = (x + importance - prefix) * (1.f / importance);
    f3 weight = sampleLobe(choice, wo, sx, sy, s1, wi, pdf, type);
    if (!(reduceMax(weight) > 0.f))
    {
      weight = mk(0.f);
      pdf = 0.f;
      type = 0;
    }
    weight *= sc;
    if (!(reduceMax(weight) > 0.f) || !(pdf > 0.f)) return mk(0.f);
    if (type & kBsdfDelta) return weight * impSum * (1.f / importance);
    f3 value = weight * pdf;
    pdf *= importance;
    for (int i = 0; i < nLobes; ++i)
    {
      if (i == choice || !(imp[i] > 0.f)) continue;
      float p;
      const f3 v = evalLobe(i, wo, wi, p);
      value += v * scale[i];
      pdf += p * imp[i];
    }
    pdf *= 1.f / impSum;
    return value * (1.f / pdf);
  }
};

// Material texture lookup: repeat in both directions (image/image_texture.h:197-226).
PRT_D f3 textureRgb(const DevTexture& t, float u, float v)
{
  return texLookup(t.rgb, t.width, t.height, u, v, true);
}

// StandardMaterial::getBsdfLobes (material/standard.cpp:410-620), the lobes implemented on
// the device: Lambertian base without specular, subsurface, coat or sheen layers.
PRT_D void resolveStandard(const DevScene& sc, const DevMaterial& m, const ShadeCtx& ctx, f3 wo, StdBsdf& b)
{
  b.fr = makeShadingFrame(ctx, wo);
  b.Ng = ctx.Ng;
  b.flags = 0;
  b.nLobes = 0;
  b.impSum = 0.f;
  const float base = clamp01(m.baseWeight);
  f3 baseColor = mk(m.baseColor[0], m.baseColor[1], m.baseColor[2]);
  if (m.baseColorTex >= 0) baseColor = textureRgb(sc.textures[m.baseColorTex], ctx.uvx, ctx.uvy) * baseColor;
  baseColor = clamp01(baseColor);
  const float metalness = clamp01(m.metalness);
  const float dielectric = 1.f - metalness;
  if (dielectric > kMatEps)
  {
    const float transmission = clamp01(m.transmissionWeight);
    const float opaque = dielectric * (1.f - transmission);
    if (opaque > kMatEps)
    {
      b.diffuse.color = baseColor * base;
      const int i = b.nLobes++;
      b.kind[i] = 0;
      b.scale[i] = opaque;
      b.imp[i] = b.diffuse.importance() * opaque;
      b.impSum += b.imp[i];
      b.flags |= kDiffuseReflection;
    }
  }
  b.albedo = b.diffuse.color;
}

} // namespace prt
