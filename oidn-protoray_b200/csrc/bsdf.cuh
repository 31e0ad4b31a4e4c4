// BSDFs of the reference's Standard material on the device.
//
// StandardMaterial::getBsdfLobes (material/standard.cpp:410-620) builds, per hit, a small
// tree: MultiBsdf{opaque base, translucent base, metal base}, optionally wrapped by a coat
// layer. Here the tree is a fixed struct: the per-hit parameters are resolved once
// (resolveStandard) and eval/sample walk the same composition with the same arithmetic as
// the reference classes, without virtual calls or a per-hit arena.
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

// ---- energy-compensation tables (bsdf/albedo_tables.h; DevTables in device_scene.h) -----------
constexpr int kGgxTableSize = 32;
constexpr int kTableSize = 16;

// math/interpolation.h interp{1,2,3,4}DLinear: clamp, floor, lerp a + s*(b - a).
PRT_D float lerpf(float a, float b, float s) { return a + s * (b - a); }

PRT_D void interpAxis(float p, int size, int& i0, int& i1, float& s)
{
  const float c = fminf(fmaxf(p, 0.f), (float)(size - 1));
  s = c - floorf(c);
  i0 = min((int)c, size - 1);
  i1 = min(i0 + 1, size - 1);
}

PRT_D float interp1D(const float* f, int size, float x)
{
  int a, b;
  float s;
  interpAxis(x, size, a, b, s);
  return lerpf(__ldg(f + a), __ldg(f + b), s);
}

PRT_D float interp2D(const float* f, int size, float x, float y)
{
  int x0, x1, y0, y1;
  float sx, sy;
  interpAxis(x, size, x0, x1, sx);
  interpAxis(y, size, y0, y1, sy);
  const float f0 = lerpf(__ldg(f + x0 + y0 * size), __ldg(f + x1 + y0 * size), sx);
  const float f1 = lerpf(__ldg(f + x0 + y1 * size), __ldg(f + x1 + y1 * size), sx);
  return lerpf(f0, f1, sy);
}

PRT_D float interp3D(const float* f, int size, float x, float y, float z)
{
  int z0, z1;
  float sz;
  interpAxis(z, size, z0, z1, sz);
  const int n2 = size * size;
  return lerpf(interp2D(f + z0 * n2, size, x, y), interp2D(f + z1 * n2, size, x, y), sz);
}

PRT_D float interp4D(const float* f, int size, float x, float y, float z, float w)
{
  int w0, w1;
  float sw;
  interpAxis(w, size, w0, w1, sw);
  const int n3 = size * size * size;
  return lerpf(interp3D(f + w0 * n3, size, x, y, z), interp3D(f + w1 * n3, size, x, y, z), sw);
}

// MicrofacetAlbedoTable (bsdf/albedo_tables.h:8-37)
PRT_D float ggxAlbedo(const DevTables& t, float cosThetaO, float roughness)
{
  const float k = (float)(kGgxTableSize - 1);
  return interp2D(t.ggxDir, kGgxTableSize, cosThetaO * k, roughness * k);
}

PRT_D float ggxAlbedoAvg(const DevTables& t, float roughness)
{
  return interp1D(t.ggxAvg, kGgxTableSize, roughness * (float)(kGgxTableSize - 1));
}

// MicrofacetDielectricAlbedoTable (bsdf/albedo_tables.h:39-130): eta <= 1 uses the eta table
// over [1/3, 1], eta > 1 the reciprocal table over [1, 3].
PRT_D float dielAlbedo(const DevTables& t, float cosThetaO, float eta, float roughness)
{
  const float k = (float)(kTableSize - 1);
  if (eta <= 1.f)
  {
    const float e = (eta - t.etaLo) / (t.etaHi - t.etaLo);
    return interp3D(t.dielEtaDir, kTableSize, cosThetaO * k, e * k, roughness * k);
  }
  const float e = (eta - 1.f) / (3.f - 1.f);
  return interp3D(t.dielRcpDir, kTableSize, cosThetaO * k, e * k, roughness * k);
}

PRT_D float dielAlbedoAvg(const DevTables& t, float eta, float roughness)
{
  const float k = (float)(kTableSize - 1);
  if (eta <= 1.f)
  {
    const float e = (eta - t.etaLo) / (t.etaHi - t.etaLo);
    return interp2D(t.dielEtaAvg, kTableSize, e * k, roughness * k);
  }
  const float e = (eta - 1.f) / (3.f - 1.f);
  return interp2D(t.dielRcpAvg, kTableSize, e * k, roughness * k);
}

// MicrofacetDielectricReflectionAlbedoTable (bsdf/albedo_tables.h:132-170)
PRT_D float reflAlbedo(const DevTables& t, float cosThetaO, float eta, float roughness)
{
  const float k = (float)(kTableSize - 1);
  const float e = (eta - t.etaLo) / (t.etaHi - t.etaLo);
  return interp3D(t.reflDir, kTableSize, cosThetaO * k, e * k, roughness * k);
}

// MicrofacetSheenAlbedoTable (bsdf/albedo_tables.h:281-300): 16 x 16 over (cos, roughness).
PRT_D float sheenAlbedo(const DevTables& t, float cosThetaO, float roughness)
{
  const float k = (float)(kTableSize - 1);
  return interp2D(t.sheenDir, kTableSize, cosThetaO * k, roughness * k);
}

PRT_D float reflAlbedoAvg(const DevTables& t, float eta, float roughness)
{
  const float k = (float)(kTableSize - 1);
  const float e = (eta - t.etaLo) / (t.etaHi - t.etaLo);
  return interp2D(t.reflAvg, kTableSize, e * k, roughness * k);
}

// ---- microfacet distribution (bsdf/ggx_distribution.h) ---------------------------------------
PRT_D float roughnessToAlpha(float r) { return fmaxf(r * r, 0.001f); }

struct GGX
{
  float ax, ay;

  PRT_D float eval(f3 wh) const
  {
    const float c2 = sqr(wh.z);
    const float e = (sqr(wh.x / ax) + sqr(wh.y / ay)) / c2;
    return 1.f / (kPi * ax * ay * sqr(c2 * (1.f + e)));
  }

  PRT_D float lambda(f3 w) const
  {
    const float c2 = sqr(w.z);
    const float invA2 = (sqr(w.x * ax) + sqr(w.y * ay)) / c2;
    return 0.5f * (-1.f + sqrtf(1.f + invA2));
  }

  PRT_D float G1(f3 w) const { return 1.f / (1.f + lambda(w)); }
  PRT_D float G2(f3 wo, f3 wi) const { return 1.f / (1.f + lambda(wo) + lambda(wi)); }

  PRT_D float evalVisible(f3 wh, f3 wo, float cosThetaOH, float& pdf) const
  {
    const float D = eval(wh);
    pdf = G1(wo) * fabsf(cosThetaOH) * D / fabsf(wo.z);
    return D;
  }

  // Visible-normal sampling (Heitz 2018), GGXDistribution::sampleVisible.
  PRT_D f3 sampleVisible(f3 wo, float& pdf, float sx, float sy) const
  {
    const f3 V = normalize(mk(ax * wo.x, ay * wo.y, wo.z));
    const f3 T1 = V.z < 0.9999f ? normalize(cross(V, mk(0.f, 0.f, 1.f))) : mk(1.f, 0.f, 0.f);
    const f3 T2 = cross(T1, V);
    const float a = 1.f / (1.f + V.z);
    const float r = sqrtf(sx);
    // phi = sy < a ? sy / a * pi : pi + (sy - a) / (1 - a) * pi
    const float phiOverPi = sy < a ? sy / a : 1.f + (sy - a) / (1.f - a);
    float sp, cp;
    sincospif(phiOverPi, &sp, &cp);
    const float P1 = r * cp;
    const float P2 = r * sp * (sy < a ? 1.f : V.z);
    f3 wh = P1 * T1 + P2 * T2 + sqrtf(fmaxf(0.f, 1.f - P1 * P1 - P2 * P2)) * V;
    wh = normalize(mk(ax * wh.x, ay * wh.y, fmaxf(0.f, wh.z)));
    pdf = G1(wo) * fabsf(dot(wo, wh)) * eval(wh) / fabsf(wo.z);
    return wh;
  }
};

// ---- Beckmann distribution (bsdf/beckmann_distribution.h:14-43) -------------------------------
// Samples a microfacet normal m with density D(m) cos(theta_m) (Walter et al. 2007, eqs. 28-29):
// tan^2(theta) = -alpha^2 log(1 - s.x), phi = 2 pi s.y, pdf = (1 - s.x) / (pi alpha^2 cos^3(theta)).
// The reference uses it for the flakes of its CarPaint material.
struct Beckmann
{
  float alpha;

  PRT_D f3 sample(float& pdf, float sx, float sy) const
  {
    const float a2 = alpha * alpha;
    const float tanTheta2 = -a2 * logf(1.f - sx);
    const float cosTheta = 1.f / sqrtf(1.f + tanTheta2);
    const float sinTheta = sqrtf(fmaxf(1.f - cosTheta * cosTheta, 0.f));
    float sinPhi, cosPhi;
    sincospif(2.f * sy, &sinPhi, &cosPhi);
    pdf = (1.f - sx) / (kPi * a2 * (cosTheta * cosTheta * cosTheta));
    return mk(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
  }
};

// ---- Fresnel (bsdf/optics.h) -------------------------------------------------------------------
PRT_D float fresnelDielectric(float cosI, float cosT, float eta)
{
  const float Rper = (eta * cosI - cosT) * (1.f / (eta * cosI + cosT));
  const float Rpar = (cosI - eta * cosT) * (1.f / (cosI + eta * cosT));
  return 0.5f * (Rpar * Rpar + Rper * Rper);
}

PRT_D float fresnelDielectric(float cosI, float eta)
{
  cosI = fmaxf(cosI, 0.f);
  const float k = 1.f - eta * eta * (1.f - cosI * cosI);
  if (!(k >= 0.f)) return 1.f;
  return fresnelDielectric(cosI, sqrtf(k), eta);
}

PRT_D float fresnelDielectricEx(float cosI, float& cosT, float eta)
{
  cosI = fabsf(cosI);
  const float k = 1.f - eta * eta * (1.f - cosI * cosI);
  if (!(k >= 0.f))
  {
    cosT = 0.f;
    return 1.f;
  }
  cosT = sqrtf(k);
  return fresnelDielectric(cosI, cosT, eta);
}

// fresnelDielectricAvg (bsdf/optics.h:137-149) depends on eta alone; it is evaluated on the host
// per material and side (DevEta::favg, favgRcp).

PRT_D float refractCos(float cosI, float eta)
{
  const float k = 1.f - eta * eta * (1.f - cosI * cosI);
  return sqrtf(fmaxf(k, 0.f));
}

PRT_D f3 refractDir(f3 I, f3 N, float cosI, float cosT, float eta) { return eta * (cosI * N - I) - cosT * N; }

PRT_D float fresnelConductor(float cosI, float eta, float k)
{
  cosI = fabsf(cosI);
  const float tmp = sqr(eta) + sqr(k);
  const float c2 = sqr(cosI);
  const float Rpar = (tmp * c2 - 2.f * eta * cosI + 1.f) * (1.f / (tmp * c2 + 2.f * eta * cosI + 1.f));
  const float Rper = (tmp - 2.f * eta * cosI + c2) * (1.f / (tmp + 2.f * eta * cosI + c2));
  return 0.5f * (Rpar + Rper);
}

// Gulbrandsen's artistic (reflectivity, edge tint) -> (eta, k).
PRT_D void artisticToIor(float r, float g, float& eta, float& k)
{
  r = fminf(r, 0.99f);
  const float nMin = (1.f - r) / (1.f + r);
  const float nMax = (1.f + sqrtf(r)) / (1.f - sqrtf(r));
  const float n = g * nMin + (1.f - g) * nMax;
  const float k2 = (sqr(n + 1.f) * r - sqr(n - 1.f)) / (1.f - r);
  eta = n;
  k = sqrtf(fmaxf(k2, 0.f));
}

PRT_D float artisticAvg(float r, float g)
{
  const float r2 = r * r, r3 = r2 * r, g2 = g * g, g3 = g2 * g;
  return 0.087237f + 0.0230685f * g - 0.0864902f * g2 + 0.0774594f * g3 + 0.782654f * r - 0.136432f * r2 +
         0.278708f * r3 + 0.19744f * g * r + 0.0360605f * g2 * r - 0.2586f * g * r2;
}

PRT_D f3 powf3(f3 c, float e) { return mk(powf(c.x, e), powf(c.y, e), powf(c.z, e)); }
PRT_D f3 lerp3(f3 a, f3 b, float s) { return a + s * (b - a); }

// ---- lobes ---------------------------------------------------------------------------------------

// DiffuseBrdf (bsdf/diffuse.h:45-82).
// R: the instance may be rough (kFeatRoughDiffuse); R = false compiles the rough branch out.
template <bool R>
struct DiffuseLobeT
{
  f3 color;
  float roughness;  // Oren-Nayar roughness (rough lobe only)
  bool rough;       // RoughDiffuseBrdf (bsdf/rough_diffuse.h:53-108) instead of DiffuseBrdf

  PRT_D int flags() const { return kDiffuseReflection; }
  PRT_D float importance() const { return reduceMax(color); }
  PRT_D f3 albedo() const { return color; }

  PRT_D f3 eval(const Frame& fr, f3 Ng, f3 wo, f3 wi, float& pdf) const
  {
    if (R && rough)
    {
      // Oren-Nayar with Fujii's simplification ("A tiny improvement of Oren-Nayar reflectance
      // model", 2012): f = color (1 + r s / t) / (pi + (pi/2 - 2/3) r), s = wo.wi - cos_o cos_i,
      // t = max(cos_o, cos_i) where s > 0, else 1.
      const float cosThetaO = fmaxf(dot(wo, fr.N), 0.f);
      const float cosThetaI = fmaxf(dot(wi, fr.N), 0.f);
      pdf = cosThetaI * kInvPi;
      const float s = dot(wo, wi) - cosThetaO * cosThetaI;
      const float sInvt = s > 0.f ? s * rcpSafe(fmaxf(cosThetaO, cosThetaI)) : s;
      return color * (cosThetaI * (1.f + roughness * sInvt) * (1.f / (kPi + (0.5f * kPi - 2.f / 3.f) * roughness)));
    }
    const float cosThetaI = fmaxf(dot(wi, fr.N), 0.f);
    pdf = cosThetaI * kInvPi;
    return color * kInvPi * cosThetaI;
  }

  PRT_D f3 sample(const Frame& fr, f3 Ng, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf, int& type) const
  {
    wi = toWorld(fr, cosineSampleHemisphere(pdf, sx, sy));
    type = kDiffuseReflection;
    if (!(dot(wi, Ng) > 0.f)) return mk(0.f);
    if (R && rough)
    {
      const f3 v = eval(fr, Ng, wo, wi, pdf);
      return v * (1.f / pdf);
    }
    return color;
  }
};

// Microfiber sheen distribution (Conty and Kulla 2017, "Production Friendly Microfacet Sheen
// BRDF"; Kulla and Conty 2017, "Revisiting Physically Based Shading at Imageworks"):
// D = (2 + 1/r) sin^(1/r)(theta) / (2 pi); Lambda from the papers' fitted curve; the incoming
// Lambda is softened near the terminator as bsdf/sheen_distribution.h:60-67 does.
struct SheenDist
{
  float r;  // alpha in (0, 1]

  PRT_D float eval(float cosTheta) const
  {
    const float sinTheta = sqrtf(fmaxf(1.f - cosTheta * cosTheta, 0.f));
    const float invr = 1.f / r;
    return (2.f + invr) * powf(sinTheta, invr) * (1.f / (2.f * kPi));
  }

  // The published fit of log Lambda, interpolated in (1 - r)^2 between its two end points.
  PRT_D float fitL(float x) const
  {
    const float w0 = (1.f - r) * (1.f - r), w1 = 1.f - w0;
    const float a = w0 * 25.3245f + w1 * 21.5473f;
    const float b = w0 * 3.32435f + w1 * 3.82987f;
    const float c = w0 * 0.16801f + w1 * 0.19823f;
    const float d = w0 * -1.27393f + w1 * -1.97760f;
    const float e = w0 * -4.85967f + w1 * -4.32054f;
    return a / (1.f + b * powf(x, c)) + d * x + e;
  }

  PRT_D float lambda(float cosTheta) const
  {
    return cosTheta < 0.5f ? expf(fitL(cosTheta)) : expf(2.f * fitL(0.5f) - fitL(1.f - cosTheta));
  }

  PRT_D float lambdaI(float cosTheta) const
  {
    const float u = 1.f - cosTheta;
    const float u2 = u * u, u4 = u2 * u2;
    return powf(lambda(cosTheta), 1.f + 2.f * u4 * u4);
  }

  // Height-correlated masking-shadowing.
  PRT_D float G2(float cosThetaO, float cosThetaI) const
  {
    return 1.f / (1.f + lambda(cosThetaO) + lambdaI(cosThetaI));
  }
};

// RoughConductorBrdf / ConductorBrdf with the artistic Fresnel (bsdf/rough_conductor.h:108-225,
// bsdf/conductor.h, bsdf/optics.h:243-268).
struct ConductorLobe
{
  f3 r, g, eta, k;
  GGX mf;
  float roughness;
  float Eavg;
  f3 fmsScale;
  bool rough;

  PRT_D void init(const DevTables& t, f3 reflectivity, f3 edgeTint, float rgh, bool isRough)
  {
    r = reflectivity;
    g = edgeTint;
    artisticToIor(r.x, g.x, eta.x, k.x);
    artisticToIor(r.y, g.y, eta.y, k.y);
    artisticToIor(r.z, g.z, eta.z, k.z);
    rough = isRough;
    roughness = rgh;
    const float a = roughnessToAlpha(rgh);
    mf.ax = mf.ay = a;
    if (rough)
    {
      Eavg = ggxAlbedoAvg(t, rgh);
      const f3 Favg = mk(artisticAvg(r.x, g.x), artisticAvg(r.y, g.y), artisticAvg(r.z, g.z));
      fmsScale = Favg * Favg * Eavg * mk(1.f / (1.f - Favg.x * (1.f - Eavg)), 1.f / (1.f - Favg.y * (1.f - Eavg)),
                                         1.f / (1.f - Favg.z * (1.f - Eavg)));
    }
  }

  PRT_D f3 F(float c) const
  {
    return mk(fresnelConductor(c, eta.x, k.x), fresnelConductor(c, eta.y, k.y), fresnelConductor(c, eta.z, k.z));
  }

  PRT_D int flags() const { return rough ? kGlossyReflection : kSpecularReflection; }
  PRT_D float importance() const { return 1.f; }
  PRT_D f3 albedo() const { return r; }

  PRT_D f3 fms(const DevTables& t, float cosThetaO, float cosThetaI) const
  {
    const float Eo = ggxAlbedo(t, cosThetaO, roughness);
    const float Ei = ggxAlbedo(t, cosThetaI, roughness);
    return fmsScale * ((1.f - Eo) * (1.f - Ei) * (1.f / (kPi * (1.f - Eavg))) * cosThetaI);
  }

  PRT_D f3 eval(const DevTables& t, const Frame& fr, f3 Ng, f3 wo, f3 wi, float& pdf) const
  {
    pdf = 0.f;
    if (!rough) return mk(0.f);
    const float cosThetaO = dot(wo, fr.N);
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaO > 0.f) || !(cosThetaI > 0.f)) return mk(0.f);
    const f3 wh = normalize(wi + wo);
    const float cosThetaOH = dot(wo, wh);
    const f3 wo0 = toLocal(fr, wo), wi0 = toLocal(fr, wi), wh0 = toLocal(fr, wh);
    float whPdf;
    const float D = mf.evalVisible(wh0, wo0, cosThetaOH, whPdf);
    const float G = mf.G2(wo0, wi0);
    pdf = whPdf * (1.f / (4.f * fabsf(cosThetaOH)));
    return F(cosThetaOH) * (D * G * (1.f / (4.f * cosThetaO))) + fms(t, cosThetaO, cosThetaI);
  }

  PRT_D f3 sample(const DevTables& t, const Frame& fr, f3 Ng, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf,
                  int& type) const
  {
    const float cosThetaO = dot(wo, fr.N);
    if (!rough)
    {
      wi = 2.f * cosThetaO * fr.N - wo;
      if (!(cosThetaO > 0.f) || !(dot(wi, Ng) > 0.f)) return mk(0.f);
      type = kSpecularReflection;
      pdf = 1.f;
      return F(cosThetaO);
    }
    if (!(cosThetaO > 0.f)) return mk(0.f);
    const f3 wo0 = toLocal(fr, wo);
    float whPdf;
    const f3 wh = toWorld(fr, mf.sampleVisible(wo0, whPdf, sx, sy));
    wi = reflect(wo, wh);
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI > 0.f) || !(dot(wi, Ng) > 0.f)) return mk(0.f);
    const float cosThetaOH = dot(wo, wh);
    const f3 wi0 = toLocal(fr, wi);
    const float G = mf.G2(wo0, wi0);
    type = kGlossyReflection;
    pdf = whPdf * (1.f / (4.f * fabsf(cosThetaOH)));
    return F(cosThetaOH) * (G * rcpSafe(mf.G1(wo0))) + fms(t, cosThetaO, cosThetaI) * (1.f / pdf);
  }
};

// RoughDielectricBsdf / DielectricBsdf (bsdf/rough_dielectric.h:265-550, bsdf/dielectric.h:56-131).
// eta = etaExt / etaInt as seen from the side wo is on.
struct DielectricLobe
{
  float eta, rcpEta, rcpEta2;
  GGX mf;
  float roughness;
  float EavgEta, EavgRcpEta, fmsRatio;
  bool rough;

  PRT_D void init(const DevTables& t, const DevEta& e, float rgh, bool isRough)
  {
    eta = e.eta;
    rcpEta = e.rcpEta;
    rcpEta2 = e.rcpEta2;
    rough = isRough;
    roughness = rgh;
    mf.ax = mf.ay = roughnessToAlpha(rgh);
    if (rough)
    {
      EavgEta = dielAlbedoAvg(t, eta, rgh);
      EavgRcpEta = dielAlbedoAvg(t, rcpEta, rgh);
      const float FavgEta = e.favg;
      const float FavgRcpEta = e.favgRcp;
      const float a = (1.f - FavgEta) * (1.f / (1.f - EavgRcpEta));
      const float b = (1.f - FavgRcpEta) * (1.f / (1.f - EavgEta));
      const float x = b * (1.f / (a + b));
      fmsRatio = 1.f - x * (1.f - FavgEta);
    }
  }

  PRT_D int flags() const
  {
    return rough ? (kGlossyReflection | kGlossyTransmission) : (kSpecularReflection | kSpecularTransmission);
  }
  PRT_D float importance() const { return 1.f; }
  PRT_D f3 albedo() const { return mk(1.f); }

  // Single-scattering part (RoughDielectricBsdfSimd::evalSingle).
  PRT_D float evalSingle(const Frame& fr, f3 Ng, f3 wo, f3 wi, float& pdf) const
  {
    pdf = 0.f;
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return 0.f;
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI * dot(wi, Ng) > 0.f)) return 0.f;
    const bool refl = cosThetaI > 0.f;
    f3 wh = normalize(refl ? wi + wo : eta * wo + wi);
    if (dot(wh, fr.N) < 0.f) wh = -wh;
    const float cosThetaOH = dot(wo, wh);
    const float cosThetaIH = dot(wi, wh);
    const float F = fresnelDielectric(cosThetaOH, eta);
    float value;
    if (refl)
    {
      pdf = F * (1.f / (4.f * fabsf(cosThetaOH)));
      value = F * (1.f / (4.f * cosThetaO));
    }
    else
    {
      pdf = (1.f - F) * rcpEta2 * fabsf(cosThetaIH) * (1.f / sqr(cosThetaOH + rcpEta * cosThetaIH));
      value = pdf * fabsf(cosThetaOH) * (1.f / cosThetaO);
    }
    const f3 wo0 = toLocal(fr, wo), wi0 = toLocal(fr, wi), wh0 = toLocal(fr, wh);
    float whPdf;
    const float D = mf.evalVisible(wh0, wo0, cosThetaOH, whPdf);
    const float G = mf.G2(wo0, wi0);
    pdf = pdf * whPdf;
    return value * D * G;
  }

  // Multiple-scattering part for a direction on the reflection or transmission side.
  PRT_D float evalFms(const DevTables& t, float Eo, float cosThetaI, float& fmsPdf) const
  {
    if (cosThetaI > 0.f)
    {
      const float Ei = dielAlbedo(t, cosThetaI, eta, roughness);
      fmsPdf = fmsRatio * (cosThetaI * kInvPi);
      return fmsRatio * (1.f - Eo) * (1.f - Ei) * (1.f / (kPi * (1.f - EavgEta))) * cosThetaI;
    }
    const float c = fabsf(cosThetaI);
    const float Ei = dielAlbedo(t, c, rcpEta, roughness);
    fmsPdf = (1.f - fmsRatio) * (c * kInvPi);
    return (1.f - fmsRatio) * (1.f - Eo) * (1.f - Ei) * (1.f / (kPi * (1.f - EavgRcpEta))) * c;
  }

  PRT_D f3 eval(const DevTables& t, const Frame& fr, f3 Ng, f3 wo, f3 wi, float& pdf) const
  {
    pdf = 0.f;
    if (!rough) return mk(0.f);
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI * dot(wi, Ng) > 0.f)) return mk(0.f);
    const float Eo = dielAlbedo(t, cosThetaO, eta, roughness);
    float fmsPdf;
    const float fmsValue = evalFms(t, Eo, cosThetaI, fmsPdf);
    float singlePdf;
    const float single = evalSingle(fr, Ng, wo, wi, singlePdf);
    pdf = Eo * singlePdf + (1.f - Eo) * fmsPdf;
    return mk(single + fmsValue);
  }

  PRT_D f3 sample(const DevTables& t, const Frame& fr, f3 Ng, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf,
                  int& type) const
  {
    pdf = 0.f;
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    if (!rough)
    {
      float cosThetaT;
      const float F = fresnelDielectricEx(cosThetaO, cosThetaT, eta);
      wi = mk(0.f);
      if (sc <= F)
      {
        wi = 2.f * cosThetaO * fr.N - wo;
        if (!(dot(wi, Ng) > 0.f)) return mk(0.f);
        type = kSpecularReflection;
        pdf = F;
        return mk(1.f);
      }
      wi = refractDir(wo, fr.N, cosThetaO, cosThetaT, eta);
      if (!(dot(wi, Ng) < 0.f)) return mk(0.f);
      type = kSpecularTransmission;
      pdf = 1.f - F;
      return mk(1.f);
    }
    const float Eo = dielAlbedo(t, cosThetaO, eta, roughness);
    bool ok;
    wi = mk(0.f);
    if (sc <= Eo)
    {
      const f3 wo0 = toLocal(fr, wo);
      float whPdf;
      const f3 wh = toWorld(fr, mf.sampleVisible(wo0, whPdf, sx, sy));
      const float cosThetaOH = dot(wo, wh);
      float cosThetaTH;
      const float F = fresnelDielectricEx(cosThetaOH, cosThetaTH, eta);
      const float sc1 = sc * (1.f / Eo);
      if (sc1 <= F)
      {
        wi = 2.f * cosThetaOH * wh - wo;
        ok = dot(wi, fr.N) > 0.f;
      }
      else
      {
        wi = refractDir(wo, wh, cosThetaOH, cosThetaTH, eta);
        ok = dot(wi, fr.N) < 0.f;
      }
    }
    else
    {
      const float sc1 = (sc - Eo) * (1.f / (1.f - Eo));
      float p;
      const f3 d = toWorld(fr, cosineSampleHemisphere(p, sx, sy));
      wi = sc1 <= fmsRatio ? d : -d;
      ok = true;
    }
    if (!ok) return mk(0.f);
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI * dot(wi, Ng) > 0.f)) return mk(0.f);
    type = cosThetaI > 0.f ? kGlossyReflection : kGlossyTransmission;
    float fmsPdf;
    const float fmsValue = evalFms(t, Eo, cosThetaI, fmsPdf);
    float singlePdf;
    const float single = evalSingle(fr, Ng, wo, wi, singlePdf);
    pdf = Eo * singlePdf + (1.f - Eo) * fmsPdf;
    return mk((single + fmsValue) * (1.f / pdf));
  }
};

// A dielectric layer over a substrate: RoughCoatingBsdf (bsdf/rough_coating.h:271-593) when
// rough, CoatingBsdf (bsdf/coating.h:189-417) when smooth.
struct CoatLayer
{
  float eta;        // <= 1
  f3 color;         // transmittance
  float thickness;
  GGX mf;
  float roughness;
  float avg;        // Ravg (rough) or Favg (smooth), times scale
  float scale;
  bool rough;

  PRT_D void init(const DevTables& t, const DevEta& e, f3 col, float thick, float rgh, bool isRough, float s)
  {
    eta = e.eta <= 1.f ? e.eta : e.rcpEta;
    color = col;
    thickness = thick;
    rough = isRough;
    roughness = rgh;
    mf.ax = mf.ay = roughnessToAlpha(rgh);
    scale = s;
    // The reference evaluates the averages with the constructor argument (before the
    // eta <= 1 fold) and the scale.
    avg = (rough ? reflAlbedoAvg(t, e.eta, rgh) : e.favg) * s;
  }

  PRT_D int flags(int baseFlags) const { return baseFlags | (rough ? kGlossyReflection : kSpecularReflection); }
  PRT_D float importance(float baseImportance) const { return fmaxf(1.f, baseImportance); }
  PRT_D f3 albedo(f3 base) const { return lerp3(base, base * powf3(color, thickness), scale); }

  // Attenuation of the substrate's value through the layer.
  PRT_D f3 attenuate(const DevTables& t, f3 baseValue, float cosThetaO, float cosThetaI, float Fo, float cosThetaO1,
                     bool diffuseBase) const
  {
    float Fi, lengthO1, lengthI1;
    if (rough)
    {
      lengthO1 = 1.f / refractCos(cosThetaO, eta);
      lengthI1 = 1.f / refractCos(fabsf(cosThetaI), eta);
      Fi = reflAlbedo(t, fabsf(cosThetaI), eta, roughness) * scale;
    }
    else
    {
      float cosThetaI1;
      Fi = fresnelDielectricEx(fabsf(cosThetaI), cosThetaI1, eta) * scale;
      lengthO1 = 1.f / cosThetaO1;
      lengthI1 = 1.f / cosThetaI1;
    }
    float length = lengthO1 + lengthI1;
    if (cosThetaI <= 0.f) length *= 0.5f;
    baseValue = lerp3(baseValue, baseValue * powf3(color, thickness * length), scale);
    float T = fminf(1.f - Fo, 1.f - Fi);
    if (diffuseBase) T = (1.f - Fo) * (1.f - Fi) * (1.f / (1.f - avg));
    return baseValue * T;
  }

  // Straight-through transmittance of the layer over a substrate transmittance (CoatingBsdf /
  // RoughCoatingBsdf::getTransparency): absorption along the refracted path, times 1 - F
  // (Fresnel, or the directional reflection albedo when rough).
  PRT_D f3 transparency(const DevTables& t, const Frame& fr, f3 wo, f3 baseT) const
  {
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    float F, length;
    if (rough)
    {
      length = 1.f / refractCos(cosThetaO, eta);
      F = reflAlbedo(t, cosThetaO, eta, roughness) * scale;
    }
    else
    {
      float cosThetaO1;
      F = fresnelDielectricEx(cosThetaO, cosThetaO1, eta) * scale;
      length = 1.f / cosThetaO1;
    }
    baseT = lerp3(baseT, baseT * powf3(color, thickness * length), scale);
    return baseT * (1.f - F);
  }

  PRT_D f3 coatValue(const Frame& fr, f3 wo, f3 wi, float cosThetaO, float& coatPdf) const
  {
    const f3 wh = normalize(wo + wi);
    const float cosThetaOH = dot(wo, wh);
    const float F = fresnelDielectric(cosThetaOH, eta) * scale;
    const f3 wo0 = toLocal(fr, wo), wi0 = toLocal(fr, wi), wh0 = toLocal(fr, wh);
    float whPdf;
    const float D = mf.evalVisible(wh0, wo0, cosThetaOH, whPdf);
    const float G = mf.G2(wo0, wi0);
    coatPdf = whPdf * (1.f / (4.f * fabsf(cosThetaOH)));
    return mk(F * D * G * (1.f / (4.f * cosThetaO)));
  }

  // `Sub` provides flags(), importance(), eval(wo, wi, pdf), sample(...).
  template <class Sub>
  PRT_D f3 eval(const DevTables& t, const Sub& base, const Frame& fr, f3 Ng, f3 wo, f3 wi, float& pdf) const
  {
    pdf = 0.f;
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI * dot(wi, Ng) > 0.f)) return mk(0.f);
    float Fo, cosThetaO1 = 0.f;
    if (rough)
      Fo = reflAlbedo(t, cosThetaO, eta, roughness) * scale;
    else
      Fo = fresnelDielectricEx(cosThetaO, cosThetaO1, eta) * scale;
    const float coatImp = Fo;
    const float baseImp = (1.f - Fo) * base.importance();
    const float coatPick = coatImp * (1.f / (coatImp + baseImp));
    const float basePick = 1.f - coatPick;
    float basePdf;
    f3 baseValue = base.eval(t, wo, wi, basePdf);
    const bool diffuseBase = (base.flags() & ~kBsdfDiffuse) == 0;
    baseValue = attenuate(t, baseValue, cosThetaO, cosThetaI, Fo, cosThetaO1, diffuseBase);
    if (rough && cosThetaI > 0.f)
    {
      float coatPdf;
      const f3 cv = coatValue(fr, wo, wi, cosThetaO, coatPdf);
      pdf = coatPick * coatPdf + basePick * basePdf;
      return cv + baseValue;
    }
    pdf = basePdf * basePick;
    return baseValue;
  }

  template <class Sub>
  PRT_D f3 sample(const DevTables& t, const Sub& base, const Frame& fr, f3 Ng, f3 wo, float sx, float sy, float sc,
                  f3& wi, float& pdf, int& type) const
  {
    pdf = 0.f;
    type = 0;
    wi = mk(0.f);
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    const bool diffuseBase = (base.flags() & ~kBsdfDiffuse) == 0;
    if (!rough)
    {
      // CoatingBsdfSimd::sample
      float cosThetaO1;
      const float Fo = fresnelDielectricEx(cosThetaO, cosThetaO1, eta) * scale;
      const float coatImp = Fo;
      const float baseImp = (1.f - Fo) * base.importance();
      const float coatPick = coatImp * (1.f / (coatImp + baseImp));
      const float basePick = 1.f - coatPick;
      if (sc <= coatPick)
      {
        wi = 2.f * cosThetaO * fr.N - wo;
        if (!(dot(wi, Ng) > 0.f)) return mk(0.f);
        type = kSpecularReflection;
        pdf = coatPick;
        return mk(Fo * (1.f / coatPick));
      }
      const float s1 = (sc - coatPick) * (1.f / basePick);
      float basePdf;
      int baseType;
      f3 bw = base.sample(t, wo, sx, sy, s1, wi, basePdf, baseType);
      type = baseType;
      const float cosThetaI = dot(wi, fr.N);
      if (!(reduceMax(bw) > 0.f) || !(cosThetaI * dot(wi, Ng) > 0.f)) return mk(0.f);
      float cosThetaI1;
      const float Fi = fresnelDielectricEx(fabsf(cosThetaI), cosThetaI1, eta) * scale;
      float length = 1.f / cosThetaO1 + 1.f / cosThetaI1;
      if (cosThetaI <= 0.f) length *= 0.5f;
      bw = lerp3(bw, bw * powf3(color, thickness * length), scale);
      float T = fminf(1.f - Fo, 1.f - Fi);
      if (diffuseBase) T = (1.f - Fo) * (1.f - Fi) * (1.f / (1.f - avg));
      pdf = basePdf * basePick;
      return bw * (T * (1.f / basePick));
    }
    // RoughCoatingBsdfSimd::sample
    const f3 wo0 = toLocal(fr, wo);
    const float Ro = reflAlbedo(t, cosThetaO, eta, roughness) * scale;
    const float coatImp = Ro;
    const float baseImp = (1.f - Ro) * base.importance();
    const float coatPick = coatImp * (1.f / (coatImp + baseImp));
    const float basePick = 1.f - coatPick;
    f3 wh = mk(0.f);
    float basePdf = 0.f;
    f3 baseValue = mk(0.f);
    if (sc <= coatPick)
    {
      float whPdf;
      wh = toWorld(fr, mf.sampleVisible(wo0, whPdf, sx, sy));
      const float cosThetaOH = dot(wo, wh);
      wi = 2.f * cosThetaOH * wh - wo;
      if (!(dot(wi, fr.N) > 0.f)) return mk(0.f);
      type = kGlossyReflection;
      baseValue = base.eval(t, wo, wi, basePdf);
    }
    else
    {
      const float s1 = (sc - coatPick) * (1.f / basePick);
      f3 baseWi;
      float basePdf2;
      int baseType;
      const f3 bw = base.sample(t, wo, sx, sy, s1, baseWi, basePdf2, baseType);
      if (!(reduceMax(bw) > 0.f)) return mk(0.f);
      wi = baseWi;
      basePdf = basePdf2;
      type = baseType;
      baseValue = bw * ((type & kBsdfDelta) != 0 ? 1.f : basePdf);
      wh = normalize(wo + wi);
    }
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI * dot(wi, Ng) > 0.f)) return mk(0.f);
    const float cosThetaOH = dot(wo, wh);
    baseValue = attenuate(t, baseValue, cosThetaO, cosThetaI, Ro, 0.f, diffuseBase);
    if (type & kBsdfDelta)
    {
      pdf = basePdf;
      return baseValue * (1.f / basePick);
    }
    if (cosThetaI <= 0.f)
    {
      pdf = basePick * basePdf;
      return baseValue * (1.f / pdf);
    }
    const float F = fresnelDielectric(cosThetaOH, eta) * scale;
    const f3 wi0 = toLocal(fr, wi), wh0 = toLocal(fr, wh);
    float whPdf;
    const float D = mf.evalVisible(wh0, wo0, cosThetaOH, whPdf);
    const float G = mf.G2(wo0, wi0);
    const float coatPdf = whPdf * (1.f / (4.f * fabsf(cosThetaOH)));
    const f3 cv = mk(F * D * G * (1.f / (4.f * cosThetaO)));
    pdf = coatPick * coatPdf + basePick * basePdf;
    return (cv + baseValue) * (1.f / pdf);
  }
};

// SheenBsdf (bsdf/sheen.h:199-451): a sheen layer over a substrate. The sheen lobe is
// sampled uniformly over the hemisphere and picked against the substrate by Ro * max(color)
// versus (1 - Ro) * importance(substrate); the substrate is scaled by min(1 - Ro, 1 - Ri), where
// R is the sheen's directional albedo.
struct SheenLayer
{
  f3 color;
  SheenDist mf;
  float roughness;
  float scale;

  PRT_D void init(f3 col, float rgh, float s)
  {
    color = col;
    roughness = rgh;
    mf.r = roughnessToAlpha(rgh);
    scale = s;
  }

  PRT_D int flags(int baseFlags) const { return baseFlags | kDiffuseReflection; }

  PRT_D f3 sheenValue(const Frame& fr, f3 wo, f3 wi, float cosThetaO, float cosThetaI) const
  {
    const f3 wh = normalize(wo + wi);
    const float D = mf.eval(dot(wh, fr.N));
    const float G = mf.G2(cosThetaO, cosThetaI);
    return color * (D * G * (1.f / (4.f * cosThetaO)) * scale);
  }

  template <class Sub>
  PRT_D f3 eval(const DevTables& t, const Sub& base, const Frame& fr, f3 Ng, f3 wo, f3 wi, float& pdf) const
  {
    pdf = 0.f;
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI * dot(wi, Ng) > 0.f)) return mk(0.f);
    float basePdf;
    f3 baseValue = base.eval(t, wo, wi, basePdf);
    const float Ro = sheenAlbedo(t, cosThetaO, roughness) * scale;
    const float Ri = sheenAlbedo(t, fabsf(cosThetaI), roughness) * scale;
    baseValue *= fminf(1.f - Ro, 1.f - Ri);
    const float coatImp = Ro * reduceMax(color);
    const float baseImp = (1.f - Ro) * base.importance();
    const float coatPick = coatImp * (1.f / (coatImp + baseImp));
    const float basePick = 1.f - coatPick;
    if (cosThetaI > 0.f)
    {
      pdf = coatPick * (1.f / (2.f * kPi)) + basePick * basePdf;
      return sheenValue(fr, wo, wi, cosThetaO, cosThetaI) + baseValue;
    }
    pdf = basePdf * basePick;
    return baseValue;
  }

  template <class Sub>
  PRT_D f3 sample(const DevTables& t, const Sub& base, const Frame& fr, f3 Ng, f3 wo, float sx, float sy, float sc,
                  f3& wi, float& pdf, int& type) const
  {
    pdf = 0.f;
    type = 0;
    wi = mk(0.f);
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    const float Ro = sheenAlbedo(t, cosThetaO, roughness) * scale;
    const float coatImp = Ro * reduceMax(color);
    const float baseImp = (1.f - Ro) * base.importance();
    const float coatPick = coatImp * (1.f / (coatImp + baseImp));
    const float basePick = 1.f - coatPick;
    float basePdf = 0.f;
    f3 baseValue = mk(0.f);
    if (sc <= coatPick)
    {
      type = kDiffuseReflection;
      // uniformSampleHemisphere: phi = 2 pi sx, cos(theta) = sy
      const float cosTheta = sy;
      const float sinTheta = sqrtf(fmaxf(1.f - sy * sy, 0.f));
      float sinPhi, cosPhi;
      sincospif(2.f * sx, &sinPhi, &cosPhi);
      wi = toWorld(fr, mk(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta));
      baseValue = base.eval(t, wo, wi, basePdf);
    }
    else
    {
      const float s1 = (sc - coatPick) * (1.f / basePick);
      f3 baseWi;
      float basePdf2;
      int baseType;
      const f3 bw = base.sample(t, wo, sx, sy, s1, baseWi, basePdf2, baseType);
      if (!(reduceMax(bw) > 0.f)) return mk(0.f);
      wi = baseWi;
      basePdf = basePdf2;
      type = baseType;
      baseValue = bw * ((type & kBsdfDelta) != 0 ? 1.f : basePdf);
    }
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI * dot(wi, Ng) > 0.f)) return mk(0.f);
    const float Ri = sheenAlbedo(t, fabsf(cosThetaI), roughness) * scale;
    baseValue *= fminf(1.f - Ro, 1.f - Ri);
    if (type & kBsdfDelta)
    {
      pdf = basePdf;
      return baseValue * (1.f / basePick);
    }
    if (cosThetaI <= 0.f)
    {
      pdf = basePick * basePdf;
      return baseValue * (1.f / pdf);
    }
    pdf = coatPick * (1.f / (2.f * kPi)) + basePick * basePdf;
    return (sheenValue(fr, wo, wi, cosThetaO, cosThetaI) + baseValue) * (1.f / pdf);
  }
};

// ---- Standard material composition -----------------------------------------------------------

enum : int
{
  kSlotOpaque = 0,
  kSlotDielectric = 1,
  kSlotConductor = 2,
  kSlotThin = 3,         // thin-walled dielectric (translucent base of a thin-walled material)
  kSlotTransparent = 4,  // TransparentBtdf (translucent base whose IOR equals the ambient IOR)
};


// DiffuseBtdf (bsdf/diffuse.h:126-166): Lambertian transmission to the far side of the shading
// normal.
struct DiffuseBtdfLobe
{
  f3 color;

  PRT_D int flags() const { return kDiffuseTransmission; }
  PRT_D float importance() const { return reduceMax(color); }
  PRT_D f3 albedo() const { return color; }

  PRT_D f3 eval(const Frame& fr, f3 Ng, f3 wo, f3 wi, float& pdf) const
  {
    const float cosThetaI = fmaxf(-dot(wi, fr.N), 0.f);
    pdf = cosThetaI * kInvPi;
    return color * kInvPi * cosThetaI;
  }

  PRT_D f3 sample(const Frame& fr, f3 Ng, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf, int& type) const
  {
    wi = -toWorld(fr, cosineSampleHemisphere(pdf, sx, sy));
    type = kDiffuseTransmission;
    if (!(dot(wi, Ng) <= 0.f)) return mk(0.f);
    return color;
  }
};

// Thin-walled dielectric: ThinDielectricBsdf (bsdf/thin_dielectric.h:74-160) when smooth,
// ThinRoughDielectricBsdf (bsdf/thin_rough_dielectric.h:166-340) when rough. Light is reflected
// (specular, or GGX with Kulla-Conty energy compensation) or passes straight through
// (unbent) attenuated by color^(thickness / cos(refracted angle)).
struct ThinDielectricLobe
{
  float eta;
  f3 color;
  float thickness;
  GGX mf;
  float roughness;
  float Eavg, fmsScale;
  bool rough;

  PRT_D void init(const DevTables& t, const DevEta& e, f3 col, float thick, float rgh, bool isRough)
  {
    eta = e.eta;
    color = col;
    thickness = thick;
    rough = isRough;
    roughness = rgh;
    mf.ax = mf.ay = roughnessToAlpha(rgh);
    if (rough)
    {
      Eavg = ggxAlbedoAvg(t, rgh);
      const float Favg = e.favg;
      fmsScale = Favg * (1.f - Eavg) * (1.f / (1.f - Favg * Eavg));
    }
  }

  PRT_D int flags() const { return (rough ? kGlossyReflection : kSpecularReflection) | kUnbentTransmission; }
  PRT_D float importance() const { return 1.f; }
  PRT_D f3 albedo() const { return powf3(color, thickness); }

  // Probability of reflection: Fresnel (smooth) or the directional reflection albedo plus the
  // compensated multiple scattering (rough).
  PRT_D float reflectance(const DevTables& t, float cosThetaO, float& cosThetaT) const
  {
    if (!rough) return fresnelDielectricEx(cosThetaO, cosThetaT, eta);
    cosThetaT = refractCos(cosThetaO, eta);
    const float Eo = ggxAlbedo(t, cosThetaO, roughness);
    return reflAlbedo(t, cosThetaO, eta, roughness) + fmsScale * (1.f - Eo);
  }

  PRT_D f3 transparency(const DevTables& t, const Frame& fr, f3 wo) const
  {
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    float cosThetaT;
    const float R = reflectance(t, cosThetaO, cosThetaT);
    return (1.f - R) * powf3(color, (1.f / cosThetaT) * thickness);
  }

  PRT_D f3 eval(const DevTables& t, const Frame& fr, f3 Ng, f3 wo, f3 wi, float& pdf) const
  {
    pdf = 0.f;
    if (!rough) return mk(0.f);
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    const float cosThetaI = dot(wi, fr.N);
    if (!(cosThetaI * dot(wi, Ng) > 0.f) || !(cosThetaI > 0.f)) return mk(0.f);
    const f3 wh = normalize(wi + wo);
    const float cosThetaOH = dot(wo, wh);
    const f3 wo0 = toLocal(fr, wo), wi0 = toLocal(fr, wi), wh0 = toLocal(fr, wh);
    const float F = fresnelDielectric(cosThetaOH, eta);
    float whPdf;
    const float D = mf.evalVisible(wh0, wo0, cosThetaOH, whPdf);
    const float G = mf.G2(wo0, wi0);
    const float Eo = ggxAlbedo(t, cosThetaO, roughness);
    const float Ei = ggxAlbedo(t, cosThetaI, roughness);
    const float fms = fmsScale * ((1.f - Eo) * (1.f - Ei) * (1.f / (kPi * (1.f - Eavg))) * cosThetaI);
    const float R = reflAlbedo(t, cosThetaO, eta, roughness) + fmsScale * (1.f - Eo);
    pdf = whPdf * (1.f / (4.f * fabsf(cosThetaOH))) * R;
    return mk(F * D * G * (1.f / (4.f * cosThetaO)) + fms);
  }

  PRT_D f3 sample(const DevTables& t, const Frame& fr, f3 Ng, f3 wo, float sx, float sy, float sc, f3& wi,
                  float& pdf, int& type) const
  {
    pdf = 0.f;
    wi = mk(0.f);
    const float cosThetaO = dot(wo, fr.N);
    if (!(cosThetaO > 0.f)) return mk(0.f);
    if (!rough)
    {
      float cosThetaT;
      const float F = fresnelDielectricEx(cosThetaO, cosThetaT, eta);
      if (sc <= F)
      {
        wi = 2.f * cosThetaO * fr.N - wo;
        type = kSpecularReflection;
        pdf = F;
        return dot(wi, Ng) > 0.f ? mk(1.f) : mk(0.f);
      }
      wi = -wo;
      type = kUnbentTransmission;
      pdf = 1.f - F;
      return dot(wi, Ng) < 0.f ? powf3(color, (1.f / cosThetaT) * thickness) : mk(0.f);
    }
    const float Eo = ggxAlbedo(t, cosThetaO, roughness);
    const float R = reflAlbedo(t, cosThetaO, eta, roughness) + fmsScale * (1.f - Eo);
    if (sc <= R)
    {
      const f3 wo0 = toLocal(fr, wo);
      float whPdf;
      const f3 wh = toWorld(fr, mf.sampleVisible(wo0, whPdf, sx, sy));
      const float cosThetaOH = dot(wo, wh);
      wi = 2.f * cosThetaOH * wh - wo;
      const float cosThetaI = dot(wi, fr.N);
      type = kGlossyReflection;
      if (!(cosThetaI > 0.f) || !(dot(wi, Ng) > 0.f)) return mk(0.f);
      const f3 wi0 = toLocal(fr, wi);
      const float F = fresnelDielectric(cosThetaOH, eta);
      const float G = mf.G2(wo0, wi0);
      const float Ei = ggxAlbedo(t, cosThetaI, roughness);
      const float fms = fmsScale * ((1.f - Eo) * (1.f - Ei) * (1.f / (kPi * (1.f - Eavg))) * cosThetaI);
      pdf = whPdf * (1.f / (4.f * fabsf(cosThetaOH))) * R;
      return mk(F * G * rcpSafe(mf.G1(wo0)) * (1.f / R) + fms * (1.f / pdf));
    }
    wi = -wo;
    type = kUnbentTransmission;
    pdf = 1.f - R;
    return dot(wi, Ng) < 0.f ? powf3(color, (1.f / refractCos(cosThetaO, eta)) * thickness) : mk(0.f);
  }
};

// MultiBsdf (bsdf/multi_bsdf.h:151-270) over two children given by callables: eval(pdf) and
// sample(sc, wi, pdf, type) for child 0 and 1, with scales s and importances i (the child's
// importance times its scale; a child with importance 0 takes no part).
template <class E0, class E1>
PRT_D f3 multi2Eval(float s0, float i0, float s1, float i1, const E0& e0, const E1& e1, float& pdf)
{
  f3 v = mk(0.f);
  pdf = 0.f;
  if (i0 > 0.f)
  {
    float p;
    v += e0(p) * s0;
    pdf += p * i0;
  }
  if (i1 > 0.f)
  {
    float p;
    v += e1(p) * s1;
    pdf += p * i1;
  }
  pdf *= 1.f / (i0 + i1);
  return v;
}

template <class S0, class S1, class E0, class E1>
PRT_D f3 multi2Sample(float s0, float i0, float s1, float i1, const S0& smp0, const S1& smp1, const E0& e0,
                      const E1& e1, float sc, f3& wi, float& pdf, int& type)
{
  pdf = 0.f;
  type = 0;
  wi = mk(0.f);
  const float isum = i0 + i1;
  if (!(isum > 0.f)) return mk(0.f);
  const float x = sc * isum;
  const int choice = x > i0 ? 1 : 0;
  const float importance = choice ? i1 : i0, prefix = choice ? i0 + i1 : i0, scale = choice ? s1 : s0;
  const float s1c = (x + importance - prefix) * (1.f / importance);
  f3 weight = choice ? smp1(s1c, wi, pdf, type) : smp0(s1c, wi, pdf, type);
  if (!(reduceMax(weight) > 0.f))
  {
    weight = mk(0.f);
    pdf = 0.f;
    type = 0;
    wi = mk(0.f);
  }
  weight *= scale;
  if (!(reduceMax(weight) > 0.f) || !(pdf > 0.f)) return mk(0.f);
  if (type & kBsdfDelta) return weight * isum * (1.f / importance);
  f3 value = weight * pdf;
  pdf *= importance;
  const float io = choice ? i0 : i1;
  if (io > 0.f)
  {
    float p;
    value += (choice ? e0(p) * s0 : e1(p) * s1);
    pdf += p * io;
  }
  pdf *= 1.f / isum;
  return value * (1.f / pdf);
}

// MultiBsdf::getAlbedo accumulated child by child (no arrays, so nothing goes to local memory).
struct AlbedoSum
{
  f3 v = mk(0.f);
  float scaleSum = 0.f, total = 0.f;
  PRT_D void add(f3 a, float s, float imp)
  {
    if (!(imp > 0.f)) return;
    total += s;
    if (!(a.x >= 0.f)) return;
    v += a * s;
    scaleSum += s;
  }
  PRT_D f3 value() const { return v * (total * rcpSafe(scaleSum)); }
  // Without transparent children the scale sums are equal and the renormalisation is 1.
  PRT_D f3 valueOpaque() const { return v; }
};

// The opaque base of the Standard material (material/standard.cpp:441-502): a Lambertian (or
// Oren-Nayar) lobe, blended with the thin-walled subsurface approximation when the material has
// one -- Multi{diffuse x (1 - subsurface), subsurface x subsurface} with subsurface =
// Multi{diffuse BRDF x (1 - t), diffuse BTDF x t} in the subsurface colour, t = (1 +
// anisotropy) / 2, each Multi collapsing to its only child when the other weight is below eps --
// optionally under the specular dielectric layer. S = false compiles the subsurface out.
template <bool R, bool S>
struct OpaqueBase
{
  DiffuseLobeT<R> diff;
  CoatLayer spec;
  bool hasSpec;
  DiffuseLobeT<R> ssRefl;
  DiffuseBtdfLobe ssTrans;
  bool hasDiff, hasSS, ssHasR, ssHasT;
  float wDiff, wSS, wR, wT;
};

// The subsurface blend alone: Multi{BRDF x wR, BTDF x wT}, or its only child.
template <bool R, bool S>
struct SubsurfaceTree
{
  const OpaqueBase<R, S>* o;
  Frame fr;
  f3 Ng;
  PRT_D float i0() const { return o->ssHasR ? o->ssRefl.importance() * o->wR : 0.f; }
  PRT_D float i1() const { return o->ssHasT ? o->ssTrans.importance() * o->wT : 0.f; }
  PRT_D int flags() const { return (o->ssHasR ? kDiffuseReflection : 0) | (o->ssHasT ? kDiffuseTransmission : 0); }
  PRT_D float importance() const
  {
    if (o->ssHasR && o->ssHasT) return i0() + i1();
    return o->ssHasR ? o->ssRefl.importance() : o->ssTrans.importance();
  }
  PRT_D f3 albedo() const
  {
    if (o->ssHasR && o->ssHasT)
    {
      AlbedoSum sum;
      sum.add(o->ssRefl.albedo(), o->wR, i0());
      sum.add(o->ssTrans.albedo(), o->wT, i1());
      return sum.value();
    }
    return o->ssHasR ? o->ssRefl.albedo() : o->ssTrans.albedo();
  }
  PRT_D f3 eval(f3 wo, f3 wi, float& pdf) const
  {
    if (!o->ssHasT) return o->ssRefl.eval(fr, Ng, wo, wi, pdf);
    if (!o->ssHasR) return o->ssTrans.eval(fr, Ng, wo, wi, pdf);
    return multi2Eval(
      o->wR, i0(), o->wT, i1(), [&](float& p) { return o->ssRefl.eval(fr, Ng, wo, wi, p); },
      [&](float& p) { return o->ssTrans.eval(fr, Ng, wo, wi, p); }, pdf);
  }
  PRT_D f3 sample(f3 wo, float sx, float sy, float sc, f3& wi, float& pdf, int& type) const
  {
    if (!o->ssHasT) return o->ssRefl.sample(fr, Ng, wo, sx, sy, sc, wi, pdf, type);
    if (!o->ssHasR) return o->ssTrans.sample(fr, Ng, wo, sx, sy, sc, wi, pdf, type);
    return multi2Sample(
      o->wR, i0(), o->wT, i1(),
      [&](float c, f3& w, float& p, int& ty) { return o->ssRefl.sample(fr, Ng, wo, sx, sy, c, w, p, ty); },
      [&](float c, f3& w, float& p, int& ty) { return o->ssTrans.sample(fr, Ng, wo, sx, sy, c, w, p, ty); },
      [&](float& p) { return o->ssRefl.eval(fr, Ng, wo, wi, p); },
      [&](float& p) { return o->ssTrans.eval(fr, Ng, wo, wi, p); }, sc, wi, pdf, type);
  }
};

// The whole opaque base below the specular layer: Multi{diffuse x wDiff, subsurface x wSS}, or
// its only child; with S = false just the diffuse lobe.
template <bool R, bool S>
struct OpaqueSub
{
  const OpaqueBase<R, S>* o;
  Frame fr;
  f3 Ng;
  PRT_D SubsurfaceTree<R, S> ss() const { return SubsurfaceTree<R, S>{o, fr, Ng}; }
  PRT_D bool blend() const { return S && o->hasSS; }
  PRT_D float i0() const { return o->hasDiff ? o->diff.importance() * o->wDiff : 0.f; }
  PRT_D float i1() const { return o->hasSS ? ss().importance() * o->wSS : 0.f; }
  PRT_D int flags() const
  {
    if (!blend()) return kDiffuseReflection;
    return (o->hasDiff ? kDiffuseReflection : 0) | ss().flags();
  }
  PRT_D float importance() const
  {
    if (!blend()) return o->diff.importance();
    if (!o->hasDiff) return ss().importance();
    return i0() + i1();
  }
  PRT_D f3 albedo() const
  {
    if (!blend()) return o->diff.albedo();
    if (!o->hasDiff) return ss().albedo();
    AlbedoSum sum;
    sum.add(o->diff.albedo(), o->wDiff, i0());
    sum.add(ss().albedo(), o->wSS, i1());
    return sum.value();
  }
  PRT_D f3 eval(const DevTables& t, f3 wo, f3 wi, float& pdf) const
  {
    if (!blend()) return o->diff.eval(fr, Ng, wo, wi, pdf);
    if (!o->hasDiff) return ss().eval(wo, wi, pdf);
    return multi2Eval(
      o->wDiff, i0(), o->wSS, i1(), [&](float& p) { return o->diff.eval(fr, Ng, wo, wi, p); },
      [&](float& p) { return ss().eval(wo, wi, p); }, pdf);
  }
  PRT_D f3 sample(const DevTables& t, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf, int& type) const
  {
    if (!blend()) return o->diff.sample(fr, Ng, wo, sx, sy, sc, wi, pdf, type);
    if (!o->hasDiff) return ss().sample(wo, sx, sy, sc, wi, pdf, type);
    return multi2Sample(
      o->wDiff, i0(), o->wSS, i1(),
      [&](float c, f3& w, float& p, int& ty) { return o->diff.sample(fr, Ng, wo, sx, sy, c, w, p, ty); },
      [&](float c, f3& w, float& p, int& ty) { return ss().sample(wo, sx, sy, c, w, p, ty); },
      [&](float& p) { return o->diff.eval(fr, Ng, wo, wi, p); }, [&](float& p) { return ss().eval(wo, wi, p); },
      sc, wi, pdf, type);
  }
};

// The Standard material's BSDF tree (material/standard.cpp:410-620): MultiBsdf over the base
// lobes (opaque, translucent, metal; bsdf/multi_bsdf.h:151-270), the outer coat, the sheen,
// and -- for opacity below 1 -- Multi{that x opacity, TransparentBtdf x (1 - opacity)}. F is the
// feature set the instance may contain (branches outside F are compiled out).
template <int F>
struct StdBsdfT
{
  static constexpr bool kR = (F & kFeatRoughDiffuse) != 0;
  static constexpr bool kS = (F & kFeatSubsurface) != 0;
  Frame fr;
  f3 Ng;
  int nLobes;
  int kind[3];
  float scale[3];
  float imp[3];
  float impSum;
  int baseFlags;
  OpaqueBase<kR, kS> opaque;
  DielectricLobe diel;
  ThinDielectricLobe thin;
  ConductorLobe cond;
  CoatLayer coat;
  bool hasCoat;
  SheenLayer sheen;
  bool hasSheen;
  bool hasTransp;    // top-level opacity blend
  bool hasInner;     // opacity > eps: the tree above takes part
  float opacityW, transpW;
  f3 albedoV;

  PRT_D OpaqueSub<kR, kS> opaqueSub() const { return OpaqueSub<kR, kS>{&opaque, fr, Ng}; }

  PRT_D int coatedFlags() const { return ((F & kFeatCoat) && hasCoat) ? coat.flags(baseFlags) : baseFlags; }
  PRT_D int innerFlags() const { return ((F & kFeatSheen) && hasSheen) ? sheen.flags(coatedFlags()) : coatedFlags(); }
  PRT_D int flags() const
  {
    if ((F & kFeatTransparent) && hasTransp) return (hasInner ? innerFlags() : 0) | kTransparency;
    return innerFlags();
  }

  PRT_D f3 evalSlot(const DevTables& t, int k, f3 wo, f3 wi, float& pdf) const
  {
    if ((F & kFeatOpaque) && k == kSlotOpaque)
    {
      if ((F & kFeatSpecular) && opaque.hasSpec) return opaque.spec.eval(t, opaqueSub(), fr, Ng, wo, wi, pdf);
      return opaqueSub().eval(t, wo, wi, pdf);
    }
    if ((F & kFeatDielectric) && k == kSlotDielectric) return diel.eval(t, fr, Ng, wo, wi, pdf);
    if ((F & kFeatThin) && k == kSlotThin) return thin.eval(t, fr, Ng, wo, wi, pdf);
    if ((F & kFeatConductor) && k == kSlotConductor) return cond.eval(t, fr, Ng, wo, wi, pdf);
    pdf = 0.f;
    return mk(0.f);
  }

  PRT_D f3 sampleSlot(const DevTables& t, int k, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf,
                      int& type) const
  {
    if ((F & kFeatOpaque) && k == kSlotOpaque)
    {
      if ((F & kFeatSpecular) && opaque.hasSpec)
        return opaque.spec.sample(t, opaqueSub(), fr, Ng, wo, sx, sy, sc, wi, pdf, type);
      return opaqueSub().sample(t, wo, sx, sy, sc, wi, pdf, type);
    }
    if ((F & kFeatDielectric) && k == kSlotDielectric) return diel.sample(t, fr, Ng, wo, sx, sy, sc, wi, pdf, type);
    if ((F & kFeatThin) && k == kSlotThin) return thin.sample(t, fr, Ng, wo, sx, sy, sc, wi, pdf, type);
    if ((F & kFeatConductor) && k == kSlotConductor) return cond.sample(t, fr, Ng, wo, sx, sy, sc, wi, pdf, type);
    if ((F & kFeatTransparent) && k == kSlotTransparent)
    {
      // TransparentBtdf::sample (bsdf/transparent.h:32-45): straight through, weight 1.
      wi = -wo;
      type = kTransparency;
      pdf = 1.f;
      return mk(1.f);
    }
    pdf = 0.f;
    return mk(0.f);
  }

  // MultiBsdfSimd::eval
  PRT_D f3 evalBase(const DevTables& t, f3 wo, f3 wi, float& pdf) const
  {
    f3 value = mk(0.f);
    pdf = 0.f;
    for (int i = 0; i < nLobes; ++i)
    {
      if (!(imp[i] > 0.f)) continue;
      float p;
      const f3 v = evalSlot(t, kind[i], wo, wi, p);
      value += v * scale[i];
      pdf += p * imp[i];
    }
    pdf *= 1.f / impSum;
    return value;
  }

  // MultiBsdfSimd::sample
  PRT_D f3 sampleBase(const DevTables& t, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf, int& type) const
  {
    pdf = 0.f;
    type = 0;
    wi = mk(0.f);
    if (!(impSum > 0.f)) return mk(0.f);
    if (nLobes == 1) return sampleSlot(t, kind[0], wo, sx, sy, sc, wi, pdf, type) * scale[0];
    const float x = sc * impSum;
    int choice = 0;
    float prefix = imp[0], importance = imp[0], sc0 = scale[0];
    for (int i = 1; i < nLobes; ++i)
    {
      if (!(x > prefix)) break;
      choice = i;
      prefix += imp[i];
      importance = imp[i];
      sc0 = scale[i];
    }
    const float s1 = (x + importance - prefix) * (1.f / importance);
    f3 weight = sampleSlot(t, kind[choice], wo, sx, sy, s1, wi, pdf, type);
    if (!(reduceMax(weight) > 0.f))
    {
      weight = mk(0.f);
      pdf = 0.f;
      type = 0;
      wi = mk(0.f);
    }
    weight *= sc0;
    if (!(reduceMax(weight) > 0.f) || !(pdf > 0.f)) return mk(0.f);
    if (type & kBsdfDelta) return weight * impSum * (1.f / importance);
    f3 value = weight * pdf;
    pdf *= importance;
    for (int i = 0; i < nLobes; ++i)
    {
      if (i == choice || !(imp[i] > 0.f)) continue;
      float p;
      const f3 v = evalSlot(t, kind[i], wo, wi, p);
      value += v * scale[i];
      pdf += p * imp[i];
    }
    pdf *= 1.f / impSum;
    return value * (1.f / pdf);
  }

  PRT_D int baseFlagsFn() const { return baseFlags; }

  struct BaseSub
  {
    const StdBsdfT* b;
    PRT_D int flags() const { return b->baseFlags; }
    PRT_D float importance() const { return b->impSum; }
    PRT_D f3 eval(const DevTables& t, f3 wo, f3 wi, float& pdf) const { return b->evalBase(t, wo, wi, pdf); }
    PRT_D f3 sample(const DevTables& t, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf, int& type) const
    {
      return b->sampleBase(t, wo, sx, sy, sc, wi, pdf, type);
    }
  };

  // The base with its coat (when present): the substrate of the sheen layer.
  PRT_D f3 evalCoated(const DevTables& t, f3 wo, f3 wi, float& pdf) const
  {
    if ((F & kFeatCoat) && hasCoat) return coat.eval(t, BaseSub{this}, fr, Ng, wo, wi, pdf);
    return evalBase(t, wo, wi, pdf);
  }

  PRT_D f3 sampleCoated(const DevTables& t, f3 wo, float sx, float sy, float sz, f3& wi, float& pdf, int& type) const
  {
    if ((F & kFeatCoat) && hasCoat) return coat.sample(t, BaseSub{this}, fr, Ng, wo, sx, sy, sz, wi, pdf, type);
    return sampleBase(t, wo, sx, sy, sz, wi, pdf, type);
  }

  PRT_D float coatedImportance() const { return ((F & kFeatCoat) && hasCoat) ? coat.importance(impSum) : impSum; }

  struct CoatedSub
  {
    const StdBsdfT* b;
    PRT_D int flags() const { return b->coatedFlags(); }
    PRT_D float importance() const { return b->coatedImportance(); }
    PRT_D f3 eval(const DevTables& t, f3 wo, f3 wi, float& pdf) const { return b->evalCoated(t, wo, wi, pdf); }
    PRT_D f3 sample(const DevTables& t, f3 wo, float sx, float sy, float sc, f3& wi, float& pdf, int& type) const
    {
      return b->sampleCoated(t, wo, sx, sy, sc, wi, pdf, type);
    }
  };

  // The tree below the opacity blend.
  PRT_D f3 evalInner(const DevTables& t, f3 wo, f3 wi, float& pdf) const
  {
    if ((F & kFeatSheen) && hasSheen) return sheen.eval(t, CoatedSub{this}, fr, Ng, wo, wi, pdf);
    return evalCoated(t, wo, wi, pdf);
  }

  PRT_D f3 sampleInner(const DevTables& t, f3 wo, float sx, float sy, float sz, f3& wi, float& pdf, int& type) const
  {
    if ((F & kFeatSheen) && hasSheen) return sheen.sample(t, CoatedSub{this}, fr, Ng, wo, sx, sy, sz, wi, pdf, type);
    return sampleCoated(t, wo, sx, sy, sz, wi, pdf, type);
  }

  // SheenBsdf::getImportance is max(max(sheen colour), substrate importance).
  PRT_D float innerImportance() const
  {
    if ((F & kFeatSheen) && hasSheen) return fmaxf(reduceMax(sheen.color), coatedImportance());
    return coatedImportance();
  }

  PRT_D f3 eval(const DevTables& t, f3 wo, f3 wi, float& pdf) const
  {
    if ((F & kFeatTransparent) && hasTransp)
    {
      if (!hasInner)
      {
        pdf = 0.f;
        return mk(0.f);
      }
      return multi2Eval(
        opacityW, innerImportance() * opacityW, transpW, transpW,
        [&](float& p) { return evalInner(t, wo, wi, p); },
        [&](float& p) {
          p = 0.f;
          return mk(0.f);
        },
        pdf);
    }
    return evalInner(t, wo, wi, pdf);
  }

  PRT_D f3 sample(const DevTables& t, f3 wo, float sx, float sy, float sz, f3& wi, float& pdf, int& type) const
  {
    if ((F & kFeatTransparent) && hasTransp)
    {
      auto transparent = [&](float c, f3& w, float& p, int& ty) {
        w = -wo;
        ty = kTransparency;
        p = 1.f;
        return mk(1.f);
      };
      if (!hasInner) return transparent(sz, wi, pdf, type);
      return multi2Sample(
        opacityW, innerImportance() * opacityW, transpW, transpW,
        [&](float c, f3& w, float& p, int& ty) { return sampleInner(t, wo, sx, sy, c, w, p, ty); }, transparent,
        [&](float& p) { return evalInner(t, wo, wi, p); },
        [&](float& p) {
          p = 0.f;
          return mk(0.f);
        },
        sz, wi, pdf, type);
    }
    return sampleInner(t, wo, sx, sy, sz, wi, pdf, type);
  }

  PRT_D f3 albedo() const { return albedoV; }
  PRT_D f3 normal() const { return ((F & kFeatTransparent) && hasTransp && !hasInner) ? mk(0.f) : fr.N; }
};

// Material texture lookup: repeat in both directions (image/image_texture.h:197-226).
PRT_D f3 textureRgb(const DevTexture& t, float u, float v)
{
  return texLookup(t.rgb, t.width, t.height, u, v, true);
}

using StdBsdf = StdBsdfT<kFeatAll>;

template <int F>
PRT_D void addSlot(StdBsdfT<F>& b, int kind, float scale, float importance, int flags)
{
  const int i = b.nLobes++;
  b.kind[i] = kind;
  b.scale[i] = scale;
  b.imp[i] = importance * scale;
  b.impSum += b.imp[i];
  b.baseFlags |= flags;
}

// The material's (textured) base colour.
PRT_D f3 standardBaseColor(const DevScene& sc, const DevMaterial& m, const ShadeCtx& ctx)
{
  f3 baseColor = mk(m.baseColor[0], m.baseColor[1], m.baseColor[2]);
  if (m.baseColorTex >= 0) baseColor = textureRgb(sc.textures[m.baseColorTex], ctx.uvx, ctx.uvy) * baseColor;
  return clamp01(baseColor);
}

// StandardMaterial::getBsdfLobes (material/standard.cpp:410-620): Lambertian or Oren-Nayar base
// with the thin-walled subsurface blend and an optional specular layer, rough or smooth
// dielectric transmission (thin-walled: unbent; IOR equal to the ambient IOR: transparent),
// rough or smooth artistic conductor, rough or smooth coat, sheen, and the opacity blend.
// `backfacing` is the medium-interface orientation (material/material.h:66-76).
template <int F>
PRT_D void resolveStandard(const DevScene& sc, const DevTables& t, const DevMaterial& m, const ShadeCtx& ctx, f3 wo,
                           bool backfacing, StdBsdfT<F>& b)
{
  b.fr = makeShadingFrame(ctx, wo);
  b.Ng = ctx.Ng;
  b.nLobes = 0;
  b.impSum = 0.f;
  b.baseFlags = 0;
  b.hasCoat = false;
  b.hasSheen = false;
  b.hasTransp = false;
  b.hasInner = true;
  b.opaque.hasSpec = false;
  b.opaque.hasSS = false;
  b.opaque.hasDiff = true;
  b.opacityW = 1.f;
  b.transpW = 0.f;
  const float opacity = (F & kFeatTransparent) ? clamp01(m.opacity) : 1.f;
  if ((F & kFeatTransparent) && 1.f - opacity > kMatEps)
  {
    b.hasTransp = true;
    b.opacityW = opacity;
    b.transpW = 1.f - opacity;
    b.hasInner = opacity > kMatEps;
    if (!b.hasInner)
    {
      b.albedoV = mk(-1.f);  // TransparentBtdf::getAlbedo
      return;
    }
  }
  const float base = clamp01(m.baseWeight);
  const f3 baseColor = standardBaseColor(sc, m, ctx);
  const float metalness = clamp01(m.metalness);
  const float specular = clamp01(m.specularWeight);
  const float specularRoughness = clamp01(m.specularRoughness);
  const bool fromOutside = m.thinWalled ? true : !backfacing;
  AlbedoSum albedoSum;
  const float dielectric = 1.f - metalness;
  if ((F & (kFeatOpaque | kFeatDielectric | kFeatThin | kFeatTransparent)) && dielectric > kMatEps)
  {
    const float transmission = clamp01(m.transmissionWeight);
    const DevEta& eta = m.spec[fromOutside ? 0 : 1];
    const float opaque = dielectric * (1.f - transmission);
    if ((F & kFeatOpaque) && opaque > kMatEps)
    {
      auto& o = b.opaque;
      o.diff.color = baseColor * base;
      o.diff.rough = m.hasDiffuseRoughness != 0;
      o.diff.roughness = clamp01(m.diffuseRoughness);
      if (F & kFeatSubsurface)
      {
        const float subsurface = clamp01(m.subsurfaceWeight);
        const float diffuse = 1.f - subsurface;
        o.hasDiff = diffuse > kMatEps;
        o.hasSS = subsurface > kMatEps;
        o.wDiff = diffuse;
        o.wSS = subsurface;
        if (o.hasSS)
        {
          const f3 ssColor = m.subsurfaceFromBase
                               ? baseColor * base
                               : clamp01(mk(m.subsurfaceColor[0], m.subsurfaceColor[1], m.subsurfaceColor[2]));
          const float aniso = fminf(fmaxf(m.subsurfaceAnisotropy, -1.f), 1.f);
          o.wT = (1.f + aniso) * 0.5f;
          o.wR = 1.f - o.wT;
          o.ssHasR = o.wR > kMatEps;
          o.ssHasT = o.wT > kMatEps;
          o.ssRefl.color = ssColor;
          o.ssRefl.rough = o.diff.rough;
          o.ssRefl.roughness = o.diff.roughness;
          o.ssTrans.color = ssColor;
        }
      }
      const auto sub = b.opaqueSub();
      f3 a = sub.albedo();
      int fl = sub.flags();
      float impo = sub.importance();
      if ((F & kFeatSpecular) && fabsf(m.specularIor - m.ambientIor) > kMatEps && specular > kMatEps)
      {
        o.hasSpec = true;
        o.spec.init(t, eta, mk(1.f), 1.f, specularRoughness, m.hasSpecularRoughness != 0, specular);
        fl = o.spec.flags(fl);
        a = o.spec.albedo(a);
        impo = o.spec.importance(impo);
      }
      addSlot(b, kSlotOpaque, opaque, impo, fl);
      albedoSum.add(a, opaque, impo * opaque);
    }
    const float translucent = dielectric * transmission * specular;
    if ((F & (kFeatDielectric | kFeatThin | kFeatTransparent)) && translucent > kMatEps)
    {
      if (fabsf(m.specularIor - m.ambientIor) > kMatEps)
      {
        if ((F & kFeatThin) && m.thinWalled)
        {
          const f3 tc = mk(m.transmissionColor[0], m.transmissionColor[1], m.transmissionColor[2]);
          b.thin.init(t, eta, tc, m.thinThickness, specularRoughness, m.hasSpecularRoughness != 0);
          addSlot(b, kSlotThin, translucent, 1.f, b.thin.flags());
          albedoSum.add(b.thin.albedo(), translucent, translucent);
        }
        else if ((F & kFeatDielectric) && !m.thinWalled)
        {
          b.diel.init(t, eta, specularRoughness, m.hasSpecularRoughness != 0);
          addSlot(b, kSlotDielectric, translucent, 1.f, b.diel.flags());
          albedoSum.add(mk(1.f), translucent, translucent);
        }
      }
      else if (F & kFeatTransparent)
      {
        addSlot(b, kSlotTransparent, translucent, 1.f, kTransparency);
        albedoSum.add(mk(-1.f), translucent, translucent);
      }
    }
  }
  const float metal = metalness * specular;
  if ((F & kFeatConductor) && metal > kMatEps)
  {
    const f3 specColor = clamp01(mk(m.specularColor[0], m.specularColor[1], m.specularColor[2]));
    b.cond.init(t, m.principled ? baseColor : baseColor * base, specColor, specularRoughness,
                m.hasSpecularRoughness != 0);
    addSlot(b, kSlotConductor, metal, 1.f, b.cond.flags());
    albedoSum.add(b.cond.albedo(), metal, metal);
  }
  f3 albedo = (F & kFeatTransparent) ? albedoSum.value() : albedoSum.valueOpaque();
  const float coat = clamp01(m.coatWeight);
  if ((F & kFeatCoat) && coat > kMatEps && fabsf(m.coatIor - m.ambientIor) > kMatEps)
  {
    const DevEta& coatEta = m.coat[fromOutside ? 0 : 1];
    const f3 coatColor = clamp01(mk(m.coatColor[0], m.coatColor[1], m.coatColor[2]));
    b.coat.init(t, coatEta, coatColor, m.coatThickness, clamp01(m.coatRoughness), m.hasCoatRoughness != 0, coat);
    b.hasCoat = true;
    albedo = b.coat.albedo(albedo);
  }
  const float sheen = clamp01(m.sheenWeight);
  if ((F & kFeatSheen) && sheen > kMatEps)
  {
    const f3 sheenColor = clamp01(mk(m.sheenColor[0], m.sheenColor[1], m.sheenColor[2]));
    const float tint = clamp01(m.sheenTint);
    b.sheen.init(sheenColor + tint * (baseColor - sheenColor), clamp01(m.sheenRoughness), sheen);
    b.hasSheen = true;
  }
  if ((F & kFeatTransparent) && b.hasTransp)
  {
    AlbedoSum top;
    top.add(albedo, b.opacityW, b.innerImportance() * b.opacityW);
    top.add(mk(-1.f), b.transpW, b.transpW);
    albedo = top.value();
  }
  b.albedoV = albedo;
}

// Material::getTransparency for a shadow ray crossing the surface (StandardMaterial,
// material/standard.cpp:626-645): 1 - opacity for materials without transmission; otherwise the
// transmittance of the BSDF tree built without its opaque and metal lobes -- thin-walled
// dielectric (1 - R) color^(thickness / cos), transparent lobe 1, solid dielectric 0, scaled by
// the translucent weight, through the coat (CoatLayer::transparency); a sheen layer passes
// nothing (SheenBsdf has no transparency) -- blended with the opacity as the BSDF is.
PRT_D f3 standardTransparency(const DevScene& sc, const DevTables& t, const DevMaterial& m, const ShadeCtx& ctx, f3 wo)
{
  const float opacity = clamp01(m.opacity);
  if (!(m.type & kMatTransmissive)) return mk(1.f - opacity);
  const bool hasTransp = 1.f - opacity > kMatEps;
  if (hasTransp && !(opacity > kMatEps)) return mk(1.f);
  const Frame fr = makeShadingFrame(ctx, wo);
  f3 T = mk(0.f);
  const float metalness = clamp01(m.metalness);
  const float specular = clamp01(m.specularWeight);
  const float dielectric = 1.f - metalness;
  if (dielectric > kMatEps)
  {
    const float transmission = clamp01(m.transmissionWeight);
    const float translucent = dielectric * transmission * specular;
    if (translucent > kMatEps)
    {
      if (fabsf(m.specularIor - m.ambientIor) > kMatEps)
      {
        if (m.thinWalled)
        {
          ThinDielectricLobe thin;
          thin.init(t, m.spec[0], mk(m.transmissionColor[0], m.transmissionColor[1], m.transmissionColor[2]),
                    m.thinThickness, clamp01(m.specularRoughness), m.hasSpecularRoughness != 0);
          T = thin.transparency(t, fr, wo) * translucent;
        }
      }
      else
        T = mk(translucent);
    }
  }
  const float coat = clamp01(m.coatWeight);
  if (coat > kMatEps && fabsf(m.coatIor - m.ambientIor) > kMatEps)
  {
    const bool fromOutside = m.thinWalled ? true : !ctx.backfacing;
    const DevEta& coatEta = m.coat[fromOutside ? 0 : 1];
    CoatLayer c;
    c.init(t, coatEta, clamp01(mk(m.coatColor[0], m.coatColor[1], m.coatColor[2])), m.coatThickness,
           clamp01(m.coatRoughness), m.hasCoatRoughness != 0, coat);
    T = c.transparency(t, fr, wo, T);
  }
  if (clamp01(m.sheenWeight) > kMatEps) T = mk(0.f);
  if (hasTransp) T = T * opacity + mk(1.f - opacity);
  return T;
}

} // namespace prt
