// Hit-point reconstruction, shading frames, sampling distributions and lights on the device.
#pragma once

#include "device_scene.h"
#include "prt_math.cuh"

namespace prt {

constexpr float kEpsScale = 0x1.fp-18f;  // core/ray.h:66
constexpr float kMatEps = 1e-4f;         // math/constants eps used by the materials

// Per-hit shading context (core/shading_context.h:111-120).
struct ShadeCtx
{
  f3 p;
  float eps;
  Frame f;       // interpolated shading frame
  f3 Ng;         // geometric normal, facing the incoming ray
  float uvx, uvy;
  bool backfacing;
  int mesh;
  int material;
  int prim;      // triangle index within its mesh
};

PRT_D f3 ldf4(const float4* p, int i)
{
  const float4 v = __ldg(p + i);
  return mk(v.x, v.y, v.z);
}

// Scene::postIntersect (render/scene.h:61-72) -> TriangleMesh::postIntersect
// (geometry/triangle_mesh.cpp:152-250), for the triangle triId hit at (t, u, v).
PRT_D void postIntersect(const DevScene& sc, f3 org, f3 dir, float t, int triId, float hu, float hv, ShadeCtx& ctx)
{
  const int4 tv = __ldg(sc.triVerts + triId);
  const int mesh = tv.w;
  ctx.mesh = mesh;
  ctx.material = __ldg(sc.meshMaterial + mesh);
  ctx.prim = triId - __ldg(sc.meshTriOffset + mesh);
  const int flags = __ldg(sc.meshFlags + mesh);
  const float b1 = hu, b2 = hv;
  const float b0 = 1.f - b1 - b2;
  // Ray::getHitPoint(eps), core/ray.h:60-67
  ctx.p = org + t * dir;
  ctx.eps = fmaxf(t, reduceMax(abs3(ctx.p))) * kEpsScale;
  const f3 p0 = ldf4(sc.pos, tv.x), p1 = ldf4(sc.pos, tv.y), p2 = ldf4(sc.pos, tv.z);
  const f3 dp1 = p1 - p0, dp2 = p2 - p0;
  const f3 Ng = normalize(cross(dp1, dp2));
  f3 N = Ng;
  if (flags & 1)
  {
    const f3 n0 = ldf4(sc.nrm, tv.x), n1 = ldf4(sc.nrm, tv.y), n2 = ldf4(sc.nrm, tv.z);
    N = normalize(b0 * n0 + b1 * n1 + b2 * n2);
    if (dot(N, Ng) < 0.f) N = -N;
  }
  ctx.Ng = Ng;
  ctx.f.N = N;
  if (flags & 2)
  {
    const float2 t0 = __ldg(sc.uv + tv.x), t1 = __ldg(sc.uv + tv.y), t2 = __ldg(sc.uv + tv.z);
    ctx.uvx = b0 * t0.x + b1 * t1.x + b2 * t2.x;
    ctx.uvy = b0 * t0.y + b1 * t1.y + b2 * t2.y;
    const float du1 = t1.x - t0.x, du2 = t2.x - t0.x;
    const float dv1 = t1.y - t0.y, dv2 = t2.y - t0.y;
    const float det = du1 * dv2 - dv1 * du2;
    const float invDet = 1.f / det;
    const f3 dpdu = (dv2 * dp1 - dv1 * dp2) * invDet;
    const f3 dpdv = (du1 * dp2 - du2 * dp1) * invDet;
    f3 U = dpdu - dot(dpdu, N) * N;
    const float Ulen2 = lengthSqr(U);
    U = U * rsqrtf(Ulen2);
    f3 V = dpdv - dot(dpdv, N) * N;
    V = V - dot(V, U) * U;
    const float Vlen2 = lengthSqr(V);
    V = V * rsqrtf(Vlen2);
    if (det == 0.f || Ulen2 == 0.f || Vlen2 == 0.f || !(Ulen2 < kPosMax) || !(Vlen2 < kPosMax))
      makeFrame(N, U, V);
    ctx.f.U = U;
    ctx.f.V = V;
  }
  else
  {
    ctx.uvx = hu;
    ctx.uvy = hv;
    makeFrame(N, ctx.f.U, ctx.f.V);
  }
  ctx.backfacing = dot(ctx.Ng, dir) > 0.f;
  if (ctx.backfacing)
  {
    ctx.Ng = -ctx.Ng;
    ctx.f.N = -ctx.f.N;
  }
}

// ShadingContextSimd::makeFrame (core/shading_context.h:144-191) for the default tangent-space
// normal (0,0,1): Keller et al. 2017 shading-normal adaptation, then Gram-Schmidt.
PRT_D Frame makeShadingFrame(const ShadeCtx& ctx, f3 wo)
{
  Frame fr;
  f3 N = ctx.f.N;
  f3 wi = reflect(wo, N);
  if (dot(wi, ctx.Ng) < 0.f)
  {
    const float a = -dot(wi, ctx.Ng);
    float b = dot(N, ctx.Ng);
    if (b < 0.f)
    {
      b = -b;
      wi = -wi;
    }
    const f3 wi1 = normalize(wi + a * rcpSafe(b) * N + 1e-5f * ctx.Ng);
    N = normalize(wo + wi1);
  }
  fr.N = N;
  f3 U = ctx.f.U - dot(ctx.f.U, N) * N;
  const float Ulen2 = lengthSqr(U);
  U = U * rsqrtf(Ulen2);
  f3 V = ctx.f.V - dot(ctx.f.V, N) * N;
  V = V - dot(V, U) * U;
  const float Vlen2 = lengthSqr(V);
  V = V * rsqrtf(Vlen2);
  if (Ulen2 == 0.f || Vlen2 == 0.f)
    makeFrame(N, U, V);
  fr.U = U;
  fr.V = V;
  return fr;
}

// ---- Distribution1D (sampling/distribution1d.{h,cpp}) -------------------------------------
PRT_D int cdfLookup(const float* cdf, int size, float s)
{
  int first = 0, len = size;
  while (len > 0)
  {
    const int half = len >> 1;
    const int mid = first + half;
    if (s < __ldg(cdf + mid))
      len = half;
    else
    {
      first = mid + 1;
      len = len - half - 1;
    }
  }
  return max(first - 1, 0);
}

PRT_D int cdfSample(const float* cdf, int size, float& pdf, float s)
{
  const int i = cdfLookup(cdf, size, s);
  pdf = __ldg(cdf + i + 1) - __ldg(cdf + i);
  return i;
}

PRT_D int cdfSampleReuse(const float* cdf, int size, float& pdf, float& s)
{
  const int i = cdfLookup(cdf, size, s);
  const float c0 = __ldg(cdf + i), c1 = __ldg(cdf + i + 1);
  pdf = c1 - c0;
  s = (s - c0) * (1.f / pdf);
  return i;
}

PRT_D float cdfPdf(const float* cdf, int size, int i)
{
  if (i < 0 || i >= size) return 0.f;
  return __ldg(cdf + i + 1) - __ldg(cdf + i);
}

// ---- shape samplers (sampling/shape_sampler.h) ----------------------------------------------
PRT_D f3 cosineSampleHemisphere(float& pdf, float sx, float sy)
{
  const float cosTheta = sqrtf(sx);
  const float sinTheta = sqrtf(1.f - sx);
  float sinPhi, cosPhi;
  sincospif(2.f * sy, &sinPhi, &cosPhi);  // phi = 2 pi sy
  pdf = cosTheta * kInvPi;
  return mk(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
}

PRT_D f3 uniformSampleSphere(float& pdf, float sx, float sy)
{
  const float cosTheta = 1.f - 2.f * sx;
  const float sinTheta = 2.f * sqrtf(sx * (1.f - sx));
  float sinPhi, cosPhi;
  sincospif(2.f * sy, &sinPhi, &cosPhi);
  pdf = 1.f / (4.f * kPi);
  return mk(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
}

PRT_D float cos2sin(float c) { return sqrtf(fmaxf(1.f - c * c, 0.f)); }

PRT_D f3 uniformSampleCone(float& pdf, float sx, float sy, float angle, float cosAngle, float conePdf)
{
  const float cosTheta = 1.f - sx * (1.f - cosAngle);
  const float sinTheta = cos2sin(cosTheta);
  float sinPhi, cosPhi;
  sincospif(2.f * sy, &sinPhi, &cosPhi);
  pdf = conePdf;
  (void)angle;
  return mk(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
}

PRT_D f3 uniformSampleTriangle(float u, float v, f3 v0, f3 v1, f3 v2)
{
  if (v > u)
  {
    u *= 0.5f;
    v -= u;
  }
  else
  {
    v *= 0.5f;
    u -= v;
  }
  return v2 + u * (v0 - v2) + v * (v1 - v2);
}

// ---- lights -------------------------------------------------------------------------------
struct Etri
{
  f3 v0, v1, v2, n, color;
};

PRT_D Etri loadEtri(const DevScene& sc, int i)
{
  const float4* p = reinterpret_cast<const float4*>(sc.etris) + 4 * i;
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
  Etri e;
  e.v0 = mk(a.x, a.y, a.z);
  e.v1 = mk(a.w, b.x, b.y);
  e.v2 = mk(b.z, b.w, c.x);
  e.n = mk(c.y, c.z, c.w);
  e.color = mk(d.x, d.y, d.z);
  return e;
}

// Bilinear texture lookup (ImageTextureImpl::get, image/image_texture.h:197-226): half-texel
// shift, repeat in u, repeat or clamp in v, a + s*(b - a) interpolation. `rgb` is stored in
// texture-row order (row 0 = the bottom image row), the order ImageTextureBuffer::store
// writes (image/image_texture.h:377-392), so v indexes rows directly.
PRT_D f3 texLookup(const float* rgb, int w, int h, float u, float v, bool repeatV)
{
  const float x = u - 0.5f / (float)w;
  const float y = v - 0.5f / (float)h;
  const float xr = (x - floorf(x)) * (float)w;
  const float yr = repeatV ? (y - floorf(y)) * (float)h : fminf(fmaxf(y * (float)h, 0.f), (float)(h - 1));
  const float sx = xr - floorf(xr), sy = yr - floorf(yr);
  const int x0 = min(max((int)xr, 0), w - 1);
  const int y0 = min(max((int)yr, 0), h - 1);
  const int x1 = x0 + 1 == w ? 0 : x0 + 1;
  const int y1 = repeatV ? (y0 + 1 == h ? 0 : y0 + 1) : min(y0 + 1, h - 1);
  const f3 c00 = ld3(rgb + 3 * ((size_t)y0 * w + x0));
  const f3 c10 = ld3(rgb + 3 * ((size_t)y0 * w + x1));
  const f3 c01 = ld3(rgb + 3 * ((size_t)y1 * w + x0));
  const f3 c11 = ld3(rgb + 3 * ((size_t)y1 * w + x1));
  const f3 c0 = c00 + sx * (c10 - c00);
  const f3 c1 = c01 + sx * (c11 - c01);
  return c0 + sy * (c1 - c0);
}

PRT_D float imageLightPdf(const DevImageLight& im, float u, float v, float sinTheta)
{
  int ix = (int)(u * (float)im.lutW);
  int iy = (int)(v * (float)im.lutH);
  ix = min(max(ix, 0), im.lutW - 1);
  iy = min(max(iy, 0), im.lutH - 1);
  const float xPdf = cdfPdf(im.xCdfs + (size_t)iy * (im.lutW + 1), im.lutW, ix);
  const float yPdf = cdfPdf(im.yCdf, im.lutH, iy);
  return xPdf * yPdf * (float)im.lutW * (float)im.lutH * (1.f / (2.f * kPi * kPi * sinTheta));
}

// One environment light's radiance and solid-angle pdf toward wi.
PRT_D f3 evalEnv(const DevScene& sc, int e, f3 wi, float& pdf)
{
  const DevEnvLight& L = sc.env[e];
  pdf = 0.f;
  if (L.kind == kEnvDistant)
  {
    // DistantLight::eval (light/distant_light.h:48-57)
    const float c = dot(wi, mk(L.dir[0], L.dir[1], L.dir[2]));
    if (!(c >= L.cosAngle)) return mk(0.f);
    pdf = L.conePdf;
    return mk(L.color[0], L.color[1], L.color[2]);
  }
  if (L.kind == kEnvAmbient)
  {
    pdf = 1.f / (4.f * kPi);
    return mk(L.color[0], L.color[1], L.color[2]);
  }
  // ImageLight::eval (light/image_light.h:79-92)
  const float theta = acosf(fminf(fmaxf(wi.y, -1.f), 1.f));
  const float phi = atan2f(wi.x, -wi.z);
  const float u = 0.5f + phi * (1.f / (2.f * kPi));
  const float v = 1.f - theta * (1.f / kPi);
  pdf = imageLightPdf(sc.image, u, v, sinf(theta));
  return texLookup(sc.image.rgb, sc.image.width, sc.image.height, u, v, false);
}

// Scene::evalEnvLight (render/scene.h:142-157).
PRT_D f3 evalEnvLights(const DevScene& sc, f3 wi, float& pdf)
{
  f3 value = mk(0.f);
  pdf = 0.f;
  for (int e = 0; e < sc.envCount; ++e)
  {
    float p;
    value += evalEnv(sc, e, wi, p);
    pdf += p * cdfPdf(sc.lightCdf, sc.lightCount, sc.areaLightCount + e);
  }
  return value;
}

// Scene::evalAreaLight + TriangleLight::eval (render/scene.h:173-195, light/triangle_light.h:91-108).
PRT_D f3 evalAreaLight(const DevScene& sc, int mesh, int prim, f3 wi, float dist, float& pdf)
{
  pdf = 0.f;
  const int lightId = __ldg(sc.meshLight + mesh);
  if (lightId < 0) return mk(0.f);
  const int cnt = __ldg(sc.areaTriCount + lightId);
  const float pickProb = cdfPdf(sc.areaCdf + __ldg(sc.areaCdfOffset + lightId), cnt, prim);
  const Etri e = loadEtri(sc, __ldg(sc.areaTriOffset + lightId) + prim);
  const float dirDotN = dot(wi, e.n);
  if (!(dirDotN < 0.f)) return mk(0.f);
  pdf = 2.f * dist * dist * rcpSafe(fabsf(dirDotN)) * pickProb;
  pdf *= cdfPdf(sc.lightCdf, sc.lightCount, lightId);
  return e.color;
}

// Light::sample of light `l` (area lights first, then environment lights). Returns the
// radiance divided by the pdf; zero on failure.
PRT_D f3 sampleOneLight(const DevScene& sc, int l, f3 p, float sx, float sy, float sc3, f3& wi, float& pdf,
                        float& dist)
{
  pdf = 0.f;
  dist = kPosMax;
  if (l < sc.areaLightCount)
  {
    // TriangleLight::sample (light/triangle_light.h:130-157)
    const int cnt = __ldg(sc.areaTriCount + l);
    float pickProb;
    const int t = cdfSample(sc.areaCdf + __ldg(sc.areaCdfOffset + l), cnt, pickProb, sc3);
    const Etri e = loadEtri(sc, __ldg(sc.areaTriOffset + l) + t);
    const f3 d = uniformSampleTriangle(sx, sy, e.v0, e.v1, e.v2) - p;
    dist = sqrtf(lengthSqr(d));
    const float dirDotN = dot(d, e.n);
    if (!(dirDotN < 0.f)) return mk(0.f);
    wi = d * (1.f / dist);
    pdf = 2.f * dist * dist * dist * rcpSafe(fabsf(dirDotN)) * pickProb;
    return e.color * (1.f / pdf);
  }
  const DevEnvLight& L = sc.env[l - sc.areaLightCount];
  if (L.kind == kEnvDistant)
  {
    // DistantLight::sample (light/distant_light.h:66-72)
    const f3 local = uniformSampleCone(pdf, sx, sy, L.halfAngle, L.cosAngle, L.conePdf);
    wi = local.x * mk(L.frameU[0], L.frameU[1], L.frameU[2]) + local.y * mk(L.frameV[0], L.frameV[1], L.frameV[2]) +
         local.z * mk(L.dir[0], L.dir[1], L.dir[2]);
    return mk(L.color[0], L.color[1], L.color[2]) * (1.f / pdf);
  }
  if (L.kind == kEnvAmbient)
  {
    wi = uniformSampleSphere(pdf, sx, sy);
    return mk(L.color[0], L.color[1], L.color[2]) * (1.f / pdf);
  }
  // ImageLight::sample (light/image_light.h:112-135)
  const DevImageLight& im = sc.image;
  float yPdf, xPdf;
  float s1 = sy, s0 = sx;
  const int iy = cdfSampleReuse(im.yCdf, im.lutH, yPdf, s1);
  const int ix = cdfSampleReuse(im.xCdfs + (size_t)iy * (im.lutW + 1), im.lutW, xPdf, s0);
  const float u = ((float)ix + s0) * (1.f / (float)im.lutW);
  const float v = ((float)iy + s1) * (1.f / (float)im.lutH);
  // theta = (1 - v) pi, phi = (u - 0.5) 2 pi
  float sinPhi, cosPhi, sinTheta, cosTheta;
  sincospif((u - 0.5f) * 2.f, &sinPhi, &cosPhi);
  sincospif(1.f - v, &sinTheta, &cosTheta);
  wi = mk(sinPhi * sinTheta, cosTheta, -cosPhi * sinTheta);
  pdf = xPdf * yPdf * (float)im.lutW * (float)im.lutH * (1.f / (2.f * kPi * kPi * sinTheta));
  return texLookup(im.rgb, im.width, im.height, u, v, false) * (1.f / pdf);
}

// Scene::sampleLight (render/scene.h:215-250).
PRT_D f3 sampleLight(const DevScene& sc, f3 p, float sx, float sy, float sz, f3& wi, float& pdf, float& dist,
                     int& light)
{
  light = 0;
  if (sc.lightCount == 1) return sampleOneLight(sc, 0, p, sx, sy, sz, wi, pdf, dist);
  float pickProb;
  float s = sz;
  const int l = cdfSampleReuse(sc.lightCdf, sc.lightCount, pickProb, s);
  light = l;
  const f3 w = sampleOneLight(sc, l, p, sx, sy, s, wi, pdf, dist);
  pdf *= pickProb;
  return w * (1.f / pickProb);
}

} // namespace prt
