// Path-replay adjoint of the frame-form path tracer (Vicini, Speierer and Jakob 2021, "Path
// Replay Backpropagation"). It differentiates the image that the wavefront kernels render
// (the estimator of render/path_renderer_stream.h:592-1010: NEE with MIS, BSDF sampling,
// Russian roulette) with respect to
//   * every texel of every scene texture used as a Lambertian base colour, and
//   * the specular roughness of every material with a specular layer over a Lambertian base.
//
// Each thread owns one path (pixel x sample). It walks the path twice from its Sobol seed,
// which makes the walk reproducible instead of stored:
//   1. primal: the path's radiance L;
//   2. replay: at every surface vertex k, the radiance still to come after k's own
//      contributions is Lrem = L - (what was added at vertices <= k). The vertex's
//      parameters pi receive
//        delta . ( dNEE_k/dpi + Lrem * (df_k(wi)/dpi) / f_k(wi) )
//      where delta = dLoss/dPixel / spp and wi is the sampled direction. Sampling pdfs, MIS
//      weights and the Russian-roulette probability are treated as constants (detached
//      sampling), which keeps the estimator unbiased.
// Lambertian base colour enters f linearly, so df/drho = f / rho exactly. For roughness the
// local derivative of the BSDF value is a central difference of two BSDF evaluations at
// roughness +- h (the BSDF is smooth in roughness between the energy-compensation table
// nodes; h = 1e-3 by default).
//
// Gradients are accumulated with warp-aggregated atomics: lanes that hit the same texel (or
// the same material) in the same step are summed with shuffles, and one lane adds the sum.
#include "wavefront.cuh"

#include <algorithm>
#include <cstring>

namespace prt {

constexpr int kAdjointFeatures = kFeatOpaque | kFeatSpecular;
constexpr int kAdjointMaxTextures = 32;

struct AdjointLaunch
{
  DevScene sc;
  DevTables tab;
  DevCamera cam;
  DevRenderer rd;
  int width, height, pixelCount;
  uint32_t firstSample;
  int spp;
  const float* dLdI;     // width * height * 3, row-major, row 0 at the top
  float* gradTex;        // concatenated textures, each width * height * 3, row 0 at the top
  float* gradRough;      // one per material
  long long texOffset[kAdjointMaxTextures];
  float step;            // roughness step of the central difference
  uint32_t* err;
};

// Adds v (3 channels) to dst[3 * key ..] once per group of active lanes with equal keys.
PRT_D void groupAdd3(bool has, uint32_t key, f3 v, float* dst)
{
  const unsigned active = __activemask();
  const unsigned grp = __match_any_sync(active, has ? key : 0xffffffffu);
  if (!has) return;
  f3 s = mk(0.f);
  for (unsigned m = grp; m; m &= m - 1u)
  {
    const int src = __ffs(m) - 1;
    s.x += __shfl_sync(grp, v.x, src);
    s.y += __shfl_sync(grp, v.y, src);
    s.z += __shfl_sync(grp, v.z, src);
  }
  if (laneId() == __ffs(grp) - 1)
  {
    float* d = dst + 3 * (size_t)key;
    if (s.x != 0.f) atomicAdd(d + 0, s.x);
    if (s.y != 0.f) atomicAdd(d + 1, s.y);
    if (s.z != 0.f) atomicAdd(d + 2, s.z);
  }
}

PRT_D void groupAdd1(bool has, uint32_t key, float v, float* dst)
{
  const unsigned active = __activemask();
  const unsigned grp = __match_any_sync(active, has ? key : 0xffffffffu);
  if (!has) return;
  float s = 0.f;
  for (unsigned m = grp; m; m &= m - 1u) s += __shfl_sync(grp, v, __ffs(m) - 1);
  if (laneId() == __ffs(grp) - 1 && s != 0.f) atomicAdd(dst + key, s);
}

// Bilinear footprint of texLookup (repeat in u and v): the four texels and their weights.
struct TexFootprint
{
  int x[2], y[2];
  float sx, sy;
};

PRT_D TexFootprint texFootprint(int w, int h, float u, float v)
{
  TexFootprint f;
  const float x = u - 0.5f / (float)w;
  const float y = v - 0.5f / (float)h;
  const float xr = (x - floorf(x)) * (float)w;
  const float yr = (y - floorf(y)) * (float)h;
  f.sx = xr - floorf(xr);
  f.sy = yr - floorf(yr);
  f.x[0] = min(max((int)xr, 0), w - 1);
  f.y[0] = min(max((int)yr, 0), h - 1);
  f.x[1] = f.x[0] + 1 == w ? 0 : f.x[0] + 1;
  f.y[1] = f.y[0] + 1 == h ? 0 : f.y[0] + 1;
  return f;
}

// One walk of a camera path. Adjoint = false: returns the path's radiance. Adjoint = true:
// replays the same path given its radiance L and scatters delta-weighted derivatives.
template <bool Adjoint>
PRT_D f3 walkPath(const AdjointLaunch& A, int x, int y, uint32_t sampleIndex, f3 L, f3 delta)
{
  using Bsdf = StdBsdfT<kAdjointFeatures>;
  const DevScene& sc = A.sc;
  uint32_t pixelId = (uint32_t)x | ((uint32_t)y << 16);
  f3 org, dir;
  float tnear;
  {
    const SobolState st = sobolSetSample(A.rd.seed, sampleIndex, pixelId);
    float sx, sy;
    sobolGet2D(st, kDimPixel, sx, sy);
    cameraRay(A.cam, ((float)x + sx) * (1.f / (float)A.width), ((float)y + sy) * (1.f / (float)A.height), org, dir,
              tnear);
  }
  f3 T = mk(1.f);
  f3 Lp = mk(0.f);     // primal radiance
  f3 Lrem = L;         // replay: radiance still to come
  float lastPdf = 1.f;
  int lastType = kSpecularReflection;
  for (int depth = 0; depth <= A.rd.maxDepth; ++depth)
  {
    const TraceHit h = traverse<false>(sc.nodes, sc.tris, org, dir, tnear, kPosMax, A.err);
    if (h.triId < 0)
    {
      float lightPdf;
      const f3 Le = evalEnvLights(sc, dir, lightPdf);
      const float w = (lastType & kBsdfSmooth) == 0 ? 1.f : misWeight(lastPdf, lightPdf);
      Lp += T * w * Le;
      break;
    }
    const int4 tv = __ldg(sc.triVerts + h.triId);
    const int matId = __ldg(sc.meshMaterial + tv.w);
    if (sc.materials[matId].type & kMatEmissive)
    {
      float lightPdf;
      const int prim = h.triId - __ldg(sc.meshTriOffset + tv.w);
      const f3 Le = evalAreaLight(sc, tv.w, prim, dir, h.t, lightPdf);
      const float w = (lastType & kBsdfSmooth) == 0 ? 1.f : misWeight(lastPdf, lightPdf);
      Lp += T * w * Le;
      break;
    }
    if (depth >= A.rd.maxDepth) break;
    ShadeCtx ctx;
    postIntersect(sc, org, dir, h.t, h.triId, h.u, h.v, ctx);
    const DevMaterial& mat = sc.materials[ctx.material];
    const f3 wo = -dir;
    Bsdf bsdf;
    resolveStandard<kAdjointFeatures>(sc, A.tab, mat, ctx, wo, false, bsdf);
    const SobolState st = sobolSetSample(A.rd.seed, sampleIndex, pixelId & kPixelIdMask);
    const uint32_t sampleDim = kDimBase + kDimBounce * (uint32_t)depth;
    const bool aov1 = (pixelId & kPathAov1Flag) == 0u;
    const bool aov2 = (pixelId & kPathAov2Flag) == 0u;
    const bool rr = !(aov1 || aov2);
    // Direct light (NEE)
    f3 dirL = mk(0.f), wiL = mk(0.f);
    bool nee = false;
    if (bsdf.flags() & kBsdfSmooth)
    {
      float lx, ly, lz;
      sobolGet3D(st, sampleDim + kDimLight, lx, ly, lz);
      float lightPdf, dist;
      const f3 Lw = sampleLight(sc, ctx.p, lx, ly, lz, wiL, lightPdf, dist);
      if (reduceMax(Lw) > 0.f && lightPdf > 0.f)
      {
        float bsdfPdf;
        const f3 bv = bsdf.eval(A.tab, wo, wiL, bsdfPdf);
        if (reduceMax(bv) > 0.f)
        {
          const f3 dirT = T * bv;
          if (depth >= A.rd.rrDepth)
          {
            const float contProb = rr ? fminf(luminance(dirT * (1.f / bsdfPdf)), 0.95f) : 1.f;
            bsdfPdf *= contProb;
          }
          dirL = dirT * misWeight(lightPdf, bsdfPdf) * Lw;
          const float far = dist - ctx.eps;
          nee = far > 0.f ? traverse<true>(sc.nodes, sc.tris, ctx.p, wiL, ctx.eps, far, A.err).triId < 0 : true;
          if (nee) Lp += dirL;
        }
      }
    }
    // BSDF sampling
    float bx, by, bz;
    sobolGet3D(st, sampleDim + kDimBsdf, bx, by, bz);
    f3 wi;
    float bsdfPdf;
    int bsdfType;
    const f3 bw = bsdf.sample(A.tab, wo, bx, by, bz, wi, bsdfPdf, bsdfType);
    bool extend = reduceMax(bw) > 0.f && bsdfPdf > 0.f;
    const int extType = extend ? bsdfType : 0;
    if (aov1) pixelId |= kPathAov1Flag;
    if (aov2 && (extType & kBsdfDelta) == 0) pixelId |= kPathAov2Flag;
    f3 Tn = T * bw;
    extend = extend && reduceMax(Tn) >= A.rd.minWeight;
    if (depth >= A.rd.rrDepth)
    {
      const float contProb = rr ? fminf(luminance(Tn), 0.95f) : 1.f;
      extend = extend && sobolGet1D(st, sampleDim + kDimTerminate) <= contProb;
      Tn *= 1.f / contProb;
      bsdfPdf *= contProb;
    }
    if (Adjoint)
    {
      if (nee) Lrem = Lrem - dirL;
      const f3 scat = extend ? Lrem : mk(0.f);   // radiance that arrives through wi
      const f3 neeL = nee ? dirL : mk(0.f);
      // Lambertian base colour from a texture.
      const bool lambert = !bsdf.opaque.hasSpec && mat.metalness == 0.f && mat.transmissionWeight == 0.f;
      if (lambert && mat.baseColorTex >= 0 && mat.baseColorTex < kAdjointMaxTextures)
      {
        const DevTexture& tex = sc.textures[mat.baseColorTex];
        const f3 rho = bsdf.opaque.diff.color;               // clamp01(texture * factor) * baseWeight
        const f3 raw = textureRgb(tex, ctx.uvx, ctx.uvy);
        const float base = clamp01(mat.baseWeight);
        const float fac[3] = {mat.baseColor[0], mat.baseColor[1], mat.baseColor[2]};
        const float r[3] = {rho.x, rho.y, rho.z}, rw[3] = {raw.x, raw.y, raw.z};
        const float num[3] = {neeL.x + scat.x, neeL.y + scat.y, neeL.z + scat.z};
        const float dl[3] = {delta.x, delta.y, delta.z};
        float g[3];
        for (int c = 0; c < 3; ++c)
        {
          const float t = rw[c] * fac[c];
          // d(pixel)/d(texture value): 0 where the colour is clamped.
          g[c] = (r[c] > 1e-6f && t > 0.f && t < 1.f) ? dl[c] * num[c] / r[c] * base * fac[c] : 0.f;
        }
        const bool has = g[0] != 0.f || g[1] != 0.f || g[2] != 0.f;
        const TexFootprint fp = texFootprint(tex.width, tex.height, ctx.uvx, ctx.uvy);
        const float wx[2] = {1.f - fp.sx, fp.sx}, wy[2] = {1.f - fp.sy, fp.sy};
        float* dst = A.gradTex + A.texOffset[mat.baseColorTex];
        for (int j = 0; j < 2; ++j)
          for (int i = 0; i < 2; ++i)
          {
            const float wgt = wx[i] * wy[j];
            // Device rows are stored bottom-up; gradients are returned top-down.
            const uint32_t key = (uint32_t)((tex.height - 1 - fp.y[j]) * tex.width + fp.x[i]);
            groupAdd3(has, key, mk(g[0] * wgt, g[1] * wgt, g[2] * wgt), dst);
          }
      }
      // Specular roughness of a specular layer over a Lambertian base.
      if (bsdf.opaque.hasSpec)
      {
        const float alpha = clamp01(mat.specularRoughness);
        const float a1 = fminf(alpha + A.step, 1.f), a0 = fmaxf(alpha - A.step, 1e-4f);
        float pdfDummy;
        const f3 f = extend ? bsdf.eval(A.tab, wo, wi, pdfDummy) : mk(0.f);
        f3 dn = mk(0.f), ds = mk(0.f);
        for (int side = 0; side < 2; ++side)
        {
          DevMaterial m2 = mat;
          m2.specularRoughness = side ? a1 : a0;
          Bsdf b2;
          resolveStandard<kAdjointFeatures>(sc, A.tab, m2, ctx, wo, false, b2);
          const float sgn = side ? 1.f : -1.f;
          if (nee) dn += sgn * b2.eval(A.tab, wo, wiL, pdfDummy);
          if (extend) ds += sgn * b2.eval(A.tab, wo, wi, pdfDummy);
        }
        const float inv = 1.f / (a1 - a0);
        float g = 0.f;
        if (nee)
        {
          float p2;
          const f3 bv = bsdf.eval(A.tab, wo, wiL, p2);
          const float b[3] = {bv.x, bv.y, bv.z}, d[3] = {dn.x, dn.y, dn.z}, n[3] = {neeL.x, neeL.y, neeL.z};
          const float dl[3] = {delta.x, delta.y, delta.z};
          for (int c = 0; c < 3; ++c)
            if (b[c] > 0.f) g += dl[c] * n[c] * d[c] * inv / b[c];
        }
        if (extend)
        {
          const float fv[3] = {f.x, f.y, f.z}, d[3] = {ds.x, ds.y, ds.z}, s[3] = {scat.x, scat.y, scat.z};
          const float dl[3] = {delta.x, delta.y, delta.z};
          for (int c = 0; c < 3; ++c)
            if (fv[c] > 0.f) g += dl[c] * s[c] * d[c] * inv / fv[c];
        }
        groupAdd1(g != 0.f, (uint32_t)ctx.material, g, A.gradRough);
      }
    }
    if (!extend) break;
    T = Tn;
    const bool update = (bsdfType & kBsdfContinuation) == 0;
    if (update)
    {
      lastPdf = bsdfPdf;
      lastType = bsdfType;
    }
    org = ctx.p;
    dir = wi;
    tnear = ctx.eps;
  }
  return Lp;
}

__global__ void __launch_bounds__(128) kAdjoint(AdjointLaunch A)
{
  const int64_t total = (int64_t)A.pixelCount * A.spp;
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total; w += (int64_t)gridDim.x * blockDim.x)
  {
    const int s = (int)(w / A.pixelCount);
    const int idx = (int)(w - (int64_t)s * A.pixelCount);
    int x, y;
    pixelOf(idx, A.width, x, y);
    const uint32_t sampleIndex = A.firstSample + (uint32_t)s;
    const float* g = A.dLdI + 3 * ((size_t)y * A.width + x);
    const float invSpp = 1.f / (float)A.spp;
    const f3 delta = mk(g[0] * invSpp, g[1] * invSpp, g[2] * invSpp);
    if (!(reduceMax(abs3(delta)) > 0.f)) continue;
    const f3 L = walkPath<false>(A, x, y, sampleIndex, mk(0.f), mk(0.f));
    walkPath<true>(A, x, y, sampleIndex, L, delta);
  }
}

__global__ void kTextureFromImage(const float* __restrict__ src, float* __restrict__ dst, int w, int h)
{
  const int64_t n = (int64_t)w * h;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int y = (int)(i / w), x = (int)(i - (int64_t)y * w);
    const int64_t d = ((int64_t)(h - 1 - y) * w + x) * 3;
    dst[d + 0] = src[3 * i + 0];
    dst[d + 1] = src[3 * i + 1];
    dst[d + 2] = src[3 * i + 2];
  }
}

cudaError_t launchAdjoint(Context& ctx, uint32_t firstSample, int spp, const float* dLdI, float* gradTex,
                          float* gradRough, float roughnessStep)
{
  AdjointLaunch A;
  std::memset(&A, 0, sizeof(A));
  A.sc = ctx.scene;
  A.tab = ctx.tables;
  A.cam = ctx.camera;
  A.rd = ctx.renderer;
  A.width = ctx.width;
  A.height = ctx.height;
  A.pixelCount = ctx.width * ctx.height;
  A.firstSample = firstSample;
  A.spp = spp;
  A.dLdI = dLdI;
  A.gradTex = gradTex;
  A.gradRough = gradRough;
  long long off = 0;
  for (size_t i = 0; i < ctx.texturesHost.size() && i < (size_t)kAdjointMaxTextures; ++i)
  {
    A.texOffset[i] = off;
    off += 3ll * ctx.texturesHost[i].width * ctx.texturesHost[i].height;
  }
  A.step = roughnessStep;
  A.err = ctx.ps.err;
  const int64_t total = (int64_t)A.pixelCount * spp;
  const int64_t blocks = std::min<int64_t>((total + 127) / 128, (int64_t)ctx.smCount * 16);
  kAdjoint<<<(int)std::max<int64_t>(blocks, 1), 128, 0, ctx.stream>>>(A);
  return cudaGetLastError();
}

cudaError_t launchTextureUpdate(Context& ctx, const DevTexture& t, const float* rgb)
{
  const int64_t n = (int64_t)t.width * t.height;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx.smCount * 8));
  kTextureFromImage<<<blocks, 256, 0, ctx.stream>>>(rgb, const_cast<float*>(t.rgb), t.width, t.height);
  return cudaGetLastError();
}

} // namespace prt
