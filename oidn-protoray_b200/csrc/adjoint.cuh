// Path-replay adjoint: the per-vertex gradient step (Vicini, Speierer and Jakob 2021, "Path
// Replay Backpropagation"), used by the replay form of the surface-shading kernel.
//
// The adjoint of an image differentiates the frame-form estimator (NEE with MIS, BSDF
// sampling, Russian roulette; render/path_renderer_stream.h:592-1010) with respect to
//   * every texel of every scene texture used as a Lambertian base colour, and
//   * the specular roughness of every material with a specular layer over a Lambertian base.
// A forward wave leaves each path's radiance L in the path state; the replay wave walks the
// same paths again from their Sobol seeds (recomputation instead of storing the paths) and
// keeps Lrem, the radiance still to come. At surface vertex k, with NEE contribution N_k
// (if unoccluded) and sampled direction wi, the parameters pi of the vertex receive
//     delta . ( dN_k/dpi + (Lrem_k - N_k) * (df_k(wi)/dpi) / f_k(wi) )
// where delta = dLoss/dPixel / spp. Sampling pdfs, MIS weights and the Russian-roulette
// probability are constants of the replay (detached sampling), which keeps the estimator
// unbiased. A Lambertian base colour enters f linearly, so df/drho = f / rho exactly. For
// roughness the local derivative of the BSDF value is a central difference of two BSDF
// evaluations at roughness +- h (h = 1e-3).
//
// Gradients are added with warp-aggregated atomics: active lanes with the same key (texel or
// material) are summed with shuffles and one lane adds the sum.
#pragma once
#include "wavefront.cuh"

namespace prt {

constexpr int kAdjointFeatures = kFeatOpaque | kFeatSpecular;

// Adds v (3 channels) to dst[3 * key ..] once per group of active lanes with the same target
// address (lanes of one warp may belong to different frames of a batch, so the address, not
// the key alone, identifies the target).
PRT_D void groupAdd3(bool has, uint32_t key, f3 v, float* dst)
{
  float* d = dst + 3 * (size_t)key;
  const unsigned active = __activemask();
  const unsigned grp = __match_any_sync(active, has ? (unsigned long long)d : 0ull);
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
    if (s.x != 0.f) atomicAdd(d + 0, s.x);
    if (s.y != 0.f) atomicAdd(d + 1, s.y);
    if (s.z != 0.f) atomicAdd(d + 2, s.z);
  }
}

PRT_D void groupAdd1(bool has, uint32_t key, float v, float* dst)
{
  float* d = dst + key;
  const unsigned active = __activemask();
  const unsigned grp = __match_any_sync(active, has ? (unsigned long long)d : 0ull);
  if (!has) return;
  float s = 0.f;
  for (unsigned m = grp; m; m &= m - 1u) s += __shfl_sync(grp, v, __ffs(m) - 1);
  if (laneId() == __ffs(grp) - 1 && s != 0.f) atomicAdd(d, s);
}

// Bilinear footprint of texLookup (repeat in u and v): the four texels and the fractions.
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

// Gradient step of one surface vertex (see the file comment). neeL = N_k (0 when occluded or
// absent), scat = Lrem_k - N_k when the path continues through wi (0 when it ends here).
template <int F>
PRT_D void adjointVertex(const AdjointView& A, const DevScene& sc, const DevTables& tab, const DevMaterial& mat,
                         const ShadeCtx& ctx, const StdBsdfT<F>& bsdf, f3 wo, f3 wi, f3 wiL, bool extend, bool nee,
                         f3 neeL, f3 scat, f3 delta)
{
  // Lambertian base colour from a texture.
  const bool lambert = !bsdf.opaque.hasSpec && mat.metalness == 0.f && mat.transmissionWeight == 0.f;
  const bool textured = lambert && mat.baseColorTex >= 0 && mat.baseColorTex < kAdjointMaxTextures;
  if (textured)
  {
    const DevTexture& tex = sc.textures[mat.baseColorTex];
    const f3 rho = bsdf.opaque.diff.color;  // clamp01(texture * factor) * baseWeight
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
  if ((F & kFeatSpecular) && bsdf.opaque.hasSpec && (nee || extend))
  {
    const float alpha = clamp01(mat.specularRoughness);
    const float a1 = fminf(alpha + A.step, 1.f), a0 = fmaxf(alpha - A.step, 1e-4f);
    float pdfDummy;
    const f3 f = extend ? bsdf.eval(tab, wo, wi, pdfDummy) : mk(0.f);
    const f3 bv = nee ? bsdf.eval(tab, wo, wiL, pdfDummy) : mk(0.f);
    f3 dn = mk(0.f), ds = mk(0.f);
    for (int side = 0; side < 2; ++side)
    {
      DevMaterial m2 = mat;
      m2.specularRoughness = side ? a1 : a0;
      StdBsdfT<F> b2;
      resolveStandard<F>(sc, tab, m2, ctx, wo, false, b2);
      const float sgn = side ? 1.f : -1.f;
      if (nee) dn += sgn * b2.eval(tab, wo, wiL, pdfDummy);
      if (extend) ds += sgn * b2.eval(tab, wo, wi, pdfDummy);
    }
    const float inv = 1.f / (a1 - a0);
    const float dl[3] = {delta.x, delta.y, delta.z};
    const float b[3] = {bv.x, bv.y, bv.z}, dnv[3] = {dn.x, dn.y, dn.z}, n[3] = {neeL.x, neeL.y, neeL.z};
    const float fv[3] = {f.x, f.y, f.z}, dsv[3] = {ds.x, ds.y, ds.z}, s[3] = {scat.x, scat.y, scat.z};
    float g = 0.f;
    for (int c = 0; c < 3; ++c)
    {
      if (nee && b[c] > 0.f) g += dl[c] * n[c] * dnv[c] * inv / b[c];
      if (extend && fv[c] > 0.f) g += dl[c] * s[c] * dsv[c] * inv / fv[c];
    }
    groupAdd1(g != 0.f, (uint32_t)ctx.material, g, A.gradRough);
  }
}

} // namespace prt
