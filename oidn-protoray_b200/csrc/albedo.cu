// Energy-compensation tables built on the device at context creation.
//
// Restates precomputeAlbedoTables (bsdf/albedo_tables.cpp:37-188) with the integrators of
// bsdf/albedo.h: each table entry is a midpoint-rule integral over an n x n grid of
// visible-normal samples (n = sqrt(1024) = 32), accumulated in the same order as the
// reference, one thread per entry; the directional-average tables integrate each row with the
// trapezoid rule over 1025 points (integrateAvg, bsdf/albedo_tables.cpp:20-31).
#include "bsdf.cuh"
#include "runtime.h"
#include "host_rcp.h"

namespace prt {

namespace {

PRT_D f3 woOf(float cosThetaO)
{
  const float c = fmaxf(cosThetaO, 1e-6f);
  return mk(cos2sin(c), 0.f, c);
}

PRT_D float sampleCoord(int i, int n) { return fminf(((float)i + 0.5f) / (float)n, 1.f - 1e-6f); }

// MicrofacetAlbedo::sample (bsdf/albedo.h:16-31)
PRT_D float ggxSample(float cosThetaO, const GGX& mf, float sx, float sy)
{
  const f3 wo = woOf(cosThetaO);
  float whPdf;
  const f3 wh = mf.sampleVisible(wo, whPdf, sx, sy);
  const float cosThetaOH = dot(wo, wh);
  const f3 wi = 2.f * cosThetaOH * wh - wo;
  if (wi.z <= 0.f) return 0.f;
  return mf.G2(wo, wi) * rcpSafe(mf.G1(wo));
}

// MicrofacetDielectricAlbedo::sample (bsdf/albedo.h:55-83)
PRT_D float dielSample(float cosThetaO, float eta, const GGX& mf, float sx, float sy)
{
  const f3 wo = woOf(cosThetaO);
  float whPdf;
  const f3 wh = mf.sampleVisible(wo, whPdf, sx, sy);
  const float cosThetaOH = dot(wo, wh);
  float cosThetaTH;
  const float F = fresnelDielectricEx(cosThetaOH, cosThetaTH, eta);
  float weight = 0.f;
  f3 wi = 2.f * cosThetaOH * wh - wo;
  if (wi.z > 0.f) weight += F * (mf.G2(wo, wi) * rcpSafe(mf.G1(wo)));
  wi = refractDir(wo, wh, cosThetaOH, cosThetaTH, eta);
  if (wi.z < 0.f) weight += (1.f - F) * (mf.G2(wo, wi) * rcpSafe(mf.G1(wo)));
  return weight;
}

// MicrofacetDielectricReflectionAlbedo::sample (bsdf/albedo.h:101-118)
PRT_D float reflSample(float cosThetaO, float eta, const GGX& mf, float sx, float sy)
{
  const f3 wo = woOf(cosThetaO);
  float whPdf;
  const f3 wh = mf.sampleVisible(wo, whPdf, sx, sy);
  const float cosThetaOH = dot(wo, wh);
  const float F = fresnelDielectric(cosThetaOH, eta);
  const f3 wi = 2.f * cosThetaOH * wh - wo;
  if (wi.z <= 0.f) return 0.f;
  return F * (mf.G2(wo, wi) * rcpSafe(mf.G1(wo)));
}

__global__ void kGgxTable(float* dir)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int size = kGgxTableSize;
  if (idx >= size * size) return;
  const int i = idx % size, j = idx / size;
  const float cosThetaO = (float)i / (size - 1);
  const float roughness = (float)j / (size - 1);
  GGX mf;
  mf.ax = mf.ay = roughnessToAlpha(roughness);
  const int n = 32;
  float sum = 0.f;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) sum += ggxSample(cosThetaO, mf, sampleCoord(a, n), sampleCoord(b, n));
  dir[idx] = fminf(sum / (float)(n * n), 1.f);
}

// kind 0: dielectric (reflection + transmission), 1: dielectric reflection only.
__global__ void kDielTable(float* dir, float minEta, float maxEta, int kind)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int size = kTableSize;
  if (idx >= size * size * size) return;
  const int i = idx % size, j = (idx / size) % size, k = idx / (size * size);
  const float cosThetaO = (float)i / (size - 1);
  const float eta = lerpf(minEta, maxEta, (float)j / (size - 1));
  const float roughness = (float)k / (size - 1);
  GGX mf;
  mf.ax = mf.ay = roughnessToAlpha(roughness);
  const int n = 32;
  float sum = 0.f;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
    {
      const float sx = sampleCoord(a, n), sy = sampleCoord(b, n);
      sum += kind == 0 ? dielSample(cosThetaO, eta, mf, sx, sy) : reflSample(cosThetaO, eta, mf, sx, sy);
    }
  dir[idx] = fminf(sum / (float)(n * n), 1.f);
}

// integrateAvg: one thread per row of `size` directional values.
// MicrofacetSheenAlbedo::integrate (bsdf/albedo.h:287-330): 32 x 32 midpoint samples of the
// uniformly sampled sheen lobe per (cos, roughness) entry.
__global__ void kSheenTable(float* dir)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kTableSize * kTableSize) return;
  const int i = idx % kTableSize, j = idx / kTableSize;
  const float cosThetaO = fmaxf((float)i / (float)(kTableSize - 1), 1e-6f);
  const float roughness = (float)j / (float)(kTableSize - 1);
  SheenDist mf;
  mf.r = roughnessToAlpha(roughness);
  const f3 wo = mk(sqrtf(fmaxf(1.f - cosThetaO * cosThetaO, 0.f)), 0.f, cosThetaO);
  const int n = 32;
  float sum = 0.f;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
    {
      const float sx = sampleCoord(a, n), sy = sampleCoord(b, n);
      const float cosThetaI = sy;
      const float sinThetaI = sqrtf(fmaxf(1.f - sy * sy, 0.f));
      float sinPhi, cosPhi;
      sincospif(2.f * sx, &sinPhi, &cosPhi);
      const f3 wi = mk(cosPhi * sinThetaI, sinPhi * sinThetaI, cosThetaI);
      const f3 wh = normalize(wo + wi);
      const float D = mf.eval(wh.z);
      const float G = mf.G2(cosThetaO, cosThetaI);
      sum += D * G * (2.f * kPi) / (4.f * cosThetaO);
    }
  dir[idx] = fminf(sum / (float)(n * n), 1.f);
}

__global__ void kAvg(const float* dir, float* avg, int rows, int size)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const float* f = dir + (size_t)r * size;
  const int n = 1024 + 1;
  float sum = 0.f;
  for (int i = 0; i < n; ++i)
  {
    const float cosThetaO = (float)i / (n - 1);
    sum += interp1D(f, size, cosThetaO * (size - 1)) * cosThetaO * ((i == 0 || i == n - 1) ? 0.5f : 1.f);
  }
  avg[r] = fminf(2.f * (sum / (n - 1)), 1.f);
}

} // namespace

cudaError_t buildAlbedoTables(DevTables& t, float** storage)
{
  const int g2 = kGgxTableSize * kGgxTableSize;
  const int t3 = kTableSize * kTableSize * kTableSize;
  const int t2 = kTableSize * kTableSize;
  const size_t total = g2 + kGgxTableSize + 3 * (t3 + t2) + (t3 + t2) + t3 * kTableSize + t2;
  float* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, total * sizeof(float));
  if (e != cudaSuccess) return e;
  e = cudaMemset(buf, 0, total * sizeof(float));
  if (e != cudaSuccess) return e;
  float* p = buf;
  auto take = [&](size_t n) {
    float* q = p;
    p += n;
    return q;
  };
  float* ggxDir = take(g2);
  float* ggxAvg = take(kGgxTableSize);
  float* dielEtaDir = take(t3);
  float* dielEtaAvg = take(t2);
  float* dielRcpDir = take(t3);
  float* dielRcpAvg = take(t2);
  float* reflDir = take(t3);
  float* reflAvg = take(t2);
  float* reflEcDir = take(t3);
  float* reflEcAvg = take(t2);
  float* condEcDir = take((size_t)t3 * kTableSize);
  float* sheenDir = take(t2);
  kGgxTable<<<(g2 + 127) / 128, 128>>>(ggxDir);
  kAvg<<<1, kGgxTableSize>>>(ggxDir, ggxAvg, kGgxTableSize, kGgxTableSize);
  // The eta <= 1 axes run over [rcp(maxIor), rcp(minIor)] with the reference CPU build's rcp
  // (bsdf/albedo_tables.cpp:96-97,111-112), which puts the last slice at 0.99999994 on x86-64.
  const float minIor = 1.f, maxIor = 3.f;
  t.etaLo = hostRcp(maxIor);
  t.etaHi = hostRcp(minIor);
  kDielTable<<<(t3 + 127) / 128, 128>>>(dielEtaDir, t.etaLo, t.etaHi, 0);
  kAvg<<<(t2 + 127) / 128, 128>>>(dielEtaDir, dielEtaAvg, t2, kTableSize);
  kDielTable<<<(t3 + 127) / 128, 128>>>(dielRcpDir, minIor, maxIor, 0);
  kAvg<<<(t2 + 127) / 128, 128>>>(dielRcpDir, dielRcpAvg, t2, kTableSize);
  kDielTable<<<(t3 + 127) / 128, 128>>>(reflDir, t.etaLo, t.etaHi, 1);
  kAvg<<<(t2 + 127) / 128, 128>>>(reflDir, reflAvg, t2, kTableSize);
  kSheenTable<<<(t2 + 127) / 128, 128>>>(sheenDir);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return e;
  t.ggxDir = ggxDir;
  t.ggxAvg = ggxAvg;
  t.dielEtaDir = dielEtaDir;
  t.dielEtaAvg = dielEtaAvg;
  t.dielRcpDir = dielRcpDir;
  t.dielRcpAvg = dielRcpAvg;
  t.reflDir = reflDir;
  t.reflAvg = reflAvg;
  t.reflEcDir = reflEcDir;
  t.reflEcAvg = reflEcAvg;
  t.condEcDir = condEcDir;
  t.sheenDir = sheenDir;
  *storage = buf;
  return cudaSuccess;
}

} // namespace prt
