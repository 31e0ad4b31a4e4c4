// Owen-scrambled, shuffled Sobol sampler (Burley 2020) on the device, bit-exact with the
// reference's SIMD sampler (sampling/sobol_burley_sampler_simd.h:36-84) that the stream
// path tracer uses.
//
// The integer pipeline follows sampling/sobol_burley.h: hashHP (:32-42), reversedBitOwen
// (:53-61), the dimension-0/1 fast paths and the direction-table XOR (:150-190), and the
// 1D/2D/3D shuffles with their seed constants (:223-297). The per-pixel scramble is
// murmurHash3Finalize(murmurHash3Mix(seed, pixelId)) (math/hash.h:13-42).
//
// The final uint -> float conversion follows the reference's default (AVX2) build, where a
// vuint8 is converted as float(x & 0x7fffffff) + (x >> 31 ? 2^31 : 0)
// (math/simd/vfloat8_avx2.h:171-178) and then scaled by 1/4294967808
// (math/simd.h:76-84). That double rounding differs from a correctly rounded conversion in
// rare ties, so it is reproduced here operation for operation.
#pragma once

#include "prt_math.cuh"

namespace prt {

// Direction numbers of Sobol dimension 2 in the reversed-bit form the Burley sampler uses
// (sampling/sobol_burley.cpp:9 stores dimensions 0-3 as a table). Dimension 0 is the
// identity and dimension 1 has a closed form, so only dimension 2 is needed. It is generated
// here from the Sobol recurrence for the primitive polynomial x^2 + x + 1 with initial
// values m1 = 1, m2 = 3:  m_k = 2 m_{k-1} ^ 4 m_{k-2} ^ m_{k-2},  entry k-1 = reverse_k(m_k).
struct SobolDirections
{
  uint32_t v[32];
};

constexpr uint32_t reverseLowBits(uint32_t x, int n)
{
  uint32_t r = 0;
  for (int i = 0; i < n; ++i)
    if ((x >> i) & 1u) r |= 1u << (n - 1 - i);
  return r;
}

constexpr SobolDirections makeSobolDim2()
{
  SobolDirections t{};
  uint32_t m[33] = {};
  m[1] = 1u;
  m[2] = 3u;
  for (int k = 3; k <= 32; ++k)
    m[k] = (2u * m[k - 1]) ^ (4u * m[k - 2]) ^ m[k - 2];
  for (int k = 1; k <= 32; ++k)
    t.v[k - 1] = reverseLowBits(m[k], k);
  return t;
}

__device__ __constant__ static const SobolDirections kSobolDim2 = makeSobolDim2();

PRT_D uint32_t hashHP(uint32_t i)
{
  i ^= i >> 16;
  i *= 0x21f0aaadu;
  i ^= i >> 15;
  i *= 0xd35a2d97u;
  i ^= i >> 15;
  return i ^ 0xe6fe3bebu;
}

PRT_D uint32_t reversedBitOwen(uint32_t n, uint32_t seed)
{
  n ^= n * 0x3d20adeau;
  n += seed;
  n *= (seed >> 16) | 1u;
  n ^= n * 0x05526c56u;
  n ^= n * 0x53a22864u;
  return n;
}

PRT_D uint32_t murmurMix(uint32_t hash, uint32_t k)
{
  k *= 0xcc9e2d51u;
  k = (k << 15) | (k >> 17);
  k *= 0x1b873593u;
  hash ^= k;
  hash = ((hash << 13) | (hash >> 19)) * 5u + 0xe6546b64u;
  return hash;
}

PRT_D uint32_t murmurFinalize(uint32_t hash)
{
  hash ^= hash >> 16;
  hash *= 0x85ebca6bu;
  hash ^= hash >> 13;
  hash *= 0xc2b2ae35u;
  hash ^= hash >> 16;
  return hash;
}

// uint -> [0,1) float exactly as the AVX2 build of the reference computes it.
PRT_D float toUnormExclAvx2(uint32_t x)
{
  const float lo = __uint2float_rn(x & 0x7fffffffu);
  const float hi = (x & 0x80000000u) ? 2147483648.0f : 0.0f;
  return __fmul_rn(__fadd_rn(lo, hi), 1.0f / 4294967808.0f);
}

// One dimension (0, 1 or 2) of the scrambled Sobol point with reversed-bit index.
PRT_D float sobolBurley(uint32_t revBitIndex, int dimension, uint32_t scrambleSeed)
{
  uint32_t result;
  if (dimension == 0)
  {
    result = __brev(revBitIndex);
  }
  else if (dimension == 1)
  {
    uint32_t v = revBitIndex;
    v ^= v << 16;
    v ^= (v & 0x00FF00FFu) << 8;
    v ^= (v & 0x0F0F0F0Fu) << 4;
    v ^= (v & 0x33333333u) << 2;
    v ^= (v & 0x55555555u) << 1;
    result = __brev(v);
  }
  else
  {
    // XOR of the direction numbers of the set bits, most significant bit first.
    result = 0u;
    uint32_t bits = revBitIndex;
    while (bits != 0u)
    {
      const int j = __clz(bits);
      result ^= kSobolDim2.v[j];
      bits &= ~(0x80000000u >> j);
    }
  }
  result = __brev(reversedBitOwen(result, scrambleSeed));
  return toUnormExclAvx2(result);
}

// Per-path sampler state: SobolBurleySamplerSimd<false>::State.
struct SobolState
{
  uint32_t index;
  uint32_t scramble;
};

PRT_D SobolState sobolSetSample(uint32_t seed, uint32_t sampleIndex, uint32_t pixelId)
{
  SobolState s;
  s.index = sampleIndex;
  s.scramble = murmurFinalize(murmurMix(seed, pixelId));
  return s;
}

PRT_D float sobolGet1D(const SobolState& st, uint32_t dim)
{
  const uint32_t seed = st.scramble ^ hashHP(dim);
  const uint32_t index = reversedBitOwen(__brev(st.index), seed ^ 0xbff95bfeu);
  return sobolBurley(index, 0, seed ^ 0x635c77bdu);
}

PRT_D void sobolGet2D(const SobolState& st, uint32_t dimSet, float& x, float& y)
{
  const uint32_t seed = st.scramble ^ hashHP(dimSet);
  const uint32_t index = reversedBitOwen(__brev(st.index), seed ^ 0xf8ade99au);
  x = sobolBurley(index, 0, seed ^ 0xe0aaaf76u);
  y = sobolBurley(index, 1, seed ^ 0x94964d4eu);
}

PRT_D void sobolGet3D(const SobolState& st, uint32_t dimSet, float& x, float& y, float& z)
{
  const uint32_t seed = st.scramble ^ hashHP(dimSet);
  const uint32_t index = reversedBitOwen(__brev(st.index), seed ^ 0xcaa726acu);
  x = sobolBurley(index, 0, seed ^ 0x9e78e391u);
  y = sobolBurley(index, 1, seed ^ 0x67c33241u);
  z = sobolBurley(index, 2, seed ^ 0x78c395c5u);
}

} // namespace prt
