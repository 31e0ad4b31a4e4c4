/* Test infrastructure: a plain-C restatement of the reference's Sobol-Burley sampler, the
 * oracle for the integer part of the path (used by the CPU tests; never linked into the
 * product).
 *
 * Follows sampling/sobol_burley.h (hashHP :32-42, reversedBitOwen :53-61, sobolBurley
 * :104-190, sobolBurleySample1D/2D/3D :223-297), math/hash.h:13-42 (MurmurHash3 mix and
 * finalizer) and the AVX2 uint -> float conversion of math/simd/vfloat8_avx2.h:171-178
 * followed by the 1/4294967808 scale of math/simd.h:76-84. Dimension 2's direction numbers
 * come from the Sobol recurrence for x^2 + x + 1 (m1 = 1, m2 = 3).
 */
#include "prt_oracle.h"

static uint32_t rev32(uint32_t x)
{
  uint32_t r = 0;
  for (int i = 0; i < 32; ++i)
    if (x & (1u << i)) r |= 1u << (31 - i);
  return r;
}

static uint32_t hash_hp(uint32_t i)
{
  i ^= i >> 16;
  i *= 0x21f0aaadu;
  i ^= i >> 15;
  i *= 0xd35a2d97u;
  i ^= i >> 15;
  return i ^ 0xe6fe3bebu;
}

static uint32_t owen(uint32_t n, uint32_t seed)
{
  n ^= n * 0x3d20adeau;
  n += seed;
  n *= (seed >> 16) | 1u;
  n ^= n * 0x05526c56u;
  n ^= n * 0x53a22864u;
  return n;
}

static uint32_t dim2_table[32];
static int dim2_ready = 0;

static void init_dim2(void)
{
  uint32_t m[33];
  m[1] = 1;
  m[2] = 3;
  for (int k = 3; k <= 32; ++k) m[k] = (2u * m[k - 1]) ^ (4u * m[k - 2]) ^ m[k - 2];
  for (int k = 1; k <= 32; ++k)
  {
    uint32_t r = 0;
    for (int i = 0; i < k; ++i)
      if ((m[k] >> i) & 1u) r |= 1u << (k - 1 - i);
    dim2_table[k - 1] = r;
  }
  dim2_ready = 1;
}

static float to_unorm_avx2(uint32_t x)
{
  volatile float lo = (float)(int32_t)(x & 0x7fffffffu);
  volatile float hi = (x & 0x80000000u) ? 2147483648.0f : 0.0f;
  volatile float sum = lo + hi;
  return sum * (1.0f / 4294967808.0f);
}

static float sobol_dim(uint32_t rev_index, int dim, uint32_t seed)
{
  uint32_t result = 0;
  if (dim == 0)
    result = rev32(rev_index);
  else if (dim == 1)
  {
    uint32_t v = rev_index;
    v ^= v << 16;
    v ^= (v & 0x00FF00FFu) << 8;
    v ^= (v & 0x0F0F0F0Fu) << 4;
    v ^= (v & 0x33333333u) << 2;
    v ^= (v & 0x55555555u) << 1;
    result = rev32(v);
  }
  else
  {
    for (int i = 0; i < 32; ++i)
      if (rev_index & (0x80000000u >> i)) result ^= dim2_table[i];
  }
  return to_unorm_avx2(rev32(owen(result, seed)));
}

static uint32_t murmur_mix(uint32_t hash, uint32_t k)
{
  k *= 0xcc9e2d51u;
  k = (k << 15) | (k >> 17);
  k *= 0x1b873593u;
  hash ^= k;
  return ((hash << 13) | (hash >> 19)) * 5u + 0xe6546b64u;
}

static uint32_t murmur_fin(uint32_t h)
{
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

void prto_sobol(uint32_t seed, int64_t n, const uint32_t* sample_index, const uint32_t* pixel_id,
                const uint32_t* dim_set, int dims, float* out)
{
  static const uint32_t shuffle[4] = {0, 0xbff95bfeu, 0xf8ade99au, 0xcaa726acu};
  static const uint32_t scr[4][3] = {{0, 0, 0},
                                     {0x635c77bdu, 0, 0},
                                     {0xe0aaaf76u, 0x94964d4eu, 0},
                                     {0x9e78e391u, 0x67c33241u, 0x78c395c5u}};
  if (!dim2_ready) init_dim2();
  for (int64_t i = 0; i < n; ++i)
  {
    const uint32_t scramble = murmur_fin(murmur_mix(seed, pixel_id[i]));
    const uint32_t s = scramble ^ hash_hp(dim_set[i]);
    const uint32_t index = owen(rev32(sample_index[i]), s ^ shuffle[dims]);
    for (int d = 0; d < dims; ++d) out[dims * i + d] = sobol_dim(index, d, s ^ scr[dims][d]);
  }
}
