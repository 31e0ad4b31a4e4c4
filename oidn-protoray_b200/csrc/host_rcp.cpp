// Host reciprocal with the reference CPU build's rounding (see host_rcp.h).
#include "host_rcp.h"

#if defined(__x86_64__) || defined(_M_X64)
#include <immintrin.h>
#elif defined(__aarch64__)
#include <arm_neon.h>
#endif

namespace prt {

float hostRcp(float x)
{
#if defined(__x86_64__) || defined(_M_X64)
  // rcpss gives ~12 bits; one Newton step, each operation rounded to float as the scalar SSE
  // instructions round it.
  const __m128 v = _mm_set_ss(x);
  const __m128 r = _mm_rcp_ss(v);
  const __m128 twoR = _mm_add_ss(r, r);
  const __m128 r2x = _mm_mul_ss(_mm_mul_ss(r, r), v);
  return _mm_cvtss_f32(_mm_sub_ss(twoR, r2x));
#elif defined(__aarch64__)
  // frecpe gives ~8 bits; frecps computes 2 - r x, two steps.
  const float32x2_t v = vdup_n_f32(x);
  float32x2_t r = vrecpe_f32(v);
  for (int i = 0; i < 2; ++i) r = vmul_f32(vrecps_f32(v, r), r);
  return vget_lane_f32(r, 0);
#else
  return 1.f / x;
#endif
}

float hostFresnelDielectricAvg(float eta)
{
  const float r = hostRcp(eta);
  if (r >= 1.f) return (r - 1.f) / (4.08567f + 1.00071f * r);
  const float r2 = r * r;
  const float r3 = r2 * r;
  return 0.997118f + 0.1014f * r - 0.965241f * r2 - 0.130607f * r3;
}

} // namespace prt
