// Device math for the B200 path tracer: float3 helpers, the fixed-operation arithmetic the
// ray/triangle test must share with the host oracle, and small utilities.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define PRT_HD __host__ __device__ __forceinline__
#define PRT_D __device__ __forceinline__

namespace prt {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kPosMax = 3.402823466e38f;  // FLT_MAX: the reference's posMax (math/constants)

struct f3
{
  float x, y, z;
};

PRT_HD f3 mk(float x, float y, float z) { return f3{x, y, z}; }
PRT_HD f3 mk(float s) { return f3{s, s, s}; }
PRT_HD f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
PRT_HD f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
PRT_HD f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
PRT_HD f3 operator*(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
PRT_HD f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
PRT_HD f3 operator*(float s, f3 a) { return f3{a.x * s, a.y * s, a.z * s}; }
PRT_HD f3& operator+=(f3& a, f3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
PRT_HD f3& operator*=(f3& a, f3 b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
PRT_HD f3& operator*=(f3& a, float s) { a.x *= s; a.y *= s; a.z *= s; return a; }
PRT_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PRT_HD f3 cross(f3 a, f3 b) { return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
PRT_HD float lengthSqr(f3 a) { return dot(a, a); }
PRT_HD float reduceMax(f3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
PRT_HD f3 fmax3(f3 a, float s) { return f3{fmaxf(a.x, s), fmaxf(a.y, s), fmaxf(a.z, s)}; }
PRT_HD f3 fmin3(f3 a, float s) { return f3{fminf(a.x, s), fminf(a.y, s), fminf(a.z, s)}; }
PRT_HD f3 clamp01(f3 a) { return fmin3(fmax3(a, 0.f), 1.f); }
PRT_HD float clamp01(float a) { return fminf(fmaxf(a, 0.f), 1.f); }
PRT_HD float sqr(float a) { return a * a; }
PRT_HD f3 abs3(f3 a) { return f3{fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }

// Linear RGB luminance, image/color.h:19-22.
PRT_HD float luminance(f3 c) { return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z; }

PRT_D f3 normalize(f3 a) { return a * rsqrtf(lengthSqr(a)); }
// math/math.h:114-117: posMax instead of infinity for 0.
PRT_D float rcpSafe(float x) { return x == 0.f ? kPosMax : 1.f / x; }

// ---- fixed-operation arithmetic shared (by definition) with the host oracle ----------------
// The oracle's CPU intersector performs exactly these IEEE operations, so the GPU's
// ray/triangle results (hit, t, u, v) are bit-identical on the same inputs:
//   cross(a,b).x = fma(a.y, b.z, -(a.z*b.y)) and cyclic; dot(a,b) = fma(a.x,b.x, fma(a.y,b.y, a.z*b.z)).
PRT_D f3 crossFx(f3 a, f3 b)
{
  return f3{__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)),
            __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
            __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x))};
}

PRT_D float dotFx(f3 a, f3 b)
{
  return __fmaf_rn(a.x, b.x, __fmaf_rn(a.y, b.y, __fmul_rn(a.z, b.z)));
}

PRT_D f3 subFx(f3 a, f3 b)
{
  return f3{__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}

// Orthonormal frame around a unit normal, math/basis3.h:173-179.
struct Frame
{
  f3 U, V, N;
};

PRT_D void makeFrame(f3 N, f3& U, f3& V)
{
  const f3 U0 = mk(0.f, N.z, -N.y);
  const f3 U1 = mk(-N.z, 0.f, N.x);
  U = normalize(lengthSqr(U0) > lengthSqr(U1) ? U0 : U1);
  V = normalize(cross(N, U));
}

PRT_D f3 toWorld(const Frame& f, f3 v) { return v.x * f.U + v.y * f.V + v.z * f.N; }
PRT_D f3 toLocal(const Frame& f, f3 v) { return mk(dot(v, f.U), dot(v, f.V), dot(v, f.N)); }

// bsdf/optics.h:12-16.
PRT_D f3 reflect(f3 v, f3 n) { return 2.f * dot(v, n) * n - v; }

PRT_D f3 ld3(const float* p) { return f3{__ldg(p), __ldg(p + 1), __ldg(p + 2)}; }

} // namespace prt
