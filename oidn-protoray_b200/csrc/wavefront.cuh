// Device helpers shared by the wavefront kernels (integrator.cu) and the path-replay adjoint
// (adjoint.cu): path flags, sample dimensions, pixel order, camera rays, radiance clamp, MIS.
#pragma once
#include "runtime.h"
#include "sobol_burley.cuh"
#include "traverse.cuh"
#include "bsdf.cuh"

namespace prt {

// Path flags kept in the high bits of pixelId (render/path_renderer_stream.h:69-79).
constexpr uint32_t kPixelIdMask = 0x0fff0fffu;
constexpr uint32_t kPathAov1Flag = 0x20000000u;
constexpr uint32_t kPathAov2Flag = 0x10000000u;
constexpr uint32_t kShadowFinish = 0x80000000u;

// Sample dimensions (render/integrator.h:52-56, render/path_renderer_stream.h:24-33).
constexpr uint32_t kDimPixel = 0, kDimLens = 2, kDimBase = 4;
constexpr uint32_t kDimBsdf = 0, kDimLight = 3, kDimTerminate = 6, kDimBounce = 7;

PRT_D int laneId() { return threadIdx.x & 31; }

// Appends `pred` lanes of the calling (converged) warp to a queue; returns the slot or -1.
PRT_D int warpAppend(int* counter, bool pred)
{
  const unsigned active = __activemask();
  const unsigned ballot = __ballot_sync(active, pred);
  if (ballot == 0u) return -1;
  const int leader = __ffs(ballot) - 1;
  int base = 0;
  if (laneId() == leader) base = atomicAdd(counter, __popc(ballot));
  base = __shfl_sync(active, base, leader);
  return pred ? base + __popc(ballot & ((1u << laneId()) - 1u)) : -1;
}

// Pixel of a slot within one sample: 8x8 Morton blocks, blocks in row-major order.
PRT_D void pixelOf(int idx, int width, int& x, int& y)
{
  const int block = idx >> 6, local = idx & 63;
  const int bw = width >> 3;
  const int bx = block % bw, by = block / bw;
  const int lx = (local & 1) | ((local >> 1) & 2) | ((local >> 2) & 4);
  const int ly = ((local >> 1) & 1) | ((local >> 2) & 2) | ((local >> 3) & 4);
  x = bx * 8 + lx;
  y = by * 8 + ly;
}

PRT_D int slotOfPixel(int x, int y, int width)
{
  const int block = (y >> 3) * (width >> 3) + (x >> 3);
  const int lx = x & 7, ly = y & 7;
  const int local = (lx & 1) | ((ly & 1) << 1) | ((lx & 2) << 1) | ((ly & 2) << 2) | ((lx & 4) << 2) | ((ly & 4) << 3);
  return block * 64 + local;
}

// IntegratorBase::clampL (render/integrator.h:28-46).
PRT_D f3 clampL(f3 L, float maxRadiance)
{
  f3 c = mk(0.f < L.x ? L.x : 0.f, 0.f < L.y ? L.y : 0.f, 0.f < L.z ? L.z : 0.f);
  const float y = luminance(c);
  if (y > maxRadiance) c *= maxRadiance * (1.f / y);
  return c;
}

// MIS power heuristic (render/path_renderer_stream.h:1077-1080).
PRT_D float misWeight(float a, float b) { return sqr(a) * rcpSafe(sqr(a) + sqr(b)); }

// PinholeCamera::getRay (camera/pinhole_camera.h:78-83).
PRT_D void cameraRay(const DevCamera& cam, float ix, float iy, f3& org, f3& dir, float& tnear)
{
  const f3 d = mk(cam.imageO[0], cam.imageO[1], cam.imageO[2]) + ix * mk(cam.imageDx[0], cam.imageDx[1], cam.imageDx[2]) +
               iy * mk(cam.imageDy[0], cam.imageDy[1], cam.imageDy[2]);
  const float len = sqrtf(lengthSqr(d));
  dir = d * (1.f / len);
  org = mk(cam.org[0], cam.org[1], cam.org[2]);
  tnear = cam.nearClip * len;
}

} // namespace prt
