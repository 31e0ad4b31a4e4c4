// Texture updates for inverse rendering: copies a caller-order image (row 0 at the top) into a
// device texture, which stores rows bottom-up (image/image_texture.h:377-392 order).
#include "runtime.h"

#include <algorithm>

namespace prt {

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

cudaError_t launchTextureUpdate(Context& ctx, const DevTexture& t, const float* rgb)
{
  const int64_t n = (int64_t)t.width * t.height;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx.smCount * 8));
  kTextureFromImage<<<blocks, 256, 0, ctx.stream>>>(rgb, const_cast<float*>(t.rgb), t.width, t.height);
  return cudaGetLastError();
}

} // namespace prt
