// C++ host wrapper of the B200 render device, mirroring the reference's render-Device API
// (render/device.h:56-114) method for method, over the C ABI in include/prt_cuda.h.
//
// Errors come back as the exception types the reference's DeviceCpu throws:
// std::invalid_argument (PRT_ERR_INVALID_ARG), std::logic_error (PRT_ERR_LOGIC, e.g. an image
// size not divisible by the 32x8 tile, render/path_renderer_stream.h:109-112), and
// std::runtime_error for CUDA, memory, state and device-abort failures.
//
// Header-only; link with libprt_cuda.so. A reference-side adapter derives the reference's
// prt::Device and forwards each virtual to the same entry points, so that `-dev cuda` selects it.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/prt_cuda.h"

namespace prt_cuda {

class DeviceCuda
{
public:
  explicit DeviceCuda(int deviceOrdinal = 0)
  {
    if (prt_cuda_create(deviceOrdinal, &ctx_) != PRT_OK)
      throw std::runtime_error("prt_cuda_create failed: no usable CUDA device");
  }

  ~DeviceCuda()
  {
    if (ctx_) prt_cuda_destroy(ctx_);
  }

  DeviceCuda(const DeviceCuda&) = delete;
  DeviceCuda& operator=(const DeviceCuda&) = delete;

  std::string getInfo() const { return "NVIDIA B200 (sm_100a) wavefront path tracer"; }

  // Device::initScene + initLights (render/device_cpu.cpp:96-107).
  void initScene(const prt_scene_desc& scene) { check(prt_cuda_scene_upload(ctx_, &scene)); }

  // Device::initRenderer for type "pathStream" / sampler "sobolBurley" (render/device_cpu.cpp:32-46).
  void initRenderer(int maxDepth = 100, int rrDepth = 8, float minWeight = 1e-4f,
                    float maxRadiance = 3.402823466e38f, int type = PRT_RENDERER_PATH, int samples = 16)
  {
    const prt_renderer_desc r{maxDepth, rrDepth, minWeight, maxRadiance, type, samples};
    check(prt_cuda_renderer(ctx_, &r));
  }

  void initSampler(uint32_t seed) { check(prt_cuda_init_sampler(ctx_, seed)); }

  void initCamera(const prt_camera_desc& camera) { check(prt_cuda_camera(ctx_, &camera)); }

  // Device::initFrame (render/device_cpu.cpp:178-232).
  void initFrame(int width, int height, int aovMask = 0)
  {
    check(prt_cuda_frame(ctx_, width, height, aovMask));
    width_ = width;
    height_ = height;
  }

  void clearFrame() { check(prt_cuda_clear(ctx_)); }

  // Device::render: one sample per pixel per call in the reference; spp samples here.
  prt_render_stats render(int spp = 1)
  {
    prt_render_stats st{};
    check(prt_cuda_render(ctx_, spp, &st));
    return st;
  }

  // Device::blitFrame (render/device_cpu.cpp:316-366): width*height RGB floats.
  std::vector<float> blitFrame(int aov = PRT_BLIT_HDR)
  {
    std::vector<float> out((size_t)width_ * height_ * 3);
    check(prt_cuda_blit(ctx_, aov, out.data()));
    return out;
  }

  void blitFrame(int aov, float* dst) { check(prt_cuda_blit(ctx_, aov, dst)); }

  prt_context* handle() const { return ctx_; }

private:
  void check(int rc) const
  {
    if (rc == PRT_OK) return;
    const std::string msg = prt_cuda_last_error(ctx_);
    if (rc == PRT_ERR_INVALID_ARG) throw std::invalid_argument(msg);
    if (rc == PRT_ERR_LOGIC) throw std::logic_error(msg);
    throw std::runtime_error("prt_cuda error " + std::to_string(rc) + ": " + msg);
  }

  prt_context* ctx_ = nullptr;
  int width_ = 0, height_ = 0;
};

} // namespace prt_cuda
