// Host runtime of the B200 render device: the context behind the C ABI and the kernel
// launchers it drives. Shared by device.cu (C ABI, scene upload) and integrator.cu (kernels).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "bvh8.h"
#include "device_scene.h"

namespace prt {

// Device memory block owned by the context.
struct DevBuf
{
  void* ptr = nullptr;
  size_t bytes = 0;
};

// Queue entries of extended paths: the path slot in bits 0-28 and the octant of the new ray's
// direction (bit k set when component k is negative) in bits 29-31. Readers mask the slot.
constexpr uint32_t kQueueOctShift = 29;
constexpr uint32_t kQueuePathMask = (1u << kQueueOctShift) - 1u;

// Path state of one wave, structure of arrays indexed by path slot.
struct PathState
{
  int64_t capacity = 0;
  float4* rayO = nullptr;   // origin, near
  float4* rayD = nullptr;   // direction, far
  float4* hit = nullptr;    // t, u, v, triangle id (int bits)
  float4* thr = nullptr;    // throughput, lastBsdfPdf
  float4* rad = nullptr;    // radiance L, lastBsdfType (int bits)
  uint4* info = nullptr;    // pixelId | path flags, sample index, medium id, -
  float4* shO = nullptr;    // shadow rays: origin, near
  float4* shD = nullptr;    // direction, far
  float4* shL = nullptr;    // unoccluded contribution, path slot | finish flag (int bits)
  float4* out = nullptr;    // final radiance per path (w = 1 when written)
  float4* aovA = nullptr;   // first-hit albedo per path (w = 1 when written)
  float4* aovN = nullptr;   // first-hit normal per path
  // SH AOV (PRT_AOV_SH), render/path_renderer_stream.h:46-52: the radiance gathered after the
  // first hit (xyz) with the irradiance scale pi / cos of the first bounce (w); the first
  // bounce's direction; the first hit's unoccluded direct light scaled to irradiance and its
  // direction; the path's SH sample (3 float4 per path: the 4 coefficients x RGB); the
  // irradiance scale of each first-hit shadow ray (per shadow-ray slot).
  float4* sphL = nullptr;
  float4* sphWi = nullptr;
  float4* sphDirL = nullptr;
  float4* sphDirWi = nullptr;
  float4* sphOut = nullptr;
  float* sphDirScale = nullptr;
  int* queue[2] = {nullptr, nullptr};
  int* classQueues = nullptr;  // kShadeClasses queues of `capacity` entries each
  int* counters = nullptr;  // per bounce: input and shadow counts, then the work counters
  int* octBins = nullptr;   // ray binning: 8 octant counts, then 8 octant cursors (frame form)
  unsigned long long* travCounts = nullptr;  // closest nodes, closest tris, shadow nodes, shadow tris
  uint32_t* err = nullptr;
};

// One frame of a batch render: its scene, camera, renderer settings, frame and range of
// work items (pixel-samples) in the batch's global work order.
struct BatchItem
{
  DevScene sc;
  DevCamera cam;
  DevRenderer rd;
  int width, height, pixelCount, aovMask;
  long long workBase;   // first work item of this frame
  long long workCount;  // pixelCount * spp
  float4* accum;        // sum rgb + weight per pixel
  float4* accA;         // first-hit albedo sums (aovMask != 0)
  float4* accN;         // first-hit normal sums
  AdjointView adj;      // gradient targets of the batch adjoint (prt_cuda_batch_adjoint)
};

// Counter block of one batch iteration (ints): [0] paths to trace, [1..kShadeClasses] paths
// per shading class, [kBatchCntShadow] shadow rays, then the two work counters.
constexpr int kBatchCntShadow = 1 + kShadeClasses;
constexpr int kBatchCntStride = 16;

// Device-side control block of a batch render (kBatchStep advances it every iteration).
struct BatchCtl
{
  long long workNext, workTotal;
  long long regenBase;
  int regenCount, regenOffset;
  int counts[2][kBatchCntStride];
  int freeCount[2];
  int done;
  int iterations;
  unsigned long long rays[2];  // closest-hit rays, shadow rays
};

// Host state of a batch render (prt_batch): the frames, their uploaded scenes, a shared
// path pool with its queues and free lists, and the captured bounce-loop graph.
struct BatchState
{
  std::vector<DevBuf> bufs;        // scene buffers and accumulation planes of every item
  std::vector<BatchItem> items;    // host copy of the items (device pointers inside)
  BatchItem* dItems = nullptr;
  long long workTotal = 0;
  int maxDepth = 0;
  int bvhDepth = 0;                // deepest BVH8 of the items (wide levels)
  bool anyAov = false;
  PathState ps;                    // path pool; ps.err is the context's error flag
  BatchCtl* ctl = nullptr;
  int* freeList[2] = {nullptr, nullptr};
  cudaGraphExec_t exec = nullptr;  // kGraphIterations bounce iterations
  int graphKernels = 0;
  // Forward render: per work item (pixel-sample) the clamped radiance and the first-hit albedo and
  // normal (the latter two when an item has AOVs), summed per pixel in sample order at the end.
  float4* workOut = nullptr;
  float4* workA = nullptr;
  float4* workN = nullptr;
  // Differentiable batches: radiance per work item (float4) and the replay graph.
  float4* pathL = nullptr;
  cudaGraphExec_t execReplay = nullptr;
  int graphKernelsReplay = 0;
  std::vector<std::vector<DevMaterial>> itemMaterials;  // host copies per item
  std::vector<std::vector<DevTexture>> itemTextures;
};

struct Context
{
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string lastError;
  int smCount = 0;
  std::vector<DevBuf> sceneBufs;  // freed on re-upload
  std::vector<DevBuf> envBufs;    // environment lights and the light CDF, replaced by prt_cuda_scene_lights
  std::vector<float> areaLightPowerHost;  // area-light powers, the head of the light CDF
  float sceneRadius = 0.f;        // half the diagonal of the scene bounds (render/scene.cpp:367)
  float boundsLo[3] = {0.f, 0.f, 0.f}, boundsHi[3] = {0.f, 0.f, 0.f};
  DevScene scene{};
  bool hasScene = false;
  Bvh8 bvh;                       // host copy of a host-built tree
  int bvhBuilder = 0;             // PRT_BVH_HOST / PRT_BVH_DEVICE of the uploaded scene
  double bvhBuildMs = 0.0;
  int64_t bvhNodes = 0, bvhTris = 0;
  int bvhDepth = 0, bvhTop = 1, bvhIterations = 0;
  std::vector<int> meshTriOffsetHost;
  std::vector<DevMaterial> materialsHost;  // host copies of the uploaded material records
  std::vector<DevTexture> texturesHost;    // device pointers and sizes of the scene's textures
  DevRenderer renderer{100, 8, 1e-4f, 3.402823466e38f, 0u, 0, 16, 0};
  bool hasRenderer = false;
  DevCamera camera{};
  bool hasCamera = false;
  int width = 0, height = 0, aovMask = 0;
  bool aovSh = false;             // PRT_AOV_SH: the SH planes of the frame and the path state
  float* accum = nullptr;         // sum rgb + weight per pixel (float4)
  float* accumA = nullptr;        // first-hit albedo sums
  float* accumN = nullptr;        // first-hit normal sums
  float* accumC = nullptr;        // checkpoint: the sums at the last power-of-two sample count
  float* accum2 = nullptr;        // squared samples (PRT_AOV_HDR_VAR)
  float* accumSH = nullptr;       // SH coefficient sums, 4 planes of float4 (PRT_AOV_SH)
  double* errPartials = nullptr;  // per-block partial sums of the frame error
  int64_t accumCount = 0;         // samples accumulated since the last clear
  int toneType = 0;               // PRT_TONE_*
  float toneExposure = 1.f, toneInvWhite2 = 0.f;
  uint32_t sampleIndex = 0;
  PathState ps;
  int waveSamples = 0;            // samples per pixel per wave
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevTables tables{};             // energy-compensation tables (albedo.cu)
  float* tableStorage = nullptr;
  int profileFlags = 0;
  int traceBlocks = 8;            // launch tuning (prt_tuning)
  int shadeBlocks = 8;
  int64_t wavePaths = 128ll << 20;
  int topStage = 0;               // stage the top BVH levels in shared memory (frame form)
  int rayBins = 0;                // group each bounce's extended rays by direction octant (frame form)
  int traceStack = 12;            // smallest traversal stack to try: 12 (shared memory), 24 or 48 (local)
  DevMaterial whiteMaterial{};    // irradiance mode: the first hit's material (white Principled)
  DevMaterial* whiteMaterialDev = nullptr;  // its device copy
  int whiteClass = 0;             // its shading class
  // Device buffers that stage host memory passed to an entry point (one per buffer argument of
  // a call, reused by later calls and grown when a call needs more; freed with the context).
  std::vector<DevBuf> stage;
  int stageNext = 0;              // slots in use by the current call
};

// Per-call statistics gathered by renderSamples.
struct RenderCounters
{
  int64_t closestRays = 0, shadowRays = 0, launches = 0, traceLaunches = 0;
  double traceMs = 0.0, shadowMs = 0.0, shadeMs = 0.0;
  unsigned long long trav[4] = {0, 0, 0, 0};
};

// Kernel launchers (integrator.cu). All are asynchronous on ctx.stream.
cudaError_t launchSobol(Context& ctx, int64_t n, const uint32_t* si, const uint32_t* pid, const uint32_t* dims,
                        int ndim, float* out);
cudaError_t launchTrace(Context& ctx, int64_t n, const float* rays, int32_t* triOut, float* t, float* u,
                        float* v);
cudaError_t launchOccluded(Context& ctx, int64_t n, const float* rays, int32_t* occ);
cudaError_t launchPrimary(Context& ctx, uint32_t sampleIndex, float* raysOut, int32_t* triOut, float* t);
// Renders samples [ctx.sampleIndex, ctx.sampleIndex + spp) and accumulates them; returns the
// number of closest + shadow rays traced.
cudaError_t renderSamples(Context& ctx, int spp, RenderCounters& rc);
cudaError_t launchBlit(Context& ctx, int aov, float* dst);
// Renders every item of a batch to completion (path regeneration over one shared path pool,
// bounce loop replayed as a CUDA graph) into the items' accumulation planes.
cudaError_t renderBatch(Context& ctx, BatchState& b, RenderCounters& rc);
// Path-replay adjoint of the last renderBatch of a differentiable batch: scatters each item's
// gradients into the targets of its BatchItem::adj (set on the device before the call).
cudaError_t replayBatch(Context& ctx, BatchState& b, RenderCounters& rc);
cudaError_t launchBlitPlane(Context& ctx, const float4* plane, int n, float* dst);
// PRT_BLIT_HDR_VAR and PRT_BLIT_LDR (film post-step).
cudaError_t launchBlitVariance(Context& ctx, float* dst);
cudaError_t launchBlitLdr(Context& ctx, uint32_t* dst);
cudaError_t launchBlitLdrRgb(Context& ctx, float* dst);
// Frame error against the checkpoint (Device::getFrameError).
cudaError_t frameError(Context& ctx, double& error);
// Path-replay adjoint (adjoint.cu): dLoss/d(texel) of every scene texture and dLoss/d(specular
// roughness) of every material for the image gradient dLdI (W*H*3, device memory).
cudaError_t launchAdjoint(Context& ctx, uint32_t firstSample, int spp, const float* dLdI, float* gradTex,
                          float* gradRough, float roughnessStep, RenderCounters& rc);
// Copies a caller-order (row 0 at the top) RGB image into a device texture (row 0 at the bottom).
cudaError_t launchTextureUpdate(Context& ctx, const DevTexture& t, const float* rgb);
cudaError_t launchClear(Context& ctx);
cudaError_t launchBsdfQuery(Context& ctx, const DevMaterial& m, int mediumId, int64_t n, const float* tuples, float* out);
cudaError_t launchMicrofacetQuery(Context& ctx, int distribution, int64_t n, const float* in, float* out);
// Builds the BSDF energy-compensation tables on the current device (albedo.cu).
cudaError_t buildAlbedoTables(DevTables& t, float** storage);

} // namespace prt
