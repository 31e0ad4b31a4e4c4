// Wavefront path tracer kernels for sm_100a and their launchers.
//
// One wave = every pixel x a run of consecutive sample indices. Each kernel walks a queue of
// path slots; slot = (sample - firstSample) * pixelCount + tileMortonIndex(pixel), so the
// paths of one sample are contiguous and neighbouring slots are neighbouring pixels (8x8
// Morton blocks, like the reference's tile order, image/morton.h:33). Per bounce:
//   trace   : closest hit of every queued ray (persistent warps pull 32 rays at a time)
//   shade   : miss / area-light / surface shading, NEE shadow ray, BSDF sampling, Russian
//             roulette; extended paths and shadow rays are appended with warp-aggregated
//             atomics (the GPU form of RayStreamChannel::packSet, core/ray_stream.h:54)
//   shadow  : any-hit test; adds the NEE contribution and finishes paths that ended
// After the last bounce, accumulate() adds each pixel's samples in sample order into the FP32
// accumulation planes, reproducing AccumBuffer3f::addSerial (image/accum_buffer.h:439-486)
// without atomics, so the image does not depend on scheduling.
#include "wavefront.cuh"
#include "adjoint.cuh"
#include "../../include/prt_cuda.h"

#include <algorithm>
#include <cstddef>
#include <cstring>

namespace prt {

struct Launch
{
  DevScene sc;
  DevTables tab;
  DevCamera cam;
  DevRenderer rd;
  PathState ps;
  int width, height, pixelCount;
  uint32_t firstSample;
  int samples;       // samples in this wave
  int aovMask;
  // Batch form only (nullptr / 0 in the frame form).
  const BatchItem* items;
  int itemCount;
  BatchCtl* ctl;
  int* freeList[2];
  // Replay form of the adjoint only (frame form; the batch form keeps one per item).
  AdjointView adj;
  // Batch form: radiance of every work item (pixel-sample) when the batch is differentiable.
  float4* pathL;
  // Batch form, forward render: each work item's clamped radiance (w = 1 once written) and its
  // first-hit albedo and normal (w = 1 where set), summed per pixel by kBatchAccumulate.
  float4* workOut;
  float4* workA;
  float4* workN;
  // Some scene of the launch has transparent materials: shadow rays take the transparency
  // filter (host-side choice of the kShadow instantiation).
  int anyTransparent;
  // Irradiance mode (DevRenderer::flags, frame form): the first hit's material (device memory)
  // and its class.
  const DevMaterial* white;
  int whiteClass;
};

template <int... Fs>
struct ShadeLaunch;
// Surface classes 1..kShadeClasses-1 in kShadeClassFeatures order.
#define PRT_SHADE_CLASS_LIST                                                                          \
  kFeatOpaque, kFeatOpaque | kFeatSpecular, kFeatConductor, kFeatDielectric, kFeatOpaque | kFeatCoat, \
    kFeatOpaque | kFeatSpecular | kFeatCoat, kFeatAll


// ---- query kernels --------------------------------------------------------------------------

__global__ void kSobol(int64_t n, const uint32_t* __restrict__ si, const uint32_t* __restrict__ pid,
                       const uint32_t* __restrict__ dims, int ndim, uint32_t seed, float* __restrict__ out)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
  {
    const SobolState st = sobolSetSample(seed, si[i], pid[i]);
    if (ndim == 1)
      out[i] = sobolGet1D(st, dims[i]);
    else if (ndim == 2)
      sobolGet2D(st, dims[i], out[2 * i], out[2 * i + 1]);
    else
      sobolGet3D(st, dims[i], out[3 * i], out[3 * i + 1], out[3 * i + 2]);
  }
}

__global__ void kTraceRays(DevScene sc, int64_t n, const float4* __restrict__ rays, int32_t* __restrict__ triOut,
                           float* __restrict__ tOut, float* __restrict__ uOut, float* __restrict__ vOut,
                           uint32_t* err)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
  {
    const float4 a = rays[2 * i], b = rays[2 * i + 1];
    const TraceHit h = traverse<false>(sc.nodes, sc.tris, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w, err);
    triOut[i] = h.triId;
    tOut[i] = h.t;
    if (uOut) uOut[i] = h.u;
    if (vOut) vOut[i] = h.v;
  }
}

__global__ void kOccludedRays(DevScene sc, int64_t n, const float4* __restrict__ rays, int32_t* __restrict__ occ,
                              uint32_t* err)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
  {
    const float4 a = rays[2 * i], b = rays[2 * i + 1];
    const TraceHit h = traverse<true>(sc.nodes, sc.tris, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w, err);
    occ[i] = h.triId >= 0 ? 1 : 0;
  }
}

// Primary rays of one sample for every pixel in row-major order, plus their closest hits.
__global__ void kPrimary(DevScene sc, DevCamera cam, int width, int height, uint32_t seed, uint32_t sampleIndex,
                         float4* __restrict__ raysOut, int32_t* __restrict__ triOut, float* __restrict__ tOut,
                         uint32_t* err)
{
  const int n = width * height;
  const float invW = 1.f / (float)width, invH = 1.f / (float)height;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    const int x = i % width, y = i / width;
    const uint32_t pixelId = (uint32_t)x | ((uint32_t)y << 16);
    const SobolState st = sobolSetSample(seed, sampleIndex, pixelId);
    float sx, sy;
    sobolGet2D(st, kDimPixel, sx, sy);
    f3 org, dir;
    float tnear;
    cameraRay(cam, ((float)x + sx) * invW, ((float)y + sy) * invH, org, dir, tnear);
    raysOut[2 * i] = make_float4(org.x, org.y, org.z, tnear);
    raysOut[2 * i + 1] = make_float4(dir.x, dir.y, dir.z, kPosMax);
    const TraceHit h = traverse<false>(sc.nodes, sc.tris, org, dir, tnear, kPosMax, err);
    triOut[i] = h.triId;
    tOut[i] = h.t;
  }
}

// Microfacet-distribution sampling queries (see prt_cuda_microfacet_query): per tuple (alpha,
// s.x, s.y, wo.x, wo.y, wo.z) -> (m.x, m.y, m.z, pdf).
__global__ void kMicrofacetQuery(int distribution, int64_t n, const float* __restrict__ in, float* __restrict__ out)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
  {
    const float* t = in + 6 * i;
    float pdf = 0.f;
    f3 m;
    if (distribution == PRT_MICROFACET_BECKMANN)
      m = Beckmann{t[0]}.sample(pdf, t[1], t[2]);
    else
      m = GGX{t[0], t[0]}.sampleVisible(mk(t[3], t[4], t[5]), pdf, t[1], t[2]);
    float* o = out + 4 * i;
    o[0] = m.x;
    o[1] = m.y;
    o[2] = m.z;
    o[3] = pdf;
  }
}

// BSDF parity queries in a canonical shading context (see prt_cuda_bsdf_query).
__global__ void kBsdfQuery(DevTables tab, DevMaterial m, int mediumId, int64_t n, const float* __restrict__ tuples,
                           float* __restrict__ out)
{
  DevScene sc;
  sc.textures = nullptr;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
  {
    const float* t = tuples + 9 * i;
    const f3 wo = mk(t[0], t[1], t[2]), wi = mk(t[3], t[4], t[5]);
    ShadeCtx ctx;
    ctx.p = mk(0.f);
    ctx.eps = 1e-6f;
    ctx.f.U = mk(1.f, 0.f, 0.f);
    ctx.f.V = mk(0.f, 1.f, 0.f);
    ctx.f.N = mk(0.f, 0.f, 1.f);
    ctx.Ng = ctx.f.N;
    ctx.uvx = ctx.uvy = 0.5f;
    ctx.backfacing = false;
    const bool backfacing = (m.type & kMatMediaInterface) ? mediumId == m.mediumInt : false;
    StdBsdf b;
    resolveStandard(sc, tab, m, ctx, wo, backfacing, b);
    float evalPdf;
    const f3 ev = b.eval(tab, wo, wi, evalPdf);
    f3 swi = mk(0.f);
    float spdf = 0.f;
    int stype = 0;
    const f3 sw = b.sample(tab, wo, t[6], t[7], t[8], swi, spdf, stype);
    float* o = out + 13 * i;
    o[0] = ev.x; o[1] = ev.y; o[2] = ev.z; o[3] = evalPdf;
    o[4] = sw.x; o[5] = sw.y; o[6] = sw.z;
    o[7] = swi.x; o[8] = swi.y; o[9] = swi.z;
    o[10] = spdf;
    o[11] = __int_as_float(stype);
    o[12] = __int_as_float(b.flags());
  }
}

// ---- wavefront kernels -----------------------------------------------------------------------
//
// Every wavefront kernel exists in two forms, selected by the template flag `Batch`:
//  * frame form (Batch = false): one scene and frame per launch (Launch::sc, ::cam, ::rd);
//    the bounce depth is uniform per launch and finished paths write ps.out, which
//    kAccumulate adds per pixel in sample order after the wave;
//  * batch form (Batch = true): paths of many scenes share the queues. info.w of a path is its
//    batch item (scene, camera, renderer, frame), info.z carries the bounce depth in bits
//    16-31, finished paths add themselves to their item's accumulation planes and return their
//    slot to the free list, and kBatchRegen refills free slots with new camera paths.

// Per-path view of the scene, renderer and frame a path belongs to.
// Per-bounce counter block (ints): [0] paths entering the bounce, [1..kShadeClasses] paths per
// shading class, [kCntShadow] shadow rays, [kCntWorkTrace], [kCntWorkShadow] work counters, [kCntShadowSun] shadow
// rays toward the distant light (frame form).
constexpr int kCntShadow = 1 + kShadeClasses;
constexpr int kCntWorkTrace = kCntShadow + 1;
constexpr int kCntWorkShadow = kCntShadow + 2;
constexpr int kCntShadowSun = kCntShadow + 3;
constexpr int kCntStride = 16;
static_assert(kCntShadowSun < kCntStride, "counter block");

template <bool Batch>
struct PathEnv;

template <>
struct PathEnv<false>
{
  const DevScene& sc;
  const DevRenderer& rd;
  const AdjointView& adj;
  int aovMask, width;
  PRT_D PathEnv(const Launch& L, uint32_t) : sc(L.sc), rd(L.rd), adj(L.adj), aovMask(L.aovMask), width(L.width) {}
};

template <>
struct PathEnv<true>
{
  const BatchItem& it;
  const DevScene& sc;
  const DevRenderer& rd;
  const AdjointView& adj;
  int aovMask, width;
  PRT_D PathEnv(const Launch& L, uint32_t item)
      : it(L.items[item]), sc(it.sc), rd(it.rd), adj(it.adj), aovMask(it.aovMask), width(it.width)
  {
  }
};

constexpr uint32_t kDepthShift = 16;
constexpr uint32_t kMediumMask = 0xffffu;

// Camera path of (sample, Morton index) in slot p (render/path_renderer_stream.h:209-262).
PRT_D void initPath(const PathState& ps, int64_t p, const DevCamera& cam, const DevRenderer& rd, int width, int height,
                    int idx, uint32_t sampleIndex, uint32_t item, bool aov)
{
  int x, y;
  pixelOf(idx, width, x, y);
  const uint32_t pixelId = (uint32_t)x | ((uint32_t)y << 16);
  const SobolState st = sobolSetSample(rd.seed, sampleIndex, pixelId);
  float sx, sy;
  sobolGet2D(st, kDimPixel, sx, sy);
  f3 org, dir;
  float tnear;
  cameraRay(cam, ((float)x + sx) * (1.f / (float)width), ((float)y + sy) * (1.f / (float)height), org, dir, tnear);
  ps.rayO[p] = make_float4(org.x, org.y, org.z, tnear);
  ps.rayD[p] = make_float4(dir.x, dir.y, dir.z, kPosMax);
  ps.thr[p] = make_float4(1.f, 1.f, 1.f, 1.f);
  ps.rad[p] = make_float4(0.f, 0.f, 0.f, __int_as_float(kSpecularReflection));
  ps.info[p] = make_uint4(pixelId, sampleIndex, 0u, item);
  if (aov)
  {
    ps.aovA[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    ps.aovN[p] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (ps.sphL)
  {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    ps.sphL[p] = z;
    ps.sphWi[p] = z;
    ps.sphDirL[p] = z;
    ps.sphDirWi[p] = z;
  }
}

// Path initialisation of a frame-form wave.
__global__ void kRaygen(Launch L)
{
  const int64_t P = (int64_t)L.pixelCount * L.samples;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x)
  {
    const int s = (int)(p / L.pixelCount);
    const int idx = (int)(p - (int64_t)s * L.pixelCount);
    initPath(L.ps, p, L.cam, L.rd, L.width, L.height, idx, L.firstSample + (uint32_t)s, 0u, L.aovMask != 0);
  }
}

// Batch form: the control step at the start of an iteration (one thread). `a` is the parity
// of the iteration: it reads queue[a], free list a and counter block a, and the paths it
// extends or frees go to queue[a ^ 1] and free list a ^ 1.
__global__ void kBatchStep(BatchCtl* ctl, int a)
{
  const int b = a ^ 1;
  int* ca = ctl->counts[a];
  int* cb = ctl->counts[b];
  ctl->rays[1] += (unsigned long long)cb[kBatchCntShadow];  // shadow rays of the previous iteration
  const long long remaining = ctl->workTotal - ctl->workNext;
  const long long freeSlots = ctl->freeCount[a];
  const int n = (int)(remaining < freeSlots ? remaining : freeSlots);
  ctl->regenCount = n;
  ctl->regenBase = ctl->workNext;
  ctl->regenOffset = ca[0];
  ctl->workNext += n;
  ca[0] += n;
  ctl->rays[0] += (unsigned long long)ca[0];
  for (int k = 1; k < kBatchCntStride; ++k) ca[k] = 0;
  cb[0] = 0;
  ctl->freeCount[b] = 0;
  ctl->iterations += 1;
  if (ca[0] == 0 && ctl->workNext >= ctl->workTotal) ctl->done = 1;
}

// Batch form: fills the slots on free list `a` with new camera paths (path regeneration) and
// appends them to queue[a] after the paths extended by the previous iteration.
template <bool Adj>
__global__ void kBatchRegen(Launch L, int a, int* __restrict__ queue)
{
  const BatchCtl* ctl = L.ctl;
  const int n = ctl->regenCount;
  const long long base = ctl->regenBase;
  const int offset = ctl->regenOffset;
  const int* freeList = L.freeList[a];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    const long long w = base + i;
    // The item whose work range holds w (items are in work order).
    int lo = 0, hi = L.itemCount - 1;
    while (lo < hi)
    {
      const int mid = (lo + hi + 1) >> 1;
      if (L.items[mid].workBase <= w) lo = mid;
      else hi = mid - 1;
    }
    const BatchItem& it = L.items[lo];
    const long long local = w - it.workBase;
    const int s = (int)(local / it.pixelCount);
    const int idx = (int)(local - (long long)s * it.pixelCount);
    const int slot = freeList[i];
    initPath(L.ps, slot, it.cam, it.rd, it.width, it.height, idx, (uint32_t)s, (uint32_t)lo, it.aovMask != 0 && !Adj);
    if (Adj) L.ps.out[slot] = L.pathL[w];  // replay: the radiance still to come is the whole path's
    queue[offset + i] = slot;
  }
}

// Copies the breadth-first top levels of the frame's BVH into shared memory (Top = true; frame
// form only, the batch form mixes scenes). Returns the number of staged nodes.
template <bool Top>
PRT_D int stageTopNodes(const Launch& L)
{
  if (!Top) return 0;
  const int n = min(L.sc.topNodes, kBvh8TopNodes);
  for (int i = threadIdx.x; i < 5 * n; i += blockDim.x) gTopNodes[i] = __ldg(L.sc.nodes + i);
  __syncthreads();
  return n;
}

// Adds one warp's traversal counts to the global totals (counting variant only).
PRT_D void addCounts(unsigned long long* dst, const TraceCount& c)
{
  unsigned long long n = (unsigned long long)c.nodes, t = (unsigned long long)c.tris;
  for (int o = 16; o > 0; o >>= 1)
  {
    n += __shfl_down_sync(0xffffffffu, n, o);
    t += __shfl_down_sync(0xffffffffu, t, o);
  }
  if (laneId() == 0)
  {
    atomicAdd(dst, n);
    atomicAdd(dst + 1, t);
  }
}

// Closest-hit traversal of the queued rays. Persistent warps fetch 32 rays at a time, write
// the hit and bin the path by the shading it needs (the GPU form of the reference's material
// sort, render/renderer_stream.h:108-181): class 0 ends the path (miss, area light, maxDepth),
// classes 1.. are the material feature classes.
template <bool Count, bool Batch, bool Top = false, int Stack = kTraceStack>
__global__ void __launch_bounds__(256) kTrace(Launch L, const int* __restrict__ queue, const int* __restrict__ count,
                                              int* __restrict__ work, int depth, int* __restrict__ classQueues,
                                              int* __restrict__ classCounts)
{
  const int n = *count;
  const int top = stageTopNodes<Top && !Batch>(L);
  TraceCount tc;
  for (;;)
  {
    int base = 0;
    if (laneId() == 0) base = atomicAdd(work, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const int i = base + laneId();
    int cls = -1, p = 0;
    if (i < n)
    {
      p = queue ? (int)((uint32_t)__ldg(queue + i) & kQueuePathMask) : i;
      const float4 a = L.ps.rayO[p], b = L.ps.rayD[p];
      uint32_t item = 0u;
      int pathDepth = depth;
      if (Batch)
      {
        const uint4 info = L.ps.info[p];
        item = info.w;
        pathDepth = (int)(info.z >> kDepthShift);
      }
      const PathEnv<Batch> E(L, item);
      const TraceHit h = traverse<false, Count, Top && !Batch, Stack>(E.sc.nodes, E.sc.tris, mk(a.x, a.y, a.z),
                                                               mk(b.x, b.y, b.z), a.w, b.w, L.ps.err, &tc, top);
      L.ps.hit[p] = make_float4(h.t, h.u, h.v, __int_as_float(h.triId));
      cls = 0;
      if (h.triId >= 0 && pathDepth < E.rd.maxDepth) cls = __ldg(E.sc.meshClass + __ldg(E.sc.triVerts + h.triId).w);
      // Irradiance mode: every surface a camera ray hits is shaded with the white material.
      if (!Batch && cls > 0 && pathDepth == 0 && (L.rd.flags & PRT_RENDERER_IRRADIANCE)) cls = L.whiteClass;
    }
    for (int c = 0; c < kShadeClasses; ++c)
    {
      const int slot = warpAppend(classCounts + c, cls == c);
      if (cls == c) classQueues[(int64_t)c * L.ps.capacity + slot] = p;
    }
  }
  if (Count) addCounts(L.ps.travCounts, tc);
}

// ---- ray binning: the next bounce's queue grouped by direction octant -------------------------
//
// kShadeSurface tags each extended path's queue entry with the octant of its new direction
// (kQueueOctShift). Two passes over the entries (a counting sort on 3 bits) rewrite the queue so
// that each octant's rays are contiguous, in their previous order within an octant. A warp of
// kTrace then takes rays that visit the children of every node in the same order, and rays
// from nearby origins walk the same subtrees at the same time. bins[0..7] count the entries of
// each octant, bins[8..15] are the octants' fill cursors; both start at zero.

// Counts the entries of each octant (one add per octant and block).
__global__ void __launch_bounds__(256) kRayBinCount(const int* __restrict__ queue, const int* __restrict__ count,
                                                    int* __restrict__ bins)
{
  __shared__ int sCount[8];
  if (threadIdx.x < 8) sCount[threadIdx.x] = 0;
  __syncthreads();
  const int n = *count;
  const int lane = laneId();
  int mine = 0;  // lane o < 8 sums octant o
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n; base += warps * 32)
  {
    const int i = base + lane;
    const uint32_t oct = i < n ? (uint32_t)__ldg(queue + i) >> kQueueOctShift : 8u;
#pragma unroll
    for (int o = 0; o < 8; ++o)
    {
      const int c = __popc(__ballot_sync(0xffffffffu, oct == (uint32_t)o));
      if (lane == o) mine += c;
    }
  }
  if (lane < 8 && mine) atomicAdd(&sCount[lane], mine);
  __syncthreads();
  if (threadIdx.x < 8 && sCount[threadIdx.x]) atomicAdd(bins + threadIdx.x, sCount[threadIdx.x]);
}

// Writes each entry's path slot into its octant's range of `out`. Tiles of 256 entries: one
// cursor add per octant and tile, ranks within the tile by warp ballots. Needs 256 threads.
__global__ void __launch_bounds__(256) kRayBinScatter(const int* __restrict__ queue, const int* __restrict__ count,
                                                      int* __restrict__ bins, int* __restrict__ out)
{
  __shared__ int sBase[8];     // first slot of each octant's range
  __shared__ int sWarp[8][8];  // [warp][octant]: the warp's count, then its first slot in the range
  const int n = *count;
  const int lane = laneId(), warp = threadIdx.x >> 5;
  if (threadIdx.x < 8)
  {
    int b = 0;
    for (int o = 0; o < (int)threadIdx.x; ++o) b += bins[o];
    sBase[threadIdx.x] = b;
  }
  for (int64_t tile = blockIdx.x; tile * 256 < n; tile += gridDim.x)
  {
    const int i = (int)(tile * 256) + (int)threadIdx.x;
    const bool active = i < n;
    const uint32_t v = active ? (uint32_t)__ldg(queue + i) : 0u;
    const uint32_t oct = active ? v >> kQueueOctShift : 8u;
    unsigned same = 0u;
    int warpCount = 0;
#pragma unroll
    for (int o = 0; o < 8; ++o)
    {
      const unsigned b = __ballot_sync(0xffffffffu, oct == (uint32_t)o);
      if (oct == (uint32_t)o) same = b;
      if (lane == o) warpCount = __popc(b);
    }
    if (lane < 8) sWarp[warp][lane] = warpCount;
    __syncthreads();
    if (threadIdx.x < 8)
    {
      const int o = threadIdx.x;
      int total = 0;
      for (int w = 0; w < 8; ++w) total += sWarp[w][o];
      int run = total ? atomicAdd(bins + 8 + o, total) : 0;
      for (int w = 0; w < 8; ++w)
      {
        const int c = sWarp[w][o];
        sWarp[w][o] = run;
        run += c;
      }
    }
    __syncthreads();
    if (active) out[sBase[oct] + sWarp[warp][oct] + __popc(same & ((1u << lane) - 1u))] = (int)(v & kQueuePathMask);
    __syncthreads();
  }
}

// Ends path p with radiance `rad`. Frame form: ps.out, summed later by kAccumulate. Batch
// form: added to the item's accumulation planes at once (with the first-hit AOVs); the
// caller returns the slot to the free list.
// Radiance-to-irradiance scale pi / cos of a first-hit direction (render/path_renderer_stream.h:
// 708, 919). The reference divides by max(cos, 0) with its approximate reciprocal, which gives NaN
// for a direction at or below the BSDF's normal, and clampL turns the product into zero: such a
// direction adds nothing, which a zero scale reproduces.
PRT_D float shIrradianceScale(float cosTheta) { return cosTheta > 0.f ? kPi / cosTheta : 0.f; }

// The path's SH sample at its end (render/path_renderer_stream.h:329-344, 1032-1041): the
// radiance gathered after the first hit (plus `extra`, what this bounce adds to it) scaled to
// irradiance along the first bounce's direction, plus the first hit's direct light along its
// direction, each as first-order SH (value, value x dir.x, value x dir.y, value x dir.z,
// math/sh.h:115-135).
PRT_D void finishSh(const Launch& L, int p, f3 extra)
{
  const float4 a = L.ps.sphL[p], w = L.ps.sphWi[p], dl = L.ps.sphDirL[p], dw = L.ps.sphDirWi[p];
  const f3 v = clampL((mk(a.x, a.y, a.z) + extra) * a.w, L.rd.maxRadiance);
  const f3 d = clampL(mk(dl.x, dl.y, dl.z), L.rd.maxRadiance);
  const f3 c1 = v * w.x + d * dw.x, c2 = v * w.y + d * dw.y, c3 = v * w.z + d * dw.z;
  const f3 c0 = v + d;
  float4* o = L.ps.sphOut + 3 * (int64_t)p;
  o[0] = make_float4(c0.x, c0.y, c0.z, c1.x);
  o[1] = make_float4(c1.y, c1.z, c2.x, c2.y);
  o[2] = make_float4(c2.z, c3.x, c3.y, c3.z);
}

template <bool Batch>
PRT_D void finishPath(const Launch& L, int p, f3 rad, const uint4& info, f3 shExtra = mk(0.f))
{
  if (!Batch)
  {
    const f3 c = clampL(rad, L.rd.maxRadiance);
    L.ps.out[p] = make_float4(c.x, c.y, c.z, 1.f);
    if (L.ps.sphOut) finishSh(L, p, shExtra);
    return;
  }
  const BatchItem& it = L.items[info.w];
  const f3 c = clampL(rad, it.rd.maxRadiance);
  const uint32_t pid = info.x;
  const int px = (int)(pid & 0x0fffu), py = (int)((pid >> 16) & 0x0fffu);
  const long long w = it.workBase + (long long)info.y * it.pixelCount + slotOfPixel(px, py, it.width);
  if (L.workOut)
  {
    L.workOut[w] = make_float4(c.x, c.y, c.z, 1.f);
    if (it.aovMask)
    {
      L.workA[w] = L.ps.aovA[p];
      L.workN[w] = L.ps.aovN[p];
    }
  }
  if (L.pathL) L.pathL[w] = make_float4(c.x, c.y, c.z, 0.f);
}

// The batch's per-pixel sums of one item: its work items' radiance (and first-hit AOVs) added in
// sample order, as kAccumulate adds a frame's, so that each frame's image does not depend on the
// order in which its paths finished. Replaces the item's planes.
__global__ void kBatchAccumulate(const BatchItem* __restrict__ items, int item, const float4* __restrict__ workOut,
                                 const float4* __restrict__ workA, const float4* __restrict__ workN)
{
  const BatchItem& it = items[item];
  const int spp = (int)(it.workCount / it.pixelCount);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < it.pixelCount; q += gridDim.x * blockDim.x)
  {
    const int x = q % it.width, y = q / it.width;
    const long long base = it.workBase + slotOfPixel(x, y, it.width);
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f), a = acc, nn = acc;
    for (int s = 0; s < spp; ++s)
    {
      const long long w = base + (long long)s * it.pixelCount;
      const float4 o = workOut[w];
      if (o.w != 0.f)
      {
        acc.x += o.x;
        acc.y += o.y;
        acc.z += o.z;
        acc.w += 1.f;
      }
      if (it.aovMask)
      {
        const float4 va = workA[w], vn = workN[w];
        if (va.w != 0.f)
        {
          a.x += va.x; a.y += va.y; a.z += va.z; a.w += 1.f;
        }
        if (vn.w != 0.f)
        {
          nn.x += vn.x; nn.y += vn.y; nn.z += vn.z; nn.w += 1.f;
        }
      }
    }
    it.accum[q] = acc;
    if (it.aovMask)
    {
      it.accA[q] = a;
      it.accN[q] = nn;
    }
  }
}

// Batch form: returns the slots of the lanes with `freed` set to free list `b` (converged
// warp, like warpAppend).
template <bool Batch>
PRT_D void freeSlots(const Launch& L, int b, bool freed, int p)
{
  if (!Batch) return;
  const int f = warpAppend(&L.ctl->freeCount[b], freed);
  if (freed) L.freeList[b][f] = p;
}

// TransparentShadowFilterSimd (render/transparent_filter.h:42-94): a shadow ray that hits a
// transparent material continues through it with its transmittance multiplied by the
// material's transparency; any other hit, or a transmittance below 1e-5, occludes it.
struct ShadowFilter
{
  const DevScene* sc;
  const DevTables* tab;
  f3 o, d;
  f3* T;

  PRT_D bool operator()(int triId, float t, float u, float v) const
  {
    const int mesh = __ldg(&sc->triVerts[triId].w);
    const DevMaterial& m = sc->materials[__ldg(sc->meshMaterial + mesh)];
    if (!(m.type & kMatTransparent))
    {
      *T = mk(0.f);
      return true;
    }
    ShadeCtx ctx;
    postIntersect(*sc, o, d, t, triId, u, v, ctx);
    *T *= standardTransparency(*sc, *tab, m, ctx, -d);
    return reduceMax(*T) < 1e-5f;
  }
};

// Any-hit test of the queued shadow rays; adds the unoccluded NEE contribution and
// finishes paths that ended at this bounce (render/path_renderer_stream.h:953-1010). Transp:
// scenes with transparent materials filter the hits (ShadowFilter).
template <bool Count, bool Batch, bool Top = false, bool Transp = false, int Stack = kTraceStack>
__global__ void __launch_bounds__(256) kShadow(Launch L, const int* __restrict__ count, int* __restrict__ work,
                                               int parity, int depth)
{
  // Frame form: the front region holds count[0] rays, the back region (from the last slot down)
  // the distant light's count[kCntShadowSun - kCntShadow]; work item j maps to front j or back.
  const int nFront = *count;
  const int n = Batch ? nFront : nFront + count[kCntShadowSun - kCntShadow];
  const int top = stageTopNodes<Top && !Batch>(L);
  TraceCount tc;
  for (;;)
  {
    int base = 0;
    if (laneId() == 0) base = atomicAdd(work, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const int j = base + laneId();
    const int i = j < nFront ? j : (int)(L.ps.capacity - 1 - (j - nFront));
    bool freed = false;
    int p = 0;
    if (j < n)
    {
      const float4 a = L.ps.shO[i], b = L.ps.shD[i], c = L.ps.shL[i];
      const uint32_t tag = __float_as_uint(c.w);
      p = (int)(tag & 0x7fffffffu);
      uint4 info = make_uint4(0u, 0u, 0u, 0u);
      if (Batch) info = L.ps.info[p];
      const PathEnv<Batch> E(L, info.w);
      bool unoccluded = b.w > 0.f;
      f3 T = mk(1.f);
      if (unoccluded)
      {
        const f3 o = mk(a.x, a.y, a.z), d = mk(b.x, b.y, b.z);
        if (Transp && E.sc.hasTransparent)
        {
          const ShadowFilter flt{&E.sc, &L.tab, o, d, &T};
          unoccluded =
            traverse<true, Count, Top && !Batch, Stack>(E.sc.nodes, E.sc.tris, o, d, a.w, b.w, L.ps.err, &tc, top, flt)
              .triId < 0;
        }
        else
          unoccluded = traverse<true, Count, Top && !Batch, Stack>(E.sc.nodes, E.sc.tris, o, d, a.w, b.w, L.ps.err, &tc, top)
                         .triId < 0;
      }
      float4 r = L.ps.rad[p];
      if (unoccluded)
      {
        r.x += c.x * T.x;
        r.y += c.y * T.y;
        r.z += c.z * T.z;
        L.ps.rad[p] = r;
        // SH AOV (render/path_renderer_stream.h:1004-1017): the first hit's direct light, scaled
        // to irradiance, with its direction; later bounces add to the gathered radiance.
        if (!Batch && L.ps.sphOut)
        {
          const f3 dl = mk(c.x * T.x, c.y * T.y, c.z * T.z);
          if (depth == 0)
          {
            const float sc = L.ps.sphDirScale[i];
            L.ps.sphDirL[p] = make_float4(dl.x * sc, dl.y * sc, dl.z * sc, 0.f);
            L.ps.sphDirWi[p] = make_float4(b.x, b.y, b.z, 0.f);
          }
          else
          {
            float4 q = L.ps.sphL[p];
            q.x += dl.x;
            q.y += dl.y;
            q.z += dl.z;
            L.ps.sphL[p] = q;
          }
        }
      }
      if (tag & kShadowFinish)
      {
        finishPath<Batch>(L, p, mk(r.x, r.y, r.z), info);
        freed = true;
      }
    }
    freeSlots<Batch>(L, parity ^ 1, freed, p);
  }
  if (Count) addCounts(L.ps.travCounts + 2, tc);
}

// Paths that end at this bounce without shading a surface (render/path_renderer_stream.h:287-582
// and the depth cut-off at :612): misses (environment lights), area-light hits, and surface
// hits at maxDepth.
template <bool Batch, bool Adj = false>
__global__ void __launch_bounds__(256) kShadeEnd(Launch L, const int* __restrict__ queue, const int* __restrict__ count,
                                                 int depth, int parity)
{
  const int n = *count;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x)
  {
    const int i = base + threadIdx.x;
    const bool active = i < n;
    const int p = active ? __ldg(queue + i) : 0;
    if (active && !Adj)
    {
      const float4 rd = L.ps.rayD[p], hh = L.ps.hit[p];
      const float4 tp = L.ps.thr[p];
      float4 ra = L.ps.rad[p];
      const uint4 info = L.ps.info[p];
      const PathEnv<Batch> E(L, info.w);
      const uint32_t pixelId = info.x;
      const f3 dir = mk(rd.x, rd.y, rd.z);
      const int triId = __float_as_int(hh.w);
      const f3 T = mk(tp.x, tp.y, tp.z);
      f3 Lr = mk(ra.x, ra.y, ra.z);
      const float lastPdf = tp.w;
      const int lastType = __float_as_int(ra.w);
      const bool aov1 = (pixelId & kPathAov1Flag) == 0u;
      f3 lightL = mk(0.f);
      // A hit on a PRT_MATERIAL_MISS material is shaded as a miss.
      const bool miss =
        triId < 0 ||
        (E.sc.materials[__ldg(E.sc.meshMaterial + __ldg(&E.sc.triVerts[triId].w))].type & kMatMiss) != 0;
      if (miss)
      {
        // Irradiance mode: a camera ray that misses sees no environment
        // (render/path_renderer_stream.h:304).
        if (Batch || depth > 0 || !(L.rd.flags & PRT_RENDERER_IRRADIANCE))
        {
          float lightPdf;
          const f3 Le = evalEnvLights(E.sc, dir, lightPdf);
          const float w = (lastType & kBsdfSmooth) == 0 ? 1.f : misWeight(lastPdf, lightPdf);
          lightL = T * w * Le;
          Lr += lightL;
        }
        if (aov1 && E.aovMask)
        {
          L.ps.aovA[p] = make_float4(0.f, 0.f, 0.f, 1.f);
          L.ps.aovN[p] = make_float4(0.f, 0.f, 0.f, 1.f);
        }
      }
      else
      {
        const int4 tv = __ldg(E.sc.triVerts + triId);
        const int mesh = tv.w;
        const int matId = __ldg(E.sc.meshMaterial + mesh);
        if (E.sc.materials[matId].type & kMatEmissive)
        {
          float lightPdf;
          const int prim = triId - __ldg(E.sc.meshTriOffset + mesh);
          const f3 Le = evalAreaLight(E.sc, mesh, prim, dir, hh.x, lightPdf);
          const float w = (lastType & kBsdfSmooth) == 0 ? 1.f : misWeight(lastPdf, lightPdf);
          lightL = T * w * Le;
          Lr += lightL;
          if (aov1 && E.aovMask)
          {
            const f3 N = normalize(-dir);
            L.ps.aovA[p] = make_float4(1.f, 1.f, 1.f, 1.f);
            L.ps.aovN[p] = make_float4(N.x, N.y, N.z, 1.f);
          }
        }
        // else: a surface at maxDepth ends the path with its current radiance.
      }
      finishPath<Batch>(L, p, Lr, info, lightL);
    }
    freeSlots<Batch>(L, parity ^ 1, active, p);
  }
}

// Surface shading of one bounce (render/path_renderer_stream.h:592-949) for materials whose
// lobes lie in feature set F: NEE with MIS, BSDF sampling, Russian roulette, medium tracking.
template <int F, bool Batch, bool Adj = false>
__global__ void __launch_bounds__(256) kShadeSurface(Launch L, const int* __restrict__ queue,
                                                     const int* __restrict__ count, int launchDepth,
                                                     int* __restrict__ queueOut, int* __restrict__ extCount,
                                                     int* __restrict__ shadowCount, int parity)
{
  const int n = *count;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x)
  {
    const int i = base + threadIdx.x;
    const bool active = i < n;
    const int p = active ? __ldg(queue + i) : 0;
    bool extend = false;
    bool shadow = false;
    bool freed = false;
    uint32_t extTag = 0u;  // direction octant of the extended ray, in the queue entry's top bits
    float4 shO = make_float4(0.f, 0.f, 0.f, 0.f), shD = shO, shL = shO;
    float shScale = 0.f;   // SH AOV: irradiance scale of a first-hit shadow ray
    bool toSun = false;    // the shadow ray goes to the distant light
    if (active)
    {
      const float4 ro = L.ps.rayO[p], rd = L.ps.rayD[p], hh = L.ps.hit[p];
      const float4 tp = L.ps.thr[p];
      float4 ra = L.ps.rad[p];
      uint4 info = L.ps.info[p];
      const PathEnv<Batch> E(L, info.w);
      const int depth = Batch ? (int)(info.z >> kDepthShift) : launchDepth;
      const uint32_t sampleDim = kDimBase + kDimBounce * (uint32_t)depth;
      const f3 org = mk(ro.x, ro.y, ro.z), dir = mk(rd.x, rd.y, rd.z);
      const int triId = __float_as_int(hh.w);
      f3 T = mk(tp.x, tp.y, tp.z);
      const f3 Lr = mk(ra.x, ra.y, ra.z);
      const float lastPdf = tp.w;
      const int lastType = __float_as_int(ra.w);
      uint32_t pixelId = info.x;
      const bool aov1 = (pixelId & kPathAov1Flag) == 0u;
      ShadeCtx ctx;
      postIntersect(E.sc, org, dir, hh.x, triId, hh.y, hh.z, ctx);
      // Irradiance mode: the first hit is shaded with the white material
      // (render/path_renderer_stream.h:598).
      const bool whiteHit = !Batch && depth == 0 && (L.rd.flags & PRT_RENDERER_IRRADIANCE);
      const DevMaterial& mat = whiteHit ? *L.white : E.sc.materials[ctx.material];
      const f3 wo = -dir;
      uint32_t mediumId = info.z & kMediumMask;
      // Material::getBsdf orientation: media interfaces take it from the medium the path
      // is in, every other material is treated as front-facing (material/material.h:66-76).
      const bool backfacing = (mat.type & kMatMediaInterface) ? (int)mediumId == mat.mediumInt : false;
      StdBsdfT<F> bsdf;
      resolveStandard<F>(E.sc, L.tab, mat, ctx, wo, backfacing, bsdf);
      const SobolState st = sobolSetSample(E.rd.seed, info.y, pixelId & kPixelIdMask);
      const bool aov2 = (pixelId & kPathAov2Flag) == 0u;
      const bool rr = !(aov1 || aov2);
      // Volume transmission (Beer's law) inside a medium.
      if (mediumId > 0u)
      {
        const f3 mc = ld3(E.sc.mediaColor + 3 * mediumId);
        T *= powf3(mc, hh.x);
      }
      // Direct light (NEE)
      bool neeVisible = false;
      f3 neeL = mk(0.f), neeWi = mk(0.f);
      if (bsdf.flags() & kBsdfSmooth)
      {
        float lx, ly, lz;
        sobolGet3D(st, sampleDim + kDimLight, lx, ly, lz);
        f3 wi;
        float lightPdf, dist;
        int light;
        const f3 Lw = sampleLight(E.sc, ctx.p, lx, ly, lz, wi, lightPdf, dist, light);
        toSun = light == E.sc.distantLight;
        if (reduceMax(Lw) > 0.f && lightPdf > 0.f)
        {
          float bsdfPdf;
          const f3 bv = bsdf.eval(L.tab, wo, wi, bsdfPdf);
          if (reduceMax(bv) > 0.f)
          {
            const f3 dirT = T * bv;
            if (depth >= E.rd.rrDepth)
            {
              const float contProb = rr ? fminf(luminance(dirT * (1.f / bsdfPdf)), 0.95f) : 1.f;
              bsdfPdf *= contProb;
            }
            const f3 dirL = dirT * misWeight(lightPdf, bsdfPdf) * Lw;
            if (Adj)
            {
              // Replay: the shadow ray is traced here, its visibility is part of the vertex.
              const float far = dist - ctx.eps;
              neeVisible = far > 0.f ? traverse<true>(E.sc.nodes, E.sc.tris, ctx.p, wi, ctx.eps, far, L.ps.err).triId < 0
                                     : true;
              neeL = neeVisible ? dirL : mk(0.f);
              neeWi = wi;
            }
            else
            {
              shadow = true;
              shO = make_float4(ctx.p.x, ctx.p.y, ctx.p.z, ctx.eps);
              shD = make_float4(wi.x, wi.y, wi.z, dist - ctx.eps);
              shL = make_float4(dirL.x, dirL.y, dirL.z, 0.f);
              // SH AOV: the first hit's direct light counts as irradiance, pi / cos of the
              // light direction times its radiance (render/path_renderer_stream.h:705-709).
              if (!Batch && L.ps.sphOut && depth == 0) shScale = shIrradianceScale(dot(wi, bsdf.normal()));
            }
          }
        }
      }
      // BSDF sampling
      float bx, by, bz;
      sobolGet3D(st, sampleDim + kDimBsdf, bx, by, bz);
      f3 wi;
      float bsdfPdf;
      int bsdfType;
      const f3 bw = bsdf.sample(L.tab, wo, bx, by, bz, wi, bsdfPdf, bsdfType);
      extend = reduceMax(bw) > 0.f && bsdfPdf > 0.f;
      const int extType = extend ? bsdfType : 0;
      if (aov1)
      {
        if (!Adj && E.aovMask)
        {
          const f3 a = bsdf.albedo(), nn = bsdf.normal();
          L.ps.aovA[p] = make_float4(a.x, a.y, a.z, 1.f);
          L.ps.aovN[p] = make_float4(nn.x, nn.y, nn.z, 1.f);
        }
        pixelId |= kPathAov1Flag;
      }
      if (aov2 && (extType & kBsdfDelta) == 0) pixelId |= kPathAov2Flag;
      T *= bw;
      extend = extend && reduceMax(T) >= E.rd.minWeight;
      if (depth >= E.rd.rrDepth)
      {
        const float contProb = rr ? fminf(luminance(T), 0.95f) : 1.f;
        extend = extend && sobolGet1D(st, sampleDim + kDimTerminate) <= contProb;
        T *= 1.f / contProb;
        bsdfPdf *= contProb;
      }
      if (Adj)
      {
        // Replay: out[p] holds the radiance still to come at this vertex.
        const float4 o = L.ps.out[p];
        const f3 rest = mk(o.x, o.y, o.z) - neeL;
        const uint32_t px = pixelId & kPixelIdMask;
        const float* g = E.adj.dLdI + 3 * ((size_t)(px >> 16) * E.width + (px & 0xffffu));
        const f3 delta = mk(g[0], g[1], g[2]) * E.adj.invSpp;
        adjointVertex<F>(E.adj, E.sc, L.tab, mat, ctx, bsdf, wo, wi, neeWi, extend, neeVisible, neeL,
                         extend ? rest : mk(0.f), delta);
        if (extend) L.ps.out[p] = make_float4(rest.x, rest.y, rest.z, o.w);
      }
      if (extend)
      {
        L.ps.rayO[p] = make_float4(ctx.p.x, ctx.p.y, ctx.p.z, ctx.eps);
        L.ps.rayD[p] = make_float4(wi.x, wi.y, wi.z, kPosMax);
        extTag = ((wi.x < 0.f ? 1u : 0u) | (wi.y < 0.f ? 2u : 0u) | (wi.z < 0.f ? 4u : 0u)) << kQueueOctShift;
        const bool update = (bsdfType & kBsdfContinuation) == 0;
        L.ps.thr[p] = make_float4(T.x, T.y, T.z, update ? bsdfPdf : lastPdf);
        ra.w = __int_as_float(update ? bsdfType : lastType);
        // Material::nextMedium (material/material.h:84-93).
        if ((mat.type & kMatMediaInterface) && dot(wo, ctx.Ng) * dot(wi, ctx.Ng) < 0.f)
          mediumId = (int)mediumId == mat.mediumInt ? (uint32_t)mat.mediumExt : (uint32_t)mat.mediumInt;
        info.z = Batch ? (mediumId | ((uint32_t)(depth + 1) << kDepthShift)) : mediumId;
        L.ps.rad[p] = ra;
        // SH AOV: the first bounce's direction and its irradiance scale
        // (render/path_renderer_stream.h:914-930).
        if (!Batch && L.ps.sphOut && depth == 0)
        {
          L.ps.sphL[p] = make_float4(0.f, 0.f, 0.f, shIrradianceScale(dot(wi, bsdf.normal())));
          L.ps.sphWi[p] = make_float4(wi.x, wi.y, wi.z, 0.f);
        }
      }
      info.x = pixelId;
      L.ps.info[p] = info;
      if (!extend && (Adj || !shadow))
      {
        if (!Adj) finishPath<Batch>(L, p, Lr, info);
        freed = true;
      }
      if (shadow) shL.w = __uint_as_float((uint32_t)p | (extend ? 0u : kShadowFinish));
    }
    const int e = warpAppend(extCount, extend);
    if (extend) queueOut[e] = (int)((uint32_t)p | extTag);
    // Frame form: shadow rays toward the distant light fill the shadow arrays from the back
    // (counter kCntShadowSun), the others from the front, so that a warp of the shadow kernel
    // takes rays of one kind: the distant light's rays are parallel and their traversal coherent.
    // The two regions never meet: together they hold at most one ray per path of this bounce.
    const bool sunQueue = !Batch && !Adj && toSun;
    const int front = warpAppend(shadowCount, shadow && !sunQueue);
    const int back = Batch ? 0 : warpAppend(shadowCount + (kCntShadowSun - kCntShadow), shadow && sunQueue);
    const int sidx = sunQueue ? (int)(L.ps.capacity - 1 - back) : front;
    if (shadow)
    {
      L.ps.shO[sidx] = shO;
      L.ps.shD[sidx] = shD;
      L.ps.shL[sidx] = shL;
      if (!Batch && L.ps.sphDirScale) L.ps.sphDirScale[sidx] = shScale;
    }
    freeSlots<Batch>(L, parity ^ 1, freed, p);
  }
}

// ---- sibling stream renderers ---------------------------------------------------------------
//
// The path tracer's simpler siblings (render/renderer_factory_stream.cpp:54-67), one thread per
// pixel-sample: the camera ray of the path tracer, then
//   Type 1 (primaryStream, render/primary_renderer_stream.h:140-176): (N + 1) / 2 of the first
//          hit's shading normal, 0.05 on a miss;
//   Type 2 (aoStream, render/ao_renderer_stream.h:150-238): the fraction of aoSamples
//          cosine-distributed rays from the first hit that escape, 0 on a miss;
//   Type 3 (diffuseStream, render/diffuse_renderer_stream.h:146-213): a white diffuse walk under
//          a white sky, throughput x 0.8 per bounce, 0 at maxDepth;
//   Type 4 (diffuse2Stream, render/diffuse2_renderer_stream.h:150-255): the same with a
//          cosine-sampled sky ray per bounce; sky seen by either ray counts half, except from
//          the camera.
// Bounce k draws its directions from dimensions 4 + 2k (4 + 4k and 4 + 4k + 2 for type 4, AO ray
// k from 4 + 2k). Writes ps.out, which kAccumulate adds in sample order.
// Fast: the "...StreamFast" variant on the simple shading context -- the geometric normal as
// computed, not flipped toward the ray, and the frame made from it.
template <int Type, bool Fast>
__global__ void __launch_bounds__(256) kSimpleRender(Launch L)
{
  const int64_t P = (int64_t)L.pixelCount * L.samples;
  unsigned long long traced = 0, occl = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x)
  {
    const int s = (int)(p / L.pixelCount);
    const int idx = (int)(p - (int64_t)s * L.pixelCount);
    int x, y;
    pixelOf(idx, L.width, x, y);
    const uint32_t pixelId = (uint32_t)x | ((uint32_t)y << 16);
    const uint32_t sampleIndex = L.firstSample + (uint32_t)s;
    const SobolState st = sobolSetSample(L.rd.seed, sampleIndex, pixelId);
    float sx, sy;
    sobolGet2D(st, kDimPixel, sx, sy);
    f3 org, dir;
    float tnear;
    cameraRay(L.cam, ((float)x + sx) * (1.f / (float)L.width), ((float)y + sy) * (1.f / (float)L.height), org, dir,
              tnear);
    f3 color = mk(0.f);
    float throughput = 1.f, Lsum = 0.f;
    for (int depth = 0;; ++depth)
    {
      const TraceHit h = traverse<false>(L.sc.nodes, L.sc.tris, org, dir, tnear, kPosMax, L.ps.err);
      ++traced;
      if (h.triId < 0)
      {
        if (Type == 1) color = mk(0.05f);
        if (Type == 3) color = mk(throughput);
        if (Type == 4) color = mk(Lsum + throughput * (depth > 0 ? 0.5f : 1.f));
        break;
      }
      ShadeCtx ctx;
      postIntersect(L.sc, org, dir, h.t, h.triId, h.u, h.v, ctx);
      if (Fast)
      {
        // SimpleShadingContextSimd: N = Ng = normalize(cross(p1 - p0, p2 - p0)), unflipped.
        const f3 Ng = ctx.backfacing ? -ctx.Ng : ctx.Ng;
        ctx.f.N = Ng;
        makeFrame(Ng, ctx.f.U, ctx.f.V);
      }
      if (Type == 1)
      {
        color = (ctx.f.N + mk(1.f)) * 0.5f;
        break;
      }
      if (Type == 2)
      {
        int open = 0;
        for (int k = 0; k < L.rd.aoSamples; ++k)
        {
          float ax, ay, pdf;
          sobolGet2D(st, kDimBase + 2u * (uint32_t)k, ax, ay);
          const f3 d = toWorld(ctx.f, cosineSampleHemisphere(pdf, ax, ay));
          open += traverse<true>(L.sc.nodes, L.sc.tris, ctx.p, d, ctx.eps, kPosMax, L.ps.err).triId < 0 ? 1 : 0;
          ++occl;
        }
        color = mk((float)open * (1.f / (float)L.rd.aoSamples));
        break;
      }
      if (depth == L.rd.maxDepth)
      {
        if (Type == 4) color = mk(Lsum);
        break;
      }
      float bx, by, pdf;
      if (Type == 4)
      {
        sobolGet2D(st, kDimBase + 4u * (uint32_t)depth, bx, by);
        const f3 ds = toWorld(ctx.f, cosineSampleHemisphere(pdf, bx, by));
        sobolGet2D(st, kDimBase + 4u * (uint32_t)depth + 2u, bx, by);
        throughput *= 0.8f;
        const bool open = traverse<true>(L.sc.nodes, L.sc.tris, ctx.p, ds, ctx.eps, kPosMax, L.ps.err).triId < 0;
        ++occl;
        if (open) Lsum += throughput * 0.5f;
      }
      else
      {
        sobolGet2D(st, kDimBase + 2u * (uint32_t)depth, bx, by);
        throughput *= 0.8f;
      }
      dir = toWorld(ctx.f, cosineSampleHemisphere(pdf, bx, by));
      org = ctx.p;
      tnear = ctx.eps;
    }
    L.ps.out[p] = make_float4(color.x, color.y, color.z, 1.f);
  }
  // Ray counts: one atomic per warp.
  for (int o = 16; o > 0; o >>= 1)
  {
    traced += __shfl_down_sync(0xffffffffu, traced, o);
    occl += __shfl_down_sync(0xffffffffu, occl, o);
  }
  if (laneId() == 0)
  {
    atomicAdd(L.ps.travCounts, traced);
    atomicAdd(L.ps.travCounts + 1, occl);
  }
}

// Adds the wave's samples of each pixel, in sample order, to the accumulation planes.
// Also keeps, per pixel, the checkpoint copy of the sums taken before every power-of-two-th
// sample (AccumBuffer::begin, image/accum_buffer.h:252-260; `count` = samples since the clear)
// and, when enabled, the sums of squared samples (addSerial, :439-486).
// overwrite: each sample replaces the pixel (AccumBuffer::set, image/accum_buffer.h:547-570), for
// the renderers that do not accumulate.
__global__ void kAccumulate(Launch L, float4* __restrict__ accum, float4* __restrict__ accA, float4* __restrict__ accN,
                            float4* __restrict__ accC, float4* __restrict__ acc2, long long countBase, int overwrite,
                            float4* __restrict__ accSH)
{
  const int n = L.pixelCount;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
  {
    const int x = q % L.width, y = q / L.width;
    const int idx = slotOfPixel(x, y, L.width);
    float4 acc = accum[q];
    float4 a = accA ? accA[q] : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 nn = accN ? accN[q] : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 sq = acc2 ? acc2[q] : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int s = 0; s < L.samples; ++s)
    {
      const long long count = countBase + s;
      if (accC && (count & (count - 1)) == 0) accC[q] = acc;
      const int64_t p = (int64_t)s * L.pixelCount + idx;
      const float4 o = L.ps.out[p];
      if (overwrite)
      {
        acc = make_float4(o.x, o.y, o.z, 1.f);
        if (acc2) sq = make_float4(o.x * o.x, o.y * o.y, o.z * o.z, 0.f);
        continue;
      }
      acc.x += o.x;
      acc.y += o.y;
      acc.z += o.z;
      acc.w += 1.f;
      if (acc2)
      {
        sq.x += o.x * o.x;
        sq.y += o.y * o.y;
        sq.z += o.z * o.z;
      }
      if (accA)
      {
        const float4 va = L.ps.aovA[p];
        if (va.w != 0.f)
        {
          a.x += va.x; a.y += va.y; a.z += va.z; a.w += 1.f;
        }
        const float4 vn = L.ps.aovN[p];
        if (vn.w != 0.f)
        {
          nn.x += vn.x; nn.y += vn.y; nn.z += vn.z; nn.w += 1.f;
        }
      }
    }
    accum[q] = acc;
    if (acc2) acc2[q] = sq;
    if (accA)
    {
      accA[q] = a;
      accN[q] = nn;
    }
    // SH AOV: the four coefficient planes (an AccumBuffer3f each, weight 1 per sample).
    if (accSH && L.ps.sphOut)
    {
      float4 h[4];
      for (int k = 0; k < 4; ++k) h[k] = accSH[(int64_t)k * n + q];
      for (int s = 0; s < L.samples; ++s)
      {
        const float4* o = L.ps.sphOut + 3 * ((int64_t)s * L.pixelCount + idx);
        const float4 u = o[0], v = o[1], w = o[2];
        const float c[12] = {u.x, u.y, u.z, u.w, v.x, v.y, v.z, v.w, w.x, w.y, w.z, w.w};
        for (int k = 0; k < 4; ++k)
        {
          h[k].x += c[3 * k];
          h[k].y += c[3 * k + 1];
          h[k].z += c[3 * k + 2];
          h[k].w += 1.f;
        }
      }
      for (int k = 0; k < 4; ++k) accSH[(int64_t)k * n + q] = h[k];
    }
  }
}

// Tone mappers (image/*_tone_mapper.h): linear, Reinhard with burn, the ACES fit used by the
// reference (RRT + ODT approximation between its input and output matrices), Hable's filmic
// curve (white point 11.2, exposure bias 1.758141), log.
struct ToneMap
{
  int type;
  float exposure, invWhite2;

  PRT_D float filmic(float x) const
  {
    const float A = 0.22f, B = 0.30f, C = 0.10f, D = 0.20f, E = 0.01f, F = 0.30f;
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F;
  }

  PRT_D f3 apply(f3 c) const
  {
    if (type == PRT_TONE_NONE) return c;
    const f3 v = c * exposure;
    if (type == PRT_TONE_LINEAR) return v;
    if (type == PRT_TONE_REINHARD)
    {
      const f3 mapped = mk(v.x * (1.f + v.x * invWhite2) * (1.f / (1.f + v.x)),
                           v.y * (1.f + v.y * invWhite2) * (1.f / (1.f + v.y)),
                           v.z * (1.f + v.z * invWhite2) * (1.f / (1.f + v.z)));
      return mk(v.x * (mapped.x * rcpSafe(v.x)), v.y * (mapped.y * rcpSafe(v.y)), v.z * (mapped.z * rcpSafe(v.z)));
    }
    if (type == PRT_TONE_ACES)
    {
      const f3 x0 = mk(0.5972782409f, 0.0760130499f, 0.0284085382f) * v.x +
                    mk(0.3545713181f, 0.9083220973f, 0.1338243154f) * v.y +
                    mk(0.0482176639f, 0.0156579968f, 0.8375684636f) * v.z;
      const float a = 1.6773f, d = 0.9714f, b = 1.1174f, cc = 0.2447f;
      const f3 x1 = mk(powf(x0.x, a) / (powf(x0.x, a * d) * b + cc), powf(x0.y, a) / (powf(x0.y, a * d) * b + cc),
                       powf(x0.z, a) / (powf(x0.z, a * d) * b + cc));
      const f3 y = mk(1.6047539945f, -0.1020831870f, -0.0032670420f) * x1.x +
                   mk(-0.5310794927f, 1.1081322801f, -0.0727552477f) * x1.y +
                   mk(-0.0736720338f, -0.0060518756f, 1.0760219533f) * x1.z;
      return clamp01(y);
    }
    if (type == PRT_TONE_FILMIC)
    {
      const float ws = 1.f / filmic(11.2f);
      return mk(filmic(v.x), filmic(v.y), filmic(v.z)) * ws;
    }
    return mk(logf(v.x + 1.f), logf(v.y + 1.f), logf(v.z + 1.f)) * (1.f / 16.f);
  }
};

// encodeBgr8 (image/pixel.h:36-40): gamma 2.2, truncation to 0..255, blue in the low byte.
PRT_D uint32_t encodeBgr8(f3 c)
{
  const float g = 1.f / 2.2f;
  const int r = min(max(__float2int_rz(powf(c.x, g) * 255.f), 0), 255);
  const int gr = min(max(__float2int_rz(powf(c.y, g) * 255.f), 0), 255);
  const int b = min(max(__float2int_rz(powf(c.z, g) * 255.f), 0), 255);
  return (uint32_t)b | ((uint32_t)gr << 8) | ((uint32_t)r << 16);
}

__global__ void kBlitLdr(const float4* __restrict__ acc, int n, ToneMap tm, uint32_t* __restrict__ dst)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
  {
    const float4 a = acc[q];
    const float r = rcpSafe(a.w);
    dst[q] = encodeBgr8(tm.apply(mk(a.x * r, a.y * r, a.z * r)));
  }
}

// AccumBuffer::blitLdr(Vec3f*) (image/accum_buffer.h:681-733): tone-mapped, clamped to [0, 1].
__global__ void kBlitLdrRgb(const float4* __restrict__ acc, int n, ToneMap tm, float* __restrict__ dst)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
  {
    const float4 a = acc[q];
    const float r = rcpSafe(a.w);
    const f3 c = clamp01(tm.apply(mk(a.x * r, a.y * r, a.z * r)));
    dst[3 * q + 0] = c.x;
    dst[3 * q + 1] = c.y;
    dst[3 * q + 2] = c.z;
  }
}

// Sample variance max(sum2 - sum^2 / w, 0) / max(w - 1, 1) (image/accum_buffer.h:627-634).
__global__ void kBlitVariance(const float4* __restrict__ acc, const float4* __restrict__ acc2, int n,
                              float* __restrict__ dst)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
  {
    const float4 a = acc[q], b = acc2[q];
    const float r = rcpSafe(a.w);
    const float k = rcpSafe(fmaxf(a.w - 1.f, 1.f));
    dst[3 * q + 0] = fmaxf(b.x - a.x * a.x * r, 0.f) * k;
    dst[3 * q + 1] = fmaxf(b.y - a.y * a.y * r, 0.f) * k;
    dst[3 * q + 2] = fmaxf(b.z - a.z * a.z * r, 0.f) * k;
  }
}

// Per-block sums of the relative L1 error against the checkpoint (AccumBuffer::getError,
// image/accum_buffer.h:752-795), in a fixed tree order.
__global__ void __launch_bounds__(256) kFrameError(const float4* __restrict__ acc, const float4* __restrict__ accC,
                                                   int n, float scale, double* __restrict__ partials)
{
  __shared__ double s[256];
  double e = 0.0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
  {
    const float4 a = acc[q], c = accC[q];
    const float ra = rcpSafe(a.w), rc = rcpSafe(c.w);
    const f3 I = mk(a.x * ra, a.y * ra, a.z * ra) * scale;
    const f3 B = mk(c.x * rc, c.y * rc, c.z * rc) * scale;
    float norm = I.x + I.y + I.z;
    if (norm < 1.f) norm = sqrtf(norm);
    e += (double)((fabsf(I.x - B.x) + fabsf(I.y - B.y) + fabsf(I.z - B.z)) / (norm + 1e-4f));
  }
  s[threadIdx.x] = e;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1)
  {
    if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = s[0];
}

// sum * rcpSafe(weight) (image/accum_buffer.h:607-650).
__global__ void kBlit(const float4* __restrict__ acc, int n, float* __restrict__ dst)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
  {
    const float4 a = acc[q];
    const float r = rcpSafe(a.w);
    dst[3 * q + 0] = a.x * r;
    dst[3 * q + 1] = a.y * r;
    dst[3 * q + 2] = a.z * r;
  }
}

// ---- launchers --------------------------------------------------------------------------------

static int gridFor(const Context& ctx, int64_t n, int block = 256)
{
  const int64_t blocks = (n + block - 1) / block;
  const int64_t cap = (int64_t)ctx.smCount * 16;
  return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, cap));
}

cudaError_t launchSobol(Context& ctx, int64_t n, const uint32_t* si, const uint32_t* pid, const uint32_t* dims,
                        int ndim, float* out)
{
  kSobol<<<gridFor(ctx, n), 256, 0, ctx.stream>>>(n, si, pid, dims, ndim, ctx.renderer.seed, out);
  return cudaGetLastError();
}

cudaError_t launchTrace(Context& ctx, int64_t n, const float* rays, int32_t* triOut, float* t, float* u, float* v)
{
  kTraceRays<<<gridFor(ctx, n, 128), 128, 0, ctx.stream>>>(ctx.scene, n, reinterpret_cast<const float4*>(rays),
                                                            triOut, t, u, v, ctx.ps.err);
  return cudaGetLastError();
}

cudaError_t launchOccluded(Context& ctx, int64_t n, const float* rays, int32_t* occ)
{
  kOccludedRays<<<gridFor(ctx, n, 128), 128, 0, ctx.stream>>>(ctx.scene, n, reinterpret_cast<const float4*>(rays),
                                                               occ, ctx.ps.err);
  return cudaGetLastError();
}

cudaError_t launchPrimary(Context& ctx, uint32_t sampleIndex, float* raysOut, int32_t* triOut, float* t)
{
  const int n = ctx.width * ctx.height;
  kPrimary<<<gridFor(ctx, n, 128), 128, 0, ctx.stream>>>(ctx.scene, ctx.camera, ctx.width, ctx.height,
                                                          ctx.renderer.seed, sampleIndex,
                                                          reinterpret_cast<float4*>(raysOut), triOut, t, ctx.ps.err);
  return cudaGetLastError();
}

cudaError_t launchMicrofacetQuery(Context& ctx, int distribution, int64_t n, const float* in, float* out)
{
  kMicrofacetQuery<<<gridFor(ctx, n, 128), 128, 0, ctx.stream>>>(distribution, n, in, out);
  return cudaGetLastError();
}

cudaError_t launchBsdfQuery(Context& ctx, const DevMaterial& m, int mediumId, int64_t n, const float* tuples, float* out)
{
  kBsdfQuery<<<gridFor(ctx, n, 128), 128, 0, ctx.stream>>>(ctx.tables, m, mediumId, n, tuples, out);
  return cudaGetLastError();
}

// SH AOV blits (DeviceCpu::blitFrame, render/device_cpu.cpp:359-364): band 0 as the mean;
// bands 1-3 as their mean over max(band-0 mean, 1e-4) per channel (AccumBuffer3f::blitRel,
// image/accum_buffer.h:735-750).
__global__ void kBlitSh(const float4* __restrict__ acc0, const float4* __restrict__ acck, int n, int rel,
                        float* __restrict__ dst)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
  {
    const float4 a = acc0[q];
    const float ia = rcpSafe(a.w);
    f3 v = mk(a.x * ia, a.y * ia, a.z * ia);
    if (rel)
    {
      const float4 b = acck[q];
      const float ib = rcpSafe(b.w);
      v = mk(b.x * ib / fmaxf(v.x, 1e-4f), b.y * ib / fmaxf(v.y, 1e-4f), b.z * ib / fmaxf(v.z, 1e-4f));
    }
    dst[3 * q] = v.x;
    dst[3 * q + 1] = v.y;
    dst[3 * q + 2] = v.z;
  }
}

cudaError_t launchBlit(Context& ctx, int aov, float* dst)
{
  const int n = ctx.width * ctx.height;
  if (aov >= PRT_BLIT_SH0 && aov <= PRT_BLIT_SH3)
  {
    const float4* sh = reinterpret_cast<const float4*>(ctx.accumSH);
    const int k = aov - PRT_BLIT_SH0;
    kBlitSh<<<gridFor(ctx, n), 256, 0, ctx.stream>>>(sh, sh + (int64_t)k * n, n, k > 0 ? 1 : 0, dst);
    return cudaGetLastError();
  }
  const float* src = aov == 0 ? ctx.accum : (aov == 1 ? ctx.accumA : ctx.accumN);
  kBlit<<<gridFor(ctx, n), 256, 0, ctx.stream>>>(reinterpret_cast<const float4*>(src), n, dst);
  return cudaGetLastError();
}

cudaError_t launchClear(Context& ctx)
{
  const size_t bytes = (size_t)ctx.width * ctx.height * sizeof(float4);
  cudaError_t e = cudaMemsetAsync(ctx.accum, 0, bytes, ctx.stream);
  if (e == cudaSuccess && ctx.accumA) e = cudaMemsetAsync(ctx.accumA, 0, bytes, ctx.stream);
  if (e == cudaSuccess && ctx.accumN) e = cudaMemsetAsync(ctx.accumN, 0, bytes, ctx.stream);
  if (e == cudaSuccess && ctx.accumC) e = cudaMemsetAsync(ctx.accumC, 0, bytes, ctx.stream);
  if (e == cudaSuccess && ctx.accum2) e = cudaMemsetAsync(ctx.accum2, 0, bytes, ctx.stream);
  if (e == cudaSuccess && ctx.accumSH) e = cudaMemsetAsync(ctx.accumSH, 0, 4 * bytes, ctx.stream);
  ctx.accumCount = 0;
  return e;
}

cudaError_t launchBlitVariance(Context& ctx, float* dst)
{
  const int n = ctx.width * ctx.height;
  kBlitVariance<<<gridFor(ctx, n), 256, 0, ctx.stream>>>(reinterpret_cast<const float4*>(ctx.accum),
                                                          reinterpret_cast<const float4*>(ctx.accum2), n, dst);
  return cudaGetLastError();
}

static ToneMap toneMapOf(const Context& ctx)
{
  ToneMap tm;
  tm.type = ctx.toneType;
  tm.exposure = ctx.toneExposure;
  tm.invWhite2 = ctx.toneInvWhite2;
  return tm;
}

cudaError_t launchBlitLdr(Context& ctx, uint32_t* dst)
{
  const int n = ctx.width * ctx.height;
  kBlitLdr<<<gridFor(ctx, n), 256, 0, ctx.stream>>>(reinterpret_cast<const float4*>(ctx.accum), n, toneMapOf(ctx), dst);
  return cudaGetLastError();
}

cudaError_t launchBlitLdrRgb(Context& ctx, float* dst)
{
  const int n = ctx.width * ctx.height;
  kBlitLdrRgb<<<gridFor(ctx, n), 256, 0, ctx.stream>>>(reinterpret_cast<const float4*>(ctx.accum), n, toneMapOf(ctx),
                                                        dst);
  return cudaGetLastError();
}

cudaError_t frameError(Context& ctx, double& error)
{
  const int n = ctx.width * ctx.height;
  const int blocks = gridFor(ctx, n);
  // The reference scales by the tone mapper's exposure (Filmic's includes its bias).
  const float scale = ctx.toneType == PRT_TONE_NONE ? 1.f : ctx.toneExposure;
  kFrameError<<<blocks, 256, 0, ctx.stream>>>(reinterpret_cast<const float4*>(ctx.accum),
                                              reinterpret_cast<const float4*>(ctx.accumC), n, scale, ctx.errPartials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  std::vector<double> part(blocks);
  e = cudaMemcpyAsync(part.data(), ctx.errPartials, sizeof(double) * blocks, cudaMemcpyDeviceToHost, ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return e;
  double sum = 0.0;
  for (double v : part) sum += v;
  error = sum / (double)n;
  return cudaSuccess;
}

using ShadeClassList = ShadeLaunch<PRT_SHADE_CLASS_LIST>;
static_assert(kShadeClassFeatures[1] == kFeatOpaque && kShadeClassFeatures[7] == kFeatAll, "class list");

// Event pair recorded around one launch when kernel timing is on.
struct TimedLaunch
{
  cudaEvent_t a, b;
  int kind;  // 0 trace, 1 shadow, 2 shade
};

// Launches one surface-shading kernel per feature class (the class list is kShadeClassFeatures).
template <int... Fs>
struct ShadeLaunch;

template <>
struct ShadeLaunch<>
{
  template <bool Batch>
  static void run(int, const Launch&, cudaStream_t, int, int*, int*, int, int*, int*, int*, int)
  {
  }
};

template <int F0, int... Fs>
struct ShadeLaunch<F0, Fs...>
{
  template <bool Batch>
  static void run(int cls, const Launch& L, cudaStream_t st, int grid, int* classQueues, int* cnt, int depth,
                  int* queueOut, int* nextCount, int* shadowCount, int parity)
  {
    kShadeSurface<F0, Batch><<<grid, 256, 0, st>>>(L, classQueues + (int64_t)cls * L.ps.capacity, cnt + 1 + cls,
                                                   depth, queueOut, nextCount, shadowCount, parity);
    ShadeLaunch<Fs...>::template run<Batch>(cls + 1, L, st, grid, classQueues, cnt, depth, queueOut, nextCount,
                                            shadowCount, parity);
  }
};

using ShadeClassList = ShadeLaunch<PRT_SHADE_CLASS_LIST>;
static_assert(kShadeClassFeatures[1] == kFeatOpaque && kShadeClassFeatures[7] == kFeatAll, "class list");


// Traces one frame-form wave (kRaygen, then per bounce: closest hit, shading by class, shadow
// rays) until no path is left. replay = true runs the adjoint's replay instead: the same paths
// with the replay form of the shading kernels (classes 1 and 2, the adjoint's material set),
// which trace their shadow rays inline and scatter gradients.
template <class Begin, class End>
static cudaError_t bounceLoop(Context& ctx, const Launch& L, int P, bool replay, bool counting, Begin begin, End end,
                              RenderCounters& rc)
{
  const int maxDepth = ctx.renderer.maxDepth;
  int* counts = ctx.ps.counters;
  const int persistent = ctx.smCount * ctx.traceBlocks;
  const int shadeGrid = ctx.smCount * ctx.shadeBlocks;
  cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * kCntStride * (maxDepth + 2), ctx.stream);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(counts, &P, sizeof(int), cudaMemcpyHostToDevice, ctx.stream);
  if (e != cudaSuccess) return e;
  kRaygen<<<gridFor(ctx, P), 256, 0, ctx.stream>>>(L);
  rc.launches++;
  const bool bins = ctx.rayBins && ctx.ps.octBins;
  // The 24-entry traversal stack where the tree fits in it (the tree's wide depth bounds the
  // stack: one node group per level).
  const bool shared = ctx.traceStack <= kTraceStackShared && ctx.bvhDepth <= kTraceStackShared;
  const bool shallow = !shared && ctx.traceStack <= kTraceStackShallow && ctx.bvhDepth <= kTraceStackShallow;
  int inBuf = 1;  // queue buffer that holds this bounce's paths (camera rays need none)
  for (int depth = 0; depth <= maxDepth; ++depth)
  {
    int* cnt = counts + kCntStride * depth;
    int* next = counts + kCntStride * (depth + 1);
    const int* q = depth == 0 ? nullptr : ctx.ps.queue[inBuf];
    int* qOut = ctx.ps.queue[inBuf ^ 1];
    begin(0);
    if (counting)
      kTrace<true, false><<<persistent, 256, 0, ctx.stream>>>(L, q, cnt, cnt + kCntWorkTrace, depth,
                                                              ctx.ps.classQueues, cnt + 1);
    else if (ctx.topStage)
      kTrace<false, false, true><<<persistent, 256, 0, ctx.stream>>>(L, q, cnt, cnt + kCntWorkTrace, depth,
                                                                     ctx.ps.classQueues, cnt + 1);
    else if (shared)
      kTrace<false, false, false, kTraceStackShared><<<persistent, 256, 0, ctx.stream>>>(
        L, q, cnt, cnt + kCntWorkTrace, depth, ctx.ps.classQueues, cnt + 1);
    else if (shallow)
      kTrace<false, false, false, kTraceStackShallow><<<persistent, 256, 0, ctx.stream>>>(
        L, q, cnt, cnt + kCntWorkTrace, depth, ctx.ps.classQueues, cnt + 1);
    else
      kTrace<false, false><<<persistent, 256, 0, ctx.stream>>>(L, q, cnt, cnt + kCntWorkTrace, depth,
                                                               ctx.ps.classQueues, cnt + 1);
    end();
    begin(2);
    if (replay)
    {
      // Paths of class 0 (misses, emitters, maxDepth) carry no parameters: they are dropped.
      kShadeSurface<kShadeClassFeatures[1], false, true><<<shadeGrid, 256, 0, ctx.stream>>>(
        L, ctx.ps.classQueues + (int64_t)1 * ctx.ps.capacity, cnt + 2, depth, qOut, next, cnt + kCntShadow, 0);
      kShadeSurface<kShadeClassFeatures[2], false, true><<<shadeGrid, 256, 0, ctx.stream>>>(
        L, ctx.ps.classQueues + (int64_t)2 * ctx.ps.capacity, cnt + 3, depth, qOut, next, cnt + kCntShadow, 0);
      rc.launches += 3;
    }
    else
    {
      kShadeEnd<false><<<shadeGrid, 256, 0, ctx.stream>>>(L, ctx.ps.classQueues, cnt + 1, depth, 0);
      ShadeClassList::run<false>(1, L, ctx.stream, shadeGrid, ctx.ps.classQueues, cnt, depth, qOut, next,
                                 cnt + kCntShadow, 0);
      rc.launches += 1 + kShadeClasses;
    }
    end();
    if (!replay)
    {
      begin(1);
      if (L.anyTransparent)
      {
        if (counting)
          kShadow<true, false, false, true><<<persistent, 256, 0, ctx.stream>>>(L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
        else if (shared)
          kShadow<false, false, false, true, kTraceStackShared><<<persistent, 256, 0, ctx.stream>>>(
            L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
        else if (shallow)
          kShadow<false, false, false, true, kTraceStackShallow><<<persistent, 256, 0, ctx.stream>>>(
            L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
        else
          kShadow<false, false, false, true><<<persistent, 256, 0, ctx.stream>>>(L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
      }
      else if (counting)
        kShadow<true, false><<<persistent, 256, 0, ctx.stream>>>(L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
      else if (ctx.topStage)
        kShadow<false, false, true><<<persistent, 256, 0, ctx.stream>>>(L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
      else if (shared)
        kShadow<false, false, false, false, kTraceStackShared><<<persistent, 256, 0, ctx.stream>>>(
          L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
      else if (shallow)
        kShadow<false, false, false, false, kTraceStackShallow><<<persistent, 256, 0, ctx.stream>>>(
          L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
      else
        kShadow<false, false><<<persistent, 256, 0, ctx.stream>>>(L, cnt + kCntShadow, cnt + kCntWorkShadow, 0, depth);
      end();
      rc.launches++;
    }
    if (bins)
    {
      // Group the extended paths by direction octant into the buffer this bounce has read.
      e = cudaMemsetAsync(ctx.ps.octBins, 0, 16 * sizeof(int), ctx.stream);
      if (e != cudaSuccess) return e;
      kRayBinCount<<<shadeGrid, 256, 0, ctx.stream>>>(qOut, next, ctx.ps.octBins);
      kRayBinScatter<<<shadeGrid, 256, 0, ctx.stream>>>(qOut, next, ctx.ps.octBins, ctx.ps.queue[inBuf]);
      rc.launches += 2;
    }
    else
      inBuf ^= 1;
    rc.traceLaunches++;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // Paths in, shadow rays and paths out of this bounce; stop once no path is left.
    int in = 0, shadow = 0, out = 0;
    e = cudaMemcpyAsync(&in, cnt, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream);
    int shadowSun = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&shadow, cnt + kCntShadow, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&shadowSun, cnt + kCntShadowSun, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&out, next, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
    if (e != cudaSuccess) return e;
    rc.closestRays += in;
    rc.shadowRays += shadow + shadowSun;
    if (out == 0) break;
  }
  return cudaSuccess;
}

static Launch frameLaunch(const Context& ctx, uint32_t firstSample, int samples)
{
  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.sc = ctx.scene;
  L.tab = ctx.tables;
  L.cam = ctx.camera;
  L.rd = ctx.renderer;
  L.ps = ctx.ps;
  L.width = ctx.width;
  L.height = ctx.height;
  L.pixelCount = ctx.width * ctx.height;
  L.firstSample = firstSample;
  L.samples = samples;
  L.aovMask = ctx.aovMask;
  L.anyTransparent = ctx.scene.hasTransparent;
  L.white = ctx.whiteMaterialDev;
  L.whiteClass = ctx.whiteClass;
  return L;
}

cudaError_t renderSamples(Context& ctx, int spp, RenderCounters& rc)
{
  rc = RenderCounters();
  const int pixelCount = ctx.width * ctx.height;
  const bool timing = (ctx.profileFlags & 1) != 0;
  const bool counting = (ctx.profileFlags & 2) != 0;
  std::vector<TimedLaunch> timed;
  auto begin = [&](int kind) {
    if (!timing) return;
    TimedLaunch t;
    cudaEventCreate(&t.a);
    cudaEventCreate(&t.b);
    t.kind = kind;
    cudaEventRecord(t.a, ctx.stream);
    timed.push_back(t);
  };
  auto end = [&]() {
    if (timing) cudaEventRecord(timed.back().b, ctx.stream);
  };
  cudaError_t e = cudaSuccess;
  if (counting) e = cudaMemsetAsync(ctx.ps.travCounts, 0, 4 * sizeof(unsigned long long), ctx.stream);
  if (e != cudaSuccess) return e;
  const int type = ctx.renderer.type;
  unsigned long long simpleRays[2] = {0, 0};
  if (type != PRT_RENDERER_PATH)
  {
    e = cudaMemsetAsync(ctx.ps.travCounts, 0, 4 * sizeof(unsigned long long), ctx.stream);
    if (e != cudaSuccess) return e;
  }
  for (int done = 0; done < spp;)
  {
    const int S = std::min(ctx.waveSamples, spp - done);
    const Launch L = frameLaunch(ctx, ctx.sampleIndex + (uint32_t)done, S);
    if (type == PRT_RENDERER_PATH)
      e = bounceLoop(ctx, L, pixelCount * S, false, counting, begin, end, rc);
    else
    {
      const int P = pixelCount * S;
      begin(0);
      const int g = gridFor(ctx, P);
      switch (type)
      {
      case PRT_RENDERER_PRIMARY: kSimpleRender<1, false><<<g, 256, 0, ctx.stream>>>(L); break;
      case PRT_RENDERER_AO: kSimpleRender<2, false><<<g, 256, 0, ctx.stream>>>(L); break;
      case PRT_RENDERER_DIFFUSE: kSimpleRender<3, false><<<g, 256, 0, ctx.stream>>>(L); break;
      case PRT_RENDERER_DIFFUSE2: kSimpleRender<4, false><<<g, 256, 0, ctx.stream>>>(L); break;
      case PRT_RENDERER_PRIMARY_FAST: kSimpleRender<1, true><<<g, 256, 0, ctx.stream>>>(L); break;
      case PRT_RENDERER_AO_FAST: kSimpleRender<2, true><<<g, 256, 0, ctx.stream>>>(L); break;
      case PRT_RENDERER_DIFFUSE_FAST: kSimpleRender<3, true><<<g, 256, 0, ctx.stream>>>(L); break;
      default: kSimpleRender<4, true><<<g, 256, 0, ctx.stream>>>(L); break;
      }
      end();
      rc.launches++;
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    kAccumulate<<<gridFor(ctx, pixelCount), 256, 0, ctx.stream>>>(
      L, reinterpret_cast<float4*>(ctx.accum), reinterpret_cast<float4*>(ctx.accumA),
      reinterpret_cast<float4*>(ctx.accumN), reinterpret_cast<float4*>(ctx.accumC),
      reinterpret_cast<float4*>(ctx.accum2), (long long)ctx.accumCount, type >= PRT_RENDERER_PRIMARY_FAST ? 1 : 0,
      ctx.aovSh ? reinterpret_cast<float4*>(ctx.accumSH) : nullptr);
    ctx.accumCount += S;
    rc.launches++;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    done += S;
  }
  ctx.sampleIndex += (uint32_t)spp;
  if (type != PRT_RENDERER_PATH)
  {
    e = cudaMemcpyAsync(simpleRays, ctx.ps.travCounts, sizeof(simpleRays), cudaMemcpyDeviceToHost, ctx.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
    if (e != cudaSuccess) return e;
    rc.closestRays = (int64_t)simpleRays[0];
    rc.shadowRays = (int64_t)simpleRays[1];
  }
  if (timing || counting)
  {
    e = cudaStreamSynchronize(ctx.stream);
    if (e != cudaSuccess) return e;
  }
  for (auto& t : timed)
  {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t.a, t.b);
    (t.kind == 0 ? rc.traceMs : t.kind == 1 ? rc.shadowMs : rc.shadeMs) += ms;
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  if (counting)
  {
    e = cudaMemcpy(rc.trav, ctx.ps.travCounts, sizeof(rc.trav), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Path-replay adjoint of samples [firstSample, firstSample + spp): per wave, a forward pass
// that leaves each path's radiance in ps.out (nothing is accumulated into the frame), then the
// replay pass over the same paths.
cudaError_t launchAdjoint(Context& ctx, uint32_t firstSample, int spp, const float* dLdI, float* gradTex,
                          float* gradRough, float roughnessStep, RenderCounters& rc)
{
  rc = RenderCounters();
  AdjointView A;
  std::memset(&A, 0, sizeof(A));
  A.dLdI = dLdI;
  A.gradTex = gradTex;
  A.gradRough = gradRough;
  long long off = 0;
  for (size_t i = 0; i < ctx.texturesHost.size() && i < (size_t)kAdjointMaxTextures; ++i)
  {
    A.texOffset[i] = off;
    off += 3ll * ctx.texturesHost[i].width * ctx.texturesHost[i].height;
  }
  A.step = roughnessStep;
  A.invSpp = 1.f / (float)spp;
  auto none = [](int) {};
  auto none0 = []() {};
  const int pixelCount = ctx.width * ctx.height;
  for (int done = 0; done < spp;)
  {
    const int S = std::min(ctx.waveSamples, spp - done);
    Launch L = frameLaunch(ctx, firstSample + (uint32_t)done, S);
    L.aovMask = 0;
    cudaError_t e = bounceLoop(ctx, L, pixelCount * S, false, false, none, none0, rc);
    if (e != cudaSuccess) return e;
    L.adj = A;
    e = bounceLoop(ctx, L, pixelCount * S, true, false, none, none0, rc);
    if (e != cudaSuccess) return e;
    done += S;
  }
  return cudaSuccess;
}

// ---- batch form ---------------------------------------------------------------------------------

__global__ void kIota(int* __restrict__ dst, int n)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = i;
}

cudaError_t launchBlitPlane(Context& ctx, const float4* plane, int n, float* dst)
{
  kBlit<<<gridFor(ctx, n), 256, 0, ctx.stream>>>(plane, n, dst);
  return cudaGetLastError();
}

namespace {

constexpr int kGraphIterations = 8;  // bounce iterations per graph launch (even: parities alternate)

int* batchCounts(BatchCtl* ctl, int parity)
{
  return reinterpret_cast<int*>(reinterpret_cast<char*>(ctl) + offsetof(BatchCtl, counts)) + parity * kBatchCntStride;
}

// One bounce iteration of the batch: control step, regeneration, closest hit, shading by
// class, shadow rays. Every count is read on the device, so the sequence can be captured once
// and replayed.
int batchIteration(const Context& ctx, const Launch& L, int a, int persistent, int shadeGrid, int regenGrid, bool replay,
                   bool shared, bool shallow)
{
  const int b = a ^ 1;
  int* ca = batchCounts(L.ctl, a);
  int* cb = batchCounts(L.ctl, b);
  cudaStream_t st = ctx.stream;
  kBatchStep<<<1, 1, 0, st>>>(L.ctl, a);
  if (replay)
    kBatchRegen<true><<<regenGrid, 256, 0, st>>>(L, a, L.ps.queue[a]);
  else
    kBatchRegen<false><<<regenGrid, 256, 0, st>>>(L, a, L.ps.queue[a]);
  if (shared)
    kTrace<false, true, false, kTraceStackShared><<<persistent, 256, 0, st>>>(
      L, L.ps.queue[a], ca, ca + kBatchCntShadow + 1, 0, L.ps.classQueues, ca + 1);
  else if (shallow)
    kTrace<false, true, false, kTraceStackShallow><<<persistent, 256, 0, st>>>(
      L, L.ps.queue[a], ca, ca + kBatchCntShadow + 1, 0, L.ps.classQueues, ca + 1);
  else
    kTrace<false, true><<<persistent, 256, 0, st>>>(L, L.ps.queue[a], ca, ca + kBatchCntShadow + 1, 0,
                                                    L.ps.classQueues, ca + 1);
  if (replay)
  {
    // Adjoint replay: class-0 paths only return their slots; classes 1 and 2 (the adjoint's
    // material set) shade with inline shadow rays and scatter gradients.
    kShadeEnd<true, true><<<shadeGrid, 256, 0, st>>>(L, L.ps.classQueues, ca + 1, 0, a);
    kShadeSurface<kShadeClassFeatures[1], true, true><<<shadeGrid, 256, 0, st>>>(
      L, L.ps.classQueues + (int64_t)1 * L.ps.capacity, ca + 2, 0, L.ps.queue[b], cb, ca + kBatchCntShadow, a);
    kShadeSurface<kShadeClassFeatures[2], true, true><<<shadeGrid, 256, 0, st>>>(
      L, L.ps.classQueues + (int64_t)2 * L.ps.capacity, ca + 3, 0, L.ps.queue[b], cb, ca + kBatchCntShadow, a);
    return 6;
  }
  kShadeEnd<true><<<shadeGrid, 256, 0, st>>>(L, L.ps.classQueues, ca + 1, 0, a);
  ShadeClassList::run<true>(1, L, st, shadeGrid, L.ps.classQueues, ca, 0, L.ps.queue[b], cb, ca + kBatchCntShadow, a);
  if (L.anyTransparent && shared)
    kShadow<false, true, false, true, kTraceStackShared><<<persistent, 256, 0, st>>>(
      L, ca + kBatchCntShadow, ca + kBatchCntShadow + 2, a, 0);
  else if (L.anyTransparent && shallow)
    kShadow<false, true, false, true, kTraceStackShallow><<<persistent, 256, 0, st>>>(
      L, ca + kBatchCntShadow, ca + kBatchCntShadow + 2, a, 0);
  else if (L.anyTransparent)
    kShadow<false, true, false, true><<<persistent, 256, 0, st>>>(L, ca + kBatchCntShadow, ca + kBatchCntShadow + 2, a, 0);
  else if (shared)
    kShadow<false, true, false, false, kTraceStackShared><<<persistent, 256, 0, st>>>(
      L, ca + kBatchCntShadow, ca + kBatchCntShadow + 2, a, 0);
  else if (shallow)
    kShadow<false, true, false, false, kTraceStackShallow><<<persistent, 256, 0, st>>>(
      L, ca + kBatchCntShadow, ca + kBatchCntShadow + 2, a, 0);
  else
    kShadow<false, true><<<persistent, 256, 0, st>>>(L, ca + kBatchCntShadow, ca + kBatchCntShadow + 2, a, 0);
  return 5 + (kShadeClasses - 1);
}

} // namespace

static cudaError_t runBatch(Context& ctx, BatchState& B, RenderCounters& rc, bool replay)
{
  rc = RenderCounters();
  cudaError_t e = cudaSuccess;
  const int64_t C = B.ps.capacity;
  if (!replay)  // the replay only scatters gradients
  {
    // Work items that never finish (none should) then add nothing to their pixel.
    const size_t bytes = (size_t)B.workTotal * sizeof(float4);
    e = cudaMemsetAsync(B.workOut, 0, bytes, ctx.stream);
    if (e == cudaSuccess && B.workA) e = cudaMemsetAsync(B.workA, 0, bytes, ctx.stream);
    if (e == cudaSuccess && B.workN) e = cudaMemsetAsync(B.workN, 0, bytes, ctx.stream);
    if (e != cudaSuccess) return e;
  }
  BatchCtl h;
  std::memset(&h, 0, sizeof(h));
  h.workTotal = B.workTotal;
  h.freeCount[0] = (int)C;
  e = cudaMemcpyAsync(B.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, ctx.stream);
  if (e != cudaSuccess) return e;
  kIota<<<gridFor(ctx, C), 256, 0, ctx.stream>>>(B.freeList[0], (int)C);
  rc.launches++;
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;

  cudaGraphExec_t& exec = replay ? B.execReplay : B.exec;
  int& graphKernels = replay ? B.graphKernelsReplay : B.graphKernels;
  if (!exec)
  {
    Launch L;
    std::memset(&L, 0, sizeof(L));
    L.tab = ctx.tables;
    L.ps = B.ps;
    L.items = B.dItems;
    L.itemCount = (int)B.items.size();
    L.ctl = B.ctl;
    L.freeList[0] = B.freeList[0];
    L.freeList[1] = B.freeList[1];
    L.pathL = B.pathL;
    if (!replay)
    {
      L.workOut = B.workOut;
      L.workA = B.workA;
      L.workN = B.workN;
    }
    for (const BatchItem& it : B.items) L.anyTransparent |= it.sc.hasTransparent;
    const int persistent = ctx.smCount * ctx.traceBlocks;
    const int shadeGrid = ctx.smCount * ctx.shadeBlocks;
    const int regenGrid = gridFor(ctx, C);
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    int kernels = 0;
    const bool shared = ctx.traceStack <= kTraceStackShared && B.bvhDepth <= kTraceStackShared;
    const bool shallow = !shared && ctx.traceStack <= kTraceStackShallow && B.bvhDepth <= kTraceStackShallow;
    for (int k = 0; k < kGraphIterations; ++k)
      kernels += batchIteration(ctx, L, k & 1, persistent, shadeGrid, regenGrid, replay, shared, shallow);
    cudaError_t launchErr = cudaGetLastError();
    e = cudaStreamEndCapture(ctx.stream, &graph);
    if (e == cudaSuccess) e = launchErr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return e;
    graphKernels = kernels;
  }

  // Each slot finishes a path at least every maxDepth + 1 iterations while work remains.
  const long long rounds = (B.workTotal + C - 1) / C;
  const long long maxIterations = (rounds + 2) * (long long)(B.maxDepth + 2) + 2 * kGraphIterations;
  int* done = nullptr;
  e = cudaMallocHost(&done, sizeof(int));
  if (e != cudaSuccess) return e;
  long long iterations = 0;
  *done = 0;
  while (!*done)
  {
    if (iterations > maxIterations)
    {
      cudaFreeHost(done);
      return cudaErrorLaunchTimeout;
    }
    e = cudaGraphLaunch(exec, ctx.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(done, reinterpret_cast<char*>(B.ctl) + offsetof(BatchCtl, done), sizeof(int),
                          cudaMemcpyDeviceToHost, ctx.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
    if (e != cudaSuccess) break;
    iterations += kGraphIterations;
    rc.launches += graphKernels;
  }
  cudaFreeHost(done);
  if (e != cudaSuccess) return e;
  if (!replay)
  {
    for (int k = 0; k < (int)B.items.size(); ++k)
      kBatchAccumulate<<<gridFor(ctx, B.items[k].pixelCount), 256, 0, ctx.stream>>>(B.dItems, k, B.workOut, B.workA,
                                                                                      B.workN);
    rc.launches += (int)B.items.size();
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  e = cudaMemcpy(&h, B.ctl, sizeof(h), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  rc.closestRays = (int64_t)h.rays[0];
  rc.shadowRays = (int64_t)h.rays[1];
  rc.traceLaunches = iterations;
  return cudaSuccess;
}

cudaError_t renderBatch(Context& ctx, BatchState& B, RenderCounters& rc) { return runBatch(ctx, B, rc, false); }

cudaError_t replayBatch(Context& ctx, BatchState& B, RenderCounters& rc) { return runBatch(ctx, B, rc, true); }

} // namespace prt
