// Device BVH8 builder: Morton sort, PLOC clustering, level-by-level collapse to the compressed
// 8-wide format. See bvh_build.h for the algorithm and bvh8.h for the node format.
#include "bvh_build.h"
#include "bvh8.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <chrono>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace prt {
namespace {

void check(cudaError_t e, const char* what)
{
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("BVH8 device build: ") + what + ": " + cudaGetErrorString(e));
}

// Device buffers of one build, freed when the build returns (or throws).
struct Scratch
{
  std::vector<void*> bufs;
  ~Scratch()
  {
    for (void* p : bufs) cudaFree(p);
  }
  template <class T>
  T* alloc(size_t n)
  {
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
    bufs.push_back(p);
    return (T*)p;
  }
};

using u64 = unsigned long long;

// ---- scans ---------------------------------------------------------------------------------
// Exclusive prefix sums over tiles of 2048 values (256 threads x 8 consecutive values), with the
// tile totals scanned recursively and added back. T is uint32_t or u64; a u64 scan carries two
// 32-bit counts at once (high and low word never carry into each other for counts < 2^32).
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class T>
__device__ T warpInclusive(T v)
{
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1)
  {
    const T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; every thread of the block must call it.
template <class T, int Threads>
__device__ T blockExclusive(T v, T& total)
{
  static_assert(Threads % 32 == 0 && Threads <= 1024, "block size");
  constexpr int kWarps = Threads / 32;
  __shared__ T warpSums[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T inc = warpInclusive(v);
  if (lane == 31) warpSums[warp] = inc;
  __syncthreads();
  if (warp == 0)
  {
    T w = lane < kWarps ? warpSums[lane] : T(0);
    w = warpInclusive(w);
    if (lane < kWarps) warpSums[lane] = w;
  }
  __syncthreads();
  const T prefix = warp > 0 ? warpSums[warp - 1] : T(0);
  total = warpSums[kWarps - 1];
  __syncthreads();
  return prefix + inc - v;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) kScanTiles(const T* in, T* out, int64_t n, T* tileSums, T* total)
{
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T s = 0;
  for (int k = 0; k < kScanItems; ++k)
  {
    v[k] = base + k < n ? in[base + k] : T(0);
    s += v[k];
  }
  T tileTotal;
  T run = blockExclusive<T, kScanThreads>(s, tileTotal);
  for (int k = 0; k < kScanItems; ++k)
  {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0)
  {
    if (tileSums) tileSums[blockIdx.x] = tileTotal;
    if (total) *total = tileTotal;
  }
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) kAddTiles(T* out, int64_t n, const T* tileOffsets)
{
  const T add = tileOffsets[blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  for (int k = threadIdx.x; k < kScanTile; k += kScanThreads)
    if (base + k < n) out[base + k] += add;
}

template <class T>
struct Scanner
{
  T* levels[4] = {nullptr, nullptr, nullptr, nullptr};
  T* total = nullptr;  // device scalar: the sum of the last scan

  void init(Scratch& s, int64_t maxN)
  {
    int64_t m = maxN;
    for (int d = 0; d < 4; ++d)
    {
      m = std::max<int64_t>((m + kScanTile - 1) / kScanTile, 1);
      levels[d] = s.alloc<T>((size_t)m);
    }
    total = s.alloc<T>(1);
  }

  // Exclusive scan of n values (in == out allowed); the sum goes to `total`.
  void run(const T* in, T* out, int64_t n, cudaStream_t st, int depth = 0)
  {
    if (n <= 0)
    {
      check(cudaMemsetAsync(total, 0, sizeof(T), st), "scan");
      return;
    }
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1)
    {
      kScanTiles<T><<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, total);
      return;
    }
    if (depth >= 3) throw std::runtime_error("BVH8 device build: scan too large");
    kScanTiles<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, levels[depth], nullptr);
    run(levels[depth], levels[depth], tiles, st, depth + 1);
    kAddTiles<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(out, n, levels[depth]);
  }
};

// ---- boxes and Morton codes ------------------------------------------------------------------

__device__ __forceinline__ uint32_t orderedBits(float f)
{
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float fromOrdered(uint32_t u)
{
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ float boxArea(float3 lo, float3 hi)
{
  const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
  if (dx < 0.f) return 0.f;
  return 2.f * (dx * dy + dy * dz + dz * dx);
}

__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }

__global__ void kFillU32(uint32_t* p, int n, uint32_t v0, uint32_t v1, int split)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i < split ? v0 : v1;
}

// Triangle boxes as the traversal sees the triangle: v0, v0 + (v1 - v0) and v0 + (v2 - v0)
// reconstructed in single precision next to v1 and v2 (the host builder's rule), plus the
// centroid bounds (ordered-integer atomics, order-independent).
__global__ void kTriBoxes(const float4* __restrict__ pos, const int4* __restrict__ tv, int64_t n,
                          float4* __restrict__ boxLo, float4* __restrict__ boxHi, uint32_t* cb)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float cmn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (t < n)
  {
    const int4 id = tv[t];
    const float4 a = pos[id.x], b = pos[id.y], c = pos[id.z];
    const float va[3] = {a.x, a.y, a.z}, vb[3] = {b.x, b.y, b.z}, vc[3] = {c.x, c.y, c.z};
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k)
    {
      const float r1 = __fadd_rn(va[k], __fsub_rn(vb[k], va[k]));
      const float r2 = __fadd_rn(va[k], __fsub_rn(vc[k], va[k]));
      lo[k] = fminf(fminf(va[k], r1), fminf(r2, fminf(vb[k], vc[k])));
      hi[k] = fmaxf(fmaxf(va[k], r1), fmaxf(r2, fmaxf(vb[k], vc[k])));
      cmn[k] = cmx[k] = 0.5f * (lo[k] + hi[k]);
    }
    boxLo[t] = make_float4(lo[0], lo[1], lo[2], 0.f);
    boxHi[t] = make_float4(hi[0], hi[1], hi[2], 0.f);
  }
  for (int k = 0; k < 3; ++k)
    for (int o = 16; o > 0; o >>= 1)
    {
      cmn[k] = fminf(cmn[k], __shfl_xor_sync(0xffffffffu, cmn[k], o));
      cmx[k] = fmaxf(cmx[k], __shfl_xor_sync(0xffffffffu, cmx[k], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k)
    {
      atomicMin(&cb[k], orderedBits(cmn[k]));
      atomicMax(&cb[3 + k], orderedBits(cmx[k]));
    }
}

// Morton codes: 21 bits per axis in a 63-bit key (PRT_MORTON_BITS 63, the default) or 10 bits
// per axis in a 30-bit key. Dense clusters of small triangles (a finely tessellated sphere
// inside one coarse cell) need the longer code: with equal keys the sort falls back to the
// triangle index, which loses their spatial order.
#ifndef PRT_MORTON_BITS
#define PRT_MORTON_BITS 63
#endif
constexpr int kMortonBits = PRT_MORTON_BITS;
static_assert(kMortonBits == 63 || kMortonBits == 30, "Morton code length");
using MortonKey = std::conditional_t<kMortonBits == 63, u64, uint32_t>;

__device__ __forceinline__ uint32_t spreadBits10(uint32_t x)
{
  x &= 1023u;
  x = (x | (x << 16)) & 0x030000FFu;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__device__ __forceinline__ u64 spreadBits21(u64 x)
{
  x &= 0x1fffffull;
  x = (x | (x << 32)) & 0x001f00000000ffffull;
  x = (x | (x << 16)) & 0x001f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// Morton code of the box centre in the centroid bounds, scaled uniformly by the largest extent
// so that a flat or long scene keeps its spatial neighbourhoods.
__global__ void kMorton(const float4* __restrict__ boxLo, const float4* __restrict__ boxHi, int64_t n,
                        const uint32_t* __restrict__ cb, MortonKey* __restrict__ keys, uint32_t* __restrict__ vals)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float4 lo = boxLo[t], hi = boxHi[t];
  const float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
  float mn[3], ext = 0.f;
  for (int k = 0; k < 3; ++k)
  {
    mn[k] = fromOrdered(cb[k]);
    ext = fmaxf(ext, fromOrdered(cb[3 + k]) - mn[k]);
  }
  constexpr int kAxisBits = kMortonBits / 3;
  constexpr uint32_t kCells = 1u << kAxisBits;
  const float scale = ext > 0.f ? (float)kCells / ext : 0.f;
  uint32_t q[3];
  for (int k = 0; k < 3; ++k)
  {
    const float f = (c[k] - mn[k]) * scale;
    q[k] = f > 0.f ? min((uint32_t)f, kCells - 1u) : 0u;
  }
  if constexpr (kMortonBits == 63)
    keys[t] = (spreadBits21(q[0]) << 2) | (spreadBits21(q[1]) << 1) | spreadBits21(q[2]);
  else
    keys[t] = (spreadBits10(q[0]) << 2) | (spreadBits10(q[1]) << 1) | spreadBits10(q[2]);
  vals[t] = (uint32_t)t;
}

// ---- stable LSD radix sort of (key, value) pairs, 8 bits per pass ------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;

// Per-tile digit counts, stored digit-major (hist[digit * tiles + tile]) so that one exclusive
// scan gives every (digit, tile) its first output position.
template <class K>
__global__ void __launch_bounds__(kSortThreads) kRadixHist(const K* __restrict__ keys, int64_t n, int shift,
                                                           uint32_t* __restrict__ hist, int tiles)
{
  __shared__ uint32_t cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kSortTile;
  for (int k = threadIdx.x; k < kSortTile; k += kSortThreads)
    if (base + k < n) atomicAdd(&cnt[(uint32_t)(keys[base + k] >> shift) & 255u], 1u);
  __syncthreads();
  hist[(int64_t)threadIdx.x * tiles + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter: warp w of a tile ranks its 256 keys in input order (8 rounds of 32, lanes
// with equal digits found with __match_any_sync), the warps' counts are prefixed in warp order,
// and the tile's base for each digit comes from the scanned histogram.
template <class K>
__global__ void __launch_bounds__(kSortThreads) kRadixScatter(const K* __restrict__ keysIn,
                                                              const uint32_t* __restrict__ valsIn,
                                                              K* __restrict__ keysOut,
                                                              uint32_t* __restrict__ valsOut, int64_t n, int shift,
                                                              const uint32_t* __restrict__ offsets, int tiles)
{
  __shared__ uint32_t warpCnt[kSortWarps][256];
  __shared__ uint32_t tileBase[256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < kSortWarps * 256; k += kSortThreads) (&warpCnt[0][0])[k] = 0u;
  tileBase[threadIdx.x] = offsets[(int64_t)threadIdx.x * tiles + blockIdx.x];
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * 32 * kSortItems;
  const unsigned below = (1u << lane) - 1u;
  K key[kSortItems];
  uint32_t val[kSortItems], rank[kSortItems];
  for (int k = 0; k < kSortItems; ++k)
  {
    const int64_t i = base + k * 32 + lane;
    const bool ok = i < n;
    key[k] = ok ? keysIn[i] : K(0);
    val[k] = ok ? valsIn[i] : 0u;
    const uint32_t digit = ok ? (uint32_t)(key[k] >> shift) & 255u : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, digit);
    const int leader = __ffs(peers) - 1;
    uint32_t prior = 0u;
    if (lane == leader && ok)
    {
      prior = warpCnt[warp][digit];
      warpCnt[warp][digit] = prior + (uint32_t)__popc(peers);
    }
    prior = __shfl_sync(0xffffffffu, prior, leader);
    rank[k] = prior + (uint32_t)__popc(peers & below);
    __syncwarp();
  }
  __syncthreads();
  {
    uint32_t run = 0u;
    for (int w = 0; w < kSortWarps; ++w)
    {
      const uint32_t c = warpCnt[w][threadIdx.x];
      warpCnt[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
  for (int k = 0; k < kSortItems; ++k)
  {
    const int64_t i = base + k * 32 + lane;
    if (i >= n) continue;
    const uint32_t digit = (uint32_t)(key[k] >> shift) & 255u;
    const uint32_t dst = tileBase[digit] + warpCnt[warp][digit] + rank[k];
    keysOut[dst] = key[k];
    valsOut[dst] = val[k];
  }
}

// ---- PLOC clustering ---------------------------------------------------------------------------
// Binary nodes: leaves 0..n-1 (one triangle each, in Morton order), inner nodes after them in
// creation order, so a node's children always have smaller indices and are complete when the
// node is made. Per node: box (lo, hi), hi.w = bits of (triangle count | kLeafFlag), child =
// (left, right) or (-1, triangle), and the table of the wide collapse below.
//
// Wide collapse (Ylitie, Karras and Laine 2017, "Efficient Incoherent Ray Traversal on GPUs
// Through Compressed Wide BVHs", section 3): C(n, i) is the least SAH cost of representing the
// subtree n by at most i children of a wide node,
//   C(n, 1) = min(Cleaf(n), Cinner(n)),   C(n, i) = min(C(n, i - 1), Cdist(n, i)),
//   Cdist(n, j) = min over k = 1..j-1 of C(left, k) + C(right, j - k),
//   Cleaf(n) = area * triangles * kTriCost for at most kMaxLeafTris triangles (else none),
//   Cinner(n) = area * kNodeCost + Cdist(n, 8),
// with the decision of each entry kept in one byte: for i = 1 kLeafDecision or kInnerDecision |
// (slots of the left child in Cdist(n, 8)); for i > 1 0 = take C(n, i - 1), k = split the i
// slots k : i - k between the children. The table is filled when a node is merged (its
// children's tables are final then), and the top-down collapse follows the decisions.
// kLeafFlag marks the nodes whose C(n, 1) is a leaf: a single triangle or a subtree stored as
// one leaf of at most kMaxLeafTris triangles.
constexpr uint32_t kLeafFlag = 0x80000000u;
constexpr uint32_t kMaxLeafTris = 3;
#ifndef PRT_TRI_COST
#define PRT_TRI_COST 0.6f
#endif
constexpr float kNodeCost = 1.0f;
constexpr float kTriCost = PRT_TRI_COST;
constexpr uint32_t kLeafDecision = 0x40u;
constexpr uint32_t kInnerDecision = 0x80u;
#ifndef PRT_PLOC_RADIUS
#define PRT_PLOC_RADIUS 16
#endif
constexpr int kPlocRadius = PRT_PLOC_RADIUS;  // neighbour window on each side in the Morton order
constexpr int kNearestThreads = 256;
constexpr int kTailThreads = 1024;     // the in-block tail: one CTA clusters the last kTailMax
constexpr int kTailItems = 4;
constexpr int kTailMax = kTailThreads * kTailItems;
constexpr size_t kTailSmem = (size_t)kTailMax * (6 * sizeof(float) + 2 * sizeof(int));

struct BinNodes
{
  float4* lo;      // xyz box minimum, w = C(n, 1)
  float4* hi;      // xyz box maximum, w = bits of (triangles | kLeafFlag)
  int2* child;     // (left, right), or (-1, triangle index) for a triangle
  float4* costA;   // C(n, 1..4)
  float4* costB;   // C(n, 5..8)
  uint2* dec;      // decision bytes of C(n, 1..8)
};

__device__ __forceinline__ bool isLeafNode(float4 hi) { return (__float_as_uint(hi.w) & kLeafFlag) != 0u; }
__device__ __forceinline__ uint32_t nodeTris(float4 hi) { return __float_as_uint(hi.w) & ~kLeafFlag; }
__device__ __forceinline__ uint32_t decisionByte(uint2 d, int i)  // i = 0..7 for C(n, i + 1)
{
  return ((i < 4 ? d.x : d.y) >> (8 * (i & 3))) & 0xffu;
}

__global__ void kInitLeaves(const uint32_t* __restrict__ sortedTri, const float4* __restrict__ boxLo,
                            const float4* __restrict__ boxHi, int64_t n, BinNodes N, int* __restrict__ cid,
                            float4* __restrict__ cLo, float4* __restrict__ cHi)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t tri = sortedTri[i];
  const float4 lo = boxLo[tri], hi = boxHi[tri];
  const float c = boxArea(xyz(lo), xyz(hi)) * kTriCost;
  N.lo[i] = make_float4(lo.x, lo.y, lo.z, c);
  N.hi[i] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(1u | kLeafFlag));
  N.child[i] = make_int2(-1, (int)tri);
  N.costA[i] = make_float4(c, c, c, c);
  N.costB[i] = make_float4(c, c, c, c);
  N.dec[i] = make_uint2(kLeafDecision, 0u);
  cid[i] = (int)i;
  cLo[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
  cHi[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
}

// Writes the inner node `id` over children l and r (merged box lo/hi) with its collapse table.
__device__ __forceinline__ void makeInner(int id, int l, int r, float3 lo, float3 hi, const BinNodes& N)
{
  const float4 la = N.costA[l], lb = N.costB[l], ra = N.costA[r], rb = N.costB[r];
  const float cl[8] = {la.x, la.y, la.z, la.w, lb.x, lb.y, lb.z, lb.w};
  const float cr[8] = {ra.x, ra.y, ra.z, ra.w, rb.x, rb.y, rb.z, rb.w};
  const uint32_t cnt = nodeTris(N.hi[l]) + nodeTris(N.hi[r]);
  const float a = boxArea(lo, hi);
  float dist[9];
  uint32_t split[9];
  for (int j = 2; j <= 8; ++j)
  {
    float best = cl[0] + cr[j - 2];
    uint32_t kb = 1u;
    for (int k = 2; k < j; ++k)
    {
      const float c = cl[k - 1] + cr[j - k - 1];
      if (c < best)
      {
        best = c;
        kb = (uint32_t)k;
      }
    }
    dist[j] = best;
    split[j] = kb;
  }
  const float cInner = a * kNodeCost + dist[8];
  const bool leaf = cnt <= kMaxLeafTris && a * (float)cnt * kTriCost <= cInner;
  float c[8];
  uint32_t d[8];
  c[0] = leaf ? a * (float)cnt * kTriCost : cInner;
  d[0] = leaf ? kLeafDecision : (kInnerDecision | split[8]);
  for (int i = 1; i < 8; ++i)
  {
    const bool take = dist[i + 1] < c[i - 1];
    c[i] = take ? dist[i + 1] : c[i - 1];
    d[i] = take ? split[i + 1] : 0u;
  }
  N.lo[id] = make_float4(lo.x, lo.y, lo.z, c[0]);
  N.hi[id] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(cnt | (leaf ? kLeafFlag : 0u)));
  N.child[id] = make_int2(l, r);
  N.costA[id] = make_float4(c[0], c[1], c[2], c[3]);
  N.costB[id] = make_float4(c[4], c[5], c[6], c[7]);
  N.dec[id] = make_uint2(d[0] | (d[1] << 8) | (d[2] << 16) | (d[3] << 24), d[4] | (d[5] << 8) | (d[6] << 16) | (d[7] << 24));
}

__device__ __forceinline__ float mergedArea(float3 alo, float3 ahi, float3 blo, float3 bhi)
{
  return boxArea(make_float3(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z)),
                 make_float3(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z)));
}

// Nearest neighbour of each cluster: the cluster j within kPlocRadius positions whose merged box
// has the smallest surface area (ties to the smaller j). With `force` set, clusters pair with
// their Morton-order neighbour (2k, 2k+1) instead: used after an iteration that merged fewer
// than 1/64 of the clusters, so that degenerate inputs (many equal boxes) still halve each time.
__global__ void __launch_bounds__(kNearestThreads) kNearest(const float4* __restrict__ cLo,
                                                            const float4* __restrict__ cHi, int count,
                                                            int* __restrict__ nn, int force)
{
  constexpr int kSpan = kNearestThreads + 2 * kPlocRadius;
  __shared__ float3 sLo[kSpan], sHi[kSpan];
  const int begin = blockIdx.x * kNearestThreads - kPlocRadius;
  for (int k = threadIdx.x; k < kSpan; k += kNearestThreads)
  {
    const int j = begin + k;
    if (j >= 0 && j < count)
    {
      sLo[k] = xyz(cLo[j]);
      sHi[k] = xyz(cHi[j]);
    }
  }
  __syncthreads();
  const int i = blockIdx.x * kNearestThreads + threadIdx.x;
  if (i >= count) return;
  if (force)
  {
    nn[i] = (i ^ 1) < count ? (i ^ 1) : i;
    return;
  }
  const int li = threadIdx.x + kPlocRadius;
  const float3 lo = sLo[li], hi = sHi[li];
  u64 best = ~0ull;
  for (int d = 1; d <= kPlocRadius; ++d)
  {
    if (i - d >= 0)
    {
      const float a = mergedArea(lo, hi, sLo[li - d], sHi[li - d]);
      best = min(best, ((u64)__float_as_uint(a) << 32) | (uint32_t)(i - d));
    }
    if (i + d < count)
    {
      const float a = mergedArea(lo, hi, sLo[li + d], sHi[li + d]);
      best = min(best, ((u64)__float_as_uint(a) << 32) | (uint32_t)(i + d));
    }
  }
  nn[i] = best == ~0ull ? i : (int)(uint32_t)best;
}

// Per cluster: (merges here << 32) | (survives). A mutual pair i < j merges at i; j disappears.
__global__ void kMergeFlags(const int* __restrict__ nn, int count, u64* __restrict__ flags)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int j = nn[i];
  const bool mutual = j != i && nn[j] == i;
  flags[i] = ((u64)(mutual && i < j) << 32) | (u64)(!(mutual && i > j));
}

// Creates the merged nodes (ids in cluster order after nodeBase) and compacts the survivors.
__global__ void kCompact(const int* __restrict__ nn, int count, const u64* __restrict__ scan,
                         const int* __restrict__ cidIn, const float4* __restrict__ cLoIn,
                         const float4* __restrict__ cHiIn, int* __restrict__ cidOut, float4* __restrict__ cLoOut,
                         float4* __restrict__ cHiOut, BinNodes N, int nodeBase)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int j = nn[i];
  const bool mutual = j != i && nn[j] == i;
  if (mutual && i > j) return;
  const u64 s = scan[i];
  const uint32_t pos = (uint32_t)s;
  if (mutual)
  {
    const int id = nodeBase + (int)(s >> 32);
    const float4 al = cLoIn[i], ah = cHiIn[i], bl = cLoIn[j], bh = cHiIn[j];
    const float3 lo = make_float3(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z));
    const float3 hi = make_float3(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z));
    makeInner(id, cidIn[i], cidIn[j], lo, hi, N);
    cidOut[pos] = id;
    cLoOut[pos] = make_float4(lo.x, lo.y, lo.z, 0.f);
    cHiOut[pos] = make_float4(hi.x, hi.y, hi.z, 0.f);
  }
  else
  {
    cidOut[pos] = cidIn[i];
    cLoOut[pos] = cLoIn[i];
    cHiOut[pos] = cHiIn[i];
  }
}

// The last <= kTailMax clusters, clustered to the root by one CTA in shared memory with the same
// rules (nearest neighbour, mutual merge, forced pairing after a poor iteration). Thread t owns
// clusters 4t..4t+3, so a block scan over the threads keeps the cluster order. All reads of an
// iteration go to registers before any write, so one buffer suffices.
// result: [0] root node, [1] iterations, [2] next free node index.
__global__ void __launch_bounds__(kTailThreads, 1) kPlocTail(int count, int force, const int* __restrict__ cid,
                                                             const float4* __restrict__ cLo,
                                                             const float4* __restrict__ cHi, BinNodes N,
                                                             int nodeBase, int* result)
{
  extern __shared__ float tailSmem[];
  float* lx = tailSmem;
  float* ly = lx + kTailMax;
  float* lz = ly + kTailMax;
  float* hx = lz + kTailMax;
  float* hy = hx + kTailMax;
  float* hz = hy + kTailMax;
  int* ids = reinterpret_cast<int*>(hz + kTailMax);
  int* nn = ids + kTailMax;
  for (int i = threadIdx.x; i < count; i += kTailThreads)
  {
    const float4 a = cLo[i], b = cHi[i];
    lx[i] = a.x; ly[i] = a.y; lz[i] = a.z;
    hx[i] = b.x; hy[i] = b.y; hz[i] = b.z;
    ids[i] = cid[i];
  }
  int iters = 0;
  while (count > 1)
  {
    __syncthreads();
    for (int k = 0; k < kTailItems; ++k)
    {
      const int i = threadIdx.x * kTailItems + k;
      if (i >= count) break;
      if (force)
      {
        nn[i] = (i ^ 1) < count ? (i ^ 1) : i;
        continue;
      }
      const float3 lo = make_float3(lx[i], ly[i], lz[i]), hi = make_float3(hx[i], hy[i], hz[i]);
      u64 best = ~0ull;
      const int j0 = max(i - kPlocRadius, 0), j1 = min(i + kPlocRadius, count - 1);
      for (int j = j0; j <= j1; ++j)
      {
        if (j == i) continue;
        const float a = mergedArea(lo, hi, make_float3(lx[j], ly[j], lz[j]), make_float3(hx[j], hy[j], hz[j]));
        best = min(best, ((u64)__float_as_uint(a) << 32) | (uint32_t)j);
      }
      nn[i] = best == ~0ull ? i : (int)(uint32_t)best;
    }
    __syncthreads();
    // (merge << 16) | survive per cluster; counts stay below 2^16.
    uint32_t f[kTailItems], sum = 0u;
    for (int k = 0; k < kTailItems; ++k)
    {
      const int i = threadIdx.x * kTailItems + k;
      f[k] = 0u;
      if (i < count)
      {
        const int j = nn[i];
        const bool mutual = j != i && nn[j] == i;
        f[k] = ((uint32_t)(mutual && i < j) << 16) | (uint32_t)(!(mutual && i > j));
      }
      sum += f[k];
    }
    uint32_t tot;
    uint32_t run = blockExclusive<uint32_t, kTailThreads>(sum, tot);
    int outId[kTailItems], outPos[kTailItems];
    float3 outLo[kTailItems], outHi[kTailItems];
    for (int k = 0; k < kTailItems; ++k)
    {
      const int i = threadIdx.x * kTailItems + k;
      outPos[k] = -1;
      if (i < count && (f[k] & 0xffffu))
      {
        outPos[k] = (int)(run & 0xffffu);
        const float3 lo = make_float3(lx[i], ly[i], lz[i]), hi = make_float3(hx[i], hy[i], hz[i]);
        if (f[k] >> 16)
        {
          const int j = nn[i];
          const float3 blo = make_float3(lx[j], ly[j], lz[j]), bhi = make_float3(hx[j], hy[j], hz[j]);
          outLo[k] = make_float3(fminf(lo.x, blo.x), fminf(lo.y, blo.y), fminf(lo.z, blo.z));
          outHi[k] = make_float3(fmaxf(hi.x, bhi.x), fmaxf(hi.y, bhi.y), fmaxf(hi.z, bhi.z));
          outId[k] = nodeBase + (int)(run >> 16);
          makeInner(outId[k], ids[i], ids[j], outLo[k], outHi[k], N);
        }
        else
        {
          outLo[k] = lo;
          outHi[k] = hi;
          outId[k] = ids[i];
        }
      }
      run += f[k];
    }
    __syncthreads();
    for (int k = 0; k < kTailItems; ++k)
    {
      const int p = outPos[k];
      if (p < 0) continue;
      lx[p] = outLo[k].x; ly[p] = outLo[k].y; lz[p] = outLo[k].z;
      hx[p] = outHi[k].x; hy[p] = outHi[k].y; hz[p] = outHi[k].z;
      ids[p] = outId[k];
    }
    const int merges = (int)(tot >> 16);
    force = merges * 64 < count;
    nodeBase += merges;
    count = (int)(tot & 0xffffu);
    ++iters;
  }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    result[0] = count == 1 ? ids[0] : -1;
    result[1] = iters;
    result[2] = nodeBase;
  }
}

// ---- collapse to 8-wide nodes ------------------------------------------------------------------
constexpr int kCollapseThreads = 128;

// Children of the wide node over binary node b, from the collapse table: a leaf-flagged b (a
// tree of at most kMaxLeafTris triangles) is one leaf child; otherwise b's eight slots are split
// between its children as C(b, 1) recorded, and each (node, slots) pair is resolved by its own
// decisions until it is one child -- a leaf or the root of a wide subtree. Children go to octant
// slots greedily by dot(child centre - node centre, slot direction), largest first (bvh8.cpp's
// assignment). slotNode[8w + s] = binary node in slot s or -1; counts[w] = (inner children << 32)
// | triangles.
__global__ void __launch_bounds__(kCollapseThreads) kCollapsePlan(const int* __restrict__ work, int m, BinNodes N,
                                                                  int* __restrict__ slotNode, u64* __restrict__ counts)
{
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= m) return;
  const int b = work[w];
  const float4 blo = N.lo[b], bhi = N.hi[b];
  int ch[8];
  bool inner[8];
  int n = 0;
  if (isLeafNode(bhi))
  {
    ch[0] = b;
    inner[0] = false;
    n = 1;
  }
  else
  {
    // Pending (node, slots) pairs; their slots sum to at most 8, so at most 8 are pending.
    int sn[8], si[8];
    int sp = 0;
    const uint32_t k0 = decisionByte(N.dec[b], 0) & 15u;
    const int2 c = N.child[b];
    sn[sp] = c.y; si[sp++] = 8 - (int)k0;
    sn[sp] = c.x; si[sp++] = (int)k0;
    while (sp > 0 && n < 8)
    {
      const int x = sn[--sp];
      int i = si[sp];
      const uint2 d = N.dec[x];
      while (i > 1 && decisionByte(d, i - 1) == 0u) --i;
      if (i <= 1)
      {
        ch[n] = x;
        inner[n] = (decisionByte(d, 0) & kInnerDecision) != 0u;
        ++n;
        continue;
      }
      const int k = (int)decisionByte(d, i - 1);
      const int2 cx = N.child[x];
      if (sp + 2 > 8) break;  // cannot happen: pending slots never exceed 8
      sn[sp] = cx.y; si[sp++] = i - k;
      sn[sp] = cx.x; si[sp++] = k;
    }
  }
  float cost[8][8];
  for (int i = 0; i < n; ++i)
  {
    const float4 lo = N.lo[ch[i]], hi = N.hi[ch[i]];
    const float d[3] = {0.5f * (lo.x + hi.x) - 0.5f * (blo.x + bhi.x), 0.5f * (lo.y + hi.y) - 0.5f * (blo.y + bhi.y),
                        0.5f * (lo.z + hi.z) - 0.5f * (blo.z + bhi.z)};
    for (int s = 0; s < 8; ++s)
    {
      float c = 0.f;
      for (int k = 0; k < 3; ++k) c += ((s >> k) & 1) ? -d[k] : d[k];
      cost[i][s] = c;
    }
  }
  int childOfSlot[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
  unsigned usedChild = 0u;
  for (int round = 0; round < n; ++round)
  {
    float best = -FLT_MAX;
    int bi = -1, bs = -1;
    for (int i = 0; i < n; ++i)
    {
      if (usedChild & (1u << i)) continue;
      for (int s = 0; s < 8; ++s)
      {
        if (childOfSlot[s] >= 0) continue;
        if (cost[i][s] > best || bi < 0)
        {
          best = cost[i][s];
          bi = i;
          bs = s;
        }
      }
    }
    usedChild |= 1u << bi;
    childOfSlot[bs] = bi;
  }
  uint32_t innerN = 0u, triN = 0u;
  for (int s = 0; s < 8; ++s)
  {
    const int ci = childOfSlot[s];
    slotNode[8 * w + s] = ci >= 0 ? ch[ci] : -1;
    if (ci < 0) continue;
    if (inner[ci]) ++innerN;
    else triN += nodeTris(N.hi[ch[ci]]);
  }
  counts[w] = ((u64)innerN << 32) | triN;
}

// Quantisation frame of one axis: origin lo and the smallest power-of-two scale 2^(e-127) with
// extent / scale <= 253, leaving room to round child bounds outward (bvh8.cpp's rule).
__device__ bool quantAxisD(float lo, float hi, float& p, uint8_t& e)
{
  p = lo;
  const double ext = (double)hi - (double)lo;
  int ex = -126;
  if (ext > 0.0)
  {
    int k;
    const double m = frexp(ext / 253.0, &k);  // ext / 253 = m * 2^k, m in [0.5, 1)
    ex = m == 0.5 ? k - 1 : k;
    while (ldexp(253.0, ex) < ext) ++ex;
    ex = max(ex, -126);
  }
  if (ex > 127) return false;
  e = (uint8_t)(ex + 127);
  return true;
}

// 8-bit child bounds, rounded outward with one extra quantum where a bound lands on the grid,
// then checked in single precision (unfused, as the host builder checks) so a box never shrinks.
__device__ void quantChildD(float p, uint8_t e, float clo, float chi, uint8_t& qlo, uint8_t& qhi)
{
  const double scale = ldexp(1.0, (int)e - 127);
  const float fs = (float)scale;
  double a = floor(((double)clo - (double)p) / scale);
  double b = ceil(((double)chi - (double)p) / scale);
  if (a > 0.0 && __dadd_rn((double)p, __dmul_rn(a, scale)) == (double)clo) a -= 1.0;
  if (__dadd_rn((double)p, __dmul_rn(b, scale)) == (double)chi) b += 1.0;
  a = fmax(a, 0.0);
  b = fmin(b, 255.0);
  while (a > 0.0 && __fadd_rn(p, __fmul_rn((float)a, fs)) > clo) a -= 1.0;
  while (b < 255.0 && __fadd_rn(p, __fmul_rn((float)b, fs)) < chi) b += 1.0;
  qlo = (uint8_t)a;
  qhi = (uint8_t)b;
}

// The 48-byte triangle record: v0 with the triangle index in w, then v1 - v0 and v2 - v0 in
// single precision (the host builder's and the oracle intersector's edges).
__device__ __forceinline__ void writeTri(float4* __restrict__ out, uint32_t slot, int t, const float4* __restrict__ pos,
                                         const int4* __restrict__ tv)
{
  const int4 id = tv[t];
  const float4 a = pos[id.x], b = pos[id.y], c = pos[id.z];
  out[3 * (size_t)slot + 0] = make_float4(a.x, a.y, a.z, __int_as_float(t));
  out[3 * (size_t)slot + 1] = make_float4(__fsub_rn(b.x, a.x), __fsub_rn(b.y, a.y), __fsub_rn(b.z, a.z), 0.f);
  out[3 * (size_t)slot + 2] = make_float4(__fsub_rn(c.x, a.x), __fsub_rn(c.y, a.y), __fsub_rn(c.z, a.z), 0.f);
}

// Writes wide node levelBase + w: quantised child boxes, leaf triangles (each leaf's subtree
// walked left to right) at triBase0 + its scanned offset, inner children at nextBase + offset in
// slot order, which also become the next level's work items.
__global__ void __launch_bounds__(kCollapseThreads) kCollapseEmit(
  const int* __restrict__ work, int m, const int* __restrict__ slotNode, const u64* __restrict__ offs, int levelBase,
  int nextBase, int64_t triBase0, BinNodes N, const float4* __restrict__ pos, const int4* __restrict__ tv,
  uint4* __restrict__ outNodes, float4* __restrict__ outTris, int* __restrict__ nextWork, int* err)
{
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= m) return;
  const int b = work[w];
  const u64 o = offs[w];
  const uint32_t innerOff = (uint32_t)(o >> 32), triOff = (uint32_t)o;
  const float4 blo = N.lo[b], bhi = N.hi[b];
  Bvh8Node node;
  memset(&node, 0, sizeof(node));
  if (!quantAxisD(blo.x, bhi.x, node.px, node.ex) || !quantAxisD(blo.y, bhi.y, node.py, node.ey) ||
      !quantAxisD(blo.z, bhi.z, node.pz, node.ez))
    atomicOr(err, 1);
  node.childBase = (uint32_t)nextBase + innerOff;
  node.triBase = (uint32_t)(triBase0 + triOff);
  uint32_t innerK = 0u, triK = 0u;
  for (int s = 0; s < 8; ++s)
  {
    const int c = slotNode[8 * w + s];
    if (c < 0) continue;
    const float4 clo = N.lo[c], chi = N.hi[c];
    quantChildD(node.px, node.ex, clo.x, chi.x, node.qlox[s], node.qhix[s]);
    quantChildD(node.py, node.ey, clo.y, chi.y, node.qloy[s], node.qhiy[s]);
    quantChildD(node.pz, node.ez, clo.z, chi.z, node.qloz[s], node.qhiz[s]);
    if (!isLeafNode(chi))
    {
      node.imask |= (uint8_t)(1u << s);
      nextWork[innerOff + innerK] = c;
      ++innerK;
      continue;
    }
    node.meta[s] = (uint8_t)((nodeTris(chi) << 5) | triK);
    int stack[4];
    int sp = 0;
    stack[sp++] = c;
    while (sp > 0)
    {
      const int x = stack[--sp];
      const int2 k = N.child[x];
      if (k.x < 0)
      {
        writeTri(outTris, node.triBase + triK, k.y, pos, tv);
        ++triK;
      }
      else if (sp + 2 <= 4)
      {
        stack[sp++] = k.y;
        stack[sp++] = k.x;
      }
      else
      {
        atomicOr(err, 2);
        break;
      }
    }
  }
  const uint4* src = reinterpret_cast<const uint4*>(&node);
  uint4* dst = outNodes + 5 * (size_t)(levelBase + w);
  for (int k = 0; k < 5; ++k) dst[k] = src[k];
}

unsigned blocksFor(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <class T>
T readScalar(const T* dev, cudaStream_t st)
{
  T v;
  check(cudaMemcpyAsync(&v, dev, sizeof(T), cudaMemcpyDeviceToHost, st), "read back");
  check(cudaStreamSynchronize(st), "build");
  return v;
}

} // namespace

void buildBvh8Device(const float4* pos, const int4* triVerts, int64_t triCount, cudaStream_t st, DeviceBvh8& out)
{
  if (triCount < 0 || triCount > (int64_t)0x3fffffff)
    throw std::invalid_argument("BVH8: triangle count out of range");
  check(cudaStreamSynchronize(st), "build");
  const auto t0 = std::chrono::steady_clock::now();
  out = DeviceBvh8();
  const int n = (int)triCount;
  Scratch s;
  if (n == 0)
  {
    // One empty node: every ray misses.
    Bvh8Node* nodes = s.alloc<Bvh8Node>(1);
    check(cudaMemsetAsync(nodes, 0, sizeof(Bvh8Node), st), "build");
    Bvh8Tri* tris = s.alloc<Bvh8Tri>(1);
    check(cudaStreamSynchronize(st), "build");
    s.bufs.clear();
    out.nodes = nodes;
    out.tris = tris;
    out.nodeCount = 1;
    out.maxDepth = 1;
    out.buildMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return;
  }
  // 1. Boxes, centroid bounds, Morton codes.
  float4* triLo = s.alloc<float4>(n);
  float4* triHi = s.alloc<float4>(n);
  uint32_t* cb = s.alloc<uint32_t>(6);
  kFillU32<<<1, 32, 0, st>>>(cb, 6, 0xffffffffu, 0u, 3);
  kTriBoxes<<<blocksFor(n, 256), 256, 0, st>>>(pos, triVerts, n, triLo, triHi, cb);
  MortonKey* keysA = s.alloc<MortonKey>(n);
  uint32_t* valsA = s.alloc<uint32_t>(n);
  MortonKey* keysB = s.alloc<MortonKey>(n);
  uint32_t* valsB = s.alloc<uint32_t>(n);
  kMorton<<<blocksFor(n, 256), 256, 0, st>>>(triLo, triHi, n, cb, keysA, valsA);
  // 2. Stable radix sort, 8 bits per pass over the code's bits.
  const int tiles = (int)blocksFor(n, kSortTile);
  uint32_t* hist = s.alloc<uint32_t>((size_t)256 * tiles);
  Scanner<uint32_t> scan32;
  scan32.init(s, (int64_t)256 * tiles);
  for (int shift = 0; shift < kMortonBits; shift += 8)
  {
    kRadixHist<<<tiles, kSortThreads, 0, st>>>(keysA, n, shift, hist, tiles);
    scan32.run(hist, hist, (int64_t)256 * tiles, st);
    kRadixScatter<<<tiles, kSortThreads, 0, st>>>(keysA, valsA, keysB, valsB, n, shift, hist, tiles);
    std::swap(keysA, keysB);
    std::swap(valsA, valsB);
  }
  // 3. PLOC: large iterations over the whole device, then the in-block tail.
  const size_t nodeCap = 2 * (size_t)n;
  BinNodes N;
  N.lo = s.alloc<float4>(nodeCap);
  N.hi = s.alloc<float4>(nodeCap);
  N.child = s.alloc<int2>(nodeCap);
  N.costA = s.alloc<float4>(nodeCap);
  N.costB = s.alloc<float4>(nodeCap);
  N.dec = s.alloc<uint2>(nodeCap);
  int* cidA = s.alloc<int>(n);
  int* cidB = s.alloc<int>(n);
  float4* cLoA = s.alloc<float4>(n);
  float4* cHiA = s.alloc<float4>(n);
  float4* cLoB = s.alloc<float4>(n);
  float4* cHiB = s.alloc<float4>(n);
  kInitLeaves<<<blocksFor(n, 256), 256, 0, st>>>(valsA, triLo, triHi, n, N, cidA, cLoA, cHiA);
  int* nn = s.alloc<int>(n);
  u64* flags = s.alloc<u64>(n);
  Scanner<u64> scan64;
  scan64.init(s, n);
  int count = n, nodeBase = n, force = 0, iters = 0;
  // Each iteration merges at least a 1/64 share of the clusters, or else forces the next one to
  // pair Morton neighbours (which merges about half); so log(n)/log(64/63) iterations bound a
  // converging run. NaN boxes could stall it, hence the cap.
  const int maxIters = 64 + 64 * (int)std::ceil(std::log2((double)std::max<int64_t>(n, 2)));
  while (count > kTailMax)
  {
    if (iters >= maxIters) throw std::runtime_error("BVH8 device build: clustering did not converge");
    kNearest<<<blocksFor(count, kNearestThreads), kNearestThreads, 0, st>>>(cLoA, cHiA, count, nn, force);
    kMergeFlags<<<blocksFor(count, 256), 256, 0, st>>>(nn, count, flags);
    scan64.run(flags, flags, count, st);
    kCompact<<<blocksFor(count, 256), 256, 0, st>>>(nn, count, flags, cidA, cLoA, cHiA, cidB, cLoB, cHiB, N,
                                                    nodeBase);
    const u64 tot = readScalar(scan64.total, st);
    const int merges = (int)(tot >> 32);
    if (merges == 0 && force) throw std::runtime_error("BVH8 device build: clustering did not converge");
    force = (int64_t)merges * 64 < count;
    nodeBase += merges;
    count = (int)(uint32_t)tot;
    ++iters;
    std::swap(cidA, cidB);
    std::swap(cLoA, cLoB);
    std::swap(cHiA, cHiB);
  }
  int* result = s.alloc<int>(3);
  check(cudaFuncSetAttribute(kPlocTail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTailSmem), "build");
  kPlocTail<<<1, kTailThreads, kTailSmem, st>>>(count, force, cidA, cLoA, cHiA, N, nodeBase, result);
  check(cudaGetLastError(), "clustering");
  int res[3];
  check(cudaMemcpyAsync(res, result, sizeof(res), cudaMemcpyDeviceToHost, st), "read back");
  check(cudaStreamSynchronize(st), "clustering");
  const int root = res[0];
  iters += res[1];
  if (root < 0 || res[2] != 2 * n - 1) throw std::runtime_error("BVH8 device build: clustering did not converge");
  // 4. Collapse, one wide level per step. Wide nodes <= max(inner binary nodes, 1) <= n.
  int* workA = s.alloc<int>(n);
  int* workB = s.alloc<int>(n);
  int* slotNode = s.alloc<int>((size_t)8 * n);
  Bvh8Node* nodesTmp = s.alloc<Bvh8Node>(n);
  Bvh8Tri* tris = s.alloc<Bvh8Tri>(n);
  int* err = s.alloc<int>(1);
  check(cudaMemsetAsync(err, 0, sizeof(int), st), "build");
  check(cudaMemcpyAsync(workA, &root, sizeof(int), cudaMemcpyHostToDevice, st), "build");
  int m = 1, levelBase = 0, depth = 0, top = 0;
  int64_t triBase = 0;
  while (m > 0)
  {
    if ((int64_t)levelBase + m > n) throw std::runtime_error("BVH8 device build: node count exceeds the bound");
    kCollapsePlan<<<blocksFor(m, kCollapseThreads), kCollapseThreads, 0, st>>>(workA, m, N, slotNode, flags);
    scan64.run(flags, flags, m, st);
    kCollapseEmit<<<blocksFor(m, kCollapseThreads), kCollapseThreads, 0, st>>>(
      workA, m, slotNode, flags, levelBase, levelBase + m, triBase, N, pos, triVerts,
      reinterpret_cast<uint4*>(nodesTmp), reinterpret_cast<float4*>(tris), workB, err);
    const u64 tot = readScalar(scan64.total, st);
    if (depth < kBvh8TopLevels) top += m;
    levelBase += m;
    triBase += (uint32_t)tot;
    m = (int)(tot >> 32);
    ++depth;
    std::swap(workA, workB);
  }
  const int errFlag = readScalar(err, st);
  if (errFlag & 1) throw std::runtime_error("BVH8: scene extent too large for 8-bit quantisation");
  if (errFlag || triBase != n) throw std::runtime_error("BVH8 device build: inconsistent leaves");
  // Exact-size node array.
  void* nodes = nullptr;
  check(cudaMalloc(&nodes, sizeof(Bvh8Node) * (size_t)levelBase), "cudaMalloc");
  s.bufs.push_back(nodes);
  check(cudaMemcpyAsync(nodes, nodesTmp, sizeof(Bvh8Node) * (size_t)levelBase, cudaMemcpyDeviceToDevice, st), "build");
  check(cudaStreamSynchronize(st), "build");
  // Hand the two outputs to the caller; the rest is freed with the scratch.
  s.bufs.erase(std::remove_if(s.bufs.begin(), s.bufs.end(), [&](void* p) { return p == nodes || p == tris; }),
               s.bufs.end());
  out.nodes = nodes;
  out.tris = tris;
  out.nodeCount = levelBase;
  out.triCount = n;
  out.topCount = std::min(top, kBvh8TopNodes);
  out.maxDepth = depth;
  out.plocIterations = iters;
  out.buildMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

} // namespace prt
