// BVH8 ray traversal on the device: closest hit and any hit.
//
// Replaces the reference's Embree queries (accel/embree_intersector_stream.h:66-131, called
// from render/path_renderer_stream.h:280 and :953). The node layout is bvh8.h's compressed
// 80-byte wide node; the walk keeps "node groups" (a base index plus the still-unvisited hit
// children of one node) on a short per-thread stack, the scheme of Ylitie et al. 2017.
//
// The ray/triangle test is the fixed-operation Moller-Trumbore form shared with the host
// oracle (crossFx/dotFx in prt_math.cuh): hit iff det != 0, u >= 0, v >= 0, u + v <= 1 and
// near <= t <= far. The closest hit keeps the smallest t and, on equal t, the smallest
// global triangle index, so the result does not depend on the tree or the visiting order.
// Box tests are conservative: quantised boxes are rounded outward and the slab interval is
// compared with a relative slack of 2e-6, so that a triangle the test accepts is never culled.
#pragma once

#include "prt_math.cuh"
#include "bvh8.h"

namespace prt {

constexpr int kTraceStack = kBvh8TraceStack;  // node-group stack entries per ray
// The shallow stack of the traversal kernels' second instantiation, taken for trees of at most
// this many wide levels (the host-built tree of the 2.6M-triangle terrain has 10): half the
// local-memory frame. On the terrain frame both instantiations run equally fast (the stack's
// upper entries are never touched there); the choice is a tuning axis for other scenes.
constexpr int kTraceStackShallow = 24;
// Stacks of at most this many entries live in shared memory instead (NodeStack), laid out
// [entry][thread] for the traversal kernels' 256-thread blocks: 12 x 256 x 8 B = 24 KB per block,
// 96 KB per SM at 4 blocks. On the terrain frame (a tree of 10 wide levels) this takes 1.5% off
// kTrace and 1% off kShadow against either local-memory stack; it is the default for trees that fit.
constexpr int kTraceStackShared = 12;
constexpr int kTraceMaxIter = 1 << 20;    // loop cap: a corrupt tree ends the ray, not the kernel
constexpr uint32_t kErrStackOverflow = 1u;
constexpr uint32_t kErrIterCap = 2u;

struct TraceHit
{
  int triId;   // global triangle index, -1 on a miss
  float t, u, v;
};

PRT_D float expToScale(uint32_t e) { return __uint_as_float(e << 23); }

PRT_D bool intersectTriFx(const float4* __restrict__ tris, uint32_t idx, f3 o, f3 d, float tnear, float tfar,
                          float& t, float& u, float& v, int& triId)
{
  const float4 a = __ldg(tris + 3 * idx + 0);
  const float4 b = __ldg(tris + 3 * idx + 1);
  const float4 c = __ldg(tris + 3 * idx + 2);
  const f3 v0 = mk(a.x, a.y, a.z);
  const f3 e1 = mk(b.x, b.y, b.z);
  const f3 e2 = mk(c.x, c.y, c.z);
  const f3 p = crossFx(d, e2);
  const float det = dotFx(e1, p);
  if (!(det != 0.f)) return false;
  const f3 s = subFx(o, v0);
  const f3 q = crossFx(s, e1);
  const float inv = __frcp_rn(det);
  const float uu = __fmul_rn(dotFx(s, p), inv);
  const float vv = __fmul_rn(dotFx(d, q), inv);
  const float tt = __fmul_rn(dotFx(e2, q), inv);
  if (!(uu >= 0.f) || !(vv >= 0.f) || !(__fadd_rn(uu, vv) <= 1.f)) return false;
  if (!(tt >= tnear) || !(tt <= tfar)) return false;
  t = tt;
  u = uu;
  v = vv;
  triId = __float_as_int(a.w);
  return true;
}

struct RayPre
{
  f3 o, invd;
  uint32_t oct;             // bit k set when direction component k is negative
  uint32_t permLo, permHi;  // byte_perm selectors: byte s of an 8-byte child row -> position s ^ oct
};

PRT_D RayPre rayPre(f3 o, f3 d)
{
  RayPre r;
  r.o = o;
  const float tiny = 8.271806e-25f;  // 2^-80: keeps 1/d finite
  const float dx = fabsf(d.x) < tiny ? copysignf(tiny, d.x) : d.x;
  const float dy = fabsf(d.y) < tiny ? copysignf(tiny, d.y) : d.y;
  const float dz = fabsf(d.z) < tiny ? copysignf(tiny, d.z) : d.z;
  r.invd = mk(__frcp_rn(dx), __frcp_rn(dy), __frcp_rn(dz));
  r.oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
  // Output byte j of a permuted row is source byte j ^ oct (bytes 0-3 from the row's low word,
  // 4-7 from its high word): nibble j of the selectors.
  r.permLo = 0u;
  r.permHi = 0u;
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j)
  {
    r.permLo |= (j ^ r.oct) << (4 * j);
    r.permHi |= ((j + 4) ^ r.oct) << (4 * j);
  }
  return r;
}

PRT_D uint32_t byteOf(uint2 w, int i)
{
  return (i < 4 ? (w.x >> (8 * i)) : (w.y >> (8 * (i - 4)))) & 0xffu;
}

// An 8-byte child row (one byte per slot) reordered so that position j holds slot j ^ oct.
PRT_D uint2 permuteRow(uint2 w, const RayPre& r)
{
  return make_uint2(__byte_perm(w.x, w.y, r.permLo), __byte_perm(w.x, w.y, r.permHi));
}

// Bit s of an 8-bit mask moved to bit s ^ oct.
PRT_D uint32_t permuteBits(uint32_t x, uint32_t oct)
{
  if (oct & 1u) x = ((x & 0x55u) << 1) | ((x >> 1) & 0x55u);
  if (oct & 2u) x = ((x & 0x33u) << 2) | ((x >> 2) & 0x33u);
  if (oct & 4u) x = ((x & 0x0fu) << 4) | ((x >> 4) & 0x0fu);
  return x;
}

// Shared-memory copy of the breadth-first top levels of the BVH (bvh8.h), filled by a
// traversal kernel that stages them; with Top = true node i < topCount is read from here.
static __shared__ uint4 gTopNodes[5 * kBvh8TopNodes];

// Intersects the 8 children of one node; returns the node group of hit inner children
// (bits 24-31: hit flags at position slot ^ oct; bits 0-7: imask) and the triangle bits.
//
// The child rows are permuted into the ray's octant order once per node, so that child j of the
// loop is slot j ^ oct and its hit flag lands at bit j, the position the node group uses. The
// slab slack (2e-6 relative, which keeps the rounded interval from culling a box the exact
// interval reaches) is applied by scaling the near planes by 1 / 1.000002 instead of scaling
// every far plane up. Empty slots (meta 0, not inner) may pass the slab test; as leaves without
// triangles they add nothing.
template <bool Top>
PRT_D void intersectNode(const uint4* __restrict__ nodes, uint32_t nodeIdx, const RayPre& r, float tnear,
                         float tfar, uint2& ngroup, uint2& tgroup, int topCount = 0)
{
  uint4 w0, w1, w2, w3, w4;
  if (Top && nodeIdx < (uint32_t)topCount)
  {
    w0 = gTopNodes[5 * nodeIdx + 0];
    w1 = gTopNodes[5 * nodeIdx + 1];
    w2 = gTopNodes[5 * nodeIdx + 2];
    w3 = gTopNodes[5 * nodeIdx + 3];
    w4 = gTopNodes[5 * nodeIdx + 4];
  }
  else
  {
    w0 = __ldg(nodes + 5 * nodeIdx + 0);
    w1 = __ldg(nodes + 5 * nodeIdx + 1);
    w2 = __ldg(nodes + 5 * nodeIdx + 2);
    w3 = __ldg(nodes + 5 * nodeIdx + 3);
    w4 = __ldg(nodes + 5 * nodeIdx + 4);
  }
  const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
  const uint32_t ex = w0.w & 0xffu, ey = (w0.w >> 8) & 0xffu, ez = (w0.w >> 16) & 0xffu;
  const uint32_t imask = (w0.w >> 24) & 0xffu;
  const uint32_t childBase = w1.x, triBase = w1.y;
  // Near plane = lo for positive directions, hi for negative ones.
  const uint2 lox = make_uint2(w2.x, w2.y), loy = make_uint2(w2.z, w2.w);
  const uint2 loz = make_uint2(w3.x, w3.y), hix = make_uint2(w3.z, w3.w);
  const uint2 hiy = make_uint2(w4.x, w4.y), hiz = make_uint2(w4.z, w4.w);
  const uint2 nx = permuteRow((r.oct & 1u) ? hix : lox, r), fx = permuteRow((r.oct & 1u) ? lox : hix, r);
  const uint2 ny = permuteRow((r.oct & 2u) ? hiy : loy, r), fy = permuteRow((r.oct & 2u) ? loy : hiy, r);
  const uint2 nz = permuteRow((r.oct & 4u) ? hiz : loz, r), fz = permuteRow((r.oct & 4u) ? loz : hiz, r);
  const float kNear = 1.f / 1.000002f;
  const float ax = __fmul_rn(px - r.o.x, r.invd.x);
  const float ay = __fmul_rn(py - r.o.y, r.invd.y);
  const float az = __fmul_rn(pz - r.o.z, r.invd.z);
  const float bx = expToScale(ex) * r.invd.x;
  const float by = expToScale(ey) * r.invd.y;
  const float bz = expToScale(ez) * r.invd.z;
  const float axn = ax * kNear, ayn = ay * kNear, azn = az * kNear;
  const float bxn = bx * kNear, byn = by * kNear, bzn = bz * kNear;
  const float tnearK = tnear * kNear;
  uint32_t hits = 0u;
#pragma unroll
  for (int j = 0; j < 8; ++j)
  {
    const float x0 = fmaf((float)byteOf(nx, j), bxn, axn), x1 = fmaf((float)byteOf(fx, j), bx, ax);
    const float y0 = fmaf((float)byteOf(ny, j), byn, ayn), y1 = fmaf((float)byteOf(fy, j), by, ay);
    const float z0 = fmaf((float)byteOf(nz, j), bzn, azn), z1 = fmaf((float)byteOf(fz, j), bz, az);
    const float tmin = fmaxf(fmaxf(x0, y0), fmaxf(z0, tnearK));
    const float tmax = fminf(fminf(x1, y1), fminf(z1, tfar));
    hits |= (tmin <= tmax ? 1u : 0u) << j;
  }
  const uint32_t imaskP = permuteBits(imask, r.oct);
  uint32_t leaves = hits & ~imaskP, tri = 0u;
  if (leaves)
  {
    const uint2 meta = permuteRow(make_uint2(w1.z, w1.w), r);
    do
    {
      const int j = __ffs(leaves) - 1;
      leaves &= leaves - 1u;
      const uint32_t m = (j < 4 ? (meta.x >> (8 * j)) : (meta.y >> (8 * (j - 4)))) & 0xffu;
      tri |= ((1u << (m >> 5)) - 1u) << (m & 31u);
    } while (leaves);
  }
  ngroup = make_uint2(childBase, ((hits & imaskP) << 24) | imask);
  tgroup = make_uint2(triBase, tri);
}

// Node visits and triangle tests of one ray (counting variant only).
struct TraceCount
{
  int nodes = 0;
  int tris = 0;
};

// Any-hit filter that accepts every hit (plain occlusion).
struct AcceptAll
{
  PRT_D bool operator()(int triId, float t, float u, float v) const { return true; }
};

// The per-ray node-group stack: a local-memory array, or for Stack <= kTraceStackShared a column
// of a shared-memory array (blocks of 256 threads only).
template <int Stack, bool Shared = (Stack <= kTraceStackShared)>
struct NodeStack
{
  uint2 e[Stack];
  PRT_D uint2& at(int i) { return e[i]; }
};

template <int Stack>
struct NodeStack<Stack, true>
{
  PRT_D uint2& at(int i)
  {
    __shared__ uint2 s[Stack][256];
    return s[i][threadIdx.x];
  }
};

// AnyHit: stop at the first hit the filter accepts (filter(triangle, t, u, v) == true); hits it
// rejects are skipped without shortening the ray. Closest hit ignores the filter.
template <bool AnyHit, bool Count = false, bool Top = false, int Stack = kTraceStack, class Filter = AcceptAll>
PRT_D TraceHit traverse(const uint4* __restrict__ nodes, const float4* __restrict__ tris, f3 o, f3 d,
                        float tnear, float tfar, uint32_t* errFlag, TraceCount* count = nullptr,
                        int topCount = 0, const Filter& filter = Filter())
{
  TraceHit h;
  h.triId = -1;
  h.t = tfar;
  h.u = h.v = 0.f;
  const RayPre r = rayPre(o, d);
  NodeStack<Stack> stack;
  int sp = 0;
  // The root as a one-child group: slot 0 is inner, at bit 24 + (0 ^ oct).
  uint2 ngroup = make_uint2(0u, (1u << (24 + r.oct)) | 1u);
  uint2 tgroup = make_uint2(0u, 0u);
  for (int iter = 0; iter < kTraceMaxIter; ++iter)
  {
    while (tgroup.y != 0u)
    {
      const int bit = __ffs(tgroup.y) - 1;
      tgroup.y &= tgroup.y - 1u;
      if (Count) count->tris++;
      float t, u, v;
      int id;
      if (intersectTriFx(tris, tgroup.x + bit, o, d, tnear, h.t, t, u, v, id))
      {
        if (AnyHit)
        {
          if (!filter(id, t, u, v)) continue;
          h.triId = id;
          h.t = t;
          return h;
        }
        if (t < h.t || h.triId < 0 || id < h.triId)
        {
          h.triId = id;
          h.t = t;
          h.u = u;
          h.v = v;
        }
      }
    }
    if (ngroup.y <= 0x00ffffffu)
    {
      if (sp == 0) return h;
      ngroup = stack.at(--sp);
    }
    const int b = 31 - __clz(ngroup.y);
    ngroup.y &= ~(1u << b);
    const uint32_t slot = (uint32_t)(b - 24) ^ r.oct;
    const uint32_t imask = ngroup.y & 0xffu;
    const uint32_t nodeIdx = ngroup.x + __popc(imask & ((1u << slot) - 1u));
    if (ngroup.y > 0x00ffffffu)
    {
      if (sp == Stack)
      {
        atomicOr(errFlag, kErrStackOverflow);
        return h;
      }
      stack.at(sp++) = ngroup;
    }
    if (Count) count->nodes++;
    intersectNode<Top>(nodes, nodeIdx, r, tnear, h.t, ngroup, tgroup, topCount);
  }
  atomicOr(errFlag, kErrIterCap);
  return h;
}

} // namespace prt
