// Test infrastructure (oracle only, never linked into the product).
//
// Stand-in for the reference's Embree stream intersectors
// (accel/embree_intersector_stream.h:9-131). Embree 4 is not installed on this machine, so
// the reference renderer is compiled against this header instead: it sits ahead of the
// reference tree on the include path and keeps the two class names and the constructor
// signature that render/intersector_factory_stream.h:31-32 instantiates.
//
// It is a plain binary SAH BVH over all triangle meshes of the scene group, traversed one
// ray at a time. The ray/triangle test is the fixed-operation Moller-Trumbore form that
// the GPU traversal kernel also uses:
//   e1 = v1 - v0, e2 = v2 - v0                (plain float subtraction)
//   p  = cross(d, e2), s = o - v0, q = cross(s, e1)
//   cross(a,b).x = fma(a.y, b.z, -(a.z*b.y))   (and cyclic)
//   dot(a,b)     = fma(a.x, b.x, fma(a.y, b.y, a.z*b.z))
//   det = dot(e1, p); inv = 1/det (IEEE); u = dot(s,p)*inv; v = dot(d,q)*inv; t = dot(e2,q)*inv
//   hit iff det != 0, u >= 0, v >= 0, u + v <= 1, near <= t <= far
// Closest hit keeps the smallest t and, on equal t, the smallest global triangle index
// (meshes concatenated in group order), so the answer does not depend on the BVH shape
// or traversal order. This is what makes the GPU's hit IDs comparable bit for bit.
// Embree's own arithmetic is not available here, so parity against Embree itself is not
// pinned; parity is defined against this intersector.
#pragma once

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <vector>

#include "sys/props.h"
#include "sys/logging.h"
#include "sys/timer.h"
#include "geometry/group.h"
#include "geometry/triangle_mesh.h"
#include "core/intersector_stream.h"

namespace prt {

namespace oracle_bvh {

struct Tri
{
  float v0[3], e1[3], e2[3];
  int geomId, primId;
};

struct Node
{
  float lo[3], hi[3];
  int left;   // inner: index of the left child (right = left + 1); leaf: first triangle
  int count;  // 0 for inner nodes, number of triangles for leaves
};

// Fixed-operation helpers shared (by definition, not by code) with the GPU kernel.
static inline void crossF(const float a[3], const float b[3], float r[3])
{
  r[0] = std::fmaf(a[1], b[2], -(a[2] * b[1]));
  r[1] = std::fmaf(a[2], b[0], -(a[0] * b[2]));
  r[2] = std::fmaf(a[0], b[1], -(a[1] * b[0]));
}

static inline float dotF(const float a[3], const float b[3])
{
  return std::fmaf(a[0], b[0], std::fmaf(a[1], b[1], a[2] * b[2]));
}

// Returns true and writes t/u/v when the ray hits the triangle within [tnear, tfar].
static inline bool intersectTri(const Tri& tri, const float o[3], const float d[3], float tnear, float tfar,
                                float& t, float& u, float& v)
{
  float p[3], s[3], q[3];
  crossF(d, tri.e2, p);
  const float det = dotF(tri.e1, p);
  if (!(det != 0.f)) return false;
  s[0] = o[0] - tri.v0[0];
  s[1] = o[1] - tri.v0[1];
  s[2] = o[2] - tri.v0[2];
  crossF(s, tri.e1, q);
  const float inv = 1.0f / det;
  const float uu = dotF(s, p) * inv;
  const float vv = dotF(d, q) * inv;
  const float tt = dotF(tri.e2, q) * inv;
  if (!(uu >= 0.f) || !(vv >= 0.f) || !(uu + vv <= 1.f)) return false;
  if (!(tt >= tnear) || !(tt <= tfar)) return false;
  t = tt; u = uu; v = vv;
  return true;
}

class Bvh
{
public:
  std::vector<Tri> tris;
  std::vector<Node> nodes;
  std::vector<int> order; // leaf triangle slots -> index into tris
  long long nodeVisits = 0;

  void build()
  {
    const int n = (int)tris.size();
    order.resize(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    centroids.resize(n);
    boxes.resize(n);
    for (int i = 0; i < n; ++i)
    {
      const Tri& t = tris[i];
      float a[3], b[3], c[3];
      for (int k = 0; k < 3; ++k)
      {
        a[k] = t.v0[k];
        b[k] = t.v0[k] + t.e1[k];
        c[k] = t.v0[k] + t.e2[k];
      }
      for (int k = 0; k < 3; ++k)
      {
        // Pad by a relative epsilon so that e1/e2 reconstruction error never shrinks a box.
        float lo = std::min(a[k], std::min(b[k], c[k]));
        float hi = std::max(a[k], std::max(b[k], c[k]));
        float pad = 1e-6f * std::max(std::fabs(lo), std::fabs(hi)) + 1e-30f;
        boxes[i].lo[k] = lo - pad;
        boxes[i].hi[k] = hi + pad;
        centroids[i].c[k] = 0.5f * (lo + hi);
      }
    }
    nodes.clear();
    nodes.reserve(2 * (size_t)std::max(n, 1));
    nodes.push_back(Node());
    if (n == 0)
    {
      for (int k = 0; k < 3; ++k) { nodes[0].lo[k] = 1.f; nodes[0].hi[k] = -1.f; }
      nodes[0].left = 0;
      nodes[0].count = 0;
      return;
    }
    buildRec(0, 0, n);
    centroids.clear();
    boxes.clear();
  }

  // Closest hit. Returns the hit triangle index or -1.
  int intersect(const float o[3], const float d[3], float tnear, float& tfar, float& u, float& v) const
  {
    float inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    int best = -1;
    float bestT = tfar;
    while (sp > 0)
    {
      const Node& node = nodes[stack[--sp]];
      if (!boxHit(node, o, inv, tnear, bestT)) continue;
      if (node.count > 0)
      {
        for (int j = 0; j < node.count; ++j)
        {
          const int ti = order[node.left + j];
          float t, uu, vv;
          if (intersectTri(tris[ti], o, d, tnear, bestT, t, uu, vv))
          {
            // intersectTri already enforces t <= bestT; equal t goes to the lower index.
            if (t < bestT || best < 0 || ti < best)
            {
              bestT = t; best = ti; u = uu; v = vv;
            }
          }
        }
      }
      else
      {
        // Visit the nearer child first.
        const Node& l = nodes[node.left];
        const Node& r = nodes[node.left + 1];
        float cl = 0.f, cr = 0.f;
        for (int k = 0; k < 3; ++k)
        {
          cl += (l.lo[k] + l.hi[k] - 2.f * o[k]) * d[k];
          cr += (r.lo[k] + r.hi[k] - 2.f * o[k]) * d[k];
        }
        if (sp + 2 > 128) throw std::runtime_error("oracle BVH stack overflow");
        if (cl < cr) { stack[sp++] = node.left + 1; stack[sp++] = node.left; }
        else         { stack[sp++] = node.left; stack[sp++] = node.left + 1; }
      }
    }
    if (best >= 0) tfar = bestT;
    return best;
  }

  bool occluded(const float o[3], const float d[3], float tnear, float tfar) const
  {
    float inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0)
    {
      const Node& node = nodes[stack[--sp]];
      if (!boxHit(node, o, inv, tnear, tfar)) continue;
      if (node.count > 0)
      {
        for (int j = 0; j < node.count; ++j)
        {
          float t, uu, vv;
          if (intersectTri(tris[order[node.left + j]], o, d, tnear, tfar, t, uu, vv))
            return true;
        }
      }
      else
      {
        if (sp + 2 > 128) throw std::runtime_error("oracle BVH stack overflow");
        stack[sp++] = node.left;
        stack[sp++] = node.left + 1;
      }
    }
    return false;
  }

  // Any-hit with an intersection filter: f(triangle, t, u, v) is called for every triangle the
  // ray hits within [tnear, tfar] (each once, in traversal order) until it returns true, which
  // makes the ray occluded; hits it rejects do not shorten the ray (Embree's occluded-filter
  // semantics).
  template <class F>
  bool occludedFiltered(const float o[3], const float d[3], float tnear, float tfar, F&& f) const
  {
    float inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0)
    {
      const Node& node = nodes[stack[--sp]];
      if (!boxHit(node, o, inv, tnear, tfar)) continue;
      if (node.count > 0)
      {
        for (int j = 0; j < node.count; ++j)
        {
          const int ti = order[node.left + j];
          float t, uu, vv;
          if (intersectTri(tris[ti], o, d, tnear, tfar, t, uu, vv) && f(ti, t, uu, vv)) return true;
        }
      }
      else
      {
        if (sp + 2 > 128) throw std::runtime_error("oracle BVH stack overflow");
        stack[sp++] = node.left;
        stack[sp++] = node.left + 1;
      }
    }
    return false;
  }

private:
  struct C3 { float c[3]; };
  struct B3 { float lo[3], hi[3]; };
  std::vector<C3> centroids;
  std::vector<B3> boxes;

  static inline bool boxHit(const Node& n, const float o[3], const float inv[3], float tnear, float tfar)
  {
    // Conservative slab test: the interval is widened by a relative 1e-5 so that a
    // triangle whose rounded t lies on the box boundary is never culled.
    float t0 = tnear, t1 = tfar;
    for (int k = 0; k < 3; ++k)
    {
      float a = (n.lo[k] - o[k]) * inv[k];
      float b = (n.hi[k] - o[k]) * inv[k];
      if (std::isnan(a)) a = -INFINITY; // 0 * inf on a slab boundary
      if (std::isnan(b)) b = INFINITY;
      float lo = std::min(a, b), hi = std::max(a, b);
      t0 = std::max(t0, lo);
      t1 = std::min(t1, hi);
    }
    return t0 * (1.f - 1e-5f) - 1e-30f <= t1 * (1.f + 1e-5f) + 1e-30f;
  }

  void buildRec(int nodeIndex, int begin, int end)
  {
    B3 bb;
    B3 cb;
    for (int k = 0; k < 3; ++k)
    {
      bb.lo[k] = cb.lo[k] = FLT_MAX;
      bb.hi[k] = cb.hi[k] = -FLT_MAX;
    }
    for (int i = begin; i < end; ++i)
    {
      const int ti = order[i];
      for (int k = 0; k < 3; ++k)
      {
        bb.lo[k] = std::min(bb.lo[k], boxes[ti].lo[k]);
        bb.hi[k] = std::max(bb.hi[k], boxes[ti].hi[k]);
        cb.lo[k] = std::min(cb.lo[k], centroids[ti].c[k]);
        cb.hi[k] = std::max(cb.hi[k], centroids[ti].c[k]);
      }
    }
    for (int k = 0; k < 3; ++k)
    {
      nodes[nodeIndex].lo[k] = bb.lo[k];
      nodes[nodeIndex].hi[k] = bb.hi[k];
    }
    const int count = end - begin;
    if (count <= 4)
    {
      nodes[nodeIndex].left = begin;
      nodes[nodeIndex].count = count;
      return;
    }
    // Binned SAH over the widest centroid axis.
    int axis = 0;
    float ext = -1.f;
    for (int k = 0; k < 3; ++k)
      if (cb.hi[k] - cb.lo[k] > ext) { ext = cb.hi[k] - cb.lo[k]; axis = k; }
    int mid = begin + count / 2;
    if (ext > 0.f)
    {
      const int nb = 32;
      B3 binBox[nb];
      int binCount[nb];
      for (int b = 0; b < nb; ++b)
      {
        binCount[b] = 0;
        for (int k = 0; k < 3; ++k) { binBox[b].lo[k] = FLT_MAX; binBox[b].hi[k] = -FLT_MAX; }
      }
      const float scale = nb / ext;
      auto binOf = [&](int ti) {
        int b = (int)((centroids[ti].c[axis] - cb.lo[axis]) * scale);
        return std::min(std::max(b, 0), nb - 1);
      };
      for (int i = begin; i < end; ++i)
      {
        const int ti = order[i];
        const int b = binOf(ti);
        binCount[b]++;
        for (int k = 0; k < 3; ++k)
        {
          binBox[b].lo[k] = std::min(binBox[b].lo[k], boxes[ti].lo[k]);
          binBox[b].hi[k] = std::max(binBox[b].hi[k], boxes[ti].hi[k]);
        }
      }
      auto area = [](const B3& b) {
        float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
        if (dx < 0.f) return 0.f;
        return dx * dy + dy * dz + dz * dx;
      };
      float rightArea[nb];
      int rightCount[nb];
      B3 acc;
      for (int k = 0; k < 3; ++k) { acc.lo[k] = FLT_MAX; acc.hi[k] = -FLT_MAX; }
      int cnt = 0;
      for (int b = nb - 1; b > 0; --b)
      {
        for (int k = 0; k < 3; ++k)
        {
          acc.lo[k] = std::min(acc.lo[k], binBox[b].lo[k]);
          acc.hi[k] = std::max(acc.hi[k], binBox[b].hi[k]);
        }
        cnt += binCount[b];
        rightArea[b] = area(acc);
        rightCount[b] = cnt;
      }
      for (int k = 0; k < 3; ++k) { acc.lo[k] = FLT_MAX; acc.hi[k] = -FLT_MAX; }
      cnt = 0;
      float bestCost = FLT_MAX;
      int bestSplit = -1;
      for (int b = 1; b < nb; ++b)
      {
        for (int k = 0; k < 3; ++k)
        {
          acc.lo[k] = std::min(acc.lo[k], binBox[b - 1].lo[k]);
          acc.hi[k] = std::max(acc.hi[k], binBox[b - 1].hi[k]);
        }
        cnt += binCount[b - 1];
        if (cnt == 0 || rightCount[b] == 0) continue;
        const float cost = area(acc) * cnt + rightArea[b] * rightCount[b];
        if (cost < bestCost) { bestCost = cost; bestSplit = b; }
      }
      if (bestSplit > 0)
      {
        int* first = order.data() + begin;
        int* last = order.data() + end;
        int* p = std::partition(first, last, [&](int ti) { return binOf(ti) < bestSplit; });
        mid = (int)(p - order.data());
        if (mid == begin || mid == end) mid = begin + count / 2;
      }
      else
      {
        std::nth_element(order.begin() + begin, order.begin() + mid, order.begin() + end,
                         [&](int a, int b) { return centroids[a].c[axis] < centroids[b].c[axis]; });
      }
    }
    const int left = (int)nodes.size();
    nodes.push_back(Node());
    nodes.push_back(Node());
    nodes[nodeIndex].left = left;
    nodes[nodeIndex].count = 0;
    buildRec(left, begin, mid);
    buildRec(left + 1, mid, end);
  }
};

} // namespace oracle_bvh

// Builds the BVH once for the group's triangle meshes and answers the reference's stream
// queries ray by ray.
class OracleIntersectorBase
{
protected:
  oracle_bvh::Bvh bvh;

public:
  OracleIntersectorBase(const std::shared_ptr<Group>& scene, bool filter, const Props& props, Props& stats)
  {
    (void)filter;
    (void)props;
    Timer timer;
    for (int g = 0; g < scene->children.getSize(); ++g)
    {
      auto mesh = std::dynamic_pointer_cast<TriangleMesh>(scene->children[g]);
      if (!mesh)
        throw std::logic_error("oracle intersector: only flat triangle meshes are supported");
      for (int i = 0; i < mesh->getPrimCount(); ++i)
      {
        const Vec3i idx = mesh->indices[i];
        const Vec3f p0 = mesh->getPosition(idx[0]);
        const Vec3f p1 = mesh->getPosition(idx[1]);
        const Vec3f p2 = mesh->getPosition(idx[2]);
        oracle_bvh::Tri t;
        t.v0[0] = p0.x; t.v0[1] = p0.y; t.v0[2] = p0.z;
        t.e1[0] = p1.x - p0.x; t.e1[1] = p1.y - p0.y; t.e1[2] = p1.z - p0.z;
        t.e2[0] = p2.x - p0.x; t.e2[1] = p2.y - p0.y; t.e2[2] = p2.z - p0.z;
        t.geomId = g;
        t.primId = i;
        bvh.tris.push_back(t);
      }
    }
    bvh.build();
    const double ms = timer.query() * 1000.0;
    stats.set("buildMs", ms);
    stats.set("buildMprim", double(bvh.tris.size()) / 1e6 / std::max(ms * 1e-3, 1e-9));
  }

  const oracle_bvh::Bvh& getBvh() const { return bvh; }

protected:
  template <int N>
  void intersectStream(RayStream<N>& rays, HitStream<N>& hits, int count, IntersectorFilterSimd* filter)
  {
    if (filter)
      throw std::logic_error("oracle intersector: intersection filters are not supported");
    for (int i = 0; i < count; ++i)
    {
      const float o[3] = {rays.org.x[i], rays.org.y[i], rays.org.z[i]};
      const float d[3] = {rays.dir.x[i], rays.dir.y[i], rays.dir.z[i]};
      float tfar = rays.far[i];
      float u = 0.f, v = 0.f;
      const int ti = bvh.intersect(o, d, rays.near[i], tfar, u, v);
      if (ti >= 0)
      {
        rays.far[i] = tfar;
        hits.primId[i] = bvh.tris[ti].primId;
        hits.geomId[i] = bvh.tris[ti].geomId;
        hits.instId[i] = -1;
        hits.u[i] = u;
        hits.v[i] = v;
      }
    }
  }

  // Shadow rays. With a filter (the transparent-shadow filter, render/transparent_filter.h:42)
  // every candidate hit is handed to it as a one-lane ray/hit pair whose far is the hit
  // distance, and the ray is occluded when the filter accepts a hit.
  template <int N>
  void occludedStream(RayStream<N>& rays, int count, IntersectorFilterSimd* filter, void* payload)
  {
    for (int i = 0; i < count; ++i)
    {
      const float o[3] = {rays.org.x[i], rays.org.y[i], rays.org.z[i]};
      const float d[3] = {rays.dir.x[i], rays.dir.y[i], rays.dir.z[i]};
      bool occ;
      if (!filter)
        occ = bvh.occluded(o, d, rays.near[i], rays.far[i]);
      else
        occ = bvh.occludedFiltered(o, d, rays.near[i], rays.far[i], [&](int ti, float t, float u, float v) {
          RaySimd ray;
          ray.org = Vec3vf(vfloat(o[0]), vfloat(o[1]), vfloat(o[2]));
          ray.dir = Vec3vf(vfloat(d[0]), vfloat(d[1]), vfloat(d[2]));
          ray.near = vfloat(rays.near[i]);
          ray.far = vfloat(t);
          HitSimd hit;
          hit.primId = vint(bvh.tris[ti].primId);
          hit.geomId = vint(bvh.tris[ti].geomId);
          hit.instId = vint(-1);
          hit.u = vfloat(u);
          hit.v = vfloat(v);
          const vbool lane0 = vint(step) == vint(0);
          return any(lane0 & filter->filter(lane0, vint(i), ray, hit, payload));
        });
      if (occ)
        rays.far[i] = 0.f;
    }
  }
};

template <int streamSize>
class EmbreeIntersectorPacketStream : public IntersectorStream<streamSize>, public OracleIntersectorBase
{
public:
  EmbreeIntersectorPacketStream(const std::shared_ptr<Group>& scene, bool filter, const Props& props, Props& stats)
    : OracleIntersectorBase(scene, filter, props, stats) {}

  void intersect(RayStream<streamSize>& rays, HitStream<streamSize>& hits, int count, RayStats& stats,
                 RayHint hint, IntersectorFilterSimd* filter, void* payload) override
  {
    (void)hint; (void)payload;
    stats.rayCount += count;
    intersectStream(rays, hits, count, filter);
  }

  void occluded(RayStream<streamSize>& rays, int count, RayStats& stats,
                RayHint hint, IntersectorFilterSimd* filter, void* payload) override
  {
    (void)hint;
    stats.rayCount += count;
    occludedStream(rays, count, filter, payload);
  }
};

template <int streamSize>
class EmbreeIntersectorSingleStream : public EmbreeIntersectorPacketStream<streamSize>
{
public:
  using EmbreeIntersectorPacketStream<streamSize>::EmbreeIntersectorPacketStream;
};

} // namespace prt
