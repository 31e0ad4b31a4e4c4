// Host BVH8 builder: binned-SAH binary BVH down to single primitives, SAH-optimal collapse to
// 8-wide nodes and leaves of at most three triangles, octant slot assignment and 8-bit child-box
// quantisation. See bvh8.h for the node format.
#include "bvh8.h"

#include <deque>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <future>
#include <stdexcept>
#include <thread>

namespace prt {
namespace {

struct Box
{
  float lo[3], hi[3];
  void reset()
  {
    for (int k = 0; k < 3; ++k) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
  }
  void grow(const Box& b)
  {
    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
  }
  float area() const
  {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (dx < 0.f) return 0.f;
    return 2.f * (dx * dy + dy * dz + dz * dx);
  }
};

// Binary node. The binary tree is split down to single primitives; which subtrees become leaves
// of at most kMaxLeaf triangles, and which binary nodes become wide nodes, is decided by the
// SAH-optimal wide collapse of Ylitie, Karras and Laine 2017 (section 3): cost[i - 1] is the
// least SAH cost of representing the subtree by at most i children of a wide node,
//   C(n, 1) = min(Cleaf(n), Cinner(n)),   C(n, i) = min(C(n, i - 1), Cdist(n, i)),
//   Cdist(n, j) = min over k = 1..j-1 of C(left, k) + C(right, j - k),
//   Cleaf(n) = area * primitives * kTriCost (at most kMaxLeaf primitives),
//   Cinner(n) = area * kNodeCost + Cdist(n, 8),
// and dec[i - 1] its decision: for i = 1 kLeafDecision, or kInnerDecision | (slots of the left
// child in Cdist(n, 8)); for i > 1 0 = take C(n, i - 1), k = split the slots k : i - k.
struct BinNode
{
  Box box;
  int left;   // -1 for single-primitive leaves
  int right;
  int first;  // leaves: index into the primitive order
  int count;  // primitives in the subtree
  float cost[8];
  uint8_t dec[8];
};

constexpr int kMaxLeaf = 3;
constexpr int kBins = 32;
constexpr float kNodeCost = 1.0f;
constexpr float kTriCost = 0.6f;
constexpr uint8_t kLeafDecision = 0x40;
constexpr uint8_t kInnerDecision = 0x80;

// Fills the collapse table of an inner node from its children's tables.
void collapseTable(BinNode& n, const BinNode& l, const BinNode& r)
{
  float dist[9];
  uint8_t split[9];
  for (int j = 2; j <= 8; ++j)
  {
    float best = l.cost[0] + r.cost[j - 2];
    int kb = 1;
    for (int k = 2; k < j; ++k)
    {
      const float c = l.cost[k - 1] + r.cost[j - k - 1];
      if (c < best)
      {
        best = c;
        kb = k;
      }
    }
    dist[j] = best;
    split[j] = (uint8_t)kb;
  }
  const float a = n.box.area();
  const float cInner = a * kNodeCost + dist[8];
  const bool leaf = n.count <= kMaxLeaf && a * (float)n.count * kTriCost <= cInner;
  n.cost[0] = leaf ? a * (float)n.count * kTriCost : cInner;
  n.dec[0] = leaf ? kLeafDecision : (uint8_t)(kInnerDecision | split[8]);
  for (int i = 1; i < 8; ++i)
  {
    const bool take = dist[i + 1] < n.cost[i - 1];
    n.cost[i] = take ? dist[i + 1] : n.cost[i - 1];
    n.dec[i] = take ? split[i + 1] : 0;
  }
}

struct BinaryBuilder
{
  const std::vector<Box>& primBox;
  std::vector<float> cx, cy, cz;
  std::vector<int> order;
  std::vector<BinNode> nodes;
  std::atomic<int> nextNode{0};
  std::atomic<int> activeTasks{0};
  int maxTasks;

  BinaryBuilder(const std::vector<Box>& boxes, int threads) : primBox(boxes)
  {
    const size_t n = boxes.size();
    cx.resize(n); cy.resize(n); cz.resize(n);
    order.resize(n);
    for (size_t i = 0; i < n; ++i)
    {
      cx[i] = 0.5f * (boxes[i].lo[0] + boxes[i].hi[0]);
      cy[i] = 0.5f * (boxes[i].lo[1] + boxes[i].hi[1]);
      cz[i] = 0.5f * (boxes[i].lo[2] + boxes[i].hi[2]);
      order[i] = (int)i;
    }
    nodes.resize(std::max<size_t>(2 * n, 1));
    maxTasks = std::max(threads, 1);
  }

  float centroid(int p, int axis) const { return axis == 0 ? cx[p] : (axis == 1 ? cy[p] : cz[p]); }

  int alloc2() { return nextNode.fetch_add(2); }

  void build(int nodeIndex, int begin, int end)
  {
    BinNode& node = nodes[nodeIndex];
    Box bb, cb;
    bb.reset();
    cb.reset();
    for (int i = begin; i < end; ++i)
    {
      const int p = order[i];
      bb.grow(primBox[p]);
      const float c[3] = {cx[p], cy[p], cz[p]};
      for (int k = 0; k < 3; ++k) { cb.lo[k] = std::min(cb.lo[k], c[k]); cb.hi[k] = std::max(cb.hi[k], c[k]); }
    }
    node.box = bb;
    const int count = end - begin;
    node.count = count;
    if (count == 1)
    {
      makeLeaf(node, begin);
      return;
    }
    // Binned SAH over all three axes.
    float bestCost = FLT_MAX;
    int bestAxis = -1, bestSplit = -1;
    for (int axis = 0; axis < 3; ++axis)
    {
      const float ext = cb.hi[axis] - cb.lo[axis];
      if (!(ext > 0.f)) continue;
      const float scale = kBins / ext;
      Box binBox[kBins];
      int binCount[kBins];
      for (int b = 0; b < kBins; ++b) { binBox[b].reset(); binCount[b] = 0; }
      for (int i = begin; i < end; ++i)
      {
        const int p = order[i];
        int b = (int)((centroid(p, axis) - cb.lo[axis]) * scale);
        b = std::min(std::max(b, 0), kBins - 1);
        binCount[b]++;
        binBox[b].grow(primBox[p]);
      }
      float rightArea[kBins];
      int rightCount[kBins];
      Box acc;
      acc.reset();
      int cnt = 0;
      for (int b = kBins - 1; b > 0; --b)
      {
        acc.grow(binBox[b]);
        cnt += binCount[b];
        rightArea[b] = acc.area();
        rightCount[b] = cnt;
      }
      acc.reset();
      cnt = 0;
      for (int b = 1; b < kBins; ++b)
      {
        acc.grow(binBox[b - 1]);
        cnt += binCount[b - 1];
        if (cnt == 0 || rightCount[b] == 0) continue;
        const float cost = acc.area() * cnt + rightArea[b] * rightCount[b];
        if (cost < bestCost) { bestCost = cost; bestAxis = axis; bestSplit = b; }
      }
    }
    int mid;
    if (bestAxis >= 0)
    {
      const float ext = cb.hi[bestAxis] - cb.lo[bestAxis];
      const float scale = kBins / ext;
      const float lo = cb.lo[bestAxis];
      const int axis = bestAxis;
      int* p = std::partition(order.data() + begin, order.data() + end, [&](int prim) {
        int b = (int)((centroid(prim, axis) - lo) * scale);
        b = std::min(std::max(b, 0), kBins - 1);
        return b < bestSplit;
      });
      mid = (int)(p - order.data());
      if (mid == begin || mid == end) mid = begin + count / 2;
    }
    else
    {
      // All centroids coincide: split the range in the middle.
      mid = begin + count / 2;
    }
    const int left = alloc2();
    node.left = left;
    node.right = left + 1;
    node.first = 0;
    const bool spawn = (end - begin) > 65536 && activeTasks.load() < maxTasks;
    if (spawn)
    {
      activeTasks++;
      auto fut = std::async(std::launch::async, [this, left, begin, mid]() { build(left, begin, mid); });
      build(left + 1, mid, end);
      fut.get();
      activeTasks--;
    }
    else
    {
      build(left, begin, mid);
      build(left + 1, mid, end);
    }
    collapseTable(nodes[nodeIndex], nodes[left], nodes[left + 1]);
  }

  void makeLeaf(BinNode& node, int begin)
  {
    node.left = node.right = -1;
    node.first = begin;
    node.count = 1;
    const float c = node.box.area() * kTriCost;
    for (int i = 0; i < 8; ++i)
    {
      node.cost[i] = c;
      node.dec[i] = 0;
    }
    node.dec[0] = kLeafDecision;
  }
};

struct WideBuilder
{
  const BinaryBuilder& bin;
  const float* verts;
  Bvh8& out;
  int maxDepth = 0;

  WideBuilder(const BinaryBuilder& b, const float* v, Bvh8& o) : bin(b), verts(v), out(o) {}

  static void quantAxis(float lo, float hi, float& p, uint8_t& e)
  {
    p = lo;
    const double ext = (double)hi - (double)lo;
    // Smallest power of two with ext / scale <= 253, leaving room to round outward.
    int ex = -126;
    if (ext > 0.0)
    {
      ex = (int)std::ceil(std::log2(ext / 253.0));
      while (std::ldexp(253.0, ex) < ext) ++ex;
      ex = std::max(ex, -126);
    }
    if (ex > 127) throw std::runtime_error("BVH8: scene extent too large for 8-bit quantisation");
    e = (uint8_t)(ex + 127);
  }

  static void quantChild(float p, uint8_t e, float clo, float chi, uint8_t& qlo, uint8_t& qhi)
  {
    const double scale = std::ldexp(1.0, (int)e - 127);
    const float fs = (float)scale;
    double a = std::floor(((double)clo - (double)p) / scale);
    double b = std::ceil(((double)chi - (double)p) / scale);
    // One extra quantum where the bound lands exactly on the grid, so that rounding in the
    // kernel's plane distances never shrinks a box; then verify in single precision.
    if (a > 0.0 && (double)p + a * scale == (double)clo) a -= 1.0;
    if ((double)p + b * scale == (double)chi) b += 1.0;
    a = std::max(a, 0.0);
    b = std::min(b, 255.0);
    while (a > 0.0 && p + (float)a * fs > clo) a -= 1.0;
    while (b < 255.0 && p + (float)b * fs < chi) b += 1.0;
    qlo = (uint8_t)a;
    qhi = (uint8_t)b;
  }

  // Emits the wide node `wideIndex` for binary node `binIndex`. Its children follow the collapse
  // table: a binary node whose C(n, 1) is a leaf is one leaf child; otherwise its eight slots are
  // split between its children as recorded, and each (node, slots) pair is resolved by its own
  // decisions until it is one child (a leaf, or the root of a wide subtree).
  void emit(int wideIndex, int binIndex, int depth)
  {
    maxDepth = std::max(maxDepth, depth + 1);
    int children[8];
    bool childInner[8];
    int n = 0;
    const BinNode& root = bin.nodes[binIndex];
    if (root.dec[0] & kLeafDecision)
    {
      children[n] = binIndex;
      childInner[n++] = false;
    }
    else
    {
      int pn[8], pi[8];
      int sp = 0;
      const int k0 = root.dec[0] & 15;
      pn[sp] = root.right; pi[sp++] = 8 - k0;
      pn[sp] = root.left; pi[sp++] = k0;
      while (sp > 0 && n < 8)
      {
        const int x = pn[--sp];
        int i = pi[sp];
        const BinNode& c = bin.nodes[x];
        while (i > 1 && c.dec[i - 1] == 0) --i;
        if (i <= 1)
        {
          children[n] = x;
          childInner[n++] = (c.dec[0] & kInnerDecision) != 0;
          continue;
        }
        const int k = c.dec[i - 1];
        pn[sp] = c.right; pi[sp++] = i - k;
        pn[sp] = c.left; pi[sp++] = k;
      }
    }
    // Node box.
    Box nb;
    nb.reset();
    for (int i = 0; i < n; ++i) nb.grow(bin.nodes[children[i]].box);
    // Slot assignment: slot s stands for the direction whose axis k is negative iff bit k of
    // s is set; a child goes to the free slot that maximises dot(child centre - node centre,
    // slot direction). A ray whose negative-axis bits are r then visits hit children by
    // descending (slot ^ r), which is approximately front to back.
    float cost[8][8];
    for (int i = 0; i < n; ++i)
    {
      const Box& b = bin.nodes[children[i]].box;
      float d[3];
      for (int k = 0; k < 3; ++k) d[k] = 0.5f * (b.lo[k] + b.hi[k]) - 0.5f * (nb.lo[k] + nb.hi[k]);
      for (int s = 0; s < 8; ++s)
      {
        float c = 0.f;
        for (int k = 0; k < 3; ++k) c += ((s >> k) & 1) ? -d[k] : d[k];
        cost[i][s] = c;
      }
    }
    int slotOf[8];
    int childOfSlot[8];
    bool usedChild[8] = {false, false, false, false, false, false, false, false};
    for (int s = 0; s < 8; ++s) childOfSlot[s] = -1;
    for (int round = 0; round < n; ++round)
    {
      float best = -FLT_MAX;
      int bi = -1, bs = -1;
      for (int i = 0; i < n; ++i)
      {
        if (usedChild[i]) continue;
        for (int s = 0; s < 8; ++s)
        {
          if (childOfSlot[s] >= 0) continue;
          if (cost[i][s] > best) { best = cost[i][s]; bi = i; bs = s; }
        }
      }
      usedChild[bi] = true;
      childOfSlot[bs] = bi;
      slotOf[bi] = bs;
    }
    (void)slotOf;

    Bvh8Node node;
    std::memset(&node, 0, sizeof(node));
    quantAxis(nb.lo[0], nb.hi[0], node.px, node.ex);
    quantAxis(nb.lo[1], nb.hi[1], node.py, node.ey);
    quantAxis(nb.lo[2], nb.hi[2], node.pz, node.ez);

    // Leaf triangles first (contiguous per node), then inner children as one block.
    node.triBase = (uint32_t)out.tris.size();
    int triOffset = 0;
    int innerSlots[8];
    int innerN = 0;
    for (int s = 0; s < 8; ++s)
    {
      const int ci = childOfSlot[s];
      if (ci < 0) continue;
      const BinNode& c = bin.nodes[children[ci]];
      quantChild(node.px, node.ex, c.box.lo[0], c.box.hi[0], node.qlox[s], node.qhix[s]);
      quantChild(node.py, node.ey, c.box.lo[1], c.box.hi[1], node.qloy[s], node.qhiy[s]);
      quantChild(node.pz, node.ez, c.box.lo[2], c.box.hi[2], node.qloz[s], node.qhiz[s]);
      if (childInner[ci])
      {
        node.imask |= (uint8_t)(1u << s);
        innerSlots[innerN++] = children[ci];
      }
      else
      {
        // The leaf's primitives, left to right (at most kMaxLeaf, so at most two inner nodes).
        int prims[kMaxLeaf];
        int np = 0;
        int stack[kMaxLeaf + 1];
        int sp = 0;
        stack[sp++] = children[ci];
        while (sp > 0)
        {
          const BinNode& x = bin.nodes[stack[--sp]];
          if (x.left < 0)
          {
            if (np < kMaxLeaf) prims[np++] = bin.order[x.first];
          }
          else if (sp + 2 <= kMaxLeaf + 1)
          {
            stack[sp++] = x.right;
            stack[sp++] = x.left;
          }
        }
        if (np != c.count) throw std::logic_error("BVH8: leaf larger than the leaf limit");
        node.meta[s] = (uint8_t)((np << 5) | triOffset);
        for (int j = 0; j < np; ++j)
        {
          const int prim = prims[j];
          const float* v = verts + 9 * (size_t)prim;
          Bvh8Tri t;
          t.v0x = v[0]; t.v0y = v[1]; t.v0z = v[2];
          t.triId = prim;
          t.e1x = v[3] - v[0]; t.e1y = v[4] - v[1]; t.e1z = v[5] - v[2];
          t.e2x = v[6] - v[0]; t.e2y = v[7] - v[1]; t.e2z = v[8] - v[2];
          t.pad1 = t.pad2 = 0.f;
          out.tris.push_back(t);
        }
        triOffset += np;
      }
    }
    node.childBase = (uint32_t)out.nodes.size();
    out.nodes.resize(out.nodes.size() + innerN);
    out.nodes[wideIndex] = node;
    const uint32_t base = node.childBase;
    // Children in the top levels are emitted breadth-first (queued), deeper ones depth-first.
    for (int i = 0; i < innerN; ++i)
    {
      if (depth + 1 < kBvh8TopLevels) pending.push_back({(int)base + i, innerSlots[i], depth + 1});
      else emit((int)base + i, innerSlots[i], depth + 1);
    }
  }

  struct Pending
  {
    int wideIndex, binIndex, depth;
  };
  std::deque<Pending> pending;

  // Emits the whole tree: the top levels level by level, then each subtree depth-first.
  void emitAll()
  {
    emit(0, 0, 0);
    while (!pending.empty())
    {
      const Pending p = pending.front();
      pending.pop_front();
      emit(p.wideIndex, p.binIndex, p.depth);
    }
  }
};

} // namespace

void buildBvh8(const float* triVerts, int64_t triCount, Bvh8& out, int threads)
{
  auto t0 = std::chrono::steady_clock::now();
  if (triCount < 0 || triCount > (int64_t)0x3fffffff)
    throw std::invalid_argument("BVH8: triangle count out of range");
  out.nodes.clear();
  out.tris.clear();
  out.maxDepth = 0;
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  const int n = (int)triCount;
  if (n == 0)
  {
    Bvh8Node empty;
    std::memset(&empty, 0, sizeof(empty));
    out.nodes.push_back(empty);
    out.maxDepth = 1;
    for (int k = 0; k < 3; ++k) { out.lo[k] = 0.f; out.hi[k] = 0.f; }
    return;
  }
  std::vector<Box> boxes(n);
  for (int i = 0; i < n; ++i)
  {
    const float* v = triVerts + 9 * (size_t)i;
    for (int k = 0; k < 3; ++k)
    {
      // Boxes of the triangle as the kernel sees it (v0 + e1, v0 + e2 reconstructed in float).
      const float a = v[k];
      const float b = v[k] + (v[3 + k] - v[k]);
      const float c = v[k] + (v[6 + k] - v[k]);
      boxes[i].lo[k] = std::min(std::min(a, b), std::min(c, std::min(v[3 + k], v[6 + k])));
      boxes[i].hi[k] = std::max(std::max(a, b), std::max(c, std::max(v[3 + k], v[6 + k])));
    }
  }
  BinaryBuilder bb(boxes, threads);
  bb.nextNode = 1;
  bb.build(0, 0, n);
  out.tris.reserve(n);
  out.nodes.reserve(n / 2 + 1);
  out.nodes.resize(1);
  WideBuilder wb(bb, triVerts, out);
  wb.emitAll();
  out.maxDepth = wb.maxDepth;
  // Nodes of the top levels: the root, then every node whose parent is in the top levels.
  {
    int count = 1, levelBegin = 0, levelEnd = 1;
    for (int level = 1; level < kBvh8TopLevels; ++level)
    {
      int next = 0;
      for (int i = levelBegin; i < levelEnd; ++i) next += __builtin_popcount(out.nodes[i].imask);
      levelBegin = levelEnd;
      levelEnd += next;
      count += next;
    }
    out.topCount = std::min(count, (int)out.nodes.size());
  }
  for (int k = 0; k < 3; ++k) { out.lo[k] = bb.nodes[0].box.lo[k]; out.hi[k] = bb.nodes[0].box.hi[k]; }
  out.buildMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// ---- host reference traversal (counting) ------------------------------------------------
namespace {

inline float fmaF(float a, float b, float c) { return std::fmaf(a, b, c); }

inline bool triTest(const Bvh8Tri& t, const float o[3], const float d[3], float tnear, float tfar,
                    float& tt, float& uu, float& vv)
{
  const float e1[3] = {t.e1x, t.e1y, t.e1z}, e2[3] = {t.e2x, t.e2y, t.e2z};
  const float p[3] = {fmaF(d[1], e2[2], -(d[2] * e2[1])), fmaF(d[2], e2[0], -(d[0] * e2[2])),
                      fmaF(d[0], e2[1], -(d[1] * e2[0]))};
  const float det = fmaF(e1[0], p[0], fmaF(e1[1], p[1], e1[2] * p[2]));
  if (!(det != 0.f)) return false;
  const float s[3] = {o[0] - t.v0x, o[1] - t.v0y, o[2] - t.v0z};
  const float q[3] = {fmaF(s[1], e1[2], -(s[2] * e1[1])), fmaF(s[2], e1[0], -(s[0] * e1[2])),
                      fmaF(s[0], e1[1], -(s[1] * e1[0]))};
  const float inv = 1.0f / det;
  const float u = fmaF(s[0], p[0], fmaF(s[1], p[1], s[2] * p[2])) * inv;
  const float v = fmaF(d[0], q[0], fmaF(d[1], q[1], d[2] * q[2])) * inv;
  const float tv = fmaF(e2[0], q[0], fmaF(e2[1], q[1], e2[2] * q[2])) * inv;
  if (!(u >= 0.f) || !(v >= 0.f) || !(u + v <= 1.f)) return false;
  if (!(tv >= tnear) || !(tv <= tfar)) return false;
  tt = tv; uu = u; vv = v;
  return true;
}

inline float expScale(uint8_t e)
{
  uint32_t bits = (uint32_t)e << 23;
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

} // namespace

int bvh8TraceCount(const Bvh8& bvh, const float org[3], const float dir[3], float tnear, float& tfar,
                   int64_t& nodeVisits, int64_t& triTests)
{
  return bvh8TraceCount(bvh.nodes.data(), bvh.tris.data(), org, dir, tnear, tfar, nodeVisits, triTests);
}

int bvh8TraceCount(const Bvh8Node* nodes, const Bvh8Tri* tris, const float org[3], const float dir[3], float tnear,
                   float& tfar, int64_t& nodeVisits, int64_t& triTests)
{
  float inv[3];
  for (int k = 0; k < 3; ++k)
  {
    float d = dir[k];
    if (std::fabs(d) < 8.271806e-25f) d = std::copysign(8.271806e-25f, d); // 2^-80
    inv[k] = 1.0f / d;
  }
  const int oct = (dir[0] < 0.f ? 1 : 0) | (dir[1] < 0.f ? 2 : 0) | (dir[2] < 0.f ? 4 : 0);
  struct Entry { uint32_t node; };
  std::vector<uint32_t> stack;
  stack.push_back(0);
  int best = -1;
  float bestT = tfar;
  while (!stack.empty())
  {
    const Bvh8Node& n = nodes[stack.back()];
    stack.pop_back();
    nodeVisits++;
    const float sx = expScale(n.ex), sy = expScale(n.ey), sz = expScale(n.ez);
    const float ax = (n.px - org[0]) * inv[0], ay = (n.py - org[1]) * inv[1], az = (n.pz - org[2]) * inv[2];
    const float bx = sx * inv[0], by = sy * inv[1], bz = sz * inv[2];
    // Hit children in traversal order (descending slot ^ oct); push inner ones far-first.
    uint32_t order[8];
    int nh = 0;
    for (int b = 7; b >= 0; --b)
    {
      const int s = b ^ oct;
      if (!(n.imask & (1 << s)) && n.meta[s] == 0) continue;
      const float x0 = fmaF((float)n.qlox[s], bx, ax), x1 = fmaF((float)n.qhix[s], bx, ax);
      const float y0 = fmaF((float)n.qloy[s], by, ay), y1 = fmaF((float)n.qhiy[s], by, ay);
      const float z0 = fmaF((float)n.qloz[s], bz, az), z1 = fmaF((float)n.qhiz[s], bz, az);
      const float tmin = std::max(std::max(std::min(x0, x1), std::min(y0, y1)), std::max(std::min(z0, z1), tnear));
      const float tmax = std::min(std::min(std::max(x0, x1), std::max(y0, y1)), std::min(std::max(z0, z1), bestT));
      if (!(tmin <= tmax * 1.000002f)) continue;
      order[nh++] = (uint32_t)s;
    }
    for (int i = nh - 1; i >= 0; --i)
    {
      const int s = (int)order[i];
      if (n.imask & (1 << s))
      {
        const uint32_t rel = (uint32_t)__builtin_popcount(n.imask & ((1u << s) - 1u));
        stack.push_back(n.childBase + rel);
      }
    }
    for (int i = 0; i < nh; ++i)
    {
      const int s = (int)order[i];
      if (n.imask & (1 << s)) continue;
      const int cnt = n.meta[s] >> 5, off = n.meta[s] & 31;
      for (int j = 0; j < cnt; ++j)
      {
        const Bvh8Tri& t = tris[n.triBase + off + j];
        triTests++;
        float tt, uu, vv;
        if (triTest(t, org, dir, tnear, bestT, tt, uu, vv))
        {
          if (tt < bestT || best < 0 || t.triId < best)
          {
            bestT = tt;
            best = t.triId;
          }
        }
      }
    }
  }
  if (best >= 0) tfar = bestT;
  return best;
}

// ---- structural check -----------------------------------------------------------------------

std::string bvh8Check(const Bvh8Node* nodes, int64_t nodeCount, const Bvh8Tri* tris, int64_t triCount,
                      const float* triVerts, int topCount, int& depth)
{
  depth = 0;
  if (nodeCount < 1 || !nodes) return "no nodes";
  if (triCount < 0 || (triCount > 0 && (!tris || !triVerts))) return "invalid triangle arrays";
  auto at = [](const char* what, int64_t i) { return std::string(what) + " (node " + std::to_string(i) + ")"; };
  // Breadth-first walk from the root: every node reached once, indices in range.
  std::vector<int> level(nodeCount, 0);
  std::vector<uint8_t> recSeen(triCount, 0);
  std::vector<int64_t> order;
  order.reserve(nodeCount);
  order.push_back(0);
  level[0] = 1;
  for (size_t q = 0; q < order.size(); ++q)
  {
    const int64_t i = order[q];
    const Bvh8Node& n = nodes[i];
    depth = std::max(depth, level[i]);
    int inner = 0;
    for (int s = 0; s < 8; ++s)
    {
      if (n.imask & (1u << s))
      {
        if (n.meta[s] != 0) return at("inner slot with leaf metadata", i);
        const int64_t c = (int64_t)n.childBase + inner++;
        if (c >= nodeCount || c <= 0) return at("child index out of range", i);
        if (level[c] != 0) return at("node reached twice", c);
        level[c] = level[i] + 1;
        order.push_back(c);
      }
      else if (n.meta[s] != 0)
      {
        const int cnt = n.meta[s] >> 5, off = n.meta[s] & 31;
        if (cnt < 1 || cnt > 3 || off + cnt > 24) return at("bad leaf metadata", i);
        for (int j = 0; j < cnt; ++j)
        {
          const int64_t r = (int64_t)n.triBase + off + j;
          if (r >= triCount) return at("triangle index out of range", i);
          if (recSeen[r]) return at("triangle record referenced twice", i);
          recSeen[r] = 1;
        }
      }
    }
  }
  if (depth > kBvh8TraceStack) return "tree deeper than the traversal stack (" + std::to_string(depth) + " levels)";
  if ((int64_t)order.size() != nodeCount) return "unreachable nodes";
  // Triangle records: every record referenced, every triangle stored once, exact vertex data.
  std::vector<uint8_t> idSeen(triCount, 0);
  auto same = [](float a, float b) { return std::memcmp(&a, &b, 4) == 0; };
  for (int64_t r = 0; r < triCount; ++r)
  {
    if (!recSeen[r]) return "triangle record " + std::to_string(r) + " never referenced";
    const Bvh8Tri& t = tris[r];
    if (t.triId < 0 || t.triId >= triCount) return "triangle id out of range (record " + std::to_string(r) + ")";
    if (idSeen[t.triId]) return "triangle " + std::to_string(t.triId) + " stored twice";
    idSeen[t.triId] = 1;
    const float* v = triVerts + 9 * (size_t)t.triId;
    const float e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]}, e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
    if (!same(t.v0x, v[0]) || !same(t.v0y, v[1]) || !same(t.v0z, v[2]) || !same(t.e1x, e1[0]) ||
        !same(t.e1y, e1[1]) || !same(t.e1z, e1[2]) || !same(t.e2x, e2[0]) || !same(t.e2y, e2[1]) ||
        !same(t.e2z, e2[2]))
      return "triangle " + std::to_string(t.triId) + " has wrong vertex data";
  }
  // Containment, children before parents: each slot's 8-bit box, dequantised in single
  // precision, holds the boxes of the triangles below it (reconstructed vertices).
  std::vector<Box> content(nodeCount);
  for (size_t q = order.size(); q-- > 0;)
  {
    const int64_t i = order[q];
    const Bvh8Node& n = nodes[i];
    const float p[3] = {n.px, n.py, n.pz};
    const uint8_t e[3] = {n.ex, n.ey, n.ez};
    const uint8_t* qlo[3] = {n.qlox, n.qloy, n.qloz};
    const uint8_t* qhi[3] = {n.qhix, n.qhiy, n.qhiz};
    Box all;
    all.reset();
    int inner = 0;
    for (int s = 0; s < 8; ++s)
    {
      Box b;
      b.reset();
      if (n.imask & (1u << s))
        b = content[n.childBase + inner++];
      else if (n.meta[s] != 0)
        for (int j = 0; j < (n.meta[s] >> 5); ++j)
        {
          const Bvh8Tri& t = tris[n.triBase + (n.meta[s] & 31) + j];
          const float v0[3] = {t.v0x, t.v0y, t.v0z}, a[3] = {t.e1x, t.e1y, t.e1z}, c[3] = {t.e2x, t.e2y, t.e2z};
          for (int k = 0; k < 3; ++k)
          {
            const float x1 = v0[k] + a[k], x2 = v0[k] + c[k];
            const float* v = triVerts + 9 * (size_t)t.triId;
            b.lo[k] = std::min(b.lo[k], std::min(std::min(v0[k], x1), std::min(x2, std::min(v[3 + k], v[6 + k]))));
            b.hi[k] = std::max(b.hi[k], std::max(std::max(v0[k], x1), std::max(x2, std::max(v[3 + k], v[6 + k]))));
          }
        }
      else
        continue;
      for (int k = 0; k < 3; ++k)
      {
        const float fs = (float)std::ldexp(1.0, (int)e[k] - 127);
        const float lo = p[k] + (float)qlo[k][s] * fs, hi = p[k] + (float)qhi[k][s] * fs;
        if (qlo[k][s] > qhi[k][s] || lo > b.lo[k] || hi < b.hi[k])
          return at("child box does not contain its subtree", i) + " slot " + std::to_string(s) + " axis " +
                 std::to_string(k);
      }
      all.grow(b);
    }
    content[i] = all;
  }
  // The first topCount nodes are exactly the first kBvh8TopLevels levels.
  if (topCount < 1 || topCount > kBvh8TopNodes || topCount > nodeCount) return "top count out of range";
  for (int64_t i = 0; i < nodeCount; ++i)
    if ((level[i] <= kBvh8TopLevels) != (i < topCount)) return at("top levels not stored first", i);
  return std::string();
}

} // namespace prt
