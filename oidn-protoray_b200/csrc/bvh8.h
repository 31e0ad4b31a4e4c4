// Host-side builder of the compressed 8-wide BVH that the GPU traversal kernels walk.
//
// Replaces the reference's Embree build (accel/embree_intersector.cpp:11-90, "bvh8.triangle4"
// with SAH). The format follows the compressed wide BVH of Ylitie, Karras and Laine 2017:
// each node is 80 bytes (five 16-byte loads) holding a quantisation origin, three power-of-two
// scale exponents and 8-bit child boxes, so a node visit costs one cache line pair. Children are
// placed in slots by ray octant at build time so that a traversal that visits hit children by
// descending (slot ^ ray octant) goes roughly front to back.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace prt {

// 80-byte compressed wide node. All offsets are element indices.
struct alignas(16) Bvh8Node
{
  float px, py, pz;        // quantisation origin (node box minimum)
  uint8_t ex, ey, ez;      // child box scale per axis = 2^(e - 127)
  uint8_t imask;           // bit s: slot s holds an inner node
  uint32_t childBase;      // first inner child; inner children are stored in slot order
  uint32_t triBase;        // first triangle of the leaf children
  uint8_t meta[8];         // leaf slot: (count << 5) | offset (count 1..3, offset 0..23); 0 = empty
  uint8_t qlox[8], qloy[8], qloz[8];
  uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(Bvh8Node) == 80, "Bvh8Node must be 80 bytes");

// 48-byte triangle record: v0 and the two edges, plus the global triangle index (meshes
// concatenated in scene order) stored in the w lane of the first vector.
struct alignas(16) Bvh8Tri
{
  float v0x, v0y, v0z;
  int32_t triId;
  float e1x, e1y, e1z, pad1;
  float e2x, e2y, e2z, pad2;
};
static_assert(sizeof(Bvh8Tri) == 48, "Bvh8Tri must be 48 bytes");

// The first kBvh8TopLevels levels of the tree are stored breadth-first at the start of the
// node array (at most 1 + 8 + 64 = kBvh8TopNodes nodes), so that a kernel can stage them in
// shared memory; deeper levels are stored depth-first, each subtree contiguous.
constexpr int kBvh8TopLevels = 3;
constexpr int kBvh8TopNodes = 73;

// Node-group stack entries of the traversal kernels. A ray holds at most one group per level
// above the node it visits, so a tree of at most kBvh8TraceStack wide levels never overflows.
constexpr int kBvh8TraceStack = 48;

struct Bvh8
{
  std::vector<Bvh8Node> nodes;
  std::vector<Bvh8Tri> tris;
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // scene bounds
  int maxDepth = 0;                             // wide levels
  int topCount = 1;                             // nodes of the first kBvh8TopLevels levels (stored first)
  double buildMs = 0.0;
};

// Builds the BVH over `triCount` triangles; positions are given per triangle as 9 floats
// (v0, v1, v2). Edges are computed as v1 - v0 and v2 - v0 in single precision, exactly as the
// oracle intersector computes them, so that intersection results agree bit for bit.
void buildBvh8(const float* triVerts, int64_t triCount, Bvh8& out, int threads = 0);

// Counting traversal on the host (scalar, same box and triangle tests as the kernels):
// returns the closest hit triangle (-1 on a miss) and adds the number of nodes visited and
// triangles tested. Used to state the algorithmic bytes per ray.
int bvh8TraceCount(const Bvh8& bvh, const float org[3], const float dir[3], float tnear, float& tfar,
                   int64_t& nodeVisits, int64_t& triTests);
int bvh8TraceCount(const Bvh8Node* nodes, const Bvh8Tri* tris, const float org[3], const float dir[3], float tnear,
                   float& tfar, int64_t& nodeVisits, int64_t& triTests);

// Structural check of a BVH8 given as arrays over triCount triangles (9 floats each): see
// prt_bvh8_check. Returns an empty string when the tree is valid, else the first violation;
// depth receives the number of wide levels.
std::string bvh8Check(const Bvh8Node* nodes, int64_t nodeCount, const Bvh8Tri* tris, int64_t triCount,
                      const float* triVerts, int topCount, int& depth);

} // namespace prt
