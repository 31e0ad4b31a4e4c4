// Device (GPU) builder of the compressed BVH8 (bvh8.h) that the traversal kernels walk.
//
// Replaces the reference's Embree build (accel/embree_intersector.cpp:68-90, rtcCommitScene,
// reported as buildMs / buildMprim) with a build that runs on the GPU from the scene arrays
// already in HBM:
//   1. triangle boxes and centroid bounds, 63-bit Morton codes of the centroids;
//   2. a stable LSD radix sort of (code, triangle) pairs;
//   3. PLOC clustering (Meister and Bittner 2018, "Parallel Locally-Ordered Clustering for
//      Bounding Volume Hierarchy Construction"): every cluster finds its nearest neighbour by
//      merged-box surface area within a window of the Morton order, mutual neighbours merge,
//      the survivors are compacted; repeated until one cluster is left. Each merge also fills
//      the node's table of the SAH-optimal wide collapse (Ylitie, Karras and Laine 2017), whose
//      inputs, the children's tables, are final by then;
//   4. a top-down collapse, one wide level per step, that follows the tables: which subtrees
//      become leaves of at most three triangles and which become wide nodes; children are
//      assigned to ray-octant slots and their boxes quantised to 8 bits exactly as the host
//      builder does.
// Wide nodes are stored breadth-first over the whole tree, so the first three levels come
// first (the shared-memory staged top levels). Every step is a scan-based, order-independent
// computation, so a build is deterministic: the same scene gives the same bytes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace prt {

struct DeviceBvh8
{
  void* nodes = nullptr;   // Bvh8Node[nodeCount], cudaMalloc'd; the caller owns it
  void* tris = nullptr;    // Bvh8Tri[triCount], cudaMalloc'd; the caller owns it
  int64_t nodeCount = 0;
  int64_t triCount = 0;
  int topCount = 1;        // nodes of the first kBvh8TopLevels levels (stored first)
  int maxDepth = 0;        // wide levels
  int plocIterations = 0;  // clustering iterations (large-phase launches + the in-block tail)
  double buildMs = 0.0;    // wall time of the build, launches and waits included
};

// Builds over triCount triangles; triangle t has the vertices pos[triVerts[t].x/y/z] (xyz of
// each float4). All work is queued on `stream`; the call returns when the build is complete.
// Throws std::runtime_error on a CUDA error or a scene the 8-bit quantisation cannot hold.
void buildBvh8Device(const float4* pos, const int4* triVerts, int64_t triCount, cudaStream_t stream,
                     DeviceBvh8& out);

} // namespace prt
