// Host loaders of the reference's scene files, producing the flat prt_scene_desc of
// include/prt_cuda.h (Scene::Scene, render/scene.cpp:65-77, picks the loader by extension):
//
// * .rkscene: a JSON document with one binary buffer (.rkbin) of vertex, index and instance
//   arrays, and image files for texture maps. Follows rkscene::load (rkscene/rkscene.h:264-905:
//   buffers, typed buffer views, materials, geometries, objects, lights) and the geometry /
//   material half of Scene::loadScene (render/scene.cpp:174-362): every file material becomes a
//   Standard material, geometries without a (valid) material get the default (Principled)
//   material, and each object adds its geometries to the scene -- once, or once per instance
//   transform with positions and normals transformed (TriangleMesh::clone,
//   geometry/triangle_mesh.cpp:326-356). The device has no two-level BVH, so instances are
//   always flattened (the reference flattens them with its "flatten" prop and for emissive
//   objects).
// * .mesh: the reference's TriangleMesh blob (sys/blob.h, geometry/triangle_mesh.cpp:362-378:
//   blob id, bounds, counts, indices, per-triangle material ids, interleaved vertex attributes,
//   material names) with the Wavefront material library of the same name (.mtl, read as
//   material/mtl_loader.cpp does), made into materials as Scene::loadMesh
//   (render/scene.cpp:136-172) and MaterialFactory::make (material/material_factory.cpp:29-96)
//   do: "Standard", "Principled", or the default "OBJ" type mapped onto a Principled material.
//   The device binds one material per mesh, so the blob's triangles are split into one mesh
//   per material, in material order.
//
// The environment lights come from the caller (Scene::initLights reads them from props, not from
// the file, whose lights list is parsed and checked only).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/prt_cuda.h"

namespace prt {

struct RkScene
{
  std::vector<std::vector<float>> positions;   // per emitted mesh
  std::vector<std::vector<float>> normals;
  std::vector<std::vector<float>> texcoords;
  std::vector<std::vector<int32_t>> indices;
  std::vector<prt_mesh> meshes;
  std::vector<prt_material> materials;
  std::vector<std::vector<float>> texturePixels;  // RGB FP32, row 0 at the top
  std::vector<prt_texture> textures;
  std::vector<std::string> texturePaths;
  int64_t triangleCount = 0;

  // Points `desc` at this scene's arrays (valid while the RkScene lives and is not changed);
  // env is zeroed and bvh_build set to PRT_BVH_HOST.
  void describe(prt_scene_desc& desc) const;
};

// Loads `path` by its extension (.rkscene or .mesh); throws std::invalid_argument (malformed
// or unsupported content) or std::runtime_error (a file that cannot be opened or read).
void loadSceneFile(const std::string& path, RkScene& out);

void loadRkScene(const std::string& path, RkScene& out);
void loadMeshScene(const std::string& path, RkScene& out);

} // namespace prt
