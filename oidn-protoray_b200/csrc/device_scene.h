// Device-resident scene, renderer and frame state shared by the host runtime and the kernels.
// Plain structs of device pointers and scalars, passed to kernels by value.
#pragma once

#include <cstdint>

namespace prt {

// Material type bits (material/material.h MaterialType).
enum : int
{
  kMatEmissive = 1 << 0,
  kMatTransmissive = 1 << 1,
  kMatMediaInterface = 1 << 2,
  kMatTransparent = 1 << 3,
  kMatMiss = 1 << 4,          // PRT_MATERIAL_MISS: hits end the path as misses
};

// Lobe features of a Standard material, known per material at upload. A shading kernel
// instantiated for a feature set compiles only those lobes; kFeatAll keeps every branch.
enum : int
{
  kFeatOpaque = 1 << 0,     // Lambertian opaque base
  kFeatSpecular = 1 << 1,   // dielectric specular layer over the opaque base
  kFeatDielectric = 1 << 2, // transmissive dielectric base
  kFeatConductor = 1 << 3,  // metal base
  kFeatCoat = 1 << 4,       // outer coat layer
  kFeatSheen = 1 << 5,      // outermost sheen layer
  kFeatRoughDiffuse = 1 << 6, // Oren-Nayar base instead of Lambert
  kFeatSubsurface = 1 << 7, // thin-walled subsurface / backlight: diffuse BRDF + BTDF in the opaque base
  kFeatThin = 1 << 8,       // thin-walled dielectric transmission (unbent)
  kFeatTransparent = 1 << 9, // transparent (continuation) lobe: opacity < 1, or transmission with ior == ambient
  kFeatAll = 1023,
};

// Shading classes: 0 ends the path (miss, area-light hit, maxDepth); 1.. shade a surface with
// the lobe features listed here. Materials whose features match no specialised class use the
// last (general) class.
constexpr int kShadeClasses = 8;
constexpr int kShadeClassFeatures[kShadeClasses] = {
  0,
  kFeatOpaque,
  kFeatOpaque | kFeatSpecular,
  kFeatConductor,
  kFeatDielectric,
  kFeatOpaque | kFeatCoat,
  kFeatOpaque | kFeatSpecular | kFeatCoat,
  kFeatAll,
};

// One side of a dielectric interface (index 0: hit from outside, 1: from inside), resolved on
// the host with hostRcp: eta = clamp(outsideIor * rcp(insideIor), 1/3, 3) as
// StandardMaterial::getBsdfLobes forms it (material/standard.cpp:217-218, 357), and the values
// the lobes derive from eta with rcp (bsdf/rough_dielectric.h:39-46,105,155;
// bsdf/rough_coating.h:41; bsdf/coating.h:33-36; bsdf/thin_rough_dielectric.h:43).
struct DevEta
{
  float eta;
  float rcpEta;    // rcp(eta)
  float rcpEta2;   // rcp(eta^2)
  float favg;      // fresnelDielectricAvg(eta)
  float favgRcp;   // fresnelDielectricAvg(rcp(eta))
};

// A Standard material with its parameters read and clamped as StandardMaterial::getBsdfLobes
// reads them (material/standard.cpp:410-620). "has*" flags mirror the MaterialParam truth
// tests that pick rough versus smooth lobes (material/material_param.h:49,181).
struct DevMaterial
{
  DevEta spec[2];        // specular interface (ambientIor | specularIor)
  DevEta coat[2];        // coat interface (ambientIor | coatIor)
  int type;
  int features;          // kFeat* lobes the material can produce
  int shadeClass;        // index into kShadeClassFeatures (0 for emissive materials)
  int baseColorTex;      // texture index or -1
  int mediumInt, mediumExt;
  float baseWeight;
  float baseColor[3];    // factor (multiplies the texture when textured)
  float metalness;
  float diffuseRoughness;
  int hasDiffuseRoughness;
  float specularWeight;
  float specularColor[3];
  float specularRoughness;
  int hasSpecularRoughness;
  float specularIor;
  float ambientIor;
  float transmissionWeight;
  float transmissionColor[3];
  float transmissionDepth;
  float subsurfaceWeight;
  float subsurfaceColor[3];
  float subsurfaceAnisotropy;
  float coatWeight;
  float coatColor[3];
  float coatRoughness;
  int hasCoatRoughness;
  float coatIor;
  float sheenWeight;
  float sheenColor[3];
  float sheenRoughness;
  float sheenTint;       // sheen colour = lerp(sheenColor, baseColor, sheenTint) (Principled)
  float coatThickness;   // 0.5 for Standard, "coatThickness" for Principled
  int principled;        // PrincipledMaterial: the conductor uses the unweighted base colour
  float emission[3];     // emissionColor * emissionLuminance
  int thinWalled;
  float opacity;
  float thinThickness;   // thin-walled transmission: thickness / transmissionDepth
  int subsurfaceFromBase; // Principled backlight: the subsurface colour is the (textured) diffuse colour
};

struct DevTexture
{
  const float* rgb;  // texture-row order: row 0 is the bottom image row
  int width, height;
};

// Environment light kinds, in Scene::initLights order (render/scene.cpp:365-450).
enum : int
{
  kEnvDistant = 1,
  kEnvAmbient = 2,
  kEnvImage = 3,
};

struct DevEnvLight
{
  int kind;
  float color[3];     // distant/ambient radiance
  float dir[3];       // distant: unit direction toward the light
  float frameU[3], frameV[3];
  float cosAngle;     // distant: cos of the cone half angle
  float conePdf;      // distant: 1 / (4 pi sin^2(angle/2))
  float halfAngle;
};

struct DevImageLight
{
  const float* rgb;       // width*height*3, texture-row order (row 0 = bottom)
  int width, height;
  int lutW, lutH;         // LUT (Distribution2D) size
  const float* yCdf;      // lutH + 1
  const float* xCdfs;     // lutH * (lutW + 1)
};

struct DevScene
{
  // BVH8 (bvh8.h)
  const uint4* nodes;
  const float4* tris;
  int64_t triCount;
  // Shading data per global triangle: vertex indices (global) and mesh index.
  const int4* triVerts;      // x, y, z: global vertex indices; w: mesh index
  const float4* pos;         // per vertex
  const float4* nrm;         // per vertex, or null where a mesh has no normals
  const float2* uv;          // per vertex, or null where a mesh has no texcoords
  const int* meshFlags;      // bit 0: has normals, bit 1: has texcoords
  const int* meshMaterial;   // material index per mesh
  const int* meshTriOffset;  // first global triangle of each mesh
  const int* meshLight;      // area light index per mesh, -1 if not emissive
  const int* meshClass;      // shading class per mesh (its material's)
  int meshCount;
  const DevMaterial* materials;
  int materialCount;
  const DevTexture* textures;
  // Lights (render/scene.h:16-30): area lights first, then environment lights.
  int lightCount;
  int areaLightCount;
  const float* lightCdf;         // lightCount + 1
  const int* areaTriOffset;      // per area light: first emissive triangle
  const int* areaTriCount;
  const int* areaCdfOffset;      // per area light: offset of its (count + 1)-entry CDF
  const float* areaCdf;
  const float* etris;            // 16 floats per emissive triangle: v0 v1 v2 normal color pad
  int envCount;
  int distantLight;              // light index of the distant environment light, -1 if none
  DevEnvLight env[4];
  DevImageLight image;
  // Media (material/medium.h): transmittance colour and IOR per medium id.
  const float* mediaColor;       // 3 per medium
  int mediaCount;
  float sceneRadius;
  int topNodes;          // BVH nodes stored breadth-first at the start (shared-memory staging)
  int hasTransparent;    // some material is transparent: shadow rays use the transparency filter
};

// BSDF energy-compensation tables (bsdf/albedo_tables.h), computed on the device at context
// creation (albedo.cu) with the integrators of bsdf/albedo.h; sizes and parameterisations are
// the reference's.
struct DevTables
{
  const float* ggxDir;        // 32 x 32   (cosThetaO, roughness)
  const float* ggxAvg;        // 32        (roughness)
  const float* dielEtaDir;    // 16^3      (cosThetaO, eta in [1/3, 1], roughness)
  const float* dielEtaAvg;    // 16^2
  const float* dielRcpDir;    // 16^3      (cosThetaO, eta in [1, 3], roughness)
  const float* dielRcpAvg;    // 16^2
  const float* reflDir;       // 16^3      dielectric reflection only, eta in [1/3, 1]
  const float* reflAvg;       // 16^2
  const float* reflEcDir;     // 16^3      with multi-scattering (specular-albedo AOV only)
  const float* reflEcAvg;     // 16^2
  const float* condEcDir;     // 16^4      (cosThetaO, r, g, roughness) (specular-albedo AOV only)
  const float* sheenDir;      // 16^2
  // Bounds of the eta in [1/3, 1] axis: rcp(3) and rcp(1) as the reference's CPU build rounds
  // them (bsdf/albedo_tables.h:66-67; hostRcp), so that lookups land on the reference's
  // coordinates. The [1, 3] axis has exact bounds.
  float etaLo, etaHi;
};

struct DevCamera
{
  float org[3];
  float imageO[3], imageDx[3], imageDy[3];
  float nearClip;
};

// Renderer settings (render/path_renderer_stream.h:114-116, render/integrator.h:60-62).
struct DevRenderer
{
  int maxDepth;
  int rrDepth;
  float minWeight;
  float maxRadiance;
  uint32_t seed;
  int type;        // PRT_RENDERER_*
  int aoSamples;
  int flags;       // PRT_RENDERER_IRRADIANCE
};

// What the adjoint's replay needs per frame besides the frame itself (csrc/adjoint.cuh).
constexpr int kAdjointMaxTextures = 32;
struct AdjointView
{
  const float* dLdI;     // width * height * 3, row-major, row 0 at the top
  float* gradTex;        // concatenated textures, each width * height * 3, row 0 at the top
  float* gradRough;      // one per material
  long long texOffset[kAdjointMaxTextures];
  float step;            // roughness step of the central difference
  float invSpp;          // 1 / samples per pixel of the differentiated image
};

} // namespace prt
