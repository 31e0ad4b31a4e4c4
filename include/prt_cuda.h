/*
 * prt_cuda.h - C ABI of the B200 render device for ProtoRay's path-tracing hot path.
 *
 * The library (libprt_cuda.so) is a new render Device that sits beside the reference's
 * DeviceCpu (render/device_cpu.h:16). Every entry point takes plain pointers and sizes;
 * no C++ or torch types cross this boundary. Host pointers are borrowed for the duration
 * of a call only. All entry points return PRT_OK (0) or a negative status; the text of the
 * last error on a context is returned by prt_cuda_last_error().
 *
 * Threading: one context per host thread; calls on one context are not re-entrant. Work is
 * issued on the context's CUDA stream, and every call that returns host-visible results is
 * synchronous (the reference's Device::render is synchronous, render/device.h:70).
 */
#ifndef PRT_CUDA_H
#define PRT_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------------
 * The reference throws std::invalid_argument / std::logic_error / std::runtime_error
 * (render/path_renderer_stream.h:109-112,154; render/renderer_factory_stream.cpp:75).
 * The C ABI maps them to distinct codes; the C++ wrapper rethrows the same types. */
#define PRT_OK                 0
#define PRT_ERR_INVALID_ARG   -1  /* std::invalid_argument */
#define PRT_ERR_LOGIC         -2  /* std::logic_error (e.g. image size not divisible by the tile) */
#define PRT_ERR_OUT_OF_MEMORY -3
#define PRT_ERR_CUDA          -4  /* a CUDA runtime call failed */
#define PRT_ERR_DEVICE_ABORT  -5  /* a device loop hit its iteration cap or a bounds check */
#define PRT_ERR_STATE         -6  /* call order violated (e.g. render before scene upload) */

typedef struct prt_context prt_context;

/* ---- scene description ----------------------------------------------------------------
 * A scene is a list of triangle meshes, each bound to one Standard material, plus the
 * environment lights. This is the flattened form of what Scene::loadScene builds from an
 * rkscene file (render/scene.cpp:174-330): one TriangleMesh per geometry, material IDs
 * remapped so that emissive materials come first (render/scene.cpp:254-268), and the
 * triangle area lights derived from emissive meshes (render/scene.cpp:79-116). */
typedef struct prt_mesh
{
  const float*   positions;   /* vertex_count * 3 */
  const float*   normals;     /* vertex_count * 3, or NULL (geometric normal is used) */
  const float*   texcoords;   /* vertex_count * 2 (UV set 0), or NULL (hit barycentrics are used) */
  const int32_t* indices;     /* tri_count * 3 */
  int32_t        vertex_count;
  int32_t        tri_count;
  int32_t        material;    /* index into prt_scene_desc.materials */
  int32_t        reserved;
} prt_mesh;

/* Parameters of the reference's "Standard" (OpenPBR-like) material, default mode
 * (material/standard.cpp:21-76). Field defaults are those of rkscene::Material
 * (rkscene/rkscene.h:161-207); prt_cuda_material_defaults() fills them. A *_texture field
 * is an index into prt_scene_desc.textures, or -1; a textured parameter is the texture
 * value times the factor (material/material_param.h:36-47). */
typedef struct prt_material
{
  float base_weight;
  float base_color[3];
  float metalness;
  float diffuse_roughness;
  float specular_weight;
  float specular_color[3];
  float specular_roughness;
  float specular_ior;
  float transmission_weight;
  float transmission_color[3];
  float transmission_depth;
  float subsurface_weight;
  float subsurface_color[3];
  float subsurface_anisotropy;
  float coat_weight;
  float coat_color[3];
  float coat_roughness;
  float coat_ior;
  float sheen_weight;
  float sheen_color[3];
  float sheen_roughness;
  float emission_luminance;
  float emission_color[3];
  float opacity;
  int32_t thin_walled;
  int32_t base_color_texture;
  int32_t model;          /* PRT_MATERIAL_STANDARD or PRT_MATERIAL_PRINCIPLED */
  float   ambient_ior;    /* Standard "ambientIOR" / Principled "outsideIor" (default 1) */
  float   coat_thickness; /* Principled "coatThickness" (Standard uses its fixed 0.5) */
  float   sheen_tint;     /* Principled "sheenTint" */
  float   backlight;      /* Principled "backlight" (thin only) */
  float   thickness;      /* "thickness" of thin-walled transmission */
  int32_t reserved[2];
} prt_material;

/* Material models. PRT_MATERIAL_PRINCIPLED is the reference's deprecated PrincipledMaterial
 * (material/principled.cpp:21-575), read from the same record: base_color = "baseColor",
 * specular_color = "edgeColor", metalness = "metallic", base_weight = "diffuse",
 * specular_weight = "specular", specular_ior = "ior", specular_roughness = "roughness" (which
 * also makes the diffuse lobe Oren-Nayar), transmission_* = "transmission*", coat_* = "coat*",
 * sheen_* = "sheen*", thin_walled = "thin", opacity = "opacity"; it has no emission.
 * prt_cuda_principled_defaults() fills its defaults. */
#define PRT_MATERIAL_STANDARD   0
#define PRT_MATERIAL_PRINCIPLED 1
/* A material whose surfaces end the path as if the ray had missed them (environment light,
 * no shading), while still blocking shadow rays. The reference's stream renderer sorts hits
 * by material id with id 0 as its miss bucket (render/renderer_stream.h:108-181); rkscene
 * scenes keep id 0 for a dummy material, but a .mesh scene gives it to its first material
 * (render/scene.cpp:136-172), whose surfaces therefore render as misses. The .mesh loader
 * marks that material so. */
#define PRT_MATERIAL_MISS       2

/* An RGB FP32 image (row 0 at the top, as stored by the reference's ImageIo). */
typedef struct prt_texture
{
  const float* rgb;   /* width * height * 3 */
  int32_t width;
  int32_t height;
} prt_texture;

/* Environment lights, in the order Scene::initLights adds them (render/scene.cpp:365-450):
 * distant, ambient, image. A sun-sky light (light/sun_sky_light.cpp:17-193) is passed as
 * its two products: the sun as the distant light and the sky as the image light. */
typedef struct prt_env_desc
{
  float   distant_color[3];     /* "distantLight"; all zero = none */
  float   distant_dir[3];       /* "distantLightDir" (toward the light) */
  float   distant_angle;        /* "distantLightAngle": angular diameter in radians */
  float   ambient_color[3];     /* "ambientLight"; all zero = none */
  const float* image_rgb;       /* "imageLight": equirectangular RGB FP32, or NULL */
  int32_t image_width;
  int32_t image_height;
  int32_t image_lut_size;       /* "imageLightLutSize"; 0 = the reference default */
  int32_t flags;                /* PRT_ENV_*; 0 = the order distant, ambient, image */
} prt_env_desc;

/* Scene::initLights (render/scene.cpp:372-440) adds its environment lights in the order
 * distantLight, ambientLight, imageLight, then a sun-sky light's sun (a distant light) and sky (an
 * image light); light selection is by power over that list, so the order decides which light a
 * given sample picks. A sun-sky light crosses this boundary as its two products in the distant and
 * image fields; when an ambient light is also present, the reference's order puts the ambient light
 * first, which this flag selects: ambient, distant, image. */
#define PRT_ENV_AMBIENT_FIRST 1

typedef struct prt_scene_desc
{
  const prt_mesh*     meshes;
  int32_t             mesh_count;
  int32_t             material_count;
  const prt_material* materials;
  const prt_texture*  textures;
  int32_t             texture_count;
  int32_t             bvh_build;   /* PRT_BVH_HOST (0) or PRT_BVH_DEVICE (1) */
  prt_env_desc        env;
} prt_scene_desc;

/* BVH8 builders. The reference builds with Embree (accel/embree_intersector.cpp:68-90). Both
 * builders emit the same compressed 8-wide format, so every ray finds the same closest hit and
 * every image is the same whichever built the tree; they differ in build time and tree quality.
 *   PRT_BVH_HOST:   binned-SAH binary build on the host threads, collapsed to 8-wide nodes;
 *   PRT_BVH_DEVICE: on the GPU from the triangles in HBM: Morton sort, PLOC clustering
 *                   (nearest neighbours within 16 positions of the Morton order), the same
 *                   8-wide collapse. Deterministic: the same scene gives the same bytes. */
#define PRT_BVH_HOST   0
#define PRT_BVH_DEVICE 1

/* Pinhole camera (camera/pinhole_camera.h:20-59). The basis is (U right, V up, N back):
 * the view direction is -N. fov is the vertical field of view in radians. */
typedef struct prt_camera_desc
{
  float position[3];
  float basis_u[3];
  float basis_v[3];
  float basis_n[3];
  float fov;
  float near_clip;
} prt_camera_desc;

/* Renderer settings: the Props keys of PathRendererStream and IntegratorBase
 * (render/path_renderer_stream.h:114-116, render/integrator.h:60-62). */
typedef struct prt_renderer_desc
{
  int32_t max_depth;      /* "maxDepth", reference default 100 */
  int32_t rr_depth;       /* "rrDepth", reference default 8 */
  float   min_weight;     /* "minWeight", reference default 1e-4 */
  float   max_radiance;   /* "maxRadiance", reference default FLT_MAX (no clamping) */
  int32_t type;           /* renderer "type": PRT_RENDERER_* (0 = pathStream) */
  int32_t samples;        /* aoStream "samples" (AO rays per pixel sample; 0 = the default 16) */
  int32_t flags;          /* PRT_RENDERER_IRRADIANCE; 0 = the standard path tracer */
} prt_renderer_desc;

/* pathStream's "irradiance" option (render/path_renderer_stream.h:130-139, 304, 598): the first
 * surface a camera path hits is shaded with a white diffuse material (Principled, base colour 1)
 * and a camera ray that misses sees no environment, so the image is the irradiance arriving at
 * the first hits. Frame form only. */
#define PRT_RENDERER_IRRADIANCE 1

/* Renderer types (render/renderer_factory_stream.cpp:54-67): the path tracer and its sibling
 * stream renderers, which reuse its camera rays and traversal:
 * PRIMARY  "primaryStream": shading normal (N + 1) / 2 of the first hit, 0.05 on a miss
 *          (render/primary_renderer_stream.h);
 * AO       "aoStream": fraction of `samples` cosine-distributed rays that escape
 *          (render/ao_renderer_stream.h);
 * DIFFUSE  "diffuseStream": white diffuse paths lit by a white sky, throughput x 0.8 per bounce
 *          (render/diffuse_renderer_stream.h);
 * DIFFUSE2 "diffuse2Stream": the same with a cosine-sampled sky ray per bounce, half-weighted
 *          (render/diffuse2_renderer_stream.h).
 * The *_FAST types are the "...StreamFast" variants: the same renderers on the simple shading
 * context (the unflipped geometric normal, SimpleShadingContextSimd, core/shading_context.h:
 * 227-243, geometry/triangle_mesh.cpp:278-298) writing each sample over the pixel instead of
 * accumulating (AccumBuffer::set, image/accum_buffer.h:547-570): the frame holds the last
 * sample. */
#define PRT_RENDERER_PATH     0
#define PRT_RENDERER_PRIMARY  1
#define PRT_RENDERER_AO       2
#define PRT_RENDERER_DIFFUSE  3
#define PRT_RENDERER_DIFFUSE2 4
#define PRT_RENDERER_PRIMARY_FAST  5
#define PRT_RENDERER_AO_FAST       6
#define PRT_RENDERER_DIFFUSE_FAST  7
#define PRT_RENDERER_DIFFUSE2_FAST 8

/* AOV selection bits for prt_cuda_frame (render/device_cpu.cpp:178-232). */
#define PRT_AOV_ALBEDO1  (1 << 0)   /* "aovAlbedo1": first-hit albedo */
#define PRT_AOV_NORMAL1  (1 << 1)   /* "aovNormal1": first-hit normal */

#define PRT_AOV_HDR_VAR  (1 << 2)   /* "aovHdrVar": per-pixel sample variance of the colour */
#define PRT_AOV_SH       (1 << 3)   /* "aovSh": first-order spherical harmonics of the radiance that
                                       reaches the first hit (render/path_renderer_stream.h:46-52,
                                       257-263, 329-344, 705-709, 914-930, 980-1059); frame form only */

/* AOV identifiers for prt_cuda_blit. */
#define PRT_BLIT_HDR      0
#define PRT_BLIT_ALBEDO1  1
#define PRT_BLIT_NORMAL1  2
#define PRT_BLIT_HDR_VAR  3   /* FrameAovs::hdrVar: sample variance (needs PRT_AOV_HDR_VAR) */
#define PRT_BLIT_LDR      4   /* Device::blitFrame(Surface&): tone-mapped 8-bit colour, one uint32
                                 per pixel (blue in bits 0-7, green 8-15, red 16-23; gamma 2.2,
                                 image/pixel.h:36-40); dst is then width * height uint32 */
#define PRT_BLIT_LDR_RGB  5   /* FrameAovs::ldr: tone-mapped colour clamped to [0, 1], RGB floats */
/* FrameAovs::sh[0..3] (needs PRT_AOV_SH), as DeviceCpu::blitFrame writes them
 * (render/device_cpu.cpp:359-364): SH0 is the mean of the band-0 coefficient (the radiance
 * scaled to irradiance, per colour channel); SH1..SH3 are the means of its products with the
 * arrival direction's x, y and z, each divided by max(SH0, 1e-4) (AccumBuffer3f::blitRel,
 * image/accum_buffer.h:735-750). RGB floats. */
#define PRT_BLIT_SH0      6
#define PRT_BLIT_SH1      7
#define PRT_BLIT_SH2      8
#define PRT_BLIT_SH3      9

/* Tone mappers for PRT_BLIT_LDR and the frame error (render/device_cpu.cpp:286-303). */
#define PRT_TONE_NONE     0
#define PRT_TONE_LINEAR   1
#define PRT_TONE_REINHARD 2
#define PRT_TONE_ACES     3
#define PRT_TONE_FILMIC   4
#define PRT_TONE_LOG      5

/* Per-call statistics, the reference's Props stats of one render() (render/path_renderer_stream.h:175-178). */
typedef struct prt_render_stats
{
  double  mray;         /* (closest + shadow rays) / 1e6 / seconds */
  int64_t rays;         /* closest + shadow rays traced */
  int64_t spp;          /* samples per pixel rendered by this call */
  double  render_ms;    /* device time of the call */
  int64_t closest_rays;
  int64_t shadow_rays;
  int64_t kernel_launches;  /* kernels this call launched */
  double  trace_ms;     /* device time of the closest-hit kernels (PRT_PROFILE_KERNELS) */
  double  shadow_ms;    /* device time of the any-hit kernels (PRT_PROFILE_KERNELS) */
  double  shade_ms;     /* device time of the shading kernels (PRT_PROFILE_KERNELS) */
  int64_t closest_nodes;    /* BVH8 node visits of closest-hit rays (PRT_PROFILE_COUNTS) */
  int64_t closest_tris;     /* triangle tests of closest-hit rays (PRT_PROFILE_COUNTS) */
  int64_t shadow_nodes;     /* node visits of shadow rays (PRT_PROFILE_COUNTS) */
  int64_t shadow_tris;      /* triangle tests of shadow rays (PRT_PROFILE_COUNTS) */
  int64_t trace_launches;   /* closest-hit traversal launches (one per bounce per wave) */
} prt_render_stats;

/* Profiling switches for prt_cuda_set_profiling. Kernel timing records CUDA events around
 * each traversal and shading launch; counting runs the counting variant of the traversal
 * kernels (the reference's nodes/prims per-ray statistic, render/path_renderer_stream.h:180-184). */
#define PRT_PROFILE_KERNELS (1 << 0)
#define PRT_PROFILE_COUNTS  (1 << 1)

/* ---- context ----------------------------------------------------------------------------- */

/* Creates a device context on the given CUDA device (Device ctor, render/device_cpu.cpp:20-23,
 * which also precomputes the BSDF albedo tables). */
int prt_cuda_create(int device_ordinal, prt_context** out_ctx);
int prt_cuda_destroy(prt_context* ctx);
const char* prt_cuda_last_error(const prt_context* ctx);

/* Fills a material with the reference's Standard defaults. */
void prt_cuda_material_defaults(prt_material* m);
/* Defaults of PrincipledMaterial's parameters (material/principled.cpp:21-60), model set. */
void prt_cuda_principled_defaults(prt_material* m);

/* ---- scene, renderer, camera, frame ----------------------------------------------------- */

/* Device::initScene + initLights (render/device_cpu.cpp:96-107): copies the scene to HBM,
 * builds the BVH8 (on the host or the device, as scene->bvh_build says) and derives area
 * lights and the light-pick distribution. */
int prt_cuda_scene_upload(prt_context* ctx, const prt_scene_desc* scene);

/* The uploaded scene's acceleration structure; the reference reports the build as
 * buildMs / buildMprim (accel/embree_intersector.cpp:88-90). */
typedef struct prt_scene_stats
{
  double  build_ms;     /* BVH build wall time (the device build includes its launches and waits) */
  int64_t node_count;   /* 80-byte wide nodes */
  int64_t tri_count;    /* 48-byte triangle records */
  int32_t builder;      /* PRT_BVH_HOST or PRT_BVH_DEVICE */
  int32_t depth;        /* wide levels */
  int32_t top_count;    /* nodes of the first three levels, stored first */
  int32_t iterations;   /* device build: clustering iterations; host build: 0 */
  float   bounds_lo[3]; /* scene bounds over all triangle vertices (Scene::getBounds) */
  float   bounds_hi[3];
} prt_scene_stats;

int prt_cuda_scene_stats(prt_context* ctx, prt_scene_stats* out);

/* Device::initLights (render/device_cpu.cpp:101-104 -> Scene::initLights, render/scene.cpp:365-450):
 * replaces the environment lights of the uploaded scene and rebuilds the light-selection table
 * (area lights first, then the environment lights); geometry, BVH, materials and area lights stay.
 * Also reached through the `env` of prt_cuda_scene_upload / prt_cuda_scene_load. */
int prt_cuda_scene_lights(prt_context* ctx, const prt_env_desc* env);

/* Copies the uploaded scene's BVH8 to host memory: min(node_capacity, node_count) 80-byte
 * nodes and min(tri_capacity, tri_count) 48-byte triangle records (bvh8.h layout; either
 * pointer may be NULL with capacity 0 to query the counts, written to *node_count / *tri_count). */
int prt_cuda_scene_bvh(prt_context* ctx, void* nodes, int64_t node_capacity, void* tris, int64_t tri_capacity,
                       int64_t* node_count, int64_t* tri_count);

/* ---- scene files -------------------------------------------------------------------------
 * The reference's scene files, read on the host into the flat description above (Scene::Scene
 * picks the loader by extension, render/scene.cpp:65-77):
 *   .rkscene -- a JSON document with one binary buffer (.rkbin) of typed arrays
 *     (rkscene/rkscene.h:264-905): every file material a Standard material, geometries
 *     without a valid material bound to the default (Principled) material appended after the
 *     file's, each object's geometries added once, or once per instance transform with
 *     positions and normals transformed (instances are always flattened), in file order
 *     (render/scene.cpp:174-362). The file's lights list is checked but, as in
 *     Scene::loadScene, not used.
 *   .mesh -- the TriangleMesh blob (geometry/triangle_mesh.cpp:362-378) with the material
 *     library <name>.mtl (material/mtl_loader.cpp): materials per Scene::loadMesh
 *     (render/scene.cpp:136-172) and MaterialFactory::make ("Standard", "Principled", or the
 *     default "OBJ" mapping onto Principled); the triangles are split into one mesh per
 *     material.
 * Texture maps are supported for the base colour only, read from little-endian colour PFM
 * images, UV set 0, no transform. The environment comes from the caller. Host-only: no GPU is
 * needed to load or describe a file. */
typedef struct prt_scene_file prt_scene_file;

/* Loads `path`. On failure returns PRT_ERR_INVALID_ARG (malformed or unsupported content) or
 * PRT_ERR_LOGIC (a file that cannot be opened or read) and writes the reason to msg
 * (msg_capacity bytes, may be 0). */
int prt_scene_file_load(const char* path, prt_scene_file** out, char* msg, int32_t msg_capacity);
/* Points desc at the loaded scene's arrays (valid until prt_scene_file_free); env is zeroed and
 * bvh_build is PRT_BVH_HOST: set them before prt_cuda_scene_upload. */
int prt_scene_file_desc(const prt_scene_file* scene, prt_scene_desc* desc);
int prt_scene_file_free(prt_scene_file* scene);

/* Device::initScene(path, props) + initLights(props) (render/device_cpu.cpp:96-110) for an
 * .rkscene or .mesh file: loads it, applies the environment lights (env may be NULL: none) and the BVH
 * builder, and uploads it as prt_cuda_scene_upload does. A file that cannot be read or parsed
 * gives PRT_ERR_INVALID_ARG with the reason in prt_cuda_last_error. */
int prt_cuda_scene_load(prt_context* ctx, const char* path, const prt_env_desc* env, int32_t bvh_build);

/* Device::initRenderer (render/device_cpu.cpp:32-46) for type "pathStream", sampler "sobolBurley". */
int prt_cuda_renderer(prt_context* ctx, const prt_renderer_desc* renderer);

/* Device::initSampler (render/device_cpu.cpp:48-51): seed, and resets the sample index to 0. */
int prt_cuda_init_sampler(prt_context* ctx, uint32_t seed);

/* Device::initCamera (render/device_cpu.cpp:110-125). */
int prt_cuda_camera(prt_context* ctx, const prt_camera_desc* camera);

/* Device::initFrame (render/device_cpu.cpp:178-232); width must be a multiple of 32 and
 * height a multiple of 8 (render/path_renderer_stream.h:109-112). */
int prt_cuda_frame(prt_context* ctx, int32_t width, int32_t height, int32_t aov_mask);

/* Device::clearFrame (render/device_cpu.cpp:304-307). */
int prt_cuda_clear(prt_context* ctx);

/* Renders spp samples per pixel: equivalent to spp calls of Device::render
 * (render/device_cpu.cpp:53-59), each advancing the sample index by one. */
int prt_cuda_render(prt_context* ctx, int32_t spp, prt_render_stats* stats);

/* No counterpart in the reference. Rendering for callers that must not allocate device memory:
 * hosts whose device memory is owned by their own pool or budget, and hosts that may not take the
 * device-wide synchronisation a cudaMalloc/cudaFree can cause in the middle of their work.
 * Renders `spp` samples per pixel numbered from `first_sample` (the same samples prt_cuda_render
 * draws at that sample index) with the current scene, camera, renderer and seed, and writes
 * their average to `hdr_out`: width*height RGB floats, row-major, in device or managed memory the
 * caller owns on the context's device (memory of another GPU is rejected). The frame size and AOV
 * mask come from prt_cuda_frame; the frame's own sums and the sample index of prt_cuda_render
 * are left untouched. The call is synchronous: it returns after the image is written.
 * No device memory is allocated or freed: path state, queues, counters and sums live in one
 * scratch area compiled into the library (about 18 MB, present on every GPU that loads it until
 * the process exits), sized for frames of at most 65,536 pixels (e.g. 256x256) and
 * maxDepth <= 1000; larger frames are rejected with PRT_ERR_INVALID_ARG.
 * The first call on a device looks up the area's device address; make that first call before
 * any stream capture. All calls on a device share the one area (each call zeroes what must start
 * at zero), so calls whose GPU work overlaps -- from several contexts or threads on one device --
 * race and must be serialised by the caller. */
int prt_cuda_render_static(prt_context* ctx, uint32_t first_sample, int32_t spp, float* hdr_out);

/* Launch tuning of the wavefront kernels; 0 in a field keeps the current value.
 * trace_blocks / shade_blocks: persistent blocks of 256 threads per SM for the traversal and
 *   shading kernels;
 * wave_paths: upper bound on paths in flight per wave (path state is ~170-240 bytes per path);
 *   134,217,728 by default (a 1920x1080 x 64-spp frame in one wave). */
typedef struct prt_tuning
{
  int32_t trace_blocks;
  int32_t shade_blocks;
  int32_t wave_paths;
  int32_t top_stage;   /* 1: traversal reads the top 3 BVH levels from shared memory; 2: from
                          global memory (the default); 0 keeps the current value */
  int32_t ray_bins;    /* 1: each bounce's extended rays are traced grouped by direction octant;
                          2: in the order shading produced them (the default); 0 keeps */
  int32_t trace_stack; /* node-group stack of the traversal kernels: 12 (the default) a 12-entry
                          stack in shared memory for trees of at most 12 wide levels, else as
                          24; 24 the 24-entry local-memory stack for trees of at most 24 levels,
                          else as 48; 48 always the 48-entry one; 0 keeps */
} prt_tuning;

int prt_cuda_set_tuning(prt_context* ctx, const prt_tuning* tuning);
int prt_cuda_get_tuning(prt_context* ctx, prt_tuning* tuning);

/* Picks the tuning that renders the current scene, camera and frame fastest: each candidate
 * renders `spp` samples per pixel once (after one warm-up), device-timed. The frame is cleared
 * and the sample index reset afterwards. Writes the chosen tuning (also made current) and its
 * Mrays/s. */
int prt_cuda_autotune(prt_context* ctx, int32_t spp, prt_tuning* chosen, double* mrays);

/* ---- batch rendering -------------------------------------------------------------------
 * No counterpart in the reference, whose Device renders one scene per call. A batch holds many
 * independent frames -- each with its own scene, camera, renderer settings, sampler seed,
 * size, sample count and AOVs -- and renders all of them in one persistent wavefront: the
 * frames' paths share one path pool, terminated paths are replaced by new camera paths of any
 * frame (path regeneration), and the bounce loop is a CUDA graph replayed until every frame
 * has all its samples. Each frame gets the image that prt_cuda_render would produce for it
 * (samples 0..spp-1 of its seed): every path's result is kept per pixel-sample and each pixel's
 * samples are added in sample order, as the frame form adds them, so repeated renders of a batch
 * are identical, the albedo1 and normal1 AOVs equal the frame form's, and the beauty image is
 * within a few ulps of it. Device memory: 48 bytes per pixel-sample of the batch, plus the scenes
 * and the path pool. */
typedef struct prt_batch prt_batch;

typedef struct prt_batch_item
{
  const prt_scene_desc* scene;   /* borrowed for prt_cuda_batch_create only */
  prt_camera_desc       camera;
  prt_renderer_desc     renderer;
  int32_t               width;   /* multiple of 32, like prt_cuda_frame */
  int32_t               height;  /* multiple of 8 */
  int32_t               spp;
  int32_t               aov_mask;  /* PRT_AOV_* */
  uint32_t              seed;      /* sampler seed (Device::initSampler) */
  int32_t               reserved;
} prt_batch_item;

/* Uploads every item's scene (BVH8 build, materials, lights) and allocates the frames and the
 * shared path pool (prt_tuning.wave_paths slots at most). */
int prt_cuda_batch_create(prt_context* ctx, const prt_batch_item* items, int32_t count, prt_batch** out_batch);
/* Clears the frames and renders every item to completion; stats count all items' rays
 * (stats->spp is 0: the items' sample counts differ). */
int prt_cuda_batch_render(prt_batch* batch, prt_render_stats* stats);
/* Device::blitFrame of one item: width*height RGB floats (host or device memory). */
int prt_cuda_batch_blit(prt_batch* batch, int32_t item, int32_t aov, float* dst);
int prt_cuda_batch_destroy(prt_batch* batch);

/* ---- batched differentiation -----------------------------------------------------------
 * No counterpart in the reference. The path-replay adjoint for a whole batch, many inverse-
 * rendering problems per launch: prt_cuda_batch_enable_adjoint makes every later
 * prt_cuda_batch_render also store each pixel-sample's radiance (16 bytes per pixel-sample);
 * prt_cuda_batch_adjoint then replays all paths of all items in one persistent wavefront and
 * writes, per item k, dLoss/d(texel) into grad_textures[k] and dLoss/d(specular roughness) into
 * grad_roughness[k] for the image gradient d_loss_d_images[k] (layouts as prt_cuda_adjoint;
 * device or managed memory). The updates change one item's parameters between steps. */
int prt_cuda_batch_enable_adjoint(prt_batch* batch);
int prt_cuda_batch_adjoint(prt_batch* batch, const float* const* d_loss_d_images, float* const* grad_textures,
                           float* const* grad_roughness, prt_render_stats* stats);
int prt_cuda_batch_update_texture(prt_batch* batch, int32_t item, int32_t texture, const float* rgb);
int prt_cuda_batch_update_material(prt_batch* batch, int32_t item, int32_t material, const prt_material* m);
int prt_cuda_batch_update_materials(prt_batch* batch, int32_t item, int32_t first, int32_t count,
                                    const prt_material* ms);

/* ---- differentiation -------------------------------------------------------------------
 * No counterpart in the reference. Path-replay adjoint of the image prt_cuda_render produces:
 * given dLoss/dImage (width*height RGB floats, row-major, row 0 at the top; host or device
 * memory), writes
 *   grad_textures: dLoss/d(texel) of every scene texture used as a Lambertian base colour,
 *                  textures concatenated in scene order, each width*height*3 floats with row 0
 *                  at the top (the layout of prt_texture); at least grad_texture_count floats;
 *   grad_roughness: dLoss/d(specular_roughness) of every material (0 for materials without a
 *                  specular layer); grad_roughness_count >= material_count.
 * Either output may be NULL. The estimate uses samples [first_sample, first_sample + spp) of the
 * current seed; each path is walked twice from its Sobol seed (primal, then replay), so nothing
 * is stored per path. Supported materials: Lambertian, optionally under a specular layer, plus
 * emitters (other lobes return PRT_ERR_INVALID_ARG). stats->render_ms is the device time. */
int prt_cuda_adjoint(prt_context* ctx, uint32_t first_sample, int32_t spp, const float* d_loss_d_image,
                     float* grad_textures, int64_t grad_texture_count, float* grad_roughness,
                     int32_t grad_roughness_count, prt_render_stats* stats);

/* Parameter updates between renders without re-uploading the scene (no BVH rebuild).
 * prt_cuda_update_texture: new contents of texture `texture` (same size; row 0 at the top;
 * host or device memory). prt_cuda_update_material: new parameters of material `material`,
 * which must keep its lobe set, emission and medium. No counterpart in the reference, which
 * reloads the scene. */
int prt_cuda_update_texture(prt_context* ctx, int32_t texture, const float* rgb);
int prt_cuda_update_material(prt_context* ctx, int32_t material, const prt_material* m);
/* The same for materials [first, first + count) in one call (one copy to the device). */
int prt_cuda_update_materials(prt_context* ctx, int32_t first, int32_t count, const prt_material* ms);

/* ---- film post-step ----------------------------------------------------------------------
 * Device::initToneMapper (render/device_cpu.cpp:286-303): `type` PRT_TONE_*, "exposure" and
 * Reinhard's "burn" (0..1). */
int prt_cuda_tone_mapper(prt_context* ctx, int32_t type, float exposure, float burn);

/* Device::getFrameError (render/device_cpu.cpp:436-439, image/accum_buffer.h:752-795): the mean
 * relative L1 difference between the current image and the image at the last power-of-two sample
 * count (the checkpoint copy every frame keeps), scaled by the tone mapper's exposure. */
int prt_cuda_frame_error(prt_context* ctx, float* error);

/* Enables PRT_PROFILE_* instrumentation for subsequent render calls (0 = off). */
int prt_cuda_set_profiling(prt_context* ctx, int32_t flags);

/* Device::blitFrame (render/device_cpu.cpp:316-366): sum * rcpSafe(weight) per pixel, as
 * width*height*3 floats. dst may be host or device memory. */
int prt_cuda_blit(prt_context* ctx, int32_t aov, float* dst);

/* ---- parity and query entry points ----------------------------------------------------- */

/* Sobol-Burley samples as the stream renderer draws them (sampling/sobol_burley_sampler_simd.h:36-84):
 * for each i, setSample(sample_index[i], pixel_id[i]) with the context seed, then a
 * `dims`-dimensional draw (1, 2 or 3) from dimension set dim_set[i]. out has n*dims floats. */
int prt_cuda_sobol(prt_context* ctx, int64_t n, const uint32_t* sample_index, const uint32_t* pixel_id,
                   const uint32_t* dim_set, int32_t dims, float* out);

/* Closest-hit query for n rays (org xyz, near, dir xyz, far per ray: 8 floats). Writes
 * geom_id, prim_id (-1 on miss), t (far on miss) and barycentrics u, v. */
int prt_cuda_trace(prt_context* ctx, int64_t n, const float* rays, int32_t* geom_id, int32_t* prim_id,
                   float* t, float* u, float* v);

/* Any-hit query: occluded[i] = 1 if a triangle lies within [near, far] of ray i. */
int prt_cuda_occluded(prt_context* ctx, int64_t n, const float* rays, int32_t* occluded);

/* Primary rays of sample `sample_index` for every pixel (render/path_renderer_stream.h:209-262)
 * and their closest hits: rays_out has width*height*8 floats, geom_id/prim_id width*height. */
int prt_cuda_query_primary(prt_context* ctx, uint32_t sample_index, float* rays_out,
                           int32_t* geom_id, int32_t* prim_id, float* t);

/* BSDF of one Standard material evaluated and sampled on the device for n tuples of
 * (wo, wi, 3D sample) (9 floats each) in a canonical shading context: identity shading frame
 * (N = z), geometric normal z, UV (0.5, 0.5), front-facing hit, path in medium `medium_id`
 * (0 = outside; 1 = inside a transmissive material's own medium). out gets 13 floats per
 * tuple: eval value (3), eval pdf, sample weight (3), sampled wi (3), sample pdf, sample type
 * and BSDF flags (int bits). Mirrors Material::getBsdf + BsdfSimd::eval/sample
 * (material/material.h:66-76, bsdf/bsdf.h:106-110); used for BSDF parity. */
int prt_cuda_bsdf_query(prt_context* ctx, const prt_material* material, int32_t medium_id, int64_t n,
                        const float* tuples, float* out);

/* Microfacet-distribution sampling on the device for n tuples of (alpha, s.x, s.y, wo.x, wo.y,
 * wo.z) (6 floats each, canonical frame N = z); out gets (m.x, m.y, m.z, pdf) per tuple.
 *   PRT_MICROFACET_BECKMANN:     BeckmannDistribution::sample (bsdf/beckmann_distribution.h:21-42),
 *                                the distribution of the reference's CarPaint flakes
 *                                (material/flakes.h:59); wo is unused.
 *   PRT_MICROFACET_GGX_VISIBLE:  GGXDistribution::sampleVisible (bsdf/ggx_distribution.h:52-82),
 *                                isotropic alpha, visible normals of wo.
 * Used for sampler parity. */
#define PRT_MICROFACET_BECKMANN    1
#define PRT_MICROFACET_GGX_VISIBLE 2
int prt_cuda_microfacet_query(prt_context* ctx, int32_t distribution, int64_t n, const float* in, float* out);

/* Copies the BSDF energy-compensation tables the context computed at creation (the
 * reference's precomputeAlbedoTables, bsdf/albedo_tables.cpp:173-188) to out, concatenated in
 * the order GGX dir (32x32), GGX avg (32), dielectric eta dir (16^3), eta avg (16^2), dielectric
 * 1/eta dir (16^3), avg (16^2), dielectric reflection dir (16^3), avg (16^2), sheen dir (16^2,
 * bsdf/albedo_tables.h:281-300). Writes at most
 * `capacity` floats and returns the total count through *count. */
int prt_cuda_albedo_tables(prt_context* ctx, float* out, int64_t capacity, int64_t* count);

/* Replaces the context's energy-compensation tables with `tables` (count floats, in the layout of
 * prt_cuda_albedo_tables): the reference application's own, which prt::DeviceCuda uploads at
 * construction (the tables the context builds agree with them to ~2e-6, and the compensation
 * terms of rough dielectrics amplify a table's last digits by 1 / (1 - E_avg)), or any other set
 * for parity studies that separate the BSDF arithmetic from the tables' values. Synchronous;
 * takes effect from the next render or query. */
int prt_cuda_set_albedo_tables(prt_context* ctx, const float* tables, int64_t count);

/* Host-only (no GPU needed): builds the BVH8 over tri_count triangles given as 9 floats each
 * (v0, v1, v2) and walks it with the counting traversal, the scalar twin of the closest-hit
 * kernel. For each of the n rays (8 floats) writes the global triangle index (-1 on a miss)
 * and t; adds the node visits and triangle tests to *node_visits / *tri_tests and stores the
 * node count. Used to state the algorithmic bytes per ray; the reference's counterpart is its
 * nodes/prims per-ray statistic (render/path_renderer_stream.h:180-184). */
int prt_bvh8_count(const float* tri_verts, int64_t tri_count, int64_t n, const float* rays, int32_t* tri_out,
                   float* t_out, int64_t* node_visits, int64_t* tri_tests, int64_t* node_count);

/* Host-only (no GPU needed): checks a BVH8 given as arrays (bvh8.h layout) over tri_count
 * triangles (tri_verts: 9 floats each, v0 v1 v2): every node reached once from the root, child
 * and triangle indices in range, every triangle stored once with v0 and the single-precision
 * edges v1 - v0 and v2 - v0, every 8-bit child box containing its subtree's triangles (as
 * dequantised in single precision), the first top_count nodes exactly the first three levels,
 * and the depth within the traversal stack. Writes the depth (wide levels) to *depth when not
 * NULL. Returns PRT_OK, or PRT_ERR_INVALID_ARG with the first violation in msg. */
int prt_bvh8_check(const void* nodes, int64_t node_count, const void* tris, int64_t tri_count,
                   const float* tri_verts, int32_t top_count, int32_t* depth, char* msg, int32_t msg_capacity);

/* Host-only: the PRT_BVH_HOST build (binned SAH, 8-wide collapse) into caller arrays of at
 * least max(tri_count, 1) nodes and tri_count triangle records; writes the node count and the
 * top-level node count. */
int prt_bvh8_build_host(const float* tri_verts, int64_t tri_count, void* nodes, int64_t node_capacity, void* tris,
                        int64_t tri_capacity, int64_t* node_count, int32_t* top_count);

/* Host-only: the counting traversal of prt_bvh8_count over a BVH8 given as arrays that pass
 * prt_bvh8_check (for instance one built on the device and copied back with
 * prt_cuda_scene_bvh). */
int prt_bvh8_trace(const void* nodes, int64_t node_count, const void* tris, int64_t tri_count, int64_t n,
                   const float* rays, int32_t* tri_out, float* t_out, int64_t* node_visits, int64_t* tri_tests);

#ifdef __cplusplus
}
#endif

#endif /* PRT_CUDA_H */
