// Test infrastructure: drives the reference-side adapter prt::DeviceCuda
// (oidn-protoray_b200/host/reference/device_cuda.h) compiled against the reference's own headers,
// with the light accessors inserted as the integration inserts them (oracle/Makefile, target
// adapter). Three entry points for the tests:
//   adapter_env    -- the environment lights the adapter forwards for a set of light Props
//                     (Scene::initLights's keys), read back from the reference's light objects;
//   adapter_tables -- the energy-compensation tables a DeviceCuda's context holds;
//   adapter_render -- a whole render through prt::Device's interface: initScene(path, props),
//                     initCamera, initFrame, initRenderer, initSampler, spp x render, blitFrame.
// Props are passed as text, one per line: "<key> f <x>" (float), "i <n>" (int),
// "v3 <x> <y> <z>" (Vec3f) or "s <text>" (string).
#include <cstring>
#include <sstream>
#include <string>

#include "device_cuda.h"

using namespace prt;

namespace {

std::string g_error;

Props parseProps(const char* spec)
{
  Props p;
  std::istringstream in(spec ? spec : "");
  std::string line;
  while (std::getline(in, line))
  {
    std::istringstream ls(line);
    std::string key, type;
    if (!(ls >> key >> type)) continue;
    if (type == "f")
    {
      float x;
      ls >> x;
      p.set(key, x);
    }
    else if (type == "i")
    {
      int x;
      ls >> x;
      p.set(key, x);
    }
    else if (type == "v3")
    {
      float x, y, z;
      ls >> x >> y >> z;
      p.set(key, Vec3f(x, y, z));
    }
    else if (type == "s")
    {
      std::string rest;
      std::getline(ls >> std::ws, rest);
      p.set(key, rest);
    }
    else
      throw std::invalid_argument("bad props line: " + line);
  }
  return p;
}

template <class F>
int guard(F&& f)
{
  try
  {
    f();
    return 0;
  }
  catch (const std::invalid_argument& e)
  {
    g_error = e.what();
    return 1;
  }
  catch (const std::logic_error& e)
  {
    g_error = e.what();
    return 2;
  }
  catch (const std::exception& e)
  {
    g_error = e.what();
    return 3;
  }
}

} // namespace

extern "C" {

const char* adapter_last_error() { return g_error.c_str(); }

// env_f: distant colour (3), direction (3), angle, ambient colour (3) = 10 floats;
// env_i: image width, height, LUT size, flags. `image` (width*height*3 floats, top row first)
// may be null to query the size.
int adapter_env(const char* props_spec, float* env_f, int32_t* env_i, float* image)
{
  return guard([&] {
    CudaEnvLights lights;
    cudaEnvLightsFromProps(parseProps(props_spec), lights);
    const prt_env_desc& e = lights.env;
    for (int k = 0; k < 3; ++k)
    {
      env_f[k] = e.distant_color[k];
      env_f[3 + k] = e.distant_dir[k];
      env_f[7 + k] = e.ambient_color[k];
    }
    env_f[6] = e.distant_angle;
    env_i[0] = e.image_rgb ? e.image_width : 0;
    env_i[1] = e.image_rgb ? e.image_height : 0;
    env_i[2] = e.image_lut_size;
    env_i[3] = e.flags;
    if (image && e.image_rgb) std::memcpy(image, e.image_rgb, sizeof(float) * 3 * e.image_width * e.image_height);
  });
}

// The energy-compensation tables of a DeviceCuda's context (prt_cuda_albedo_tables layout), as
// constructed with hostTables = host_tables. Writes at most `capacity` floats; *count gets the
// total.
int adapter_tables(int host_tables, float* out, int64_t capacity, int64_t* count)
{
  return guard([&] {
    DeviceCuda device(0, host_tables != 0);
    if (prt_cuda_albedo_tables(device.handle(), out, capacity, count) != PRT_OK)
      throw std::runtime_error(prt_cuda_last_error(device.handle()));
  });
}

// camera: position, basis U, V, N, fov, nearClip (14 floats). renderer: maxDepth, rrDepth.
// hdr (and, when aov_mask asks for them, albedo1 / normal1): width*height*3 floats.
// stats: rays traced, Mrays/s of the last call.
int adapter_render(const char* scene_path, const char* light_props, const float* camera, int width, int height,
                   int aov_mask, const int* renderer, uint32_t seed, int spp, float* hdr, float* albedo1,
                   float* normal1, double* stats)
{
  return guard([&] {
    DeviceCuda device(0);
    device.initScene(scene_path, parseProps(light_props));
    // The reference application's order: frame, then camera (main/render/render_window.cpp:317,745).
    Props frame;
    if (aov_mask & PRT_AOV_ALBEDO1) frame.set("aovAlbedo1");
    if (aov_mask & PRT_AOV_NORMAL1) frame.set("aovNormal1");
    device.initFrame(Vec2i(width, height), frame);
    Props cam;
    cam.set("type", "pinhole");
    cam.set("position", Vec3f(camera[0], camera[1], camera[2]));
    cam.set("basis", Basis3f(Vec3f(camera[3], camera[4], camera[5]), Vec3f(camera[6], camera[7], camera[8]),
                             Vec3f(camera[9], camera[10], camera[11])));
    cam.set("fov", camera[12]);
    cam.set("nearClip", camera[13]);
    cam.set("width", width);
    cam.set("height", height);
    device.initCamera(cam);
    Props filter;
    filter.set("filter", "box");
    device.initFilter(filter);
    Props r, st;
    r.set("type", "pathStream");
    r.set("sampler", "sobolBurley");
    r.set("maxDepth", renderer[0]);
    r.set("rrDepth", renderer[1]);
    device.initRenderer(r, st);
    device.initSampler(seed);
    device.clearFrame();
    double rays = 0.0, mray = 0.0;
    for (int i = 0; i < spp; ++i)
    {
      Props s;
      device.render(s);
      rays += (double)s.get<int64_t>("ray");
      mray = s.get<double>("mray");
    }
    FrameAovs aovs;
    aovs.hdr = reinterpret_cast<Vec3f*>(hdr);
    aovs.albedo1 = (aov_mask & PRT_AOV_ALBEDO1) ? reinterpret_cast<Vec3f*>(albedo1) : nullptr;
    aovs.normal1 = (aov_mask & PRT_AOV_NORMAL1) ? reinterpret_cast<Vec3f*>(normal1) : nullptr;
    device.blitFrame(aovs);
    const Box3f b = device.getSceneBounds();
    stats[0] = rays;
    stats[1] = mray;
    stats[2] = b.low.x;
    stats[3] = b.high.y;
  });
}

} // extern "C"
