// Scene-file loaders: the rkscene JSON reader, typed buffer reads and material / geometry /
// object mapping; the TriangleMesh blob and Wavefront material-library reader. See scene_file.h.
#include "scene_file.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <sstream>
#include <stdexcept>

namespace prt {
namespace {

// ---- JSON -----------------------------------------------------------------------------------
// A complete RFC 8259 reader (objects keep their member order; numbers are doubles).

struct JVal
{
  enum Type { Null, Bool, Num, Str, Arr, Obj } type = Null;
  bool b = false;
  double n = 0.0;
  std::string s;
  std::vector<JVal> a;
  std::vector<std::pair<std::string, JVal>> o;

  const JVal* get(const char* key) const
  {
    if (type != Obj) return nullptr;
    for (const auto& kv : o)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

class JsonReader
{
public:
  JsonReader(const char* begin, const char* end) : p(begin), e(end) {}

  JVal document()
  {
    JVal v = value(0);
    skipSpace();
    if (p != e) fail("trailing characters");
    return v;
  }

private:
  const char* p;
  const char* e;

  [[noreturn]] void fail(const char* what) const
  {
    throw std::invalid_argument(std::string("rkscene: invalid JSON: ") + what);
  }

  void skipSpace()
  {
    while (p != e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
  }

  bool literal(const char* word)
  {
    const size_t k = std::strlen(word);
    if ((size_t)(e - p) < k || std::memcmp(p, word, k) != 0) return false;
    p += k;
    return true;
  }

  JVal value(int depth)
  {
    if (depth > 512) fail("nesting too deep");
    skipSpace();
    if (p == e) fail("unexpected end");
    JVal v;
    const char c = *p;
    if (c == '{')
    {
      v.type = JVal::Obj;
      ++p;
      skipSpace();
      if (p != e && *p == '}')
      {
        ++p;
        return v;
      }
      for (;;)
      {
        skipSpace();
        if (p == e || *p != '"') fail("expected a member name");
        std::string key = string();
        skipSpace();
        if (p == e || *p != ':') fail("expected ':'");
        ++p;
        v.o.emplace_back(std::move(key), value(depth + 1));
        skipSpace();
        if (p != e && *p == ',')
        {
          ++p;
          continue;
        }
        if (p != e && *p == '}')
        {
          ++p;
          return v;
        }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[')
    {
      v.type = JVal::Arr;
      ++p;
      skipSpace();
      if (p != e && *p == ']')
      {
        ++p;
        return v;
      }
      for (;;)
      {
        v.a.push_back(value(depth + 1));
        skipSpace();
        if (p != e && *p == ',')
        {
          ++p;
          continue;
        }
        if (p != e && *p == ']')
        {
          ++p;
          return v;
        }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"')
    {
      v.type = JVal::Str;
      v.s = string();
      return v;
    }
    if (literal("true"))
    {
      v.type = JVal::Bool;
      v.b = true;
      return v;
    }
    if (literal("false"))
    {
      v.type = JVal::Bool;
      return v;
    }
    if (literal("null")) return v;
    if (c == '-' || (c >= '0' && c <= '9'))
    {
      v.type = JVal::Num;
      v.n = number();
      return v;
    }
    fail("unexpected character");
  }

  double number()
  {
    const char* start = p;
    if (*p == '-') ++p;
    if (p == e) fail("bad number");
    if (*p == '0')
      ++p;
    else if (*p >= '1' && *p <= '9')
      while (p != e && *p >= '0' && *p <= '9') ++p;
    else
      fail("bad number");
    if (p != e && *p == '.')
    {
      ++p;
      if (p == e || !(*p >= '0' && *p <= '9')) fail("bad number");
      while (p != e && *p >= '0' && *p <= '9') ++p;
    }
    if (p != e && (*p == 'e' || *p == 'E'))
    {
      ++p;
      if (p != e && (*p == '+' || *p == '-')) ++p;
      if (p == e || !(*p >= '0' && *p <= '9')) fail("bad number");
      while (p != e && *p >= '0' && *p <= '9') ++p;
    }
    const std::string text(start, p);
    return std::strtod(text.c_str(), nullptr);
  }

  static void appendUtf8(std::string& out, uint32_t cp)
  {
    if (cp < 0x80)
      out += (char)cp;
    else if (cp < 0x800)
    {
      out += (char)(0xC0 | (cp >> 6));
      out += (char)(0x80 | (cp & 0x3F));
    }
    else if (cp < 0x10000)
    {
      out += (char)(0xE0 | (cp >> 12));
      out += (char)(0x80 | ((cp >> 6) & 0x3F));
      out += (char)(0x80 | (cp & 0x3F));
    }
    else
    {
      out += (char)(0xF0 | (cp >> 18));
      out += (char)(0x80 | ((cp >> 12) & 0x3F));
      out += (char)(0x80 | ((cp >> 6) & 0x3F));
      out += (char)(0x80 | (cp & 0x3F));
    }
  }

  uint32_t hex4()
  {
    if (e - p < 4) fail("bad \\u escape");
    uint32_t v = 0;
    for (int k = 0; k < 4; ++k, ++p)
    {
      const char h = *p;
      v <<= 4;
      if (h >= '0' && h <= '9') v |= (uint32_t)(h - '0');
      else if (h >= 'a' && h <= 'f') v |= (uint32_t)(h - 'a' + 10);
      else if (h >= 'A' && h <= 'F') v |= (uint32_t)(h - 'A' + 10);
      else fail("bad \\u escape");
    }
    return v;
  }

  std::string string()
  {
    ++p;  // opening quote
    std::string out;
    while (p != e && *p != '"')
    {
      const unsigned char c = (unsigned char)*p;
      if (c < 0x20) fail("control character in string");
      if (c != '\\')
      {
        out += (char)c;
        ++p;
        continue;
      }
      ++p;
      if (p == e) fail("bad escape");
      const char esc = *p++;
      switch (esc)
      {
      case '"': out += '"'; break;
      case '\\': out += '\\'; break;
      case '/': out += '/'; break;
      case 'b': out += '\b'; break;
      case 'f': out += '\f'; break;
      case 'n': out += '\n'; break;
      case 'r': out += '\r'; break;
      case 't': out += '\t'; break;
      case 'u':
      {
        uint32_t cp = hex4();
        if (cp >= 0xD800 && cp <= 0xDBFF)
        {
          if (e - p < 6 || p[0] != '\\' || p[1] != 'u') fail("unpaired surrogate");
          p += 2;
          const uint32_t lo = hex4();
          if (lo < 0xDC00 || lo > 0xDFFF) fail("unpaired surrogate");
          cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
        }
        else if (cp >= 0xDC00 && cp <= 0xDFFF)
          fail("unpaired surrogate");
        appendUtf8(out, cp);
        break;
      }
      default: fail("bad escape");
      }
    }
    if (p == e) fail("unterminated string");
    ++p;
    return out;
  }
};

// ---- typed values -------------------------------------------------------------------------------

[[noreturn]] void bad(const std::string& what) { throw std::invalid_argument("rkscene: " + what); }

double num(const JVal& v, const std::string& what)
{
  if (v.type != JVal::Num) bad(what + " must be a number");
  return v.n;
}

const std::string& str(const JVal& v, const std::string& what)
{
  if (v.type != JVal::Str) bad(what + " must be a string");
  return v.s;
}

void vec(const JVal& v, int n, float* out, const std::string& what)
{
  if (v.type != JVal::Arr || (int)v.a.size() < n) bad(what + " must be an array of " + std::to_string(n) + " numbers");
  for (int k = 0; k < n; ++k) out[k] = (float)num(v.a[k], what);
}

// The elements of a list member; null counts as an empty list (rkscene::save writes an empty list
// as null, and rkscene::load iterates it as empty).
const std::vector<JVal>& items(const JVal& v, const std::string& what)
{
  static const std::vector<JVal> none;
  if (v.type == JVal::Null) return none;
  if (v.type != JVal::Arr) bad(what + " must be an array");
  return v.a;
}

int64_t count(const JVal& v, const std::string& what)
{
  const double d = num(v, what);
  if (!(d >= 0.0) || d > 9.0e15 || std::floor(d) != d) bad(what + " must be a non-negative integer");
  return (int64_t)d;
}

// ---- binary buffer ------------------------------------------------------------------------------

class BinBuffer
{
public:
  BinBuffer(const std::string& path, int64_t byteLength) : length(byteLength)
  {
    file.open(path, std::ios::binary);
    if (!file)
    {
      std::ifstream gz(path + ".gz", std::ios::binary);
      if (gz) throw std::runtime_error("rkscene: gzip-compressed buffer not supported: " + path + ".gz");
      throw std::runtime_error("rkscene: failed to open file: " + path);
    }
  }

  // A buffer view {"type", "count", "byteOffset"} of `elemWords` 4-byte values per element.
  template <class T>
  void read(const JVal& view, const char* type, int elemWords, std::vector<T>& out)
  {
    const JVal* t = view.get("type");
    const JVal* c = view.get("count");
    const JVal* o = view.get("byteOffset");
    if (!t || !c || !o) bad("buffer view needs type, count and byteOffset");
    if (str(*t, "buffer type") != type) bad(std::string("unexpected buffer type (expected ") + type + ")");
    const int64_t n = count(*c, "buffer count"), off = count(*o, "buffer byteOffset");
    if (n > ((int64_t)1 << 40) / (elemWords * 4)) bad("buffer access out of bounds");
    const int64_t bytes = n * elemWords * 4;
    if (off + bytes > length) bad("buffer access out of bounds");
    out.resize((size_t)n * elemWords);
    file.seekg(off);
    if (bytes) file.read(reinterpret_cast<char*>(out.data()), bytes);
    if (!file) throw std::runtime_error("rkscene: failed to read binary data from file");
  }

private:
  std::ifstream file;
  int64_t length;
};

std::string directoryOf(const std::string& path)
{
  const size_t k = path.find_last_of('/');
  return k == std::string::npos ? std::string(".") : path.substr(0, k);
}

std::string resolve(const std::string& dir, const std::string& uri)
{
  return (!uri.empty() && uri[0] == '/') ? uri : dir + "/" + uri;
}

// Little-endian colour PFM ("PF", width, height, negative scale), bottom row first in the file;
// returned top row first.
void readPfm(const std::string& path, std::vector<float>& rgb, int& w, int& h)
{
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("rkscene: failed to open image: " + path);
  std::string magic;
  double scale = 0.0;
  f >> magic >> w >> h >> scale;
  if (!f || magic != "PF" || w <= 0 || h <= 0 || (int64_t)w * h > ((int64_t)1 << 31) || !(scale < 0.0))
    bad("unsupported image (only little-endian colour PFM): " + path);
  f.get();  // the single whitespace byte after the header
  rgb.resize((size_t)w * h * 3);
  std::vector<float> row((size_t)w * 3);
  for (int y = 0; y < h; ++y)
  {
    f.read(reinterpret_cast<char*>(row.data()), (std::streamsize)(row.size() * sizeof(float)));
    if (!f) throw std::runtime_error("rkscene: truncated image: " + path);
    std::memcpy(&rgb[(size_t)(h - 1 - y) * w * 3], row.data(), row.size() * sizeof(float));
  }
}

// ---- materials -----------------------------------------------------------------------------------

struct Loader
{
  RkScene& out;
  std::string dir;
  std::map<std::string, int> textureIndex;

  int texture(const std::string& uri)
  {
    const std::string path = resolve(dir, uri);
    auto it = textureIndex.find(path);
    if (it != textureIndex.end()) return it->second;
    std::vector<float> rgb;
    int w = 0, h = 0;
    readPfm(path, rgb, w, h);
    const int id = (int)out.texturePixels.size();
    out.texturePixels.push_back(std::move(rgb));
    out.texturePaths.push_back(path);
    prt_texture t;
    t.rgb = nullptr;  // pointed at the pixels once loading is done
    t.width = w;
    t.height = h;
    out.textures.push_back(t);
    textureIndex[path] = id;
    return id;
  }

  // A Texture1f / Texture3f parameter (rkscene.h:444-497): a number or array is the factor, a
  // string is an image (factor 1), an object may carry type, image, factor, swizzle, texcoord
  // and transform. The device reads texture maps for the base colour only, with UV set 0 and no
  // transform or swizzle.
  void param(const JVal& m, const char* name, int n, float* factor, int* tex = nullptr)
  {
    const JVal* v = m.get(name);
    if (!v) return;
    std::string image;
    if (v->type == JVal::Str)
    {
      image = v->s;
      for (int k = 0; k < n; ++k) factor[k] = 1.f;
    }
    else if (v->type == JVal::Num)
    {
      if (n != 1) bad(std::string(name) + " must be an array of 3 numbers");
      factor[0] = (float)v->n;
    }
    else if (v->type == JVal::Arr)
    {
      if (n == 1) bad(std::string(name) + " must be a number");
      vec(*v, n, factor, name);
    }
    else if (v->type == JVal::Obj)
    {
      if (const JVal* t = v->get("type"))
        if (str(*t, "texture type") != "bump") bad("unsupported texture type for material parameter");
      if (const JVal* im = v->get("image"))
      {
        image = str(*im, "texture image");
        for (int k = 0; k < n; ++k) factor[k] = 1.f;
      }
      if (const JVal* f = v->get("factor"))
      {
        if (n == 1) factor[0] = (float)num(*f, std::string(name) + " factor");
        else vec(*f, n, factor, std::string(name) + " factor");
      }
      if (!image.empty())
      {
        if (const JVal* sw = v->get("swizzle"))
          if (!str(*sw, "swizzle").empty()) bad(std::string(name) + ": texture swizzles are not supported on the device");
        if (const JVal* tc = v->get("texcoord"))
          if (count(*tc, "texcoord") != 0) bad(std::string(name) + ": only UV set 0 is supported on the device");
        if (const JVal* tf = v->get("transform"))
        {
          float off[2] = {0.f, 0.f}, sc[2] = {1.f, 1.f};
          if (const JVal* o = tf->get("offset")) vec(*o, 2, off, "texture offset");
          if (const JVal* s = tf->get("scale")) vec(*s, 2, sc, "texture scale");
          if (off[0] != 0.f || off[1] != 0.f || sc[0] != 1.f || sc[1] != 1.f)
            bad(std::string(name) + ": texture transforms are not supported on the device");
        }
      }
    }
    else
      bad(std::string(name) + " has an invalid value");
    if (!image.empty())
    {
      if (!tex) bad(std::string(name) + ": texture maps are supported for baseColor only on the device");
      *tex = texture(image);
    }
  }

  // rkscene::Material (rkscene.h:161-207, loadMaterial :500-540) as the Standard material of
  // Scene::loadScene (render/scene.cpp:204-233).
  prt_material material(const JVal& m)
  {
    if (m.type != JVal::Obj) bad("material must be an object");
    prt_material r;
    prt_cuda_material_defaults(&r);
    if (const JVal* nm = m.get("name")) str(*nm, "material name");
    param(m, "baseWeight", 1, &r.base_weight);
    param(m, "baseColor", 3, r.base_color, &r.base_color_texture);
    param(m, "metalness", 1, &r.metalness);
    param(m, "diffuseRoughness", 1, &r.diffuse_roughness);
    if (m.get("normal")) bad("normal and bump maps are not supported on the device");
    param(m, "specularWeight", 1, &r.specular_weight);
    param(m, "specularColor", 3, r.specular_color);
    param(m, "specularRoughness", 1, &r.specular_roughness);
    if (const JVal* v = m.get("specularIOR")) r.specular_ior = (float)num(*v, "specularIOR");
    param(m, "transmissionWeight", 1, &r.transmission_weight);
    param(m, "transmissionColor", 3, r.transmission_color);
    if (const JVal* v = m.get("transmissionDepth")) r.transmission_depth = (float)num(*v, "transmissionDepth");
    param(m, "subsurfaceWeight", 1, &r.subsurface_weight);
    param(m, "subsurfaceColor", 3, r.subsurface_color);
    param(m, "subsurfaceAnisotropy", 1, &r.subsurface_anisotropy);
    param(m, "coatWeight", 1, &r.coat_weight);
    param(m, "coatColor", 3, r.coat_color);
    param(m, "coatRoughness", 1, &r.coat_roughness);
    if (const JVal* v = m.get("coatIOR")) r.coat_ior = (float)num(*v, "coatIOR");
    if (m.get("coatNormal")) bad("coat normal and bump maps are not supported on the device");
    param(m, "sheenWeight", 1, &r.sheen_weight);
    param(m, "sheenColor", 3, r.sheen_color);
    param(m, "sheenRoughness", 1, &r.sheen_roughness);
    param(m, "emissionLuminance", 1, &r.emission_luminance);
    param(m, "emissionColor", 3, r.emission_color);
    if (const JVal* v = m.get("thinWalled"))
    {
      if (v->type != JVal::Bool) bad("thinWalled must be a boolean");
      r.thin_walled = v->b ? 1 : 0;
    }
    param(m, "opacity", 1, &r.opacity);
    return r;
  }
};

struct Geometry
{
  std::vector<float> positions, normals, texcoords;  // texcoords: UV set 0
  std::vector<uint32_t> indices;
  int material = -1;
};

// The vertex transform of TriangleMesh::clone: positions by the affine map (x U + y V + z N + P),
// normals by the inverse transpose of its linear part (math/affine3.h:93-108, basis3.h:154-169).
void transformMesh(const float* m, const std::vector<float>& pos, const std::vector<float>& nrm,
                   std::vector<float>& posOut, std::vector<float>& nrmOut)
{
  const float* U = m;
  const float* V = m + 3;
  const float* N = m + 6;
  const float* P = m + 9;
  posOut.resize(pos.size());
  for (size_t i = 0; i + 2 < pos.size(); i += 3)
    for (int k = 0; k < 3; ++k)
      posOut[i + k] = pos[i] * U[k] + pos[i + 1] * V[k] + pos[i + 2] * N[k] + P[k];
  nrmOut.clear();
  if (nrm.empty()) return;
  // Inverse transpose of the basis (U V N as columns): rows of the inverse are the cross
  // products V x N, N x U, U x V over the determinant, so the inverse transpose has them as
  // columns.
  const float cx[3] = {V[1] * N[2] - V[2] * N[1], V[2] * N[0] - V[0] * N[2], V[0] * N[1] - V[1] * N[0]};
  const float cy[3] = {N[1] * U[2] - N[2] * U[1], N[2] * U[0] - N[0] * U[2], N[0] * U[1] - N[1] * U[0]};
  const float cz[3] = {U[1] * V[2] - U[2] * V[1], U[2] * V[0] - U[0] * V[2], U[0] * V[1] - U[1] * V[0]};
  const float det = U[0] * cx[0] + U[1] * cx[1] + U[2] * cx[2];
  const float inv = 1.f / det;
  nrmOut.resize(nrm.size());
  for (size_t i = 0; i + 2 < nrm.size(); i += 3)
    for (int k = 0; k < 3; ++k)
      nrmOut[i + k] = (nrm[i] * cx[k] + nrm[i + 1] * cy[k] + nrm[i + 2] * cz[k]) * inv;
}

} // namespace

void RkScene::describe(prt_scene_desc& desc) const
{
  std::memset(&desc, 0, sizeof(desc));
  desc.meshes = meshes.data();
  desc.mesh_count = (int32_t)meshes.size();
  desc.materials = materials.data();
  desc.material_count = (int32_t)materials.size();
  desc.textures = textures.data();
  desc.texture_count = (int32_t)textures.size();
  desc.bvh_build = PRT_BVH_HOST;
}

void loadRkScene(const std::string& path, RkScene& out)
{
  out = RkScene();
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("rkscene: failed to open file: " + path);
  const std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  const JVal doc = JsonReader(text.data(), text.data() + text.size()).document();
  if (doc.type != JVal::Obj) bad("the document must be an object");
  const std::string dir = directoryOf(path);

  // Buffers: exactly one (rkscene.h:850-866).
  const JVal* buffers = doc.get("buffers");
  if (!buffers) bad("no buffers specified");
  if (buffers->type != JVal::Arr || buffers->a.size() != 1) bad("currently only single buffer is supported");
  const JVal* uri = buffers->a[0].get("uri");
  const JVal* byteLength = buffers->a[0].get("byteLength");
  if (!uri || !byteLength) bad("the buffer needs uri and byteLength");
  BinBuffer bin(resolve(dir, str(*uri, "buffer uri")), count(*byteLength, "buffer byteLength"));

  Loader L{out, dir, {}};
  if (const JVal* mats = doc.get("materials"))
    for (const JVal& m : items(*mats, "materials")) out.materials.push_back(L.material(m));
  const int fileMaterials = (int)out.materials.size();
  int defaultMaterial = -1;

  std::vector<Geometry> geoms;
  if (const JVal* gs = doc.get("geometries"))
    for (const JVal& g : items(*gs, "geometries"))
    {
      if (g.type != JVal::Obj) bad("geometry must be an object");
      const JVal* type = g.get("type");
      if (!type || str(*type, "geometry type") != "triangle") bad("unsupported geom type");
      if (const JVal* nm = g.get("name")) str(*nm, "geometry name");
      Geometry G;
      if (const JVal* v = g.get("positions")) bin.read(*v, "float3", 3, G.positions);
      if (const JVal* v = g.get("normals")) bin.read(*v, "float3", 3, G.normals);
      if (const JVal* v = g.get("texcoords"))
      {
        if (v->type == JVal::Arr)
        {
          if (!v->a.empty()) bin.read(v->a[0], "float2", 2, G.texcoords);
          std::vector<float> extra;
          for (size_t k = 1; k < v->a.size(); ++k) bin.read(v->a[k], "float2", 2, extra);  // checked, unused
        }
        else
          bin.read(*v, "float2", 2, G.texcoords);
      }
      if (const JVal* v = g.get("indices")) bin.read(*v, "uint", 1, G.indices);
      if (const JVal* v = g.get("material")) G.material = (int)num(*v, "geometry material");
      const size_t verts = G.positions.size() / 3;
      if (!G.normals.empty() && G.normals.size() != 3 * verts) bad("normals and positions differ in count");
      if (!G.texcoords.empty() && G.texcoords.size() != 2 * verts) bad("texcoords and positions differ in count");
      if (verts > 0x7fffffffu || G.indices.size() / 3 > 0x7fffffffu) bad("geometry too large");
      for (uint32_t idx : G.indices)
        if (idx >= verts) bad("triangle index out of range");
      geoms.push_back(std::move(G));
    }

  // Material of a geometry: its file material, or the default (Principled) material, appended
  // after the file's materials, for none or an unknown one (render/scene.cpp:237-240, 283-290).
  auto materialOf = [&](const Geometry& G) {
    if (G.material >= 0 && G.material < fileMaterials) return G.material;
    if (defaultMaterial < 0)
    {
      prt_material d;
      prt_cuda_principled_defaults(&d);
      defaultMaterial = (int)out.materials.size();
      out.materials.push_back(d);
    }
    return defaultMaterial;
  };

  // Meshes, in the order the reference adds them to its scene group: objects in file order,
  // per object its instances (if any), per instance the object's geometries.
  auto addMesh = [&](const Geometry& G, const std::vector<float>& pos, const std::vector<float>& nrm) {
    out.positions.push_back(pos);
    out.normals.push_back(nrm);
    out.texcoords.push_back(G.texcoords);
    out.indices.emplace_back(G.indices.begin(), G.indices.end());
    prt_mesh m;
    std::memset(&m, 0, sizeof(m));
    m.vertex_count = (int32_t)(pos.size() / 3);
    m.tri_count = (int32_t)(G.indices.size() / 3);
    m.material = materialOf(G);
    out.meshes.push_back(m);
    out.triangleCount += m.tri_count;
  };
  if (const JVal* objs = doc.get("objects"))
    for (const JVal& o : items(*objs, "objects"))
    {
      if (o.type != JVal::Obj) bad("object must be an object");
      if (const JVal* nm = o.get("name")) str(*nm, "object name");
      std::vector<int> ids;
      if (const JVal* gl = o.get("geometries"))
        for (const JVal& id : items(*gl, "object geometries"))
        {
          const int64_t k = count(id, "geometry index");
          if (k >= (int64_t)geoms.size()) bad("geometry index out of range");
          ids.push_back((int)k);
        }
      std::vector<float> xf;
      if (const JVal* inst = o.get("instances")) bin.read(*inst, "float3x4", 12, xf);
      if (xf.empty())
        for (int id : ids) addMesh(geoms[id], geoms[id].positions, geoms[id].normals);
      else
        for (size_t t = 0; t + 11 < xf.size(); t += 12)
          for (int id : ids)
          {
            std::vector<float> pos, nrm;
            transformMesh(&xf[t], geoms[id].positions, geoms[id].normals, pos, nrm);
            addMesh(geoms[id], pos, nrm);
          }
    }
  // Lights: checked as rkscene::load checks them (rkscene.h:809-823); the environment comes
  // from the caller, as Scene::initLights takes it from props.
  if (const JVal* lights = doc.get("lights"))
    for (const JVal& l : items(*lights, "lights"))
    {
      const JVal* type = l.get("type");
      if (!type || str(*type, "light type") != "sunSky") bad("unsupported light type");
      if (const JVal* d = l.get("direction"))
      {
        float v[3];
        vec(*d, 3, v, "light direction");
      }
    }
  if (out.materials.empty())
  {
    prt_material d;
    prt_cuda_principled_defaults(&d);
    out.materials.push_back(d);
  }
  // Point the meshes and textures at the stored arrays.
  for (size_t i = 0; i < out.meshes.size(); ++i)
  {
    prt_mesh& m = out.meshes[i];
    m.positions = out.positions[i].empty() ? nullptr : out.positions[i].data();
    m.normals = out.normals[i].empty() ? nullptr : out.normals[i].data();
    m.texcoords = out.texcoords[i].empty() ? nullptr : out.texcoords[i].data();
    m.indices = out.indices[i].empty() ? nullptr : out.indices[i].data();
  }
  for (size_t i = 0; i < out.textures.size(); ++i) out.textures[i].rgb = out.texturePixels[i].data();
}

namespace {

// ---- .mesh: TriangleMesh blob + .mtl ------------------------------------------------------------

constexpr int32_t kTriangleMeshBlobId = 0x04df8666;  // geometry/triangle_mesh.h:21

class BlobReader
{
public:
  explicit BlobReader(const std::string& path) : f(path, std::ios::binary)
  {
    if (!f) throw std::runtime_error("mesh: failed to open file: " + path);
  }
  template <class T>
  T get()
  {
    T v;
    raw(&v, sizeof(T));
    return v;
  }
  void raw(void* dst, size_t bytes)
  {
    if (bytes && !f.read(reinterpret_cast<char*>(dst), (std::streamsize)bytes))
      throw std::runtime_error("mesh: unexpected end of stream");
  }
  std::string str()
  {
    const int32_t n = get<int32_t>();
    if (n < 0 || n > (1 << 20)) throw std::invalid_argument("mesh: invalid string size in stream");
    std::string s((size_t)n, '\0');
    raw(&s[0], (size_t)n);
    return s;
  }

private:
  std::ifstream f;
};

// One material's statements from a material library: key -> value, the value kept as the
// reference's MtlLoader keeps it (material/mtl_loader.cpp:66-90): three or two numbers as a
// vector, anything else as the text after the key.
struct MtlValue
{
  int kind = 0;  // 0 text, 2 vec2, 3 vec3
  std::string text;
  float v[3] = {0.f, 0.f, 0.f};
};
using MtlProps = std::map<std::string, MtlValue>;

void parseMtl(const std::string& path, std::map<std::string, MtlProps>& lib)
{
  std::ifstream f(path);
  if (!f) return;
  std::string name, line;
  while (std::getline(f, line))
  {
    std::istringstream ls(line);
    std::string head;
    if (!(ls >> head)) continue;
    std::string rest;
    std::getline(ls, rest);
    if (head == "newmtl")
    {
      std::istringstream rs(rest);
      if (!(rs >> name)) throw std::invalid_argument("mesh: invalid material in " + path);
      continue;
    }
    if (head[0] == '#') continue;
    MtlValue val;
    const int n = std::sscanf(rest.c_str(), "%f %f %f", &val.v[0], &val.v[1], &val.v[2]);
    if (n == 3 || n == 2)
      val.kind = n;
    else
    {
      const size_t b = rest.find_first_not_of(" \t\r");
      if (b == std::string::npos) throw std::invalid_argument("mesh: invalid statement in " + path);
      val.text = rest.substr(b);
      while (!val.text.empty() && (val.text.back() == '\r' || val.text.back() == ' ')) val.text.pop_back();
    }
    lib[name][head] = val;
  }
}

// Typed reads with the conversions of the reference's Props values (sys/value.h:200-276):
// text converts as a stream read (a lone number fills all three components of a vector).
struct MtlReader
{
  const MtlProps& p;
  bool has(const char* k) const { return p.count(k) != 0; }
  float f(const char* k, float def) const
  {
    auto it = p.find(k);
    if (it == p.end()) return def;
    if (it->second.kind != 0) throw std::invalid_argument(std::string("mesh: ") + k + " has an incompatible type");
    std::istringstream s(it->second.text);
    float x = 0.f;
    s >> x;
    return x;
  }
  void v3(const char* k, float* out) const
  {
    auto it = p.find(k);
    if (it == p.end()) return;
    if (it->second.kind == 3)
      for (int c = 0; c < 3; ++c) out[c] = it->second.v[c];
    else if (it->second.kind == 0)
    {
      std::istringstream s(it->second.text);
      float x = 0.f;
      s >> x;
      out[0] = out[1] = out[2] = x;
    }
    else
      throw std::invalid_argument(std::string("mesh: ") + k + " has an incompatible type");
  }
  std::string text(const char* k) const
  {
    auto it = p.find(k);
    if (it == p.end()) return std::string();
    if (it->second.kind != 0) throw std::invalid_argument(std::string("mesh: ") + k + " must be text");
    return it->second.text;
  }
};

// MaterialFactory::make (material/material_factory.cpp:29-96) for the types the device has.
prt_material mtlMaterial(const MtlProps& props, Loader& L)
{
  MtlReader r{props};
  std::string type = r.has("type") ? r.text("type") : std::string("OBJ");
  MtlProps p2 = props;  // the OBJ mapping adds Principled keys
  if (type == "OBJ")
  {
    auto copy = [&](const char* to, const char* from) {
      if (props.count(from)) p2[to] = props.at(from);
    };
    if (!r.has("baseColor") && !r.has("baseColorMap"))
    {
      copy("baseColor", "Kd");
      copy("baseColorMap", "map_Kd");
    }
    if (!r.has("bumpMap") && !r.has("normalMap"))
    {
      copy("bumpMap", "map_Bump");
      copy("normalMap", "map_bump");
    }
    if (!r.has("opacityMap")) copy("opacityMap", "map_d");
    if (!r.has("roughness") && r.has("Ns"))
    {
      MtlValue v;
      std::ostringstream s;
      s.precision(9);
      s << std::sqrt(std::sqrt(2.f / (r.f("Ns", 0.f) + 2.f)));  // Walter et al. 2007
      v.text = s.str();
      p2["roughness"] = v;
    }
    if (!r.has("transmission") && r.has("Tf"))
    {
      float tf[3] = {1.f, 1.f, 1.f};
      r.v3("Tf", tf);
      if (std::min(tf[0], std::min(tf[1], tf[2])) < 1.f)
      {
        MtlValue one, col;
        one.text = "1";
        col.kind = 3;
        for (int c = 0; c < 3; ++c) col.v[c] = 1.f - tf[c];  // 3ds Max convention
        p2["transmission"] = one;
        p2["transmissionColor"] = col;
      }
    }
    if (!r.has("ior") && r.has("Ks"))
    {
      float ks[3] = {0.f, 0.f, 0.f};
      r.v3("Ks", ks);
      const float f0 = (ks[0] + ks[1] + ks[2]) * (1.f / 3.f) * 0.08f;
      MtlValue v;
      std::ostringstream s;
      s.precision(9);
      s << (1.f + std::sqrt(f0)) / (1.f - std::sqrt(f0));
      v.text = s.str();
      p2["ior"] = v;
    }
    type = "Principled";
  }
  MtlReader q{p2};
  for (const char* k : {"normalMap", "bumpMap", "coatNormalMap", "coatBumpMap", "baseNormalMap", "baseBumpMap"})
    if (q.has(k)) throw std::invalid_argument("mesh: normal and bump maps are not supported on the device");
  if (q.has("opacityMap")) throw std::invalid_argument("mesh: opacity maps are not supported on the device");
  for (const auto& kv : p2)
    if (kv.first.size() > 3 && kv.first.compare(kv.first.size() - 3, 3, "Map") == 0 && kv.first != "baseColorMap")
      throw std::invalid_argument("mesh: texture maps are supported for baseColor only on the device");
  prt_material m;
  auto base = [&](float* color, int* tex) {
    if (q.has("baseColorMap"))
    {
      *tex = L.texture(q.text("baseColorMap"));
      if (!q.has("baseColor")) color[0] = color[1] = color[2] = 1.f;
    }
  };
  if (type == "Standard")
  {
    prt_cuda_material_defaults(&m);
    m.ambient_ior = q.f("ambientIOR", 1.f);
    m.base_weight = q.f("baseWeight", 1.f);
    q.v3("baseColor", m.base_color);
    base(m.base_color, &m.base_color_texture);
    m.metalness = q.f("metalness", 0.f);
    m.diffuse_roughness = q.f("diffuseRoughness", 0.f);
    m.specular_weight = q.f("specularWeight", 1.f);
    q.v3("specularColor", m.specular_color);
    m.specular_roughness = q.f("specularRoughness", 0.3f);
    m.specular_ior = q.f("specularIOR", 1.5f);
    m.transmission_weight = q.f("transmissionWeight", 0.f);
    q.v3("transmissionColor", m.transmission_color);
    m.transmission_depth = q.f("transmissionDepth", 1.f);
    m.subsurface_weight = q.f("subsurfaceWeight", 0.f);
    q.v3("subsurfaceColor", m.subsurface_color);
    m.subsurface_anisotropy = q.f("subsurfaceAnisotropy", 0.f);
    m.coat_weight = q.f("coatWeight", 0.f);
    q.v3("coatColor", m.coat_color);
    m.coat_roughness = q.f("coatRoughness", 0.f);
    m.coat_ior = q.f("coatIOR", 1.6f);
    m.sheen_weight = q.f("sheenWeight", 0.f);
    q.v3("sheenColor", m.sheen_color);
    m.sheen_roughness = q.f("sheenRoughness", 0.3f);
    m.emission_luminance = q.f("emissionLuminance", 0.f);
    q.v3("emissionColor", m.emission_color);
    m.thin_walled = (int)q.f("thinWalled", 0.f);
    m.opacity = q.f("opacity", 1.f);
    return m;
  }
  if (type == "Principled")
  {
    prt_cuda_principled_defaults(&m);
    q.v3("baseColor", m.base_color);
    base(m.base_color, &m.base_color_texture);
    q.v3("edgeColor", m.specular_color);
    m.metalness = q.f("metallic", 0.f);
    m.base_weight = q.f("diffuse", 1.f);
    m.specular_weight = q.f("specular", 1.f);
    m.ambient_ior = q.f("outsideIor", 1.f);
    m.specular_ior = q.f("ior", m.ambient_ior);
    m.transmission_weight = q.f("transmission", 0.f);
    q.v3("transmissionColor", m.transmission_color);
    m.transmission_depth = q.f("transmissionDepth", 1.f);
    m.specular_roughness = q.f("roughness", 0.f);
    m.coat_weight = q.f("coat", 0.f);
    m.coat_ior = q.f("coatIor", 1.5f);
    q.v3("coatColor", m.coat_color);
    m.coat_thickness = q.f("coatThickness", 1.f);
    m.coat_roughness = q.f("coatRoughness", 0.f);
    m.sheen_weight = q.f("sheen", 0.f);
    q.v3("sheenColor", m.sheen_color);
    m.sheen_tint = q.f("sheenTint", 0.f);
    m.sheen_roughness = q.f("sheenRoughness", 0.2f);
    m.thin_walled = (int)q.f("thin", 0.f);
    m.backlight = q.f("backlight", 0.f);
    m.thickness = q.f("thickness", 1.f);
    m.opacity = q.f("opacity", 1.f);
    return m;
  }
  throw std::invalid_argument("mesh: material type " + type + " is not supported on the device");
}

} // namespace

void loadMeshScene(const std::string& path, RkScene& out)
{
  out = RkScene();
  BlobReader b(path);
  if (b.get<int32_t>() != kTriangleMeshBlobId) throw std::invalid_argument("mesh: file has wrong blob ID: " + path);
  float bounds[6];
  b.raw(bounds, sizeof(bounds));
  const int32_t triCount = b.get<int32_t>(), vertexCount = b.get<int32_t>();
  const uint8_t hasNormals = b.get<uint8_t>();
  const int8_t numTexcoords = b.get<int8_t>();
  if (triCount < 0 || vertexCount < 0 || numTexcoords < 0)
    throw std::invalid_argument("mesh: invalid triangle mesh data in stream");
  std::vector<int32_t> idx((size_t)triCount * 3);
  b.raw(idx.data(), idx.size() * sizeof(int32_t));
  std::vector<int32_t> matIds((size_t)triCount);  // one per triangle (TriangleMesh::alloc's default)
  b.raw(matIds.data(), matIds.size() * sizeof(int32_t));
  const int stride = 3 + (hasNormals ? 3 : 0) + 2 * numTexcoords;
  std::vector<float> attribs((size_t)vertexCount * stride);
  b.raw(attribs.data(), attribs.size() * sizeof(float));
  const int32_t nameCount = b.get<int32_t>();
  if (nameCount < 0 || nameCount > (1 << 20)) throw std::invalid_argument("mesh: invalid array size in stream");
  std::vector<std::string> names;
  for (int i = 0; i < nameCount; ++i) names.push_back(b.str());
  for (int32_t v : idx)
    if (v < 0 || v >= vertexCount) throw std::invalid_argument("mesh: triangle index out of range");

  // Materials (Scene::loadMesh): one per material name, from <path without extension>.mtl,
  // the default (Principled) material for names the library lacks or for a blob without names.
  const size_t dot = path.find_last_of('.');
  const size_t slash = path.find_last_of('/');
  const std::string stem = (dot != std::string::npos && (slash == std::string::npos || dot > slash)) ? path.substr(0, dot) : path;
  std::map<std::string, MtlProps> lib;
  parseMtl(stem + ".mtl", lib);
  Loader L{out, directoryOf(path), {}};
  prt_material def;
  prt_cuda_principled_defaults(&def);
  if (names.empty())
    out.materials.push_back(def);
  for (const std::string& n : names)
  {
    auto it = lib.find(n);
    out.materials.push_back(it != lib.end() ? mtlMaterial(it->second, L) : def);
  }
  const int matCount = (int)out.materials.size();
  // Scene::Scene (render/scene.cpp:119-130) needs the emissive materials at ids 1..k.
  int lightMaterials = 0;
  for (int i = 1; i < matCount; ++i)
  {
    const prt_material& m = out.materials[i];
    if (m.model == PRT_MATERIAL_STANDARD && m.emission_luminance > 0.f)
    {
      ++lightMaterials;
      if (i > lightMaterials) throw std::invalid_argument("mesh: the material IDs must be remapped");
    }
  }
  for (int32_t& m : matIds)
    if (m < 0 || m >= matCount) throw std::invalid_argument("mesh: material id out of range");
  // Id 0 is the stream renderer's miss bucket (PRT_MATERIAL_MISS).
  out.materials[0].model = PRT_MATERIAL_MISS;

  // Vertex arrays (positions, normals, UV set 0) shared by the per-material meshes.
  std::vector<float> pos((size_t)vertexCount * 3), nrm, uv;
  if (hasNormals) nrm.resize((size_t)vertexCount * 3);
  if (numTexcoords > 0) uv.resize((size_t)vertexCount * 2);
  for (int64_t v = 0; v < vertexCount; ++v)
  {
    const float* a = &attribs[(size_t)v * stride];
    for (int k = 0; k < 3; ++k) pos[3 * v + k] = a[k];
    if (hasNormals)
      for (int k = 0; k < 3; ++k) nrm[3 * v + k] = a[3 + k];
    if (numTexcoords > 0)
      for (int k = 0; k < 2; ++k) uv[2 * v + k] = a[3 + (hasNormals ? 3 : 0) + k];
  }
  for (int m = 0; m < matCount; ++m)
  {
    std::vector<int32_t> tri;
    for (int32_t t = 0; t < triCount; ++t)
      if (matIds[t] == m) tri.insert(tri.end(), {idx[3 * t], idx[3 * t + 1], idx[3 * t + 2]});
    if (tri.empty()) continue;
    out.positions.push_back(pos);
    out.normals.push_back(nrm);
    out.texcoords.push_back(uv);
    out.indices.push_back(std::move(tri));
    prt_mesh mesh;
    std::memset(&mesh, 0, sizeof(mesh));
    mesh.vertex_count = vertexCount;
    mesh.tri_count = (int32_t)(out.indices.back().size() / 3);
    mesh.material = m;
    out.meshes.push_back(mesh);
    out.triangleCount += mesh.tri_count;
  }
  for (size_t i = 0; i < out.meshes.size(); ++i)
  {
    prt_mesh& m = out.meshes[i];
    m.positions = out.positions[i].empty() ? nullptr : out.positions[i].data();
    m.normals = out.normals[i].empty() ? nullptr : out.normals[i].data();
    m.texcoords = out.texcoords[i].empty() ? nullptr : out.texcoords[i].data();
    m.indices = out.indices[i].data();
  }
  for (size_t i = 0; i < out.textures.size(); ++i) out.textures[i].rgb = out.texturePixels[i].data();
}

void loadSceneFile(const std::string& path, RkScene& out)
{
  auto endsWith = [&](const char* ext) {
    const size_t n = std::strlen(ext);
    return path.size() >= n && path.compare(path.size() - n, n, ext) == 0;
  };
  if (endsWith(".rkscene")) return loadRkScene(path, out);
  if (endsWith(".mesh")) return loadMeshScene(path, out);
  throw std::invalid_argument("unknown scene format: " + path);
}

} // namespace prt
