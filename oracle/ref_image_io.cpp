// Test infrastructure (oracle only): replacement for the reference's OpenImageIO-backed
// image/image_io.cpp, which cannot be built here (OpenImageIO is not installed). It keeps
// the interface of image/image_io.h:13-31 and reads/writes little-endian colour PFM
// (RGB FP32), which is all the oracle needs for albedo textures and environment maps.
// Rows are returned top row first, the order OpenImageIO hands to the reference.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sys/logging.h"
#include "image/image_io.h"

namespace prt {

struct ImageIo::HandleSt
{
  ImageIo::Desc desc;
  std::vector<float> rgb; // top row first
};

ImageIo::Handle ImageIo::open(const std::string& filename)
{
  FILE* f = std::fopen(filename.c_str(), "rb");
  if (!f)
  {
    LogError() << "Could not load image: " << filename;
    return 0;
  }
  char magic[3] = {0, 0, 0};
  int w = 0, h = 0;
  float scale = 0.f;
  if (std::fscanf(f, "%2s %d %d %f", magic, &w, &h, &scale) != 4 || std::strcmp(magic, "PF") != 0 ||
      w <= 0 || h <= 0 || scale >= 0.f)
  {
    std::fclose(f);
    LogError() << "Unsupported image file format (only little-endian colour PFM): " << filename;
    return 0;
  }
  std::fgetc(f); // the single whitespace byte after the header
  Handle h2 = new HandleSt;
  h2->desc.size = Vec2i(w, h);
  h2->desc.format = PixelFormat::Rgb32f;
  h2->rgb.resize((size_t)w * h * 3);
  std::vector<float> row((size_t)w * 3);
  for (int y = 0; y < h; ++y)
  {
    if (std::fread(row.data(), sizeof(float), row.size(), f) != row.size())
    {
      std::fclose(f);
      delete h2;
      LogError() << "Truncated PFM file: " << filename;
      return 0;
    }
    // PFM stores the bottom row first.
    std::memcpy(&h2->rgb[(size_t)(h - 1 - y) * w * 3], row.data(), row.size() * sizeof(float));
  }
  std::fclose(f);
  return h2;
}

ImageIo::Desc ImageIo::getDesc(Handle h)
{
  return h->desc;
}

void ImageIo::getData(Handle h, void* data)
{
  std::memcpy(data, h->rgb.data(), h->rgb.size() * sizeof(float));
}

void ImageIo::close(Handle h)
{
  delete h;
}

bool ImageIo::save(const std::string& filename, const Desc& desc, const void* data)
{
  if (desc.format != PixelFormat::Rgb32f)
    return false;
  FILE* f = std::fopen(filename.c_str(), "wb");
  if (!f) return false;
  const int w = desc.size.x, h = desc.size.y;
  std::fprintf(f, "PF\n%d %d\n-1.0\n", w, h);
  const float* src = (const float*)data;
  for (int y = h - 1; y >= 0; --y)
    std::fwrite(src + (size_t)y * w * 3, sizeof(float), (size_t)w * 3, f);
  std::fclose(f);
  return true;
}

} // namespace prt
