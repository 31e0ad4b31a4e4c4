// Test infrastructure (oracle only): exports the two lights the reference's sun-sky model
// produces (light/sun_sky_light.cpp:17-193): the sun as a DistantLight (radiance, direction,
// angular diameter) and the sky as a 512x256 RGB image for an ImageLight with a 128 LUT.
// The members are private in the reference classes, so this translation unit alone opens
// them for reading; it changes no behaviour.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "sys/props.h"
#include "sys/logging.h"
#include "sys/tasking.h"
#include "sampling/distribution2d.h"
#include "sampling/shape_sampler.h"
#include "image/color.h"
#include "image/image_texture.h"
#define private public
#define protected public
#include "light/distant_light.h"
#include "light/image_light.h"
#include "light/sun_sky_light.h"
#undef private
#undef protected

using namespace prt;

extern "C" {

// dir: direction toward the sun; outputs: sun radiance (3), sun angular diameter, and the
// sky image (width*height*3 floats, row 0 at the top) with its size.
int ref_sunsky(const float* dir, float turbidity, float albedo, float* sunColor, float* sunAngle, float* sky,
               int* width, int* height)
{
  try
  {
    Props p;
    p.set("direction", Vec3f(dir[0], dir[1], dir[2]));
    p.set("turbidity", turbidity);
    p.set("albedo", albedo);
    SunSkyLight ss(p, 1.f);
    auto sun = std::dynamic_pointer_cast<DistantLight>(ss.getSunLight());
    auto skyL = std::dynamic_pointer_cast<ImageLight>(ss.getSkyLight());
    if (!sun || !skyL) return -1;
    for (int k = 0; k < 3; ++k) sunColor[k] = sun->color[k];
    *sunAngle = sun->angle * 2.f;  // the light stores the half angle
    const Vec2i size = skyL->color->getSize();
    *width = size.x;
    *height = size.y;
    if (sky)
    {
      // Texture rows are stored flipped (texture row t = image row H-1-t); return image rows.
      for (int y = 0; y < size.y; ++y)
        for (int x = 0; x < size.x; ++x)
        {
          const Vec3f c = skyL->color->get3f(Vec2i(x, size.y - 1 - y));
          float* o = sky + 3 * ((size_t)y * size.x + x);
          o[0] = c.x;
          o[1] = c.y;
          o[2] = c.z;
        }
    }
    return 0;
  }
  catch (...)
  {
    return -2;
  }
}

} // extern "C"
