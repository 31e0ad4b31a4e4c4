// Test infrastructure (oracle only). DeviceCpu::initRenderer (render/device_cpu.cpp:32-46)
// links the single-ray and packet renderer factories, whose intersectors need Embree.
// The oracle only drives the stream renderer ("pathStream"), so those two factories are
// replaced by stubs that reject every type, as the reference does for unknown types
// (render/renderer_factory_stream.cpp:75).
#include <stdexcept>
#include "render/renderer_factory_single.h"
#include "render/renderer_factory_packet.h"

namespace prt {

std::shared_ptr<Renderer> RendererFactorySingle::make(const std::string& type, const std::shared_ptr<const Scene>&,
                                                      const std::shared_ptr<Intersector>&, const Props&, Props&)
{
  throw std::invalid_argument("oracle build: only stream renderers are available, not " + type);
}

std::shared_ptr<Renderer> RendererFactoryPacket::make(const std::string& type, const std::shared_ptr<const Scene>&,
                                                      const std::shared_ptr<Intersector>&, const Props&, Props&)
{
  throw std::invalid_argument("oracle build: only stream renderers are available, not " + type);
}

} // namespace prt
