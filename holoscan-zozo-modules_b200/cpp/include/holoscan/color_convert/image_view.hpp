// image_view.hpp - holoscan::color_convert::ImageView for C++ callers of the
// B200 converter: the reference module's borrowed image
// (include/holoscan/color_convert/image_view.hpp:15-44).
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>

#include "holoscan/color_convert/pixel_format.hpp"

namespace holoscan::color_convert {

enum class MemoryLocation : std::uint8_t { kHost = CC_HOST, kDevice = CC_DEVICE };

struct PlaneView {
  std::uint8_t* data{};
  std::size_t pitch{};
};

struct ImageView {
  PixelFormat format{PixelFormat::kRgb8};
  int width{};
  int height{};
  std::array<PlaneView, 3> planes{};
  MemoryLocation location{MemoryLocation::kDevice};
};

// A view of a packed image at `base`: each plane's rows without padding,
// the planes one after the other.
[[nodiscard]] inline ImageView packed_view(void* base, PixelFormat format, int width, int height,
                                           MemoryLocation location) noexcept {
  ImageView view{format, width, height, {}, location};
  auto* next = static_cast<std::uint8_t*>(base);
  for (int plane = 0; plane < format_info(format).planes; ++plane) {
    const PlaneSize size = plane_size(format, width, height, plane);
    view.planes[static_cast<std::size_t>(plane)] = {next, size.row_bytes};
    next += size.row_bytes * static_cast<std::size_t>(size.rows);
  }
  return view;
}

namespace detail {
inline cc_image_c to_c(const ImageView& v) noexcept {
  cc_image_c c{};
  c.format = static_cast<int32_t>(v.format);
  c.width = v.width;
  c.height = v.height;
  c.location = static_cast<int32_t>(v.location);
  for (std::size_t k = 0; k < 3; ++k) c.planes[k] = {v.planes[k].data, v.planes[k].pitch};
  return c;
}
}  // namespace detail

}  // namespace holoscan::color_convert
