// conversion.hpp - what one conversion does, for C++ callers of the B200
// converter: the reference module's ResizeMode, Rect, ConversionParams,
// Mapping, compute_mapping and validate_conversion
// (include/holoscan/color_convert/conversion.hpp:40-95), with the same
// exceptions and messages, over the C ABI.
#pragma once

#include <array>
#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>

#include "holoscan/color_convert/image_view.hpp"
#include "holoscan/color_convert/pixel_format.hpp"

namespace holoscan::color_convert {

enum class ResizeMode : std::uint8_t { kNearest = CC_NEAREST, kBilinear = CC_BILINEAR, kArea = CC_AREA };

[[nodiscard]] inline std::string_view resize_mode_name(ResizeMode mode) noexcept {
  return detail::name_or_unknown(cc_b200_resize_mode_name(static_cast<int32_t>(mode)));
}
[[nodiscard]] inline std::optional<ResizeMode> parse_resize_mode(std::string_view name) noexcept {
  return detail::parsed<ResizeMode>(cc_b200_parse_resize_mode(std::string(name).c_str()));
}

struct Rect {
  int x{};
  int y{};
  int width{};
  int height{};

  friend constexpr bool operator==(const Rect& a, const Rect& b) noexcept {
    return a.x == b.x && a.y == b.y && a.width == b.width && a.height == b.height;
  }
};

struct ConversionParams {
  ColorMatrix matrix{ColorMatrix::kBt601};
  ColorRange range{ColorRange::kLimited};
  ResizeMode mode{ResizeMode::kBilinear};
  std::optional<Rect> crop;
  bool letterbox{false};
  std::array<std::uint8_t, 3> fill_rgb{0, 0, 0};
};

struct Mapping {
  Rect source;
  Rect content;
};

namespace detail {
inline cc_params_c to_c(const ConversionParams& p) noexcept {
  cc_params_c c{};
  cc_b200_params_default(&c);
  c.matrix = static_cast<int32_t>(p.matrix);
  c.range = static_cast<int32_t>(p.range);
  c.mode = static_cast<int32_t>(p.mode);
  if (p.crop) {
    c.has_crop = 1;
    c.crop = {p.crop->x, p.crop->y, p.crop->width, p.crop->height};
  }
  c.letterbox = p.letterbox ? 1 : 0;
  for (int k = 0; k < 3; ++k) c.fill_rgb[k] = p.fill_rgb[static_cast<std::size_t>(k)];
  return c;
}

// ISP_EINVAL -> std::invalid_argument, anything else -> std::runtime_error,
// each with the library's message.
inline void check(int status) {
  if (status == ISP_OK) return;
  const std::string what = isp_b200_last_error();
  if (status == ISP_EINVAL) throw std::invalid_argument(what);
  throw std::runtime_error(what);
}
}  // namespace detail

// The mapping of a source_width x source_height image into a width x height
// one of `destination` format (letterbox, crop).
// @throws std::invalid_argument for sizes that are not positive or a crop
//         that is not inside the source.
[[nodiscard]] inline Mapping compute_mapping(int source_width, int source_height, int width, int height,
                                             PixelFormat destination, const ConversionParams& params) {
  const cc_params_c c = detail::to_c(params);
  cc_mapping_c m{};
  detail::check(cc_b200_compute_mapping(source_width, source_height, width, height,
                                        static_cast<int32_t>(destination), &c, &m));
  return {{m.source.x, m.source.y, m.source.width, m.source.height},
          {m.content.x, m.content.y, m.content.width, m.content.height}};
}

// @throws std::invalid_argument naming the first problem.
inline void validate_conversion(const ImageView& source, const ImageView& destination,
                                const ConversionParams& params) {
  const cc_image_c s = detail::to_c(source);
  const cc_image_c d = detail::to_c(destination);
  const cc_params_c c = detail::to_c(params);
  detail::check(cc_b200_validate(&s, &d, &c));
}

}  // namespace holoscan::color_convert
