// pixel_format.hpp - holoscan::color_convert's pixel formats, matrices and
// ranges for C++ callers of the B200 converter: the reference module's
// names, numbering and layouts (include/holoscan/color_convert/
// pixel_format.hpp:15-146), header-only over libisp_b200.so's C ABI
// (include/cc_b200.h).
#pragma once

#include <cstddef>
#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>

#include "cc_b200.h"

namespace holoscan::color_convert {

enum class PixelFormat : std::uint8_t {
  kNv12 = CC_NV12,
  kNv16 = CC_NV16,
  kI420 = CC_I420,
  kYuyv = CC_YUYV,
  kUyvy = CC_UYVY,
  kRgb8 = CC_RGB8,
  kBgr8 = CC_BGR8,
  kRgba8 = CC_RGBA8,
  kBgra8 = CC_BGRA8,
  kMono8 = CC_MONO8,
  kMono16 = CC_MONO16,
  kRgb16 = CC_RGB16,
};

inline constexpr PixelFormat kAllFormats[] = {
    PixelFormat::kNv12,  PixelFormat::kNv16,  PixelFormat::kI420,   PixelFormat::kYuyv,
    PixelFormat::kUyvy,  PixelFormat::kRgb8,  PixelFormat::kBgr8,   PixelFormat::kRgba8,
    PixelFormat::kBgra8, PixelFormat::kMono8, PixelFormat::kMono16, PixelFormat::kRgb16,
};

enum class ColorMatrix : std::uint8_t { kBt601 = CC_BT601, kBt709 = CC_BT709, kBt2020 = CC_BT2020 };
enum class ColorRange : std::uint8_t { kLimited = CC_RANGE_LIMITED, kFull = CC_RANGE_FULL };
enum class ColorModel : std::uint8_t { kYuv, kRgb, kGray };

struct FormatInfo {
  ColorModel model;
  int planes;
  int chroma_shift_x;
  int chroma_shift_y;
  int bytes_per_sample;
  int channels;
};

[[nodiscard]] inline FormatInfo format_info(PixelFormat format) noexcept {
  cc_format_info_c c{};
  cc_b200_format_info(static_cast<int32_t>(format), &c);
  return {static_cast<ColorModel>(c.model), c.planes, c.chroma_shift_x, c.chroma_shift_y, c.bytes_per_sample,
          c.channels};
}

[[nodiscard]] inline bool is_yuv(PixelFormat f) noexcept { return format_info(f).model == ColorModel::kYuv; }
[[nodiscard]] inline bool is_planar(PixelFormat f) noexcept { return format_info(f).planes > 1; }
[[nodiscard]] inline bool is_subsampled(PixelFormat f) noexcept {
  const FormatInfo i = format_info(f);
  return i.chroma_shift_x != 0 || i.chroma_shift_y != 0;
}
[[nodiscard]] inline bool has_alpha(PixelFormat f) noexcept {
  return f == PixelFormat::kRgba8 || f == PixelFormat::kBgra8;
}
[[nodiscard]] inline bool needs_even_width(PixelFormat f) noexcept {
  return f == PixelFormat::kYuyv || f == PixelFormat::kUyvy;
}

struct PlaneSize {
  std::size_t row_bytes;
  int rows;
};

[[nodiscard]] inline PlaneSize plane_size(PixelFormat format, int width, int height, int plane) noexcept {
  std::size_t row_bytes = 0;
  int32_t rows = 0;
  if (cc_b200_plane_size(static_cast<int32_t>(format), width, height, plane, &row_bytes, &rows) != ISP_OK) return {0, 0};
  return {row_bytes, rows};
}

[[nodiscard]] inline std::size_t packed_size(PixelFormat format, int width, int height) noexcept {
  return cc_b200_packed_size(static_cast<int32_t>(format), width, height);
}

namespace detail {
inline std::string_view name_or_unknown(const char* n) noexcept { return n != nullptr ? std::string_view(n) : "unknown"; }
template <class E>
std::optional<E> parsed(int32_t v) noexcept {
  return v < 0 ? std::nullopt : std::optional<E>(static_cast<E>(v));
}
}  // namespace detail

[[nodiscard]] inline std::string_view format_name(PixelFormat f) noexcept {
  return detail::name_or_unknown(cc_b200_format_name(static_cast<int32_t>(f)));
}
[[nodiscard]] inline std::optional<PixelFormat> parse_format(std::string_view name) noexcept {
  return detail::parsed<PixelFormat>(cc_b200_parse_format(std::string(name).c_str()));
}
[[nodiscard]] inline std::string_view matrix_name(ColorMatrix m) noexcept {
  return detail::name_or_unknown(cc_b200_matrix_name(static_cast<int32_t>(m)));
}
[[nodiscard]] inline std::optional<ColorMatrix> parse_matrix(std::string_view name) noexcept {
  return detail::parsed<ColorMatrix>(cc_b200_parse_matrix(std::string(name).c_str()));
}
[[nodiscard]] inline std::string_view range_name(ColorRange r) noexcept {
  return detail::name_or_unknown(cc_b200_range_name(static_cast<int32_t>(r)));
}
[[nodiscard]] inline std::optional<ColorRange> parse_range(std::string_view name) noexcept {
  return detail::parsed<ColorRange>(cc_b200_parse_range(std::string(name).c_str()));
}

}  // namespace holoscan::color_convert
