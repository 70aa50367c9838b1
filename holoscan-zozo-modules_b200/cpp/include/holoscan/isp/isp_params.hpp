// isp_params.hpp - the holoscan::isp settings, views and statistics layout,
// for C++ callers of the B200 ISP.
//
// The same names, fields, defaults and numbering as the reference module's
// include/holoscan/isp/isp_params.hpp, so that code written against it
// compiles unchanged; the checks and the tone table come from
// libisp_b200.so's C ABI (include/isp_b200.h), which restates
// modules/isp/src/isp_params.cpp. Header-only: link libisp_b200.so.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "isp_b200.h"

namespace holoscan::isp {

// isp_params.hpp:21-61 of the reference, with its numbering.
enum class BayerPattern : std::uint8_t { kRGGB, kBGGR, kGRBG, kGBRG };
enum class RawFormat : std::uint8_t { kUint8, kUint16, kRaw10, kRaw12 };
enum class DemosaicMethod : std::uint8_t { kBilinear, kMalvar };
enum class WhiteBalanceMode : std::uint8_t { kManual, kGrayWorld, kWhitePatch };
enum class ToneCurve : std::uint8_t { kSrgb, kGamma, kLinear, kLut };
enum class OutputFormat : std::uint8_t { kRgb8, kRgba8, kRgb16, kRgb32f };
// kCuda: this build's GPU pipeline. kCpu is the reference's host backend,
// which this build does not ship (the constructor rejects it). kAuto: kCuda
// when a CUDA device is usable.
enum class Backend : std::uint8_t { kCuda, kCpu, kAuto };

inline constexpr int kChannelR = 0;
inline constexpr int kChannelGr = 1;
inline constexpr int kChannelGb = 2;
inline constexpr int kChannelB = 3;

struct LensShading {
  int width{};
  int height{};
  int channels{1};
  std::vector<float> gains;  // [height][width][channels], each in (0, 16]
};

struct AutoExposureParams {
  float target{0.18F};
  float damping{0.5F};
  std::int64_t min_exposure_ns{10'000};
  std::int64_t max_exposure_ns{33'000'000};
  float min_gain{1.0F};
  float max_gain{16.0F};
};

struct IspParams {
  float black_level{0.0F};
  std::optional<std::array<float, 4>> channel_black_levels;
  float white_level{0.0F};
  std::optional<LensShading> lens_shading;
  WhiteBalanceMode white_balance{WhiteBalanceMode::kManual};
  std::array<float, 3> wb_gains{1.0F, 1.0F, 1.0F};
  float awb_smoothing{0.25F};
  float white_patch_percentile{0.99F};
  DemosaicMethod demosaic{DemosaicMethod::kMalvar};
  std::array<float, 9> ccm{1.0F, 0.0F, 0.0F, 0.0F, 1.0F, 0.0F, 0.0F, 0.0F, 1.0F};
  ToneCurve tone_curve{ToneCurve::kSrgb};
  float gamma{2.2F};
  std::vector<float> lut;
  float sharpen{0.0F};
  AutoExposureParams auto_exposure;
};

inline constexpr int kToneLutSize = ISP_TONE_LUT_SIZE;

struct RawImageView {
  const void* data{};
  int width{};
  int height{};
  std::size_t pitch{};
  RawFormat format{RawFormat::kUint16};
  int bit_depth{};
  BayerPattern pattern{BayerPattern::kRGGB};
};

struct RgbImageView {
  void* data{};
  std::size_t pitch{};
  OutputFormat format{OutputFormat::kRgb8};
};

struct StatsOutput {
  std::uint32_t* histogram{};
  float* stats{};
};

struct FrameExposure {
  std::int64_t exposure_ns{};
  float gain{};
};

inline constexpr int kHistogramBins = ISP_HISTOGRAM_BINS;
inline constexpr int kHistogramChannels = ISP_HISTOGRAM_CHANNELS;
inline constexpr int kHistogramLuma = 0;
inline constexpr int kHistogramRed = 1;
inline constexpr int kHistogramGreen = 2;
inline constexpr int kHistogramBlue = 3;

namespace stats {
inline constexpr int kLayoutVersion = ISP_STATS_LAYOUT_VERSION;
inline constexpr int kMeanR = 0;
inline constexpr int kMeanG = 1;
inline constexpr int kMeanB = 2;
inline constexpr int kMeanLuma = 3;
inline constexpr int kAeErrorEv = 4;
inline constexpr int kExposureScale = 5;
inline constexpr int kSuggestedExposureNs = 6;
inline constexpr int kSuggestedGain = 7;
inline constexpr int kWbGainR = 8;
inline constexpr int kWbGainG = 9;
inline constexpr int kWbGainB = 10;
inline constexpr int kSaturatedFraction = 11;
inline constexpr int kStatsSize = ISP_STATS_SIZE;
}  // namespace stats

struct PlatformFacts {
  bool cuda_device{};
};

[[nodiscard]] constexpr Backend resolve_auto(const PlatformFacts& facts) noexcept {
  return facts.cuda_device ? Backend::kCuda : Backend::kCpu;
}

[[nodiscard]] constexpr int output_channels(OutputFormat format) noexcept {
  return format == OutputFormat::kRgba8 ? 4 : 3;
}
[[nodiscard]] constexpr int output_channel_bytes(OutputFormat format) noexcept {
  return format == OutputFormat::kRgb16 ? 2 : format == OutputFormat::kRgb32f ? 4 : 1;
}

// ---- Names ------------------------------------------------------------------

namespace detail {
template <class E, std::size_t N>
constexpr std::string_view name_of(E value, const std::array<std::string_view, N>& names) noexcept {
  const auto i = static_cast<std::size_t>(value);
  return i < N ? names[i] : std::string_view{};
}
template <class E, std::size_t N>
constexpr std::optional<E> parse_of(std::string_view name, const std::array<std::string_view, N>& names) noexcept {
  for (std::size_t i = 0; i < N; ++i) {
    if (names[i] == name) return static_cast<E>(i);
  }
  return std::nullopt;
}
inline constexpr std::array<std::string_view, 3> kBackendNames{"cuda", "cpu", "auto"};
inline constexpr std::array<std::string_view, 2> kDemosaicNames{"bilinear", "malvar"};
inline constexpr std::array<std::string_view, 4> kPatternNames{"RGGB", "BGGR", "GRBG", "GBRG"};
inline constexpr std::array<std::string_view, 3> kWhiteBalanceNames{"manual", "gray-world", "white-patch"};
}  // namespace detail

[[nodiscard]] inline std::string_view backend_name(Backend b) noexcept { return detail::name_of(b, detail::kBackendNames); }
[[nodiscard]] inline std::optional<Backend> parse_backend(std::string_view name) noexcept {
  return detail::parse_of<Backend>(name, detail::kBackendNames);
}
[[nodiscard]] inline std::string_view demosaic_name(DemosaicMethod m) noexcept {
  return detail::name_of(m, detail::kDemosaicNames);
}
[[nodiscard]] inline std::optional<DemosaicMethod> parse_demosaic(std::string_view name) noexcept {
  return detail::parse_of<DemosaicMethod>(name, detail::kDemosaicNames);
}
[[nodiscard]] inline std::string_view pattern_name(BayerPattern p) noexcept {
  return detail::name_of(p, detail::kPatternNames);
}
[[nodiscard]] inline std::optional<BayerPattern> parse_pattern(std::string_view name) noexcept {
  return detail::parse_of<BayerPattern>(name, detail::kPatternNames);
}
[[nodiscard]] inline std::string_view white_balance_name(WhiteBalanceMode m) noexcept {
  return detail::name_of(m, detail::kWhiteBalanceNames);
}
[[nodiscard]] inline std::optional<WhiteBalanceMode> parse_white_balance(std::string_view name) noexcept {
  return detail::parse_of<WhiteBalanceMode>(name, detail::kWhiteBalanceNames);
}

// ---- The C ABI underneath -------------------------------------------------

namespace detail {

// The C ABI's view of `p`; its pointers borrow p's vectors.
inline isp_params_c to_c(const IspParams& p) {
  isp_params_c c{};
  isp_b200_params_default(&c);
  c.black_level = p.black_level;
  c.has_channel_black_levels = p.channel_black_levels.has_value() ? 1 : 0;
  if (p.channel_black_levels) {
    for (int i = 0; i < 4; ++i) c.channel_black_levels[i] = (*p.channel_black_levels)[i];
  }
  c.white_level = p.white_level;
  c.has_lens_shading = p.lens_shading.has_value() ? 1 : 0;
  if (p.lens_shading) {
    c.lsc_width = p.lens_shading->width;
    c.lsc_height = p.lens_shading->height;
    c.lsc_channels = p.lens_shading->channels;
    c.lsc_gains = p.lens_shading->gains.data();
    c.lsc_gains_count = p.lens_shading->gains.size();
  }
  c.white_balance = static_cast<int32_t>(p.white_balance);
  for (int i = 0; i < 3; ++i) c.wb_gains[i] = p.wb_gains[i];
  c.awb_smoothing = p.awb_smoothing;
  c.white_patch_percentile = p.white_patch_percentile;
  c.demosaic = static_cast<int32_t>(p.demosaic);
  for (int i = 0; i < 9; ++i) c.ccm[i] = p.ccm[i];
  c.tone_curve = static_cast<int32_t>(p.tone_curve);
  c.gamma = p.gamma;
  c.lut = p.lut.data();
  c.lut_size = p.lut.size();
  c.sharpen = p.sharpen;
  c.auto_exposure.target = p.auto_exposure.target;
  c.auto_exposure.damping = p.auto_exposure.damping;
  c.auto_exposure.min_exposure_ns = p.auto_exposure.min_exposure_ns;
  c.auto_exposure.max_exposure_ns = p.auto_exposure.max_exposure_ns;
  c.auto_exposure.min_gain = p.auto_exposure.min_gain;
  c.auto_exposure.max_gain = p.auto_exposure.max_gain;
  return c;
}

inline isp_raw_view_c to_c(const RawImageView& v) {
  return isp_raw_view_c{v.data, v.width, v.height, v.pitch, static_cast<int32_t>(v.format), v.bit_depth,
                        static_cast<int32_t>(v.pattern)};
}

inline isp_rgb_view_c to_c(const RgbImageView& v) { return isp_rgb_view_c{v.data, v.pitch, static_cast<int32_t>(v.format)}; }

// The reference's exceptions for a C-ABI status: invalid_argument for an
// unusable setting or view, runtime_error for everything else.
inline void check(int status) {
  if (status == ISP_OK) return;
  const std::string what = isp_b200_last_error();
  if (status == ISP_EINVAL) throw std::invalid_argument(what);
  throw std::runtime_error(what);
}

}  // namespace detail

// @throws std::invalid_argument naming the first unusable field.
inline void validate_params(const IspParams& params) {
  const isp_params_c c = detail::to_c(params);
  detail::check(isp_b200_validate_params(&c));
}

// The tone table the pipeline interpolates: kToneLutSize entries for the
// built-in curves, the configured table for kLut.
[[nodiscard]] inline std::vector<float> tone_lut(const IspParams& params) {
  const isp_params_c c = detail::to_c(params);
  std::vector<float> out(params.tone_curve == ToneCurve::kLut ? params.lut.size() : kToneLutSize);
  std::size_t n = 0;
  detail::check(isp_b200_tone_lut(&c, out.data(), out.size(), &n));
  out.resize(n);
  return out;
}

[[nodiscard]] inline std::size_t raw_row_bytes(RawFormat format, int width) noexcept {
  return isp_b200_raw_row_bytes(static_cast<int32_t>(format), width);
}

// @throws std::invalid_argument if `raw` cannot be processed with `params`.
inline void validate_raw(const RawImageView& raw, const IspParams& params) {
  const isp_params_c c = detail::to_c(params);
  const isp_raw_view_c r = detail::to_c(raw);
  detail::check(isp_b200_validate_raw(&r, &c));
}

}  // namespace holoscan::isp
