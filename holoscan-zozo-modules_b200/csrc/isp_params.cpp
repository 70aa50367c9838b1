// isp_params.cpp - settings of the B200 ISP on the host: defaults,
// validation, raw row sizes and the tone table, with the holoscan::isp
// semantics and messages (modules/isp/src/isp_params.cpp:85-237).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "isp_b200.h"
#include "isp_host.hpp"

namespace isp_b200 {

namespace {

bool finite_in(float v, float lo, float hi) { return std::isfinite(v) && v >= lo && v <= hi; }

}  // namespace

void params_default(isp_params_c* p) {
  // IspParams{} (isp_params.hpp:95-121).
  *p = isp_params_c{};
  p->black_level = 0.0F;
  p->white_level = 0.0F;
  p->white_balance = ISP_WB_MANUAL;
  p->wb_gains[0] = p->wb_gains[1] = p->wb_gains[2] = 1.0F;
  p->awb_smoothing = 0.25F;
  p->white_patch_percentile = 0.99F;
  p->demosaic = ISP_DEMOSAIC_MALVAR;
  const float identity[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int k = 0; k < 9; ++k) p->ccm[k] = identity[k];
  p->tone_curve = ISP_TONE_SRGB;
  p->gamma = 2.2F;
  p->sharpen = 0.0F;
  p->auto_exposure.target = 0.18F;
  p->auto_exposure.damping = 0.5F;
  p->auto_exposure.min_exposure_ns = 10'000;
  p->auto_exposure.max_exposure_ns = 33'000'000;
  p->auto_exposure.min_gain = 1.0F;
  p->auto_exposure.max_gain = 16.0F;
}

const char* validate_params(const isp_params_c& p) {
  if (!finite_in(p.black_level, 0.0F, 65535.0F)) return "black_level must be 0..65535";
  if (p.has_channel_black_levels) {
    for (const float level : p.channel_black_levels) {
      if (!finite_in(level, 0.0F, 65535.0F)) return "channel_black_levels must be 0..65535";
    }
  }
  if (!finite_in(p.white_level, 0.0F, 65535.0F)) {
    return "white_level must be 0 (from the bit depth) or up to 65535";
  }
  if (p.has_lens_shading) {
    if (p.lsc_width < 2 || p.lsc_height < 2 || p.lsc_width > 256 || p.lsc_height > 256) {
      return "lens_shading grid must be 2x2 to 256x256 points";
    }
    if (p.lsc_channels != 1 && p.lsc_channels != 4) return "lens_shading channels must be 1 or 4";
    if (p.lsc_gains_count != static_cast<size_t>(p.lsc_width) * p.lsc_height * p.lsc_channels ||
        p.lsc_gains == nullptr) {
      return "lens_shading gains must hold width x height x channels values";
    }
    for (size_t i = 0; i < p.lsc_gains_count; ++i) {
      const float g = p.lsc_gains[i];
      if (!(std::isfinite(g) && g > 0.0F && g <= 16.0F)) return "lens_shading gains must be in (0, 16]";
    }
  }
  for (const float g : p.wb_gains) {
    if (!(std::isfinite(g) && g > 0.0F && g <= 64.0F)) return "wb_gains must be in (0, 64]";
  }
  if (p.white_balance < ISP_WB_MANUAL || p.white_balance > ISP_WB_WHITE_PATCH) return "white_balance mode unknown";
  if (!(std::isfinite(p.awb_smoothing) && p.awb_smoothing > 0.0F && p.awb_smoothing <= 1.0F)) {
    return "awb_smoothing must be in (0, 1]";
  }
  if (!(std::isfinite(p.white_patch_percentile) && p.white_patch_percentile >= 0.5F &&
        p.white_patch_percentile < 1.0F)) {
    return "white_patch_percentile must be in [0.5, 1)";
  }
  if (p.demosaic != ISP_DEMOSAIC_BILINEAR && p.demosaic != ISP_DEMOSAIC_MALVAR) return "demosaic method unknown";
  for (const float v : p.ccm) {
    if (!finite_in(v, -16.0F, 16.0F)) return "ccm entries must be finite, -16..16";
  }
  if (p.tone_curve < ISP_TONE_SRGB || p.tone_curve > ISP_TONE_LUT) return "tone_curve unknown";
  if (p.tone_curve == ISP_TONE_GAMMA && !finite_in(p.gamma, 0.1F, 10.0F)) return "gamma must be 0.1..10";
  if (p.tone_curve == ISP_TONE_LUT) {
    if (p.lut_size < 2 || p.lut_size > 65536 || p.lut == nullptr) return "lut must have 2..65536 entries";
    for (size_t i = 0; i < p.lut_size; ++i) {
      if (!finite_in(p.lut[i], 0.0F, 1.0F)) return "lut entries must be 0..1";
    }
  }
  if (!finite_in(p.sharpen, 0.0F, 4.0F)) return "sharpen must be 0..4";
  const isp_auto_exposure_c& ae = p.auto_exposure;
  if (!(std::isfinite(ae.target) && ae.target > 0.0F && ae.target < 1.0F)) {
    return "auto_exposure.target must be in (0, 1)";
  }
  if (!finite_in(ae.damping, 0.0F, 1.0F)) return "auto_exposure.damping must be 0..1";
  if (ae.min_exposure_ns <= 0 || ae.max_exposure_ns < ae.min_exposure_ns) {
    return "auto_exposure needs 0 < min_exposure_ns <= max_exposure_ns";
  }
  if (!(std::isfinite(ae.min_gain) && std::isfinite(ae.max_gain) && ae.min_gain > 0.0F &&
        ae.max_gain >= ae.min_gain)) {
    return "auto_exposure needs 0 < min_gain <= max_gain";
  }
  return nullptr;
}

size_t raw_row_bytes(int32_t format, int32_t width) {
  const auto w = static_cast<size_t>(width < 0 ? 0 : width);
  switch (format) {
    case ISP_RAW_U8: return w;
    case ISP_RAW_U16: return 2U * w;
    case ISP_RAW_RAW10: return 5U * ((w + 3U) / 4U);
    case ISP_RAW_RAW12: return 3U * ((w + 1U) / 2U);
    default: return 0;
  }
}

float white_level_of(const isp_params_c& p, int bit_depth) {
  return p.white_level > 0.0F ? p.white_level : static_cast<float>((1U << static_cast<unsigned>(bit_depth)) - 1U);
}

std::string validate_raw(const isp_raw_view_c& raw, const isp_params_c& p) {
  if (raw.data == nullptr) return "raw image has no data";
  if (raw.width < 2 || raw.height < 2 || raw.width > 16384 || raw.height > 16384) {
    return "raw image must be 2x2 to 16384x16384";
  }
  if (raw.format < ISP_RAW_U8 || raw.format > ISP_RAW_RAW12) return "raw sample format unknown";
  if (raw.pattern < ISP_BAYER_RGGB || raw.pattern > ISP_BAYER_GBRG) return "raw Bayer pattern unknown";
  if (raw.pitch < raw_row_bytes(raw.format, raw.width)) return "raw image pitch is shorter than a row";
  if (raw.format == ISP_RAW_U16 &&
      (raw.pitch % 2U != 0U || reinterpret_cast<std::uintptr_t>(raw.data) % 2U != 0U)) {
    return "uint16 raw samples must be aligned to 2 bytes, rows too";
  }
  const int max_bits = raw.format == ISP_RAW_U8      ? 8
                       : raw.format == ISP_RAW_RAW10 ? 10
                       : raw.format == ISP_RAW_RAW12 ? 12
                                                     : 16;
  const bool packed = raw.format == ISP_RAW_RAW10 || raw.format == ISP_RAW_RAW12;
  if (raw.bit_depth < 1 || raw.bit_depth > max_bits || (packed && raw.bit_depth != max_bits)) {
    return "raw bit depth " + std::to_string(raw.bit_depth) + " does not fit its sample format";
  }
  const float white = white_level_of(p, raw.bit_depth);
  if (white > static_cast<float>((1U << static_cast<unsigned>(raw.bit_depth)) - 1U)) {
    return "white_level exceeds the raw bit depth";
  }
  for (int k = 0; k < 4; ++k) {
    const float level = p.has_channel_black_levels ? p.channel_black_levels[k] : p.black_level;
    if (!(level < white)) return "black levels must be below the white level";
  }
  return {};
}

std::string validate_out(const isp_raw_view_c& raw, const isp_rgb_view_c& out) {
  if (out.data == nullptr) return "output image has no data";
  if (out.format < ISP_OUT_RGB8 || out.format > ISP_OUT_RGB32F) return "output format unknown";
  const size_t cb = out.format == ISP_OUT_RGB16 ? 2U : out.format == ISP_OUT_RGB32F ? 4U : 1U;
  const size_t row = static_cast<size_t>(raw.width) * (out.format == ISP_OUT_RGBA8 ? 4U : 3U) * cb;
  if (out.pitch < row || out.pitch % cb != 0U ||
      (cb > 1 && reinterpret_cast<std::uintptr_t>(out.data) % cb != 0U)) {
    return "output image pitch is shorter than a row or misaligned";
  }
  return {};
}

size_t tone_table(const isp_params_c& p, float* out) {
  // isp_params.cpp:166-182: the user's table verbatim, else 4097 points of
  // the curve evaluated in double and rounded to float.
  if (p.tone_curve == ISP_TONE_LUT) {
    for (size_t i = 0; i < p.lut_size; ++i) out[i] = p.lut[i];
    return p.lut_size;
  }
  for (int i = 0; i < ISP_TONE_LUT_SIZE; ++i) {
    const double x = static_cast<double>(i) / (ISP_TONE_LUT_SIZE - 1);
    double y = x;
    if (p.tone_curve == ISP_TONE_SRGB) {
      y = x <= 0.0031308 ? 12.92 * x : 1.055 * std::pow(x, 1.0 / 2.4) - 0.055;
    } else if (p.tone_curve == ISP_TONE_GAMMA) {
      y = std::pow(x, 1.0 / static_cast<double>(p.gamma));
    }
    out[i] = static_cast<float>(y < 0.0 ? 0.0 : y > 1.0 ? 1.0 : y);
  }
  return ISP_TONE_LUT_SIZE;
}

std::vector<float> tone_lut(const isp_params_c& p) {
  std::vector<float> lut(p.tone_curve == ISP_TONE_LUT ? p.lut_size : size_t{ISP_TONE_LUT_SIZE});
  tone_table(p, lut.data());
  return lut;
}

}  // namespace isp_b200
