// cc_plan.cpp - the colour converter's host side: format tables and names,
// the letterbox geometry, the checks of a conversion (with the reference's
// messages) and its plan. The plan's colour maps are composed in double
// precision and rounded to single once, as the reference does
// (modules/color-convert/src/conversion.cpp:93-209, :362-447), so that the
// kernels' coefficients are the same floats.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../isp_host.hpp"
#include "cc_common.cuh"

namespace cc_b200 {
namespace {

const char* const kFormatNames[CC_FORMAT_COUNT] = {"nv12",  "nv16",  "i420",  "yuyv",  "uyvy",   "rgb8",
                                                   "bgr8",  "rgba8", "bgra8", "mono8", "mono16", "rgb16"};
const char* const kMatrixNames[3] = {"bt601", "bt709", "bt2020"};
const char* const kRangeNames[2] = {"limited", "full"};
const char* const kModeNames[3] = {"nearest", "bilinear", "area"};

template <int N>
const char* name_in(const char* const (&names)[N], int v) {
  return v >= 0 && v < N ? names[v] : "unknown";
}

template <int N>
int parse_in(const char* const (&names)[N], const char* text) {
  if (text == nullptr) return -1;
  for (int i = 0; i < N; ++i) {
    if (std::strcmp(names[i], text) == 0) return i;
  }
  return -1;
}

// A 3x4 affine map on colour samples: rows out, columns in plus offset.
struct Affine34 {
  double m[3][4];
};

Affine34 unit_map() { return {{{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}}}; }

// outer after inner; each entry summed from the offset (or 0), then over k in order.
Affine34 chain(const Affine34& outer, const Affine34& inner) {
  Affine34 r{};
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 4; ++j) {
      double acc = j == 3 ? outer.m[i][3] : 0.0;
      for (int k = 0; k < 3; ++k) acc += outer.m[i][k] * inner.m[k][j];
      r.m[i][j] = acc;
    }
  }
  return r;
}

// Luma weights (kr, kb) of BT.601, BT.709 and BT.2020.
void weights_of(int matrix, double* kr, double* kb) {
  if (matrix == CC_BT709) {
    *kr = 0.2126;
    *kb = 0.0722;
  } else if (matrix == CC_BT2020) {
    *kr = 0.2627;
    *kb = 0.0593;
  } else {
    *kr = 0.299;
    *kb = 0.114;
  }
}

// Code scales: Y codes per unit luma, its offset, chroma codes per unit.
void levels_of(int range, double* ys, double* yo, double* cs) {
  if (range == CC_RANGE_LIMITED) {
    *ys = 219.0;
    *yo = 16.0;
    *cs = 224.0;
  } else {
    *ys = 255.0;
    *yo = 0.0;
    *cs = 255.0;
  }
}

// Samples of `model` to R, G, B on 0..255.
Affine34 into_rgb(int model, int matrix, int range) {
  if (model == kRgb) return unit_map();
  if (model == kGray) return {{{1, 0, 0, 0}, {1, 0, 0, 0}, {1, 0, 0, 0}}};
  double kr, kb, ys, yo, cs;
  weights_of(matrix, &kr, &kb);
  levels_of(range, &ys, &yo, &cs);
  const double kg = 1.0 - kr - kb;
  // y = (Y - yo) / ys, cb = (Cb - 128) / cs, cr likewise; R = y + 2 (1 - kr) cr,
  // B = y + 2 (1 - kb) cb, G = (y - kr R - kb B) / kg.
  const double inv_y = 1.0 / ys;
  const double inv_c = 1.0 / cs;
  const double r_cr = 2.0 * (1.0 - kr);
  const double b_cb = 2.0 * (1.0 - kb);
  const double g_cb = -kb * b_cb / kg;
  const double g_cr = -kr * r_cr / kg;
  const double y_shift = -yo * inv_y;
  Affine34 a{};
  a.m[0][0] = inv_y;
  a.m[0][1] = 0.0;
  a.m[0][2] = r_cr * inv_c;
  a.m[0][3] = y_shift - r_cr * inv_c * 128.0;
  a.m[1][0] = inv_y;
  a.m[1][1] = g_cb * inv_c;
  a.m[1][2] = g_cr * inv_c;
  a.m[1][3] = y_shift - (g_cb + g_cr) * inv_c * 128.0;
  a.m[2][0] = inv_y;
  a.m[2][1] = b_cb * inv_c;
  a.m[2][2] = 0.0;
  a.m[2][3] = y_shift - b_cb * inv_c * 128.0;
  for (auto& row : a.m) {
    for (double& v : row) v *= 255.0;
  }
  return a;
}

// R, G, B on 0..255 to the samples of `model`.
Affine34 out_of_rgb(int model, int matrix, int range) {
  if (model == kRgb) return unit_map();
  double kr, kb;
  weights_of(matrix, &kr, &kb);
  const double kg = 1.0 - kr - kb;
  if (model == kGray) return {{{kr, kg, kb, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}}};
  double ys, yo, cs;
  levels_of(range, &ys, &yo, &cs);
  // y = kr r + kg g + kb b; cb = (b - y) / (2 (1 - kb)); cr = (r - y) / (2 (1 - kr)).
  const double den_b = 2.0 * (1.0 - kb);
  const double den_r = 2.0 * (1.0 - kr);
  const double sy = ys / 255.0;
  const double sc = cs / 255.0;
  return {{
      {kr * sy, kg * sy, kb * sy, yo},
      {-kr / den_b * sc, -kg / den_b * sc, (1.0 - kb) / den_b * sc, 128.0},
      {(1.0 - kr) / den_r * sc, -kg / den_r * sc, -kb / den_r * sc, 128.0},
  }};
}

// One letterboxed axis: the content's size and offset for a scaled extent.
void fit(double scaled, int size, bool even, int* content, int* offset) {
  int c = std::clamp(static_cast<int>(std::lround(scaled)), 1, size);
  if (c == size) {
    *content = size;
    *offset = 0;
    return;
  }
  if (even) c = std::max(2, c & ~1);
  int o = (size - c) / 2;
  if (even) o &= ~1;
  *content = c;
  *offset = o;
}

int check_image(const cc_image_c* v, const char* which) {
  const std::string name(which);
  if (v->width <= 0 || v->height <= 0) return isp_b200::fail(ISP_EINVAL, name + " image size must be positive");
  if ((v->format == CC_YUYV || v->format == CC_UYVY) && v->width % 2 != 0) {
    return isp_b200::fail(ISP_EINVAL, name + " image: " + kFormatNames[v->format] + " needs an even width, not " +
                                          std::to_string(v->width));
  }
  const int planes = info_of(v->format).planes;
  for (int k = 0; k < planes; ++k) {
    size_t row_bytes = 0;
    int32_t rows = 0;
    cc_b200_plane_size(v->format, v->width, v->height, k, &row_bytes, &rows);
    if (v->planes[k].data == nullptr) {
      return isp_b200::fail(ISP_EINVAL, name + " image plane " + std::to_string(k) + " has no data");
    }
    if (v->planes[k].pitch < row_bytes) {
      return isp_b200::fail(ISP_EINVAL, name + " image plane " + std::to_string(k) + " pitch " +
                                            std::to_string(v->planes[k].pitch) + " is shorter than a row of " +
                                            std::to_string(row_bytes) + " bytes");
    }
  }
  return ISP_OK;
}

}  // namespace

bool known_format(int f) { return f >= 0 && f < CC_FORMAT_COUNT; }

int compute_mapping(int sw, int sh, int w, int h, int dst_format, const cc_params_c* params, cc_mapping_c* out) {
  if (sw <= 0 || sh <= 0 || w <= 0 || h <= 0) return isp_b200::fail(ISP_EINVAL, "image sizes must be positive");
  cc_rect_c source{0, 0, sw, sh};
  if (params->has_crop) {
    const cc_rect_c& c = params->crop;
    if (c.width <= 0 || c.height <= 0 || c.x < 0 || c.y < 0 || c.x > sw - c.width || c.y > sh - c.height) {
      return isp_b200::fail(ISP_EINVAL, "crop " + std::to_string(c.width) + "x" + std::to_string(c.height) + "+" +
                                            std::to_string(c.x) + "+" + std::to_string(c.y) +
                                            " is not inside the " + std::to_string(sw) + "x" + std::to_string(sh) +
                                            " source");
    }
    source = c;
  }
  cc_rect_c content{0, 0, w, h};
  if (params->letterbox) {
    const double scale = std::min(static_cast<double>(w) / source.width, static_cast<double>(h) / source.height);
    const FormatInfo fi = info_of(dst_format);
    fit(source.width * scale, w, fi.shift_x != 0, &content.width, &content.x);
    fit(source.height * scale, h, fi.shift_y != 0, &content.height, &content.y);
  }
  out->source = source;
  out->content = content;
  return ISP_OK;
}

int validate(const cc_image_c* src, const cc_image_c* dst, const cc_params_c* params) {
  if (src == nullptr || dst == nullptr || params == nullptr) return isp_b200::fail(ISP_EINVAL, "null argument");
  if (!known_format(src->format)) return isp_b200::fail(ISP_EINVAL, "source image has an unknown pixel format");
  if (!known_format(dst->format)) return isp_b200::fail(ISP_EINVAL, "destination image has an unknown pixel format");
  if (params->matrix < 0 || params->matrix > CC_BT2020 || params->range < 0 || params->range > CC_RANGE_FULL ||
      params->mode < 0 || params->mode > CC_AREA) {
    return isp_b200::fail(ISP_EINVAL, "unknown colour matrix, range or resize mode");
  }
  if (int s = check_image(src, "source"); s != ISP_OK) return s;
  if (int s = check_image(dst, "destination"); s != ISP_OK) return s;
  cc_mapping_c m;
  return compute_mapping(src->width, src->height, dst->width, dst->height, dst->format, params, &m);
}

int make_plan(const cc_image_c* src, const cc_image_c* dst, const cc_params_c* params, Plan* plan) {
  if (int s = validate(src, dst, params); s != ISP_OK) return s;
  cc_mapping_c map;
  compute_mapping(src->width, src->height, dst->width, dst->height, dst->format, params, &map);
  Plan p{};
  const cc_image_c* views[2] = {src, dst};
  Image* images[2] = {&p.src, &p.dst};
  for (int i = 0; i < 2; ++i) {
    images[i]->format = views[i]->format;
    images[i]->width = views[i]->width;
    images[i]->height = views[i]->height;
    for (int k = 0; k < 3; ++k) {
      images[i]->data[k] = views[i]->planes[k].data;
      images[i]->pitch[k] = views[i]->planes[k].pitch;
    }
  }
  p.mode = params->mode;
  p.sx0 = map.source.x;
  p.sy0 = map.source.y;
  p.sx1 = map.source.x + map.source.width - 1;
  p.sy1 = map.source.y + map.source.height - 1;
  p.scale_x = static_cast<float>(static_cast<double>(map.source.width) / static_cast<double>(map.content.width));
  p.scale_y = static_cast<float>(static_cast<double>(map.source.height) / static_cast<double>(map.content.height));
  p.cx0 = map.content.x;
  p.cy0 = map.content.y;
  p.cx1 = map.content.x + map.content.width;
  p.cy1 = map.content.y + map.content.height;

  const int from = info_of(src->format).model;
  const int to = info_of(dst->format).model;
  p.identity = from == to ? 1 : 0;
  const Affine34 out = out_of_rgb(to, params->matrix, params->range);
  const Affine34 both = chain(out, into_rgb(from, params->matrix, params->range));
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) p.m[i * 3 + j] = static_cast<float>(both.m[i][j]);
    p.o[i] = static_cast<float>(both.m[i][3]);
  }
  for (int i = 0; i < 3; ++i) {
    double v = out.m[i][3];
    for (int k = 0; k < 3; ++k) v += out.m[i][k] * params->fill_rgb[k];
    p.fill[i] = static_cast<float>(v);
  }
  p.fill[3] = 255.0F;
  const FormatInfo fi = info_of(dst->format);
  p.bsx = fi.model == kYuv ? fi.shift_x : 0;
  p.bsy = fi.model == kYuv ? fi.shift_y : 0;
  *plan = p;
  return ISP_OK;
}

}  // namespace cc_b200

extern "C" {

ISP_B200_API void cc_b200_params_default(cc_params_c* params) {
  if (params == nullptr) return;
  std::memset(params, 0, sizeof(*params));
  params->matrix = CC_BT601;
  params->range = CC_RANGE_LIMITED;
  params->mode = CC_BILINEAR;
}

ISP_B200_API int cc_b200_format_info(int32_t format, cc_format_info_c* info) {
  if (!cc_b200::known_format(format) || info == nullptr) return isp_b200::fail(ISP_EINVAL, "unknown pixel format");
  const cc_b200::FormatInfo f = cc_b200::info_of(format);
  *info = {f.model, f.planes, f.shift_x, f.shift_y, f.bytes, f.channels};
  return ISP_OK;
}

ISP_B200_API int cc_b200_plane_size(int32_t format, int32_t width, int32_t height, int32_t plane, size_t* row_bytes,
                                    int32_t* rows) {
  if (!cc_b200::known_format(format) || row_bytes == nullptr || rows == nullptr) {
    return isp_b200::fail(ISP_EINVAL, "unknown pixel format");
  }
  const cc_b200::FormatInfo f = cc_b200::info_of(format);
  if (plane < 0 || plane >= f.planes) return isp_b200::fail(ISP_EINVAL, "no such plane");
  const size_t w = static_cast<size_t>(width < 0 ? 0 : width);
  if (plane == 0) {
    *row_bytes = w * static_cast<size_t>(f.channels * f.bytes);
    *rows = height;
    return ISP_OK;
  }
  // Subsampled extents round up: an odd last column or row keeps its own sample.
  const size_t chroma_w = (w + ((1U << f.shift_x) - 1U)) >> f.shift_x;
  *rows = (height + (1 << f.shift_y) - 1) >> f.shift_y;
  *row_bytes = chroma_w * (f.planes == 2 ? 2U : 1U);
  return ISP_OK;
}

ISP_B200_API size_t cc_b200_packed_size(int32_t format, int32_t width, int32_t height) {
  if (!cc_b200::known_format(format)) return 0;
  size_t total = 0;
  for (int k = 0; k < cc_b200::info_of(format).planes; ++k) {
    size_t row_bytes = 0;
    int32_t rows = 0;
    cc_b200_plane_size(format, width, height, k, &row_bytes, &rows);
    total += row_bytes * static_cast<size_t>(rows < 0 ? 0 : rows);
  }
  return total;
}

ISP_B200_API int cc_b200_packed_view(void* base, int32_t format, int32_t width, int32_t height, int32_t location,
                                     cc_image_c* view) {
  if (!cc_b200::known_format(format) || view == nullptr) return isp_b200::fail(ISP_EINVAL, "unknown pixel format");
  std::memset(view, 0, sizeof(*view));
  view->format = format;
  view->width = width;
  view->height = height;
  view->location = location;
  uint8_t* next = static_cast<uint8_t*>(base);
  for (int k = 0; k < cc_b200::info_of(format).planes; ++k) {
    size_t row_bytes = 0;
    int32_t rows = 0;
    cc_b200_plane_size(format, width, height, k, &row_bytes, &rows);
    view->planes[k] = {next, row_bytes};
    next += row_bytes * static_cast<size_t>(rows < 0 ? 0 : rows);
  }
  return ISP_OK;
}

ISP_B200_API const char* cc_b200_format_name(int32_t format) { return cc_b200::name_in(cc_b200::kFormatNames, format); }
ISP_B200_API int32_t cc_b200_parse_format(const char* name) { return cc_b200::parse_in(cc_b200::kFormatNames, name); }
ISP_B200_API const char* cc_b200_matrix_name(int32_t matrix) { return cc_b200::name_in(cc_b200::kMatrixNames, matrix); }
ISP_B200_API int32_t cc_b200_parse_matrix(const char* name) { return cc_b200::parse_in(cc_b200::kMatrixNames, name); }
ISP_B200_API const char* cc_b200_range_name(int32_t range) { return cc_b200::name_in(cc_b200::kRangeNames, range); }
ISP_B200_API int32_t cc_b200_parse_range(const char* name) { return cc_b200::parse_in(cc_b200::kRangeNames, name); }
ISP_B200_API const char* cc_b200_resize_mode_name(int32_t mode) { return cc_b200::name_in(cc_b200::kModeNames, mode); }
ISP_B200_API int32_t cc_b200_parse_resize_mode(const char* name) { return cc_b200::parse_in(cc_b200::kModeNames, name); }

ISP_B200_API int cc_b200_compute_mapping(int32_t source_width, int32_t source_height, int32_t width, int32_t height,
                                         int32_t destination_format, const cc_params_c* params,
                                         cc_mapping_c* mapping) {
  if (params == nullptr || mapping == nullptr) return isp_b200::fail(ISP_EINVAL, "null argument");
  if (!cc_b200::known_format(destination_format)) return isp_b200::fail(ISP_EINVAL, "unknown pixel format");
  return cc_b200::compute_mapping(source_width, source_height, width, height, destination_format, params, mapping);
}

ISP_B200_API int cc_b200_validate(const cc_image_c* source, const cc_image_c* destination, const cc_params_c* params) {
  return cc_b200::validate(source, destination, params);
}

}  // extern "C"
