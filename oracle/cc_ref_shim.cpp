// cc_ref_shim.cpp - TEST INFRASTRUCTURE ONLY. A C ABI over the reference's
// own colour converter, compiled with its unmodified sources by
// oracle/Makefile:
//   _ref/libcc_ref.so       modules/color-convert/src/conversion.cpp and
//                           reference.cpp: reference_convert,
//                           compute_mapping, validate_conversion and
//                           draw_test_pattern on the CPU. Pins the C oracle
//                           (oracle/cc_oracle.c), generates tests/golden/,
//                           and is the CPU arm of the converter benchmark.
//   _ref/libcc_ref_cuda.so  the same plus converter.cpp, kernels.cu and
//                           vic_unavailable.cpp (built with -DCC_REF_CUDA):
//                           the reference's CUDA kernel for sm_100a, timed
//                           beside the B200 converter as the GPU bar.
// Images cross as cc_image_c (include/cc_b200.h); errors come back as
// ISP_EINVAL / ISP_ECUDA with the exception's message copied into `err`.

#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>

#include "cc_b200.h"
#include "holoscan/color_convert/conversion.hpp"
#include "holoscan/color_convert/reference.hpp"
#ifdef CC_REF_CUDA
#include "holoscan/color_convert/converter.hpp"
#endif

namespace cc = holoscan::color_convert;

namespace {

cc::ImageView view_of(const cc_image_c& c) {
  cc::ImageView v;
  v.format = static_cast<cc::PixelFormat>(c.format);
  v.width = c.width;
  v.height = c.height;
  for (int k = 0; k < 3; ++k) v.planes[k] = {c.planes[k].data, c.planes[k].pitch};
  v.location = c.location == CC_DEVICE ? cc::MemoryLocation::kDevice : cc::MemoryLocation::kHost;
  return v;
}

cc::ConversionParams params_of(const cc_params_c& p) {
  cc::ConversionParams r;
  r.matrix = static_cast<cc::ColorMatrix>(p.matrix);
  r.range = static_cast<cc::ColorRange>(p.range);
  r.mode = static_cast<cc::ResizeMode>(p.mode);
  if (p.has_crop) r.crop = cc::Rect{p.crop.x, p.crop.y, p.crop.width, p.crop.height};
  r.letterbox = p.letterbox != 0;
  r.fill_rgb = {p.fill_rgb[0], p.fill_rgb[1], p.fill_rgb[2]};
  return r;
}

template <class F>
int guarded(char* err, size_t errlen, F&& f) {
  try {
    f();
    return ISP_OK;
  } catch (const std::invalid_argument& e) {
    if (err != nullptr && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return ISP_EINVAL;
  } catch (const std::exception& e) {
    if (err != nullptr && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return ISP_ECUDA;
  }
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) int cc_ref_convert(const cc_image_c* src, const cc_image_c* dst,
                                                          const cc_params_c* params, char* err, size_t errlen) {
  return guarded(err, errlen, [&] { cc::reference_convert(view_of(*src), view_of(*dst), params_of(*params)); });
}

__attribute__((visibility("default"))) int cc_ref_mapping(int sw, int sh, int w, int h, int dst_format,
                                                          const cc_params_c* params, cc_mapping_c* out, char* err,
                                                          size_t errlen) {
  return guarded(err, errlen, [&] {
    const cc::Mapping m =
        cc::compute_mapping(sw, sh, w, h, static_cast<cc::PixelFormat>(dst_format), params_of(*params));
    out->source = {m.source.x, m.source.y, m.source.width, m.source.height};
    out->content = {m.content.x, m.content.y, m.content.width, m.content.height};
  });
}

__attribute__((visibility("default"))) int cc_ref_validate(const cc_image_c* src, const cc_image_c* dst,
                                                           const cc_params_c* params, char* err, size_t errlen) {
  return guarded(err, errlen, [&] { cc::validate_conversion(view_of(*src), view_of(*dst), params_of(*params)); });
}

__attribute__((visibility("default"))) int cc_ref_test_pattern(const cc_image_c* rgb8, uint32_t frame, char* err,
                                                               size_t errlen) {
  return guarded(err, errlen, [&] { cc::draw_test_pattern(view_of(*rgb8), frame); });
}

#ifdef CC_REF_CUDA
// Converter(Backend::kCuda)::convert on device images, queued on `stream`.
__attribute__((visibility("default"))) int cc_ref_cuda_convert(const cc_image_c* src, const cc_image_c* dst,
                                                               const cc_params_c* params, void* stream, char* err,
                                                               size_t errlen) {
  static cc::Converter* converter = new cc::Converter(cc::Backend::kCuda);
  return guarded(err, errlen, [&] {
    converter->convert(view_of(*src), view_of(*dst), params_of(*params), static_cast<cudaStream_t>(stream));
  });
}
#endif

}  // extern "C"
