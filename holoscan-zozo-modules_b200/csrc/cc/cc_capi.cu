// cc_capi.cu - the colour converter's device entry points: a conversion and
// the synthetic camera pattern, both queued on the caller's stream. Nothing
// is allocated and nothing is kept between calls: the plan travels in the
// kernel's parameters.
#include <cuda_runtime.h>

#include <string>

#include "../isp_host.hpp"
#include "../isp_trace.hpp"
#include "cc_common.cuh"

extern "C" {

// Converter(Backend::kCuda)::convert
// (modules/color-convert/src/converter.cpp:84-111): both images on the
// device, checked, planned, one kernel launched.
ISP_B200_API int cc_b200_convert(const cc_image_c* source, const cc_image_c* destination, const cc_params_c* params,
                                 void* stream) {
  const isp_b200::TraceRange range("cc.convert", isp_b200::kTraceKernel);
  isp_b200::clear_error();
  if (source == nullptr || destination == nullptr || params == nullptr) {
    return isp_b200::fail(ISP_EINVAL, "null argument");
  }
  if (source->location != CC_DEVICE) return isp_b200::fail(ISP_EINVAL, "source image must be in CUDA device memory");
  if (destination->location != CC_DEVICE) {
    return isp_b200::fail(ISP_EINVAL, "destination image must be in CUDA device memory");
  }
  cc_b200::Plan plan;
  if (int s = cc_b200::make_plan(source, destination, params, &plan); s != ISP_OK) return s;
  const int e = cc_b200::launch_convert(plan, stream);
  if (e != 0) return isp_b200::fail_cuda(static_cast<cudaError_t>(e), "conversion kernel");
  return ISP_OK;
}

// launch_test_pattern (modules/color-convert/src/kernels.cu:70-83): a device
// RGB8 view with a packed row at least.
ISP_B200_API int cc_b200_test_pattern(const cc_image_c* rgb8, uint32_t frame, void* stream) {
  isp_b200::clear_error();
  if (rgb8 == nullptr || rgb8->format != CC_RGB8 || rgb8->location != CC_DEVICE || rgb8->width <= 0 ||
      rgb8->height <= 0 || rgb8->planes[0].data == nullptr ||
      rgb8->planes[0].pitch < static_cast<size_t>(rgb8->width) * 3U) {
    return isp_b200::fail(ISP_EINVAL, "the test pattern needs a device RGB8 image");
  }
  const int e = cc_b200::launch_pattern(rgb8->planes[0].data, rgb8->planes[0].pitch, rgb8->width, rgb8->height,
                                        frame, stream);
  if (e != 0) return isp_b200::fail_cuda(static_cast<cudaError_t>(e), "test pattern kernel");
  return ISP_OK;
}

}  // extern "C"
