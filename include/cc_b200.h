/*
 * cc_b200.h - the C ABI of the B200 colour converter: the step after the ISP
 * in a camera graph. A device image in one pixel format (NV12, NV16, I420,
 * YUYV, UYVY, RGB8, BGR8, RGBA8, BGRA8, MONO8, MONO16, RGB16) becomes a
 * device image in another, optionally cropped, resized (nearest, bilinear,
 * area) and letterboxed, computed by sm_100a kernels byte for byte as the
 * holoscan::color_convert CPU reference computes it.
 *
 * Statuses and error messages are the ISP library's (isp_b200.h): 0 on
 * success, ISP_EINVAL for an unusable image or setting (the reference's
 * std::invalid_argument, with the same message), ISP_ECUDA for a CUDA
 * failure (its std::runtime_error); the calling thread's last message is in
 * isp_b200_last_error().
 *
 * Reference interfaces replaced (paths inside the holoscan-zozo-modules tree):
 *   modules/color-convert/include/holoscan/color_convert/pixel_format.hpp:15-146
 *       PixelFormat, ColorMatrix, ColorRange, format_info, plane_size,
 *       packed_size, the format/matrix/range names
 *   modules/color-convert/include/holoscan/color_convert/image_view.hpp:15-44
 *       PlaneView, ImageView, packed_view
 *   modules/color-convert/include/holoscan/color_convert/conversion.hpp:40-94
 *       ResizeMode, Rect, ConversionParams, Mapping, compute_mapping,
 *       validate_conversion
 *   modules/color-convert/include/holoscan/color_convert/converter.hpp:31-72
 *       launch_test_pattern, Converter(Backend::kCuda)::convert
 */
#ifndef CC_B200_H_
#define CC_B200_H_

#include <stddef.h>
#include <stdint.h>

#include "isp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* PixelFormat, ColorMatrix, ColorRange, ResizeMode with the reference's
 * numbering (pixel_format.hpp:17-30, :43, :47; conversion.hpp:40). */
enum {
  CC_NV12 = 0,
  CC_NV16 = 1,
  CC_I420 = 2,
  CC_YUYV = 3,
  CC_UYVY = 4,
  CC_RGB8 = 5,
  CC_BGR8 = 6,
  CC_RGBA8 = 7,
  CC_BGRA8 = 8,
  CC_MONO8 = 9,
  CC_MONO16 = 10,
  CC_RGB16 = 11
};
#define CC_FORMAT_COUNT 12
enum { CC_BT601 = 0, CC_BT709 = 1, CC_BT2020 = 2 };
enum { CC_RANGE_LIMITED = 0, CC_RANGE_FULL = 1 };
enum { CC_NEAREST = 0, CC_BILINEAR = 1, CC_AREA = 2 };
enum { CC_HOST = 0, CC_DEVICE = 1 }; /* MemoryLocation (image_view.hpp:15) */

/* PlaneView and ImageView (image_view.hpp:17-29): format_info(format).planes
 * planes are used; pitch is the bytes from one row to the next. */
typedef struct cc_plane_c {
  uint8_t* data;
  size_t pitch;
} cc_plane_c;

typedef struct cc_image_c {
  int32_t format;
  int32_t width;
  int32_t height;
  int32_t location; /* CC_HOST or CC_DEVICE */
  cc_plane_c planes[3];
} cc_image_c;

/* Rect (conversion.hpp:47-54): columns x .. x + width - 1, rows y .. y + height - 1. */
typedef struct cc_rect_c {
  int32_t x;
  int32_t y;
  int32_t width;
  int32_t height;
} cc_rect_c;

/* ConversionParams (conversion.hpp:56-67); the optional crop carries has_crop. */
typedef struct cc_params_c {
  int32_t matrix;
  int32_t range;
  int32_t mode;
  int32_t has_crop;
  cc_rect_c crop;
  int32_t letterbox;
  uint8_t fill_rgb[3];
} cc_params_c;

/* Mapping (conversion.hpp:71-74): where the source rectangle lands. */
typedef struct cc_mapping_c {
  cc_rect_c source;
  cc_rect_c content;
} cc_mapping_c;

/* FormatInfo (pixel_format.hpp:49-56); model 0 YCbCr, 1 RGB, 2 gray (:46). */
typedef struct cc_format_info_c {
  int32_t model;
  int32_t planes;
  int32_t chroma_shift_x;
  int32_t chroma_shift_y;
  int32_t bytes_per_sample;
  int32_t channels;
} cc_format_info_c;

/* ConversionParams' defaults: BT.601, limited range, bilinear, no crop, no
 * letterbox, black fill. */
ISP_B200_API void cc_b200_params_default(cc_params_c* params);

/* format_info (pixel_format.hpp:58-84). ISP_EINVAL for an unknown format. */
ISP_B200_API int cc_b200_format_info(int32_t format, cc_format_info_c* info);

/* plane_size and packed_size (pixel_format.hpp:112-138); 0 for an unknown
 * format or plane. */
ISP_B200_API int cc_b200_plane_size(int32_t format, int32_t width, int32_t height, int32_t plane,
                                    size_t* row_bytes, int32_t* rows);
ISP_B200_API size_t cc_b200_packed_size(int32_t format, int32_t width, int32_t height);

/* packed_view (image_view.hpp:33-44): a view of a packed image at base. */
ISP_B200_API int cc_b200_packed_view(void* base, int32_t format, int32_t width, int32_t height,
                                     int32_t location, cc_image_c* view);

/* format_name / parse_format, matrix_name / parse_matrix, range_name /
 * parse_range, resize_mode_name / parse_resize_mode (pixel_format.hpp:140-146,
 * conversion.hpp:42-44). Names are static strings ("unknown" for a bad
 * value); parse returns the value or -1. */
ISP_B200_API const char* cc_b200_format_name(int32_t format);
ISP_B200_API int32_t cc_b200_parse_format(const char* name);
ISP_B200_API const char* cc_b200_matrix_name(int32_t matrix);
ISP_B200_API int32_t cc_b200_parse_matrix(const char* name);
ISP_B200_API const char* cc_b200_range_name(int32_t range);
ISP_B200_API int32_t cc_b200_parse_range(const char* name);
ISP_B200_API const char* cc_b200_resize_mode_name(int32_t mode);
ISP_B200_API int32_t cc_b200_parse_resize_mode(const char* name);

/* compute_mapping (conversion.hpp:76-89). ISP_EINVAL with the reference's
 * message for sizes that are not positive or a crop outside the source. */
ISP_B200_API int cc_b200_compute_mapping(int32_t source_width, int32_t source_height, int32_t width,
                                         int32_t height, int32_t destination_format,
                                         const cc_params_c* params, cc_mapping_c* mapping);

/* validate_conversion (conversion.hpp:91-95): ISP_EINVAL naming the first
 * problem, with the reference's message. */
ISP_B200_API int cc_b200_validate(const cc_image_c* source, const cc_image_c* destination,
                                  const cc_params_c* params);

/* Converter(Backend::kCuda)::convert (converter.hpp:61-71): converts source
 * into destination, both in device memory, queued on stream (a
 * cudaStream_t; NULL for the legacy default stream) after its earlier work.
 * Allocates nothing and keeps no state between calls. ISP_EINVAL for host
 * images ("source image must be in CUDA device memory") and whatever
 * validate rejects; ISP_ECUDA if the launch fails. */
ISP_B200_API int cc_b200_convert(const cc_image_c* source, const cc_image_c* destination,
                                 const cc_params_c* params, void* stream);

/* launch_test_pattern (converter.hpp:31-34): fills a device RGB8 view with
 * the synthetic camera's frame `frame` (moving colour bars over two ramps,
 * reference.hpp:40-55). ISP_EINVAL for any other view. */
ISP_B200_API int cc_b200_test_pattern(const cc_image_c* rgb8, uint32_t frame, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CC_B200_H_ */
