// isp_main_bilinear_short.cu - instances of the fused tile kernel: bilinear demosaic, sharpening off, 32-row tiles.
#include "isp_main.cuh"

namespace isp_b200 {

const void* main_kernel_bn_short(int layout, bool lut_smem, int out_format) {
  return main_instance<false, false, kTHShort>(layout, lut_smem, out_format);
}

}  // namespace isp_b200
