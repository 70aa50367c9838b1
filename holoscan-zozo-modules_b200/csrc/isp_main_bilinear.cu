// isp_main_bilinear.cu - instances of the fused tile kernel: bilinear demosaic, sharpening off, 64-row tiles.
#include "isp_main.cuh"

namespace isp_b200 {

const void* main_kernel_bn(int layout, bool lut_smem, int out_format) {
  return main_instance<false, false, kTH>(layout, lut_smem, out_format);
}

}  // namespace isp_b200
