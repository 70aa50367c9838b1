// isp_main_malvar_short.cu - instances of the fused tile kernel: Malvar-He-Cutler demosaic, sharpening off, 32-row tiles.
#include "isp_main.cuh"

namespace isp_b200 {

const void* main_kernel_mn_short(int layout, bool lut_smem, int out_format) {
  return main_instance<true, false, kTHShort>(layout, lut_smem, out_format);
}

}  // namespace isp_b200
