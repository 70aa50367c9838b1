// isp_main_malvar_sharpen_short.cu - instances of the fused tile kernel: Malvar-He-Cutler demosaic, sharpening on, 32-row tiles.
#include "isp_main.cuh"

namespace isp_b200 {

const void* main_kernel_ms_short(int layout, bool lut_smem, int out_format) {
  return main_instance<true, true, kTHShort>(layout, lut_smem, out_format);
}

}  // namespace isp_b200
