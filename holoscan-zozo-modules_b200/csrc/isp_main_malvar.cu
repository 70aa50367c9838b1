// isp_main_malvar.cu - instances of the fused tile kernel: Malvar-He-Cutler demosaic, sharpening off.
#include "isp_main.cuh"

namespace isp_b200 {

const void* main_kernel_mn(int layout, bool lut_smem) {
  return main_instance<true, false>(layout, lut_smem);
}

}  // namespace isp_b200
