// isp_batch_short_global_lut.cu - the batch tile pass over 32-row tiles, tone
// tables read from global memory (isp_batch.cuh).
#include "isp_batch.cuh"

namespace isp_b200 {

const void* batch_kernel_global_lut_short() {
  return reinterpret_cast<const void*>(&isp_batch_kernel<false, kTHShort>);
}

}  // namespace isp_b200
