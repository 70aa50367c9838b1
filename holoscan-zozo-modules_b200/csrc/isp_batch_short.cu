// isp_batch_short.cu - the batch tile pass over 32-row tiles, tone tables in
// shared memory (isp_batch.cuh).
#include "isp_batch.cuh"

namespace isp_b200 {

const void* batch_kernel_shared_lut_short() {
  return reinterpret_cast<const void*>(&isp_batch_kernel<true, kTHShort>);
}

}  // namespace isp_b200
