// isp_batch.cu - instances of the batch passes: the statistics pass and the
// tile pass with tone tables in shared memory (isp_batch.cuh).
#include "isp_batch.cuh"

namespace isp_b200 {

const void* batch_kernel_shared_lut() { return reinterpret_cast<const void*>(&isp_batch_kernel<true>); }

const void* awb_batch_kernel() { return reinterpret_cast<const void*>(&isp_awb_batch_kernel); }

size_t batch_kernel_smem(bool lut_smem) {
  return static_cast<size_t>(layout_of(true, box_row_bytes(kRawU16), lut_smem ? kBatchLutEntries : 0).total) + 128U;
}

}  // namespace isp_b200
