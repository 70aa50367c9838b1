// isp_batch_global_lut.cu - the batch tile pass reading tone tables from
// global memory, for batches with a table over kBatchLutEntries entries;
// 64-row tiles.
#include "isp_batch.cuh"

namespace isp_b200 {

const void* batch_kernel_global_lut() { return reinterpret_cast<const void*>(&isp_batch_kernel<false, kTH>); }

}  // namespace isp_b200
