// isp_batch.cu - instances of the batch passes: the statistics pass and the
// tile pass with tone tables in shared memory, 64-row tiles (isp_batch.cuh).
#include "isp_batch.cuh"

namespace isp_b200 {

const void* batch_kernel_shared_lut() { return reinterpret_cast<const void*>(&isp_batch_kernel<true, kTH>); }

const void* awb_batch_kernel() { return reinterpret_cast<const void*>(&isp_awb_batch_kernel); }

// Copies a batch's descriptors and work ranges from pinned host memory, read
// over PCIe by the SMs, to the device buffers the passes read: one 16-byte
// word per thread over two spans. The copy engines are left to the frames'
// own transfers: a descriptor copy queued on them would wait behind those.
__global__ void isp_batch_stage_kernel(const uint4* __restrict__ frames_src, uint4* __restrict__ frames_dst,
                                       int frame_words, const uint4* __restrict__ ranges_src,
                                       uint4* __restrict__ ranges_dst, int range_words) {
  const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  if (i < frame_words) {
    frames_dst[i] = frames_src[i];
  } else if (i - frame_words < range_words) {
    ranges_dst[i - frame_words] = ranges_src[i - frame_words];
  }
}

const void* batch_stage_kernel() { return reinterpret_cast<const void*>(&isp_batch_stage_kernel); }

size_t batch_kernel_smem(bool lut_smem, int tile_rows) {
  return static_cast<size_t>(layout_of(true, box_row_bytes(kRawU16), lut_smem ? kBatchLutEntries : 0, tile_rows).total) +
         128U;
}

}  // namespace isp_b200
