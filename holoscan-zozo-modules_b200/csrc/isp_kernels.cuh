// isp_kernels.cuh - host-side handles of the kernels in isp_kernels.cu.
#pragma once

#include <cstddef>

#include "isp_types.cuh"

namespace isp_b200 {

// Tone tables up to this many entries are copied into shared memory.
constexpr int kLutSmemEntries = 4097;

// The fused tile kernel for a demosaic method, sharpening on or off, and an
// output format; launch with kernel_threads() threads and
// main_kernel_smem() bytes of dynamic shared memory; arguments
// (FrameDesc, int tiles_x, int tiles).
const void* main_kernel(bool malvar, bool sharpen, int out_format);
size_t main_kernel_smem(bool sharpen, int tone_size);
int main_kernel_tiles(int width, int height, int* tiles_x);
int kernel_threads();

// The white balance statistics kernel; arguments (FrameDesc, const float* lsc).
const void* awb_kernel(bool white_patch);

}  // namespace isp_b200
