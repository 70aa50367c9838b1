// isp_kernels.cuh - host-side handles of the kernels in isp_kernels.cu.
#pragma once

#include <cstddef>

#include "isp_types.cuh"

namespace isp_b200 {

// The fused tile kernel for a demosaic method, sharpening on or off, an
// output format, a Bayer pattern and the tone table's place (shared or global); launch with kernel_threads() threads and
// main_kernel_smem() bytes of dynamic shared memory; arguments
// (const CUtensorMap raw_map, FrameDesc, int tiles_x, int tiles, int use_tma,
// int lut_in_smem). The raw map's box is main_box_row_bytes() bytes (or half
// as many uint16 samples) by main_box_rows() rows.
// Each comes in two tile heights, tile_rows 64 (two CTAs per SM) or 32
// (three CTAs per SM); tile_rows_valid() maps anything else to 0.
const void* main_kernel(bool malvar, bool sharpen, int pattern, bool lut_smem, int out_format, int tile_rows = 64);
size_t main_kernel_smem(bool sharpen, int raw_format, int lut_entries, int tile_rows = 64);
int main_box_rows(bool sharpen, int tile_rows = 64);
int main_box_row_bytes(int raw_format);
int main_kernel_tiles(int width, int height, int* tiles_x, int tile_rows = 64);
int tile_rows_valid(int tile_rows);
int kernel_threads();

// The white balance statistics kernel; arguments (const CUtensorMap raw_map,
// FrameDesc, int strips, int tiles_y, int band_tiles, int use_tma), one CTA
// per band of a strip (awb_kernel_bands); box awb_box_row_bytes() by 64 rows.
const void* awb_kernel(bool white_patch, int pattern);
size_t awb_kernel_smem();
int awb_box_row_bytes(int raw_format);
// Tiles of 64 x 64 samples over the complete quads (the batch statistics pass).
int awb_kernel_tiles(int width, int height, int* tiles_x);
// The single-frame statistics pass's strips and bands for about `ctas` CTAs;
// returns the CTA count (strips x bands).
int awb_kernel_bands(int width, int height, int ctas, int* strips, int* tiles_y, int* band_tiles);

// The bounded-wait check (arguments Scratch*, unsigned int polls; one CTA):
// a barrier nothing completes, waited for `polls` times, then the pipeline's
// error flag set as a pass that gave up sets it.
const void* wait_check_kernel();

// Tone tables up to this many entries may be copied into shared memory.
constexpr int kLutSmemEntries = 4097;
// In a batch, tone tables up to this many entries go to shared memory.
constexpr int kBatchLutEntries = 1024;

// The batch passes (isp_batch.cu): arguments (const BatchFrame* frames, int
// nframes, const int2* ranges), one range of work items per CTA. The tile
// pass's dynamic shared memory is batch_kernel_smem(); the statistics pass's
// is awb_kernel_smem().
const void* batch_kernel(bool lut_smem, int tile_rows = 64);
size_t batch_kernel_smem(bool lut_smem, int tile_rows = 64);
const void* awb_batch_kernel();
// Descriptor staging (isp_batch.cu): arguments (const uint4* frames_src,
// uint4* frames_dst, int frame_words, const uint4* ranges_src, uint4*
// ranges_dst, int range_words), one word per thread.
const void* batch_stage_kernel();
constexpr int kStageThreads = 256;

}  // namespace isp_b200
