// isp_kernels.cu - host-side dispatch and launch geometry of the B200 ISP's
// kernels (isp_main_*.cu, isp_awb.cu).
#include <algorithm>

#include "isp_common.cuh"

namespace isp_b200 {

namespace {

// The bounded wait of the tile and statistics passes, made to run out: one
// thread announces bytes on a barrier that no copy will ever complete, every
// thread waits `polls` times, gives up, and the pipeline's error flag is set
// as a real pass sets it. No copy is issued, so nothing is in flight when
// the kernel returns.
__global__ void isp_wait_check_kernel(Scratch* scratch, unsigned int polls) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&bar)), "r"(16U) : "memory");
  }
  __syncthreads();
  if (!mbar_wait(&bar, 0, polls) && threadIdx.x == 0) {
#ifdef ISP_CHECKED
    report_wait_timeout(make_span(scratch, 1, &scratch->check));
#else
    report_wait_timeout(scratch);
#endif
  }
}

}  // namespace

const void* wait_check_kernel() { return reinterpret_cast<const void*>(&isp_wait_check_kernel); }

const void* main_kernel_bn(int layout, bool lut_smem, int out_format);
const void* main_kernel_bs(int layout, bool lut_smem, int out_format);
const void* main_kernel_mn(int layout, bool lut_smem, int out_format);
const void* main_kernel_ms(int layout, bool lut_smem, int out_format);
const void* main_kernel_bn_short(int layout, bool lut_smem, int out_format);
const void* main_kernel_bs_short(int layout, bool lut_smem, int out_format);
const void* main_kernel_mn_short(int layout, bool lut_smem, int out_format);
const void* main_kernel_ms_short(int layout, bool lut_smem, int out_format);
const void* batch_kernel_shared_lut();
const void* batch_kernel_global_lut();
const void* batch_kernel_shared_lut_short();
const void* batch_kernel_global_lut_short();

int tile_rows_valid(int tile_rows) { return tile_rows == kTH ? kTH : tile_rows == kTHShort ? kTHShort : 0; }

const void* batch_kernel(bool lut_smem, int tile_rows) {
  if (tile_rows == kTHShort) return lut_smem ? batch_kernel_shared_lut_short() : batch_kernel_global_lut_short();
  return lut_smem ? batch_kernel_shared_lut() : batch_kernel_global_lut();
}

const void* main_kernel(bool malvar, bool sharpen, int pattern, bool lut_smem, int out_format, int tile_rows) {
  // RGGB and BGGR share a layout (red/blue on the quad's diagonal), as do
  // GRBG and GBRG; the kernel swaps red and blue for BGGR and GBRG.
  const int layout = pattern >> 1;
  if (tile_rows == kTHShort) {
    if (malvar) {
      return sharpen ? main_kernel_ms_short(layout, lut_smem, out_format)
                     : main_kernel_mn_short(layout, lut_smem, out_format);
    }
    return sharpen ? main_kernel_bs_short(layout, lut_smem, out_format)
                   : main_kernel_bn_short(layout, lut_smem, out_format);
  }
  if (malvar) {
    return sharpen ? main_kernel_ms(layout, lut_smem, out_format) : main_kernel_mn(layout, lut_smem, out_format);
  }
  return sharpen ? main_kernel_bs(layout, lut_smem, out_format) : main_kernel_bn(layout, lut_smem, out_format);
}

size_t main_kernel_smem(bool sharpen, int raw_format, int lut_entries, int tile_rows) {
  return static_cast<size_t>(layout_of(sharpen, box_row_bytes(raw_format), lut_entries, tile_rows).total) + 128U;
}

int main_box_rows(bool sharpen, int tile_rows) { return sharpen ? tile_rows + 8 : tile_rows + 4; }
int main_box_row_bytes(int raw_format) { return box_row_bytes(raw_format); }

int main_kernel_tiles(int width, int height, int* tiles_x, int tile_rows) {
  *tiles_x = (width + kTW - 1) / kTW;
  return *tiles_x * ((height + tile_rows - 1) / tile_rows);
}

int kernel_threads() { return kThreads; }

size_t awb_kernel_smem() {
  // two boxes of 64 x 128, lens shading table, column maps (64) and row maps
  // (a band's rows), white-patch histogram, the frame's lens shading grid.
  return 2U * 64U * 128U + kLscTableRows * 2U * kSW * 4U + 3U * 64U * 4U + 3U * kAwbBandRows * 4U +
         3U * kAwbBins * 4U + kGridSmemGains * 4U + 128U;
}

int awb_kernel_bands(int width, int height, int ctas, int* strips, int* tiles_y, int* band_tiles) {
  // Strips of 64 columns over the complete quads, cut into bands of whole
  // 64-row tiles: as many bands as let every strip's bands fill `ctas`, each
  // band at most kAwbBandRows rows, no band empty.
  const int qw = (width / 2) * 2;
  const int qh = (height / 2) * 2;
  *strips = std::max(1, (qw + 63) / 64);
  *tiles_y = std::max(1, (qh + 63) / 64);
  int bands = std::max(1, std::min(*tiles_y, ctas / *strips));
  *band_tiles = std::min((*tiles_y + bands - 1) / bands, kAwbBandRows / 64);
  bands = (*tiles_y + *band_tiles - 1) / *band_tiles;
  return *strips * bands;
}

int awb_box_row_bytes(int raw_format) {
  return raw_format == kRawU8 ? 64 : raw_format == kRawU16 ? 128 : raw_format == kRawRaw10 ? 80 : 96;
}

int awb_kernel_tiles(int width, int height, int* tiles_x) {
  // Tiles of 64 x 64 samples over the complete quads.
  const int qw = (width / 2) * 2;
  const int qh = (height / 2) * 2;
  *tiles_x = (qw + 63) / 64;
  return *tiles_x * ((qh + 63) / 64);
}

}  // namespace isp_b200
