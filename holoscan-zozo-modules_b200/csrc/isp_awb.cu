// isp_awb.cu - the white balance statistics kernel of the B200 ISP
// (gray world and white patch): each CTA takes one band of a 64-column strip,
// whose tiles of 64x64 samples arrive by TMA; the complete 2x2 quads without
// a saturated sample are summed per colour (and binned for white patch) in
// the block, then flushed once; the last CTA to finish forms the frame's
// estimate (finish_white_balance, isp_math.hpp:357-384) and clears the sums
// for the next frame.
#include "isp_awb.cuh"

namespace isp_b200 {
namespace {


// ---- White balance statistics ----------------------------------------------

// A band's lens shading maps and table: build_lsc's columns, rows, grid-row
// range and table (the same arithmetic: top + (bottom - top) * ty from
// T[k] = g + (g' - g) * tx, isp_math.hpp:121-140), for 64 columns and up to
// kAwbBandRows rows, the rows looped over the block's threads.
__device__ LscTile build_band_lsc(const FrameDesc& p, Span<const float> grid, int pattern, int x_first, int y_first,
                                  int nrows, Span<int> col_mx, Span<int> col_ix, Span<float> col_tx, Span<int> row_my, Span<int> row_k,
                                  Span<float> row_ty, Span<float> table, int* minmax) {
  constexpr int kCols = 64;
  const int t = threadIdx.x;
  if (t == 0) {
    minmax[0] = 0x7FFFFFFF;
    minmax[1] = -1;
  }
  __syncthreads();
  if (t < kCols) {
    const int x = x_first + t;
    col_mx[t] = x;
    if (p.lsc != nullptr) {
      const float fx = static_cast<float>(x) * p.lsc_sx;
      int ix = static_cast<int>(fx);
      ix = ix > p.lsc_width - 2 ? p.lsc_width - 2 : ix;
      col_ix[t] = ix;
      col_tx[t] = fx - static_cast<float>(ix);
    }
  }
  int iy_lo = 0x7FFFFFFF;
  int iy_hi = -1;
  for (int j = t; j < nrows; j += kThreads) {
    const int y = y_first + j;
    row_my[j] = y;
    if (p.lsc != nullptr) {
      const float fy = static_cast<float>(y) * p.lsc_sy;
      int iy = static_cast<int>(fy);
      iy = iy > p.lsc_height - 2 ? p.lsc_height - 2 : iy;
      row_k[j] = iy;
      row_ty[j] = fy - static_cast<float>(iy);
      iy_lo = iy < iy_lo ? iy : iy_lo;
      iy_hi = iy > iy_hi ? iy : iy_hi;
    }
  }
  if (p.lsc != nullptr) {
    iy_lo = __reduce_min_sync(0xFFFFFFFFU, iy_lo);
    iy_hi = __reduce_max_sync(0xFFFFFFFFU, iy_hi);
    if ((t & 31) == 0 && iy_hi >= 0) {
      atomicMin(&minmax[0], iy_lo);
      atomicMax(&minmax[1], iy_hi);
    }
  }
  __syncthreads();
  LscTile lt{0, 0};
  if (p.lsc == nullptr) return lt;
  lt.iy0 = minmax[0];
  lt.rows = minmax[1] - minmax[0] + 2;
  if (lt.rows > kLscTableRows) return lt;
  const int step = p.lsc_channels;
  const int planes = step == 4 ? 2 : 1;
  for (int e = t; e < lt.rows * planes * kCols; e += kThreads) {
    const int i = e % kCols;
    const int kp = e / kCols;
    const int par = kp % planes;
    const int k = kp / planes;
    const int ch = step == 4 ? cfa_of(pattern, (par << 1) | (col_mx[i] & 1)) : 0;
    Span<const float> g = grid + ((lt.iy0 + k) * p.lsc_width + col_ix[i]) * step + ch;
    table[(k * 2 + par) * kSW + i] = g[0] + (g[step] - g[0]) * col_tx[i];
  }
  for (int j = t; j < nrows; j += kThreads) row_k[j] -= lt.iy0;
  __syncthreads();
  return lt;
}

// One CTA per band of a strip: columns [64 s, 64 s + 64) of the complete
// quads, tiles [b band_tiles, (b + 1) band_tiles) of 64 rows. The band's lens
// shading maps and table are built once; its tiles then stream through a
// double-buffered TMA box with one block barrier each (buffer reuse).
template <bool kWhitePatch, int kPat>
__global__ void __launch_bounds__(kThreads, 3) isp_awb_kernel(const __grid_constant__ CUtensorMap map, FrameDesc p,
                                                         int strips, int tiles_y, int band_tiles, int use_tma) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128U - (smem_u32(smem_raw) & 127U)) & 127U);
  constexpr int kBoxRows = 64;
  constexpr int kTableAt = 2 * 64 * 128;                          // boxes: [2][64][128], a double buffer
  constexpr int kColsAt = kTableAt + kLscTableRows * 2 * kSW * 4;  // table: [kLscTableRows][2][kSW]
  constexpr int kRowsAt = kColsAt + 3 * 64 * 4;                    // col_mx, col_ix, col_tx: [64] each
  constexpr int kHistAt = kRowsAt + 3 * kAwbBandRows * 4;          // row_my, row_k, row_ty: [kAwbBandRows] each
  constexpr int kGridAt = kHistAt + 3 * kAwbBins * 4;              // hist: [3][1024]; grid_s: [kGridSmemGains]
  CheckRecord* rec = span_rec(p.scratch);
  Span<uint8_t> boxes = carve_span<uint8_t>(smem, 0, kTableAt, rec);
  Span<float> table = carve_span<float>(smem, kTableAt, kColsAt - kTableAt, rec);
  Span<int> col_mx = carve_span<int>(smem, kColsAt, 64 * 4, rec);
  Span<int> col_ix = carve_span<int>(smem, kColsAt + 64 * 4, 64 * 4, rec);
  Span<float> col_tx = carve_span<float>(smem, kColsAt + 128 * 4, 64 * 4, rec);
  Span<int> row_my = carve_span<int>(smem, kRowsAt, kAwbBandRows * 4, rec);
  Span<int> row_k = carve_span<int>(smem, kRowsAt + kAwbBandRows * 4, kAwbBandRows * 4, rec);
  Span<float> row_ty = carve_span<float>(smem, kRowsAt + 2 * kAwbBandRows * 4, kAwbBandRows * 4, rec);
  Span<unsigned int> hist = carve_span<unsigned int>(smem, kHistAt, kGridAt - kHistAt, rec);
  Span<float> grid_s = carve_span<float>(smem, kGridAt, kGridSmemGains * 4, rec);
  __shared__ uint64_t bars[2];
  __shared__ u64 red[kWarps];
  __shared__ int minmax[2];
  __shared__ int first;
  __shared__ bool last;
  Span<Scratch> s = p.scratch;
  const int tid = threadIdx.x;
  const int box_bytes = awb_box_bytes(p.raw_format);
  // The tile pass that follows may launch now: it waits (griddepcontrol.wait)
  // for this grid's completion before it does anything, but its CTAs become
  // resident on the SMs this pass leaves while the last bands are summed.
  griddep_launch_dependents();
  if constexpr (kWhitePatch) {
    for (int i = tid; i < 3 * kAwbBins; i += kThreads) hist[i] = 0U;
  }
  // The lens shading gains in shared memory for the frame, when they fit.
  Span<const float> grid = p.lsc;
  const int gains = p.lsc_width * p.lsc_height * p.lsc_channels;
  if (p.lsc != nullptr && gains <= kGridSmemGains) {
    for (int i = tid; i < gains; i += kThreads) cp_async4(&grid_s[i], &p.lsc[i]);
    grid = grid_s;
  }
  if (tid == 0 && use_tma) {
    mbar_init(&bars[0]);
    mbar_init(&bars[1]);
  }
  float black[4], inv[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    black[k] = p.black[cfa_of(kPat, k)];
    inv[k] = p.inv_range[cfa_of(kPat, k)];
  }
  const int strip = static_cast<int>(blockIdx.x) % strips;
  const int ty0 = (static_cast<int>(blockIdx.x) / strips) * band_tiles;
  const int ty1 = min(ty0 + band_tiles, tiles_y);
  const int x0 = strip * 64;
  const auto issue = [&](int ty, int b) {
    tma_load_2d(&map, boxes + b * 64 * 128, &bars[b], awb_box_x(p.raw_format, x0), ty * 64,
                static_cast<unsigned int>(kBoxRows * box_bytes));
  };
  cp_async_wait_all();
  __syncthreads();  // barriers initialised, the gains in shared memory
  if (use_tma && tid == 0 && ty0 < ty1) issue(ty0, 0);
  // The band's maps and table (block-synchronised inside), while the first
  // box is in flight.
  const LscTile lt = build_band_lsc(p, grid, kPat, x0, ty0 * 64, (ty1 - ty0) * 64, col_mx, col_ix, col_tx, row_my,
                                    row_k, row_ty, table, minmax);
  u64 acc[4] = {0, 0, 0, 0};
  uint32_t phases = 0;  // bit b: parity of buffer b's next completion
  for (int ty = ty0; ty < ty1; ++ty) {
    const int buf = (ty - ty0) & 1;
    // The other buffer was read by the previous tile (the block synchronised
    // since): load the next tile into it while this one is summed.
    if (use_tma && tid == 0 && ty + 1 < ty1) {
      fence_async_shared();
      issue(ty + 1, buf ^ 1);
    }
    if (use_tma && !mbar_wait(&bars[buf], (phases >> buf) & 1U)) {
      if (tid == 0) report_wait_timeout(s);
    }
    phases ^= 1U << buf;
    Span<const uint8_t> box = boxes + buf * 64 * 128;
    const int rows = (ty - ty0) * 64;  // the tile's first row within the band
    unsigned int sum[3] = {0U, 0U, 0U};
    unsigned int quads = 0;
    if (use_tma) {
      awb_tile_fmt<0, kWhitePatch, kPat>(p, box, box_bytes, x0, ty * 64, lt, row_k + rows, row_ty + rows, table, black,
                                          inv, hist, sum, quads);
    } else {
      awb_tile_fmt<1, kWhitePatch, kPat>(p, box, box_bytes, x0, ty * 64, lt, row_k + rows, row_ty + rows, table, black,
                                          inv, hist, sum, quads);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] += sum[k];
    acc[3] += quads;
    __syncthreads();
  }
  awb_flush<true>(p, acc, hist, kWhitePatch, red, &first, &last, static_cast<unsigned int>(ty1 > ty0 ? ty1 - ty0 : 0),
            static_cast<unsigned int>(strips * tiles_y));
}

template <bool kWhitePatch>
const void* awb_by_pattern(int pattern) {
  switch (pattern) {
    case 0: return reinterpret_cast<const void*>(&isp_awb_kernel<kWhitePatch, 0>);
    case 1: return reinterpret_cast<const void*>(&isp_awb_kernel<kWhitePatch, 1>);
    case 2: return reinterpret_cast<const void*>(&isp_awb_kernel<kWhitePatch, 2>);
    default: return reinterpret_cast<const void*>(&isp_awb_kernel<kWhitePatch, 3>);
  }
}

}  // namespace

const void* awb_kernel(bool white_patch, int pattern) {
  return white_patch ? awb_by_pattern<true>(pattern) : awb_by_pattern<false>(pattern);
}

}  // namespace isp_b200
