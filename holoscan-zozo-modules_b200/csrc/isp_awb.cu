// isp_awb.cu - the white balance statistics kernel of the B200 ISP
// (gray world and white patch): tiles of 64x64 samples arrive by TMA, the
// complete 2x2 quads without a saturated sample are summed per colour (and
// binned for white patch) in the block, then flushed once; the last CTA to
// finish forms the frame's estimate (finish_white_balance, isp_math.hpp:357-384)
// and clears the sums for the next frame.
#include "isp_awb.cuh"

namespace isp_b200 {
namespace {


// ---- White balance statistics ----------------------------------------------

template <bool kWhitePatch, int kPat>
__global__ void __launch_bounds__(kThreads, 3) isp_awb_kernel(const __grid_constant__ CUtensorMap map, FrameDesc p,
                                                         int tiles_x, int tiles, int use_tma) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128U - (smem_u32(smem_raw) & 127U)) & 127U);
  constexpr int kBoxRows = 64;
  uint8_t* boxes = smem;                                                  // [2][64][128]: double buffer
  float* table = reinterpret_cast<float*>(smem + 2 * 64 * 128);           // [kLscTableRows][2][kSW]
  int* col_mx = reinterpret_cast<int*>(table + kLscTableRows * 2 * kSW);  // [64] x 3
  int* col_ix = col_mx + 64;
  float* col_tx = reinterpret_cast<float*>(col_ix + 64);
  int* row_my = reinterpret_cast<int*>(col_tx + 64);                      // [64] x 3
  int* row_k = row_my + 64;
  float* row_ty = reinterpret_cast<float*>(row_k + 64);
  unsigned int* hist = reinterpret_cast<unsigned int*>(row_ty + 64);      // [3][1024]
  float* grid_s = reinterpret_cast<float*>(hist + 3 * kAwbBins);          // [kGridSmemGains]
  __shared__ uint64_t bars[2];
  __shared__ u64 red[kWarps];
  __shared__ int minmax[2];
  __shared__ int first;
  __shared__ bool last;
  Scratch* s = p.scratch;
  const int tid = threadIdx.x;
  const int box_bytes = awb_box_bytes(p.raw_format);
  // The tile pass that follows may launch now: it waits (griddepcontrol.wait)
  // for this grid's completion before it does anything, but its CTAs become
  // resident on the SMs this pass leaves while the last tiles are summed.
  griddep_launch_dependents();
  if constexpr (kWhitePatch) {
    for (int i = tid; i < 3 * kAwbBins; i += kThreads) hist[i] = 0U;
  }
  // The lens shading gains in shared memory for the frame, when they fit.
  const float* grid = p.lsc;
  const int gains = p.lsc_width * p.lsc_height * p.lsc_channels;
  if (p.lsc != nullptr && gains <= kGridSmemGains) {
    for (int i = tid; i < gains; i += kThreads) grid_s[i] = p.lsc[i];
    grid = grid_s;
  }
  if (tid == 0 && use_tma) {
    mbar_init(&bars[0]);
    mbar_init(&bars[1]);
  }
  __syncthreads();
  float black[4], inv[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    black[k] = p.black[cfa_of(kPat, k)];
    inv[k] = p.inv_range[cfa_of(kPat, k)];
  }
  u64 acc[4] = {0, 0, 0, 0};
  uint32_t phases = 0;  // bit b: parity of buffer b's next completion
  unsigned int done = 0;  // tiles this CTA summed; its k-th tile uses buffer k & 1
  int tile = blockIdx.x;
  const auto issue = [&](int t, int b) {
    const int ty = t / tiles_x;
    const int x0 = (t - ty * tiles_x) * 64;
    tma_load_2d(&map, boxes + b * 64 * 128, &bars[b], awb_box_x(p.raw_format, x0), ty * 64,
                static_cast<unsigned int>(kBoxRows * box_bytes));
  };
  if (use_tma && tid == 0 && tile < tiles) issue(tile, 0);
  for (; tile < tiles; tile += gridDim.x) {
    const int ty = tile / tiles_x;
    const int x0 = (tile - ty * tiles_x) * 64;
    const int y0 = ty * 64;
    const int buf = static_cast<int>(done & 1U);
    // The other buffer was read by the previous tile (the block synchronised
    // since): load the next tile into it while this one is summed.
    if (use_tma && tid == 0 && tile + static_cast<int>(gridDim.x) < tiles) {
      fence_async_shared();
      issue(tile + gridDim.x, buf ^ 1);
    }
    const LscTile lt = build_lsc(p, grid, kPat, x0, 64, y0, 64, false, 0, 0, col_mx, col_ix, col_tx, row_my, row_k,
                                 row_ty, table, minmax);
    if (use_tma && !mbar_wait(&bars[buf], (phases >> buf) & 1U)) {
      if (tid == 0) atomicExch(&s->error, 1);
    }
    phases ^= 1U << buf;
    const uint8_t* box = boxes + buf * 64 * 128;
    unsigned int sum[3] = {0U, 0U, 0U};
    unsigned int quads = 0;
    if (use_tma) {
      awb_tile_fmt<0, kWhitePatch, kPat>(p, box, box_bytes, x0, y0, lt, row_k, row_ty, table, black, inv, hist, sum, quads);
    } else {
      awb_tile_fmt<1, kWhitePatch, kPat>(p, box, box_bytes, x0, y0, lt, row_k, row_ty, table, black, inv, hist, sum, quads);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] += sum[k];
    acc[3] += quads;
    __syncthreads();
    ++done;
  }
  awb_flush(p, acc, hist, kWhitePatch, red, &first, &last, done, static_cast<unsigned int>(tiles));
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
