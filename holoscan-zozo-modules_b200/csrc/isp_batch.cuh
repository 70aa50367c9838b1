// isp_batch.cuh - frames of uneven size, format, Bayer pattern and settings
// in one launch per pass: the statistics pass over the auto-white-balance
// frames' tiles, then the tile pass over every frame's tiles.
//
// Each pass is a persistent kernel over a work list: CTA i owns the
// contiguous items ranges[i] (sized by the host so the estimated cost is
// even), walks them frame by frame, keeps the frame's FrameDesc and tone
// table in shared memory, prefetches the next item's raw box by TMA
// (whichever frame it belongs to), and flushes a frame's sums when it leaves
// it; the CTA that completes a frame's count of tiles finishes that frame
// (its statistics and histogram, or its white balance estimate). Every tile
// runs the same device code as the single-frame kernels (isp_main.cuh,
// isp_awb.cuh), so a frame's bytes are the same alone or in a batch.
#pragma once

#include "isp_awb.cuh"
#include "isp_main.cuh"

namespace isp_b200 {
namespace {

__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}

// Copies a frame's FrameDesc to shared memory (all threads; the caller syncs).
__device__ __forceinline__ void load_desc(FrameDesc* dst, const FrameDesc* src) {
  constexpr int kWords = sizeof(FrameDesc) / 4;
  static_assert(sizeof(FrameDesc) % 4 == 0, "FrameDesc words");
  const unsigned int* s = reinterpret_cast<const unsigned int*>(src);
  unsigned int* d = reinterpret_cast<unsigned int*>(dst);
  for (int i = threadIdx.x; i < kWords; i += kThreads) d[i] = s[i];
}

// The frame holding work item `item`, searching forward from frame `from`.
__device__ __forceinline__ int frame_of_item(Span<const BatchFrame> frames, int nframes, int from, int item, bool awb) {
  int f = from;
  while (f + 1 < nframes && item >= (awb ? frames[f + 1].awb_begin : frames[f + 1].tile_begin)) ++f;
  return f;
}

template <bool kLutSmem, int kTileH>
__global__ void __launch_bounds__(kThreads, kTileH == kTH ? 2 : 3)
    isp_batch_kernel(const BatchFrame* frames_in, int nframes, const int2* ranges_in) {
  using GS = Geom<true, kTileH>;  // the sharpening geometry holds every variant's
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128U - (smem_u32(smem_raw) & 127U)) & 127U);
#ifdef ISP_CHECKED
  CheckRecord* const rec = span_rec(frames_in[0].desc.scratch);
#else
  CheckRecord* const rec = nullptr;
#endif
  const Span<const BatchFrame> frames = make_span(frames_in, static_cast<size_t>(nframes), rec);
  const Span<const int2> ranges = make_span(ranges_in, static_cast<size_t>(gridDim.x), rec);
  const TileSmem m =
      carve(smem, layout_of(true, box_row_bytes(kRawU16), kLutSmem ? kBatchLutEntries : 0, kTileH), GS::kSH, rec);
  __shared__ uint64_t bar;
  __shared__ u64 red[4 * kWarps];
  __shared__ int minmax[2];
  __shared__ bool last;
  __shared__ __align__(16) FrameDesc fd;
  // A programmatic dependent of the statistics batch: resident early, it
  // waits here for that batch's completion (and the gains it wrote).
  griddep_wait();
  const int2 r = ranges[blockIdx.x];
  if (r.x >= r.y) return;
  const int tid = threadIdx.x;
  if (tid == 0) mbar_init(&bar);
  int f = frame_of_item(frames, nframes, 0, r.x, false);
  load_desc(&fd, &frames[f].desc);
  __syncthreads();
  FrameSetup fs = setup_frame<kLutSmem>(fd, m);
  __syncthreads();

  const auto issue = [&](int g, int item) {
    const BatchFrame& bf = frames[g];
    const int local = item - bf.tile_begin;
    const int ty = local / bf.tiles_x;
    const int x0 = (local - ty * bf.tiles_x) * kTW;
    const int halo = (bf.variant & 2) ? 4 : 2;
    const int fmt = bf.desc.raw_format;
    tensormap_acquire(&bf.main_map);
    tma_load_2d(&bf.main_map, m.box, &bar, box_x(fmt, x0), ty * kTileH - halo,
                static_cast<unsigned int>((kTileH + 2 * halo) * box_row_bytes(fmt)));
  };
  if (tid == 0 && frames[f].use_tma) issue(f, r.x);
  uint32_t phase = 0;
  u64 acc[4] = {0, 0, 0, 0};
  unsigned int done = 0;
  for (int item = r.x; item < r.y; ++item) {
    if (item >= frames[f].tile_begin + frames[f].tiles) {
      flush_frame(fd, fs, acc, m.hist, red, &last, done, static_cast<unsigned int>(frames[f].tiles));
      __syncthreads();
      f = frame_of_item(frames, nframes, f, item, false);
      load_desc(&fd, &frames[f].desc);
      __syncthreads();
      fs = setup_frame<kLutSmem>(fd, m);
      __syncthreads();
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] = 0;
      done = 0;
    }
    const BatchFrame& bf = frames[f];
    const int local = item - bf.tile_begin;
    const int ty = local / bf.tiles_x;
    const int x0 = (local - ty * bf.tiles_x) * kTW;
    const bool use_tma = bf.use_tma != 0;
    const auto prefetch = [&] {
      if (tid == 0 && item + 1 < r.y) {
        const int g = frame_of_item(frames, nframes, f, item + 1, false);
        if (frames[g].use_tma) {
          fence_async_shared();
          issue(g, item + 1);
        }
      }
    };
    switch (bf.variant) {
      case 0: run_tile<false, false, 0, kLutSmem, decltype(prefetch), -1, kTileH>(fd, fs, m, minmax, x0, ty * kTileH, use_tma, &bar, phase, acc, prefetch); break;
      case 1: run_tile<true, false, 0, kLutSmem, decltype(prefetch), -1, kTileH>(fd, fs, m, minmax, x0, ty * kTileH, use_tma, &bar, phase, acc, prefetch); break;
      case 2: run_tile<false, true, 0, kLutSmem, decltype(prefetch), -1, kTileH>(fd, fs, m, minmax, x0, ty * kTileH, use_tma, &bar, phase, acc, prefetch); break;
      case 3: run_tile<true, true, 0, kLutSmem, decltype(prefetch), -1, kTileH>(fd, fs, m, minmax, x0, ty * kTileH, use_tma, &bar, phase, acc, prefetch); break;
      case 4: run_tile<false, false, 1, kLutSmem, decltype(prefetch), -1, kTileH>(fd, fs, m, minmax, x0, ty * kTileH, use_tma, &bar, phase, acc, prefetch); break;
      case 5: run_tile<true, false, 1, kLutSmem, decltype(prefetch), -1, kTileH>(fd, fs, m, minmax, x0, ty * kTileH, use_tma, &bar, phase, acc, prefetch); break;
      case 6: run_tile<false, true, 1, kLutSmem, decltype(prefetch), -1, kTileH>(fd, fs, m, minmax, x0, ty * kTileH, use_tma, &bar, phase, acc, prefetch); break;
      default: run_tile<true, true, 1, kLutSmem, decltype(prefetch), -1, kTileH>(fd, fs, m, minmax, x0, ty * kTileH, use_tma, &bar, phase, acc, prefetch); break;
    }
    ++done;
  }
  flush_frame(fd, fs, acc, m.hist, red, &last, done, static_cast<unsigned int>(frames[f].tiles));
}

// The statistics tile of a frame for its Bayer pattern and mode.
template <int kSrc>
__device__ __forceinline__ void awb_tile_any(const FrameDesc& p, int pattern, bool white_patch, Span<const uint8_t> box,
                                             int box_bytes, int x0, int y0, const LscTile& lt, Span<const int> row_k,
                                             Span<const float> row_ty, Span<const float> table, const float (&black)[4],
                                             const float (&inv)[4], Span<unsigned int> hist, unsigned int (&sum)[3],
                                             unsigned int& quads) {
#define ISP_AWB_CASE(P, W) \
  awb_tile_fmt<kSrc, W, P>(p, box, box_bytes, x0, y0, lt, row_k, row_ty, table, black, inv, hist, sum, quads)
  switch (pattern * 2 + (white_patch ? 1 : 0)) {
    case 0: ISP_AWB_CASE(0, false); break;
    case 1: ISP_AWB_CASE(0, true); break;
    case 2: ISP_AWB_CASE(1, false); break;
    case 3: ISP_AWB_CASE(1, true); break;
    case 4: ISP_AWB_CASE(2, false); break;
    case 5: ISP_AWB_CASE(2, true); break;
    case 6: ISP_AWB_CASE(3, false); break;
    default: ISP_AWB_CASE(3, true); break;
  }
#undef ISP_AWB_CASE
}

__global__ void __launch_bounds__(kThreads, 3) isp_awb_batch_kernel(const BatchFrame* frames_in, int nframes,
                                                               const int2* ranges_in) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128U - (smem_u32(smem_raw) & 127U)) & 127U);
#ifdef ISP_CHECKED
  CheckRecord* const rec = span_rec(frames_in[0].desc.scratch);
#else
  CheckRecord* const rec = nullptr;
#endif
  const Span<const BatchFrame> frames = make_span(frames_in, static_cast<size_t>(nframes), rec);
  const Span<const int2> ranges = make_span(ranges_in, static_cast<size_t>(gridDim.x), rec);
  constexpr int kTableAt = 2 * 64 * 128;                          // boxes: [2][64][128], a double buffer
  constexpr int kColsAt = kTableAt + kLscTableRows * 2 * kSW * 4;  // table: [kLscTableRows][2][kSW]
  constexpr int kRowsAt = kColsAt + 3 * 64 * 4;                    // col_mx, col_ix, col_tx: [64] each
  constexpr int kHistAt = kRowsAt + 3 * 64 * 4;                    // row_my, row_k, row_ty: [64] each
  Span<uint8_t> boxes = carve_span<uint8_t>(smem, 0, kTableAt, rec);
  Span<float> table = carve_span<float>(smem, kTableAt, kColsAt - kTableAt, rec);
  Span<int> col_mx = carve_span<int>(smem, kColsAt, 64 * 4, rec);
  Span<int> col_ix = carve_span<int>(smem, kColsAt + 64 * 4, 64 * 4, rec);
  Span<float> col_tx = carve_span<float>(smem, kColsAt + 128 * 4, 64 * 4, rec);
  Span<int> row_my = carve_span<int>(smem, kRowsAt, 64 * 4, rec);
  Span<int> row_k = carve_span<int>(smem, kRowsAt + 64 * 4, 64 * 4, rec);
  Span<float> row_ty = carve_span<float>(smem, kRowsAt + 128 * 4, 64 * 4, rec);
  Span<unsigned int> hist = carve_span<unsigned int>(smem, kHistAt, 3 * kAwbBins * 4, rec);  // [3][1024]
  __shared__ uint64_t bars[2];
  __shared__ u64 red[4 * kWarps];
  __shared__ int minmax[2];
  __shared__ int first;
  __shared__ bool last;
  __shared__ __align__(16) FrameDesc fd;
  griddep_launch_dependents();  // the tile batch may become resident as this one finishes
  const int2 r = ranges[blockIdx.x];
  if (r.x >= r.y) return;
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bars[0]);
    mbar_init(&bars[1]);
  }
  for (int i = tid; i < 3 * kAwbBins; i += kThreads) hist[i] = 0U;
  int f = frame_of_item(frames, nframes, 0, r.x, true);
  load_desc(&fd, &frames[f].desc);
  __syncthreads();
  const auto issue = [&](int g, int item, int b) {
    const BatchFrame& bf = frames[g];
    const int local = item - bf.awb_begin;
    const int ty = local / bf.awb_tiles_x;
    const int x0 = (local - ty * bf.awb_tiles_x) * 64;
    const int fmt = bf.desc.raw_format;
    tensormap_acquire(&bf.awb_map);
    tma_load_2d(&bf.awb_map, boxes + b * 64 * 128, &bars[b], awb_box_x(fmt, x0), ty * 64,
                static_cast<unsigned int>(64 * awb_box_bytes(fmt)));
  };
  if (tid == 0 && frames[f].use_tma) issue(f, r.x, 0);
  // Item i of the range uses buffer (i - r.x) & 1, whether or not its frame
  // uses TMA, so the prefetching thread and the waiting block always agree.
  uint32_t phases = 0;  // bit b: parity of buffer b's next completion
  u64 acc[4] = {0, 0, 0, 0};
  unsigned int done = 0;
  for (int item = r.x; item < r.y; ++item) {
    if (item >= frames[f].awb_begin + frames[f].awb_tiles) {
      awb_flush(fd, acc, hist, fd.awb_mode == kWbWhitePatch, red, &first, &last, done,
                static_cast<unsigned int>(frames[f].awb_tiles));
      f = frame_of_item(frames, nframes, f, item, true);
      load_desc(&fd, &frames[f].desc);
      for (int i = tid; i < 3 * kAwbBins; i += kThreads) hist[i] = 0U;
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] = 0;
      done = 0;
      __syncthreads();
    }
    const BatchFrame& bf = frames[f];
    const int buf = (item - r.x) & 1;
    // The other buffer was read by the previous item (the block synchronised
    // since): load the next item into it while this one is summed.
    if (tid == 0 && item + 1 < r.y) {
      const int g = frame_of_item(frames, nframes, f, item + 1, true);
      if (frames[g].use_tma) {
        fence_async_shared();
        issue(g, item + 1, buf ^ 1);
      }
    }
    const int local = item - bf.awb_begin;
    const int ty = local / bf.awb_tiles_x;
    const int x0 = (local - ty * bf.awb_tiles_x) * 64;
    const int y0 = ty * 64;
    const LscTile lt = build_lsc(fd, fd.lsc, fd.pattern, x0, 64, y0, 64, false, 0, 0, col_mx, col_ix, col_tx, row_my, row_k,
                                 row_ty, table, minmax);
    const bool use_tma = bf.use_tma != 0;
    if (use_tma) {
      if (!mbar_wait(&bars[buf], (phases >> buf) & 1U) && tid == 0) report_wait_timeout(fd.scratch);
      phases ^= 1U << buf;
    }
    float black[4], inv[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      black[k] = fd.black[fd.cfa[k]];
      inv[k] = fd.inv_range[fd.cfa[k]];
    }
    unsigned int sum[3] = {0U, 0U, 0U};
    unsigned int quads = 0;
    const int box_bytes = awb_box_bytes(fd.raw_format);
    const bool wp = fd.awb_mode == kWbWhitePatch;
    if (use_tma) {
      awb_tile_any<0>(fd, fd.pattern, wp, boxes + buf * 64 * 128, box_bytes, x0, y0, lt, row_k, row_ty, table, black,
                      inv, hist, sum, quads);
    } else {
      awb_tile_any<1>(fd, fd.pattern, wp, boxes + buf * 64 * 128, box_bytes, x0, y0, lt, row_k, row_ty, table, black,
                      inv, hist, sum, quads);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] += sum[k];
    acc[3] += quads;
    __syncthreads();
    ++done;
  }
  awb_flush(fd, acc, hist, fd.awb_mode == kWbWhitePatch, red, &first, &last, done,
            static_cast<unsigned int>(frames[f].awb_tiles));
}

}  // namespace
}  // namespace isp_b200
