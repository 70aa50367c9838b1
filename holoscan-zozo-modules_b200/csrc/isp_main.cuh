// isp_main.cuh - the fused tile pass of the B200 ISP as device templates: a
// frame's per-CTA setup, one 64x64 tile (phases A, B, C), and the per-frame
// flush with the last-tile finish. The single-frame kernel here and the
// batch kernel (isp_batch.cu) are both built from them, so every frame gets
// the same arithmetic however it is launched. Each isp_main_*.cu
// translation unit instantiates one demosaic method and sharpening setting,
// so the instances compile in parallel.
#pragma once

#include "isp_pairs.cuh"

namespace isp_b200 {
namespace {

// Shared memory of a CTA, carved from one dynamic allocation.
struct TileSmem {
  Span<uint8_t> box;
  Span<float2> P;  // paired samples
  Span<float2> R;  // paired RGB planes (sharpening)
  Span<float2> G;
  Span<float2> B;
  Span<float2> table;  // paired lens shading table
  Span<int> col_mx;
  Span<int> col_ix;
  Span<float> col_tx;
  Span<int> row_my;
  Span<int> row_k;
  Span<float> row_ty;
  Span<unsigned int> hist;
  Span<float> grid;
  Span<float2> lut_s;
};

// Each region spans the bytes up to the next (the checked build holds its
// accesses to them; `rec` is where it counts violations).
__device__ __forceinline__ TileSmem carve(unsigned char* smem, const Layout& L, int sample_rows, CheckRecord* rec) {
  TileSmem m;
  m.box = carve_span<uint8_t>(smem, L.raw, L.samples - L.raw, rec);
  m.P = carve_span<float2>(smem, L.samples, L.r - L.samples, rec);
  m.R = carve_span<float2>(smem, L.r, L.g - L.r, rec);
  m.G = carve_span<float2>(smem, L.g, L.b - L.g, rec);
  m.B = carve_span<float2>(smem, L.b, L.lsc - L.b, rec);
  m.table = carve_span<float2>(smem, L.lsc, L.cols - L.lsc, rec);
  m.col_mx = carve_span<int>(smem, L.cols, kSW * 4, rec);
  m.col_ix = carve_span<int>(smem, L.cols + kSW * 4, kSW * 4, rec);
  m.col_tx = carve_span<float>(smem, L.cols + 2 * kSW * 4, kSW * 4, rec);
  m.row_my = carve_span<int>(smem, L.rows, sample_rows * 4, rec);
  m.row_k = carve_span<int>(smem, L.rows + sample_rows * 4, sample_rows * 4, rec);
  m.row_ty = carve_span<float>(smem, L.rows + 2 * sample_rows * 4, sample_rows * 4, rec);
  m.hist = carve_span<unsigned int>(smem, L.hist, L.grid - L.hist, rec);
  m.grid = carve_span<float>(smem, L.grid, L.lut - L.grid, rec);
  m.lut_s = carve_span<float2>(smem, L.lut, L.total - L.lut, rec);
  return m;
}

// What every tile of a frame reads, set up once per frame by a CTA.
struct FrameSetup {
  float gains[3];  // the white balance the frame is processed with
  float qblack[4];  // per quad position
  float qinv[4];
  float qgain[4];
  Span<const float2> lut;
  Span<const float> grid;  // lens shading gains: shared memory when they fit
  float lut_scale;
  bool swap_rb;
  bool want_hist;
  bool want_stats;
};

// The frame's shared-memory copies: the lens shading gains (when they fit),
// the tone table (kLutSmem) and the cleared block histogram. They read only
// the pipeline's own tables, never what the statistics pass writes. The
// tables arrive by asynchronous copies: each thread calls cp_async_wait_all()
// before the block barrier that publishes them.
template <bool kLutSmem>
__device__ __forceinline__ void fill_frame_smem(const FrameDesc& p, const TileSmem& m) {
  const int gains = p.lsc_width * p.lsc_height * p.lsc_channels;
  if (p.lsc != nullptr && gains <= kGridSmemGains) {
    for (int i = threadIdx.x; i < gains; i += kThreads) cp_async4(&m.grid[i], &p.lsc[i]);
  }
  if constexpr (kLutSmem) {
    for (int i = threadIdx.x; i < p.tone_size; i += kThreads) cp_async8(&m.lut_s[i], &p.tone[i]);
  }
  if (p.hist_out != nullptr) {
    for (int i = threadIdx.x; i < kHistChannels * kHistBins; i += kThreads) m.hist[i] = 0U;
  }
}

// The frame's lens shading gains as the tiles read them: the shared-memory
// copy when the grid fits, else the pipeline's grid in device memory.
__device__ __forceinline__ Span<const float> frame_grid(const FrameDesc& p, const TileSmem& m) {
  const int gains = p.lsc_width * p.lsc_height * p.lsc_channels;
  return p.lsc != nullptr && gains <= kGridSmemGains ? Span<const float>(m.grid) : p.lsc;
}

// Reads the frame's gains (its estimate, for auto white balance) and, with
// kFill, fills the frame's shared memory (fill_frame_smem, its copies waited
// for; without kFill the caller filled it before and waits for the copies).
// The caller synchronises the block before the first tile.
template <bool kLutSmem, bool kFill = true>
__device__ __forceinline__ FrameSetup setup_frame(const FrameDesc& p, const TileSmem& m) {
  if constexpr (kFill) fill_frame_smem<kLutSmem>(p, m);
  FrameSetup f;
#pragma unroll
  for (int k = 0; k < 3; ++k) f.gains[k] = p.auto_wb ? __ldcg(&p.scratch->awb_gains[k]) : p.wb[k];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int ch = p.cfa[k];
    f.qblack[k] = p.black[ch];
    f.qinv[k] = p.inv_range[ch];
    f.qgain[k] = f.gains[color_of(ch)];
  }
  f.grid = frame_grid(p, m);
  f.lut = kLutSmem ? m.lut_s : p.tone;
  f.lut_scale = static_cast<float>(p.tone_size - 1);
  // The demosaic runs as the layout's canonical pattern (RGGB or GRBG); for
  // BGGR and GBRG its red and blue outputs trade places before the colour
  // matrix (the estimates' arithmetic is the same at either site).
  f.swap_rb = (p.pattern & 1) != 0;
  f.want_hist = p.hist_out != nullptr;
  f.want_stats = p.stats_out != nullptr;
  if constexpr (kFill) cp_async_wait_all();
  return f;
}

// Output units u (0..511) of phase C: an output row r and group uc of four
// pairs. A warp's 32 units are 4 rows x 8 groups, and each quarter-warp
// (whose 16-byte loads share one pass through the banks) takes groups 0..3
// or 4..7 of two rows. With sharpening the two rows are r and r + 1: the
// RGB planes' row stride is an odd number of 16-byte chunks, so they meet
// different banks. Without sharpening a warp keeps one row parity (the
// Bayer sites are compile-time) and the rows are r and r + 2, which the
// sample plane's swizzle (psw) sends to different banks.
// With sharpening, thread t takes output rows r and r + 1 (r even) of group
// uc: a warp covers 8 rows x 8 groups, and each quarter-warp groups 0..3 or
// 4..7 of two neighbouring row pairs (the RGB planes' swizzle, csw, sends
// them to different banks).
__device__ __forceinline__ void unit_rows2(int t, int& r, int& uc) {
  const int w = t >> 5;
  const int l = t & 31;
  uc = (l & 3) | (((l >> 3) & 1) << 2);
  r = 8 * w + 2 * (((l >> 2) & 1) + ((l >> 4) << 1));
}

__device__ __forceinline__ void unit_rc(int u, bool same_parity, int& r, int& uc) {
  const int w = u >> 5;
  const int l = u & 31;
  const int ro = ((l >> 2) & 1) + ((l >> 4) << 1);  // 0..3
  uc = (l & 3) | (((l >> 3) & 1) << 2);
  r = same_parity ? ((w >> 1) << 3) + 2 * ro + (w & 1) : 4 * w + ro;
}

// The per-pixel tail of four pairs of one output row (pixels x .. x + 3 and
// x + 32 .. x + 35 of row y): colour matrix, statistics, tone, store and
// histograms, with the per-pixel guards only where the row leaves the image
// or the output rows are not 16-byte aligned. kOutSel: the output format
// fixed at compile time (the single-frame kernels), or -1 to choose it per
// unit (the batch kernel).
template <int kOutSel, bool kLutSmem>
__device__ __forceinline__ void finish_row(const FrameDesc& p, const FrameSetup& f, Span<unsigned int> hist,
                                           const float2 (&rgb)[4][3], int x, int y, unsigned int (&sums)[3],
                                           unsigned int& npix) {
  if (y >= p.height) return;
  const int nl = min(max(p.width - x, 0), 4);
  const int nr = min(max(p.width - x - kHalf, 0), 4);
  if (nl == 4 && nr == 4 && p.out_vector) {
    if constexpr (kOutSel < 0) {
      finish_pairs_any<kLutSmem, true>(p, rgb, x, y, nl, nr, f.lut, f.lut_scale, f.want_stats, f.want_hist, hist, sums,
                                       npix);
    } else {
      finish_pairs<kOutSel, kLutSmem, true>(p, rgb, x, y, nl, nr, f.lut, f.lut_scale, f.want_stats, f.want_hist, hist,
                                            sums, npix);
    }
  } else {
    if constexpr (kOutSel < 0) {
      finish_pairs_any<kLutSmem, false>(p, rgb, x, y, nl, nr, f.lut, f.lut_scale, f.want_stats, f.want_hist, hist,
                                        sums, npix);
    } else {
      finish_pairs<kOutSel, kLutSmem, false>(p, rgb, x, y, nl, nr, f.lut, f.lut_scale, f.want_stats, f.want_hist,
                                             hist, sums, npix);
    }
  }
}

// A hook that does nothing (run_tile's default hooks).
struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};

// One 64x64 tile at (x0, y0) (kTileH rows). Its box is waited for on `bar`.
// Hooks, all run by every thread: `after_lsc()` once the tile's lens shading
// maps and table are built, before the box wait and phase A (the frame's
// gains may be read there); `after_a()` after phase A, when the box is free
// again (to claim or prefetch the next tile); `before_c()` before phase C.
// Adds the tile's statistics sums and saturated count to `acc` (per thread).

template <bool kMalvar, bool kSharpen, int kLayout, bool kLutSmem, class AfterA, int kOutSel = -1, int kTileH = kTH,
          class BeforeC = NoHook, class AfterLsc = NoHook>
__device__ __forceinline__ void run_tile(const FrameDesc& p, const FrameSetup& f, const TileSmem& m, int* minmax,
                                         int x0, int y0, bool use_tma, uint64_t* bar, uint32_t& phase,
                                         u64 (&acc)[4], AfterA after_a, BeforeC before_c = BeforeC{},
                                         AfterLsc after_lsc = AfterLsc{}) {
  using G = Geom<kSharpen, kTileH>;
  constexpr int kPat = kLayout * 2;
  const int tid = threadIdx.x;
  const int box_bytes = box_row_bytes(p.raw_format);
  const bool interior = x0 >= 4 && y0 >= G::kHalo && x0 + kSW - 4 <= p.width && y0 + kTileH + G::kHalo <= p.height;
  TileCtx t;
  t.x0 = x0;
  t.y0 = y0;
  t.box = m.box;
  t.col_mx = m.col_mx;
  t.row_my = m.row_my;
  t.row_k = m.row_k;
  t.row_ty = m.row_ty;
  t.table = m.table;
  t.grid = f.grid;
  t.lt = interior ? build_lsc_inner(p, f.grid, p.pattern, x0 - 4, y0 - G::kHalo, G::kSH, m.col_mx, m.col_ix,
                                    m.col_tx, m.row_my, m.row_k, m.row_ty, span_cast<float>(m.table), minmax)
                  : build_lsc<true>(p, f.grid, p.pattern, x0 - 4, kSW, y0 - G::kHalo, G::kSH, true, p.width + 3,
                                    p.height + G::kHalo - 1, m.col_mx, m.col_ix, m.col_tx, m.row_my, m.row_k, m.row_ty,
                                    span_cast<float>(m.table), minmax);
  after_lsc();
  if (use_tma) {
    if (!mbar_wait(bar, phase) && tid == 0) report_wait_timeout(p.scratch);
    phase ^= 1U;
  }

  // A. Samples of the tile and its halo, preprocessed once, as pairs.
  unsigned int saturated;
  if (!use_tma) {
    saturated = phase_a2_fmt<2, G::kHalo, kTileH>(p, t, m.P, box_bytes, f.qblack, f.qinv, f.qgain, f.want_stats);
  } else if (interior) {
    saturated = phase_a2_fmt<0, G::kHalo, kTileH>(p, t, m.P, box_bytes, f.qblack, f.qinv, f.qgain, f.want_stats);
  } else {
    saturated = phase_a2_fmt<1, G::kHalo, kTileH>(p, t, m.P, box_bytes, f.qblack, f.qinv, f.qgain, f.want_stats);
  }
  acc[3] += saturated;
  __syncthreads();
  after_a();

  // B. (Sharpening) RGB of the tile and its ring; BGGR and GBRG write the
  //    demosaic's red into the blue plane and its blue into the red.
  if constexpr (kSharpen) {
    phase_b2<kMalvar, kPat, kTileH>(m.P, f.swap_rb ? m.B : m.R, m.G, f.swap_rb ? m.R : m.B);
    __syncthreads();
  }
  before_c();

  // C. The statistics sums stay below 2^32 per thread and tile (16 pixels
  //    of at most 2^20).
  unsigned int sums[3] = {0U, 0U, 0U};
  unsigned int npix = 0;
  if constexpr (kSharpen && kOutSel >= 0 && kTileH == kTH) {
    // One unit per thread: output rows r and r + 1 of group uc, whose RGB
    // rows r .. r + 3 each plane loads once.
    int r, uc;
    unit_rows2(tid, r, uc);
    const float2 amount = bc2(p.sharpen);
    float2 rgb0[4][3], rgb1[4][3];
    float2 o0[4], o1[4];
    sharpen_rows2(m.R, r, uc, amount, o0, o1);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      rgb0[i][0] = o0[i];
      rgb1[i][0] = o1[i];
    }
    sharpen_rows2(m.G, r, uc, amount, o0, o1);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      rgb0[i][1] = o0[i];
      rgb1[i][1] = o1[i];
    }
    sharpen_rows2(m.B, r, uc, amount, o0, o1);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      rgb0[i][2] = o0[i];
      rgb1[i][2] = o1[i];
    }
    finish_row<kOutSel, kLutSmem>(p, f, m.hist, rgb0, x0 + 4 * uc, y0 + r, sums, npix);
    finish_row<kOutSel, kLutSmem>(p, f, m.hist, rgb1, x0 + 4 * uc, y0 + r + 1, sums, npix);
  } else {
    // Units of four pairs of one row, kTileH / 32 per thread: sharpened (the
    // batch kernel, whose output format is chosen per unit, keeps one call
    // site of the finish; and short tiles), or demosaiced straight from the
    // samples.
#pragma unroll 1
    for (int k = 0; k < kTileH / 32; ++k) {
      int r, uc;
      unit_rc(tid + k * kThreads, true, r, uc);
      float2 rgb[4][3];
      if constexpr (kSharpen) {
        const float2 amount = bc2(p.sharpen);
        float2 o[4];
        sharpen_row1(m.R, r, uc, amount, o);
#pragma unroll
        for (int i = 0; i < 4; ++i) rgb[i][0] = o[i];
        sharpen_row1(m.G, r, uc, amount, o);
#pragma unroll
        for (int i = 0; i < 4; ++i) rgb[i][1] = o[i];
        sharpen_row1(m.B, r, uc, amount, o);
#pragma unroll
        for (int i = 0; i < 4; ++i) rgb[i][2] = o[i];
      } else {
        if (r & 1) {
          demosaic_row4<kMalvar, kPat, 1>(m.P, r, uc, rgb);
        } else {
          demosaic_row4<kMalvar, kPat, 0>(m.P, r, uc, rgb);
        }
        if (f.swap_rb) {
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float2 red = rgb[i][0];
            rgb[i][0] = rgb[i][2];
            rgb[i][2] = red;
          }
        }
      }
      finish_row<kOutSel, kLutSmem>(p, f, m.hist, rgb, x0 + 4 * uc, y0 + r, sums, npix);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) acc[k] += sums[k] - npix * kTwo23Bits;  // mod 2^32: the true sum
  __syncthreads();  // the next tile overwrites the tables, P and the planes
}

// The main pass's flush of one frame by one CTA, after it processed
// `tiles_done` of the frame's `tiles_total` tiles: block sums and histogram
// into the frame's scratch; the CTA that completes the frame's tile count
// writes the user's histogram and statistics and clears the scratch (and
// the tile claims of the single-frame pass). `red` holds 4 x kWarps values.
__device__ void flush_frame(const FrameDesc& p, const FrameSetup& f, const u64 (&acc)[4], Span<unsigned int> hist,
                            u64* red, bool* last, unsigned int tiles_done, unsigned int tiles_total) {
  Span<Scratch> sc = p.scratch;
  const int tid = threadIdx.x;
  if (!f.want_stats && !f.want_hist) {
    // Nothing to finish, but the last CTA still clears the counters.
    __syncthreads();
    if (tid == 0 && atomicAdd(&sc->main_done, tiles_done) + tiles_done == tiles_total) {
      sc->main_done = 0;
      sc->tile_next = 0;
    }
    return;
  }
  if (f.want_stats) {
    u64 total[4];
    block_sum4(acc, red, total);
    if (tid < 4 && total[tid] != 0) atomicAdd(tid < 3 ? &sc->sum[tid] : &sc->saturated, total[tid]);
  }
  if (f.want_hist) {
    __syncthreads();
    // Two bins per 64-bit atomic: a bin's count over a frame stays below
    // 2^32, so no carry crosses into its neighbour.
    static_assert(offsetof(Scratch, hist) % 8 == 0, "histogram pairs are 8-byte aligned");
    const Span<unsigned long long> pairs =
        span_cast<unsigned long long>(sub_span(sc, &sc->hist[0], kHistChannels * kHistBins));
    for (int i = tid; i < kHistChannels * kHistBins / 2; i += kThreads) {
      const uint2 h = span_cast<const uint2>(hist)[i];
      if ((h.x | h.y) != 0U) atomicAdd(&pairs[i], (static_cast<unsigned long long>(h.y) << 32) | h.x);
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) *last = atomicAdd(&sc->main_done, tiles_done) + tiles_done == tiles_total;
  __syncthreads();
  if (!*last) return;
  __threadfence();
  if (f.want_hist) {
    const Span<unsigned int> bins = sub_span(sc, &sc->hist[0], kHistChannels * kHistBins);
    for (int i = tid; i < kHistChannels * kHistBins; i += kThreads) {
      p.hist_out[i] = __ldcg(&bins[i]);
      bins[i] = 0U;
    }
  }
  if (f.want_stats && tid == 0) {
    const u64 sum[3] = {__ldcg(&sc->sum[0]), __ldcg(&sc->sum[1]), __ldcg(&sc->sum[2])};
    finish_stats(p, sum, __ldcg(&sc->saturated), f.gains);
    sc->sum[0] = sc->sum[1] = sc->sum[2] = 0;
    sc->saturated = 0;
  }
  if (tid == 0) {
    sc->main_done = 0;
    sc->tile_next = 0;
  }
}

template <bool kMalvar, bool kSharpen, int kLayout, bool kLutSmem, int kOut, int kTileH>
__global__ void __launch_bounds__(kThreads, kTileH == kTH ? 2 : 3)
    isp_main_kernel(const __grid_constant__ CUtensorMap map, FrameDesc p, int tiles_x, int tiles, int use_tma,
                    int lut_in_smem) {
  using G = Geom<kSharpen, kTileH>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128U - (smem_u32(smem_raw) & 127U)) & 127U);
  const int box_bytes = box_row_bytes(p.raw_format);
  const TileSmem m =
      carve(smem, layout_of(kSharpen, box_bytes, kLutSmem ? p.tone_size : 0, kTileH), G::kSH, span_rec(p.scratch));
  __shared__ uint64_t bar;
  __shared__ u64 red[4 * kWarps];
  __shared__ int minmax[2];
  __shared__ int next_tile;
  __shared__ bool last;
  static_cast<void>(lut_in_smem);

  const int fmt = p.raw_format;
  const auto issue = [&](int t) {
    const int ty = t / tiles_x;
    const int x0 = (t - ty * tiles_x) * kTW;
    tma_load_2d(&map, m.box, &bar, box_x(fmt, x0), ty * kTileH - G::kHalo, static_cast<unsigned int>(G::kSH * box_bytes));
  };
  // The first tile's box reads only the input frame: it is requested before
  // the wait below (the barrier initialised and made visible to the copy
  // engine first; the other threads meet it after the block barrier).
  if (use_tma && threadIdx.x == 0) {
    mbar_init(&bar);
    fence_async_shared();
    if (static_cast<int>(blockIdx.x) < tiles) issue(blockIdx.x);
  }
  fill_frame_smem<kLutSmem>(p, m);
  // The frame's set-up waits for the statistics pass (its gains); the first
  // tile's lens shading maps and table read only the pipeline's own grid, so
  // they are built before that wait (run_tile calls wait_frame after them).
  FrameSetup f;
  f.grid = frame_grid(p, m);
  cp_async_wait_all();
  __syncthreads();
  bool waited = false;
  const auto wait_frame = [&] {
    if (waited) return;
    // Launched as a programmatic dependent of the statistics pass, this
    // kernel becomes resident on the SMs that pass leaves while it finishes;
    // the wait returns once the pass has completed and its writes (the gains
    // that setup_frame reads) are visible. Without a programmatic launch it
    // returns at once.
    griddep_wait();
    // The next frame's statistics pass may launch now (when queued right
    // behind this kernel): it sums its own raw frame on the SMs this pass
    // leaves as it finishes, and waits for this pass's completion before its
    // estimate touches the white balance state read here.
    griddep_launch_dependents();
    f = setup_frame<kLutSmem, false>(p, m);
    waited = true;
  };

  u64 acc[4] = {0, 0, 0, 0};  // linear R, G, B in 2^-20 units; saturated samples
  uint32_t phase = 0;
  unsigned int done = 0;
  // Tiles are claimed as CTAs free up: the first per CTA is its index, the
  // rest come from the frame's counter, so CTAs that meet slower tiles
  // (edges, mirrored borders) take fewer and all finish together.
  int tile = blockIdx.x;
  while (tile < tiles) {
    const int ty = tile / tiles_x;
    const int x0 = (tile - ty * tiles_x) * kTW;
    // The CTA's next tile. With sharpening it is claimed once this tile's
    // box is free (after phase A) and its box requested before phase C (the
    // claim's round trip hidden behind phase B, the copy behind phase C), so
    // that claims are made as late as the box allows and the frame's last
    // tiles go to the CTAs that are free first; without sharpening (no phase
    // B) it is claimed at the tile's start and its box requested after A.
    unsigned int claim = 0;
    if (!kSharpen && threadIdx.x == 0) claim = gridDim.x + atomicAdd(&p.scratch->tile_next, 1U);
    const auto request = [&] {
      if (threadIdx.x == 0) {
        next_tile = static_cast<int>(claim);
        if (use_tma && static_cast<int>(claim) < tiles) {
          fence_async_shared();
          issue(static_cast<int>(claim));
        }
      }
    };
    const auto after_a = [&] {
      if constexpr (kSharpen) {
        if (threadIdx.x == 0) claim = gridDim.x + atomicAdd(&p.scratch->tile_next, 1U);
      } else {
        request();
      }
    };
    const auto before_c = [&] {
      if constexpr (kSharpen) request();
    };
    run_tile<kMalvar, kSharpen, kLayout, kLutSmem, decltype(after_a), kOut, kTileH, decltype(before_c),
             decltype(wait_frame)>(p, f, m, minmax, x0, ty * kTileH, use_tma != 0, &bar, phase, acc, after_a, before_c,
                                   wait_frame);
    ++done;
    tile = next_tile;  // written before run_tile's closing barrier
  }
  wait_frame();  // a CTA without a tile still takes part in the flush
  flush_frame(p, f, acc, m.hist, red, &last, done, static_cast<unsigned int>(tiles));
}

template <bool kMalvar, bool kSharpen, int kOut, int kTileH>
const void* main_instance_out(int layout, bool lut_smem) {
  if (layout == 0) {
    return lut_smem ? reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, 0, true, kOut, kTileH>)
                    : reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, 0, false, kOut, kTileH>);
  }
  return lut_smem ? reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, 1, true, kOut, kTileH>)
                  : reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, 1, false, kOut, kTileH>);
}

// The tile kernel of one tile height for a layout, tone-table placement and
// output format (one instance per format, so that each holds only its own
// store code).
template <bool kMalvar, bool kSharpen, int kTileH>
const void* main_instance(int layout, bool lut_smem, int out_format) {
  switch (out_format) {
    case kOutRgb8: return main_instance_out<kMalvar, kSharpen, kOutRgb8, kTileH>(layout, lut_smem);
    case kOutRgba8: return main_instance_out<kMalvar, kSharpen, kOutRgba8, kTileH>(layout, lut_smem);
    case kOutRgb16: return main_instance_out<kMalvar, kSharpen, kOutRgb16, kTileH>(layout, lut_smem);
    default: return main_instance_out<kMalvar, kSharpen, kOutRgb32f, kTileH>(layout, lut_smem);
  }
}

}  // namespace
}  // namespace isp_b200
