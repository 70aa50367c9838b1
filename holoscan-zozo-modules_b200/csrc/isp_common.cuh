// isp_common.cuh - device building blocks shared by the ISP's kernels: tile
// geometry and shared-memory layout, TMA and mbarrier helpers, raw unpacking,
// lens shading tables, stores, block reductions and the last-CTA finishers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "isp_device.cuh"
#include "isp_kernels.cuh"
#include "isp_ops.cuh"

namespace isp_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTW = 64;  // tile: output pixels across
constexpr int kTH = 64;  // and down
constexpr int kSW = 72;  // samples per tile row: x0 - 4 .. x0 + 67
constexpr int kUnitsRow = kSW / 4;
constexpr unsigned int kWaitLimit = 1U << 22;  // bounded mbarrier polls
// Grid rows a tile's lens shading table holds; tiles that need more compute
// each gain from the grid directly.
constexpr int kLscTableRows = 8;

// The channel (kChR, kChGr, kChGb, kChB) at quad position (y & 1) * 2 + (x & 1)
// of each Bayer pattern, packed two bits per entry so that a run-time lookup
// is a shift (a constant array indexed at run time would live in local memory).
__host__ __device__ constexpr unsigned int cfa_word() {
  constexpr int t[4][4] = {{kChR, kChGr, kChGb, kChB},
                           {kChB, kChGb, kChGr, kChR},
                           {kChGr, kChR, kChB, kChGb},
                           {kChGb, kChB, kChR, kChGr}};
  unsigned int w = 0;
  for (int p = 0; p < 4; ++p) {
    for (int q = 0; q < 4; ++q) w |= static_cast<unsigned int>(t[p][q]) << (8 * p + 2 * q);
  }
  return w;
}
constexpr unsigned int kCfaWord = cfa_word();
__host__ __device__ constexpr int cfa_of(int pattern, int pos) {
  return static_cast<int>((kCfaWord >> (8 * pattern + 2 * pos)) & 3U);
}
static_assert(cfa_of(0, 0) == kChR && cfa_of(1, 3) == kChR && cfa_of(2, 1) == kChR && cfa_of(3, 2) == kChR &&
                  cfa_of(2, 0) == kChGr && cfa_of(3, 1) == kChB && cfa_of(1, 1) == kChGb,
              "Bayer channel table");

// Lens shading grids of at most this many gains are kept in shared memory
// for the frame (a 17 x 13 x 4 grid is 884).
constexpr int kGridSmemGains = 1024;

// Paired pixels. The tile pass computes two pixels in the two lanes of every
// f32x2 operation: columns c and c + kHalf of the same row, which have the
// same Bayer colour and so the same arithmetic. Samples and RGB values live
// in shared memory as float2 pairs {v(c), v(c + kHalf)}, so that each operand
// is one aligned 8-byte element and neighbours are neighbouring pairs.
constexpr int kHalf = 32;
// Paired sample columns: pair s (0..39) holds tile samples s and s + 32
// (sample s is image column x0 - 4 + s).
constexpr int kPW = 40;
// Paired RGB columns (sharpening): pair q (0..33) holds pixels q - 1 and q + 31.
constexpr int kCW2 = 34;

// Tile heights the kernels are compiled for: kTH rows (the default) or
// kTHShort rows (more, smaller tiles: a frame of few tiles spreads over more
// SMs, and three CTAs share an SM).
constexpr int kTHShort = 32;

template <bool kSharpen, int kTileH = kTH>
struct Geom {
  static constexpr int kHalo = kSharpen ? 4 : 2;  // sample rows above and below the tile
  static constexpr int kSH = kTileH + 2 * kHalo;
  static constexpr int kCH = kTileH + 2;  // RGB rows: y0 - 1 .. y0 + kTileH
};

// ---- Shared memory layout -------------------------------------------------

struct Layout {
  int raw;      // TMA box: box rows x box bytes
  int samples;  // float2 [kSH][kPW]
  int r, g, b;  // float2 [kCH][kCW2] each (sharpening)
  int lsc;      // float2 [kLscTableRows][2][kPW]
  int cols;     // int col_mx[kSW]; int col_ix[kSW]; float col_tx[kSW]
  int rows;     // int row_my[kSH]; int row_k[kSH]; float row_ty[kSH]
  int hist;     // u32 [4][256]
  int grid;     // float [kGridSmemGains]: the frame's lens shading grid, when it fits
  int lut;      // float2 [tone_size] when in shared memory
  int total;
};

__host__ __device__ constexpr int align128(int v) { return (v + 127) & ~127; }

__host__ __device__ constexpr Layout layout_of(bool sharpen, int box_bytes_row, int lut_entries, int tile_h = kTH) {
  const int halo = sharpen ? 4 : 2;
  const int sh = tile_h + 2 * halo;
  const int plane = align128((tile_h + 2) * kCW2 * 8);
  Layout l{};
  int o = 0;
  l.raw = o;
  o = align128(o + sh * box_bytes_row);
  l.samples = o;
  o = align128(o + sh * kPW * 8);
  l.r = o;
  l.g = o + (sharpen ? plane : 0);
  l.b = o + (sharpen ? 2 * plane : 0);
  if (sharpen) o += 3 * plane;
  l.lsc = o;
  o = align128(o + kLscTableRows * 2 * kPW * 8);
  l.cols = o;
  o = align128(o + 3 * kSW * 4);
  l.rows = o;
  o = align128(o + 3 * sh * 4);
  l.hist = o;
  o = align128(o + kHistChannels * kHistBins * 4);
  l.grid = o;
  o = align128(o + kGridSmemGains * 4);
  l.lut = o;
  o = align128(o + lut_entries * 8);
  l.total = o;
  return l;
}

// Bytes per box row of each raw format (TMA inner extent, multiple of 16),
// and the byte of the box row where sample x0 - 4 starts.
__host__ __device__ constexpr int box_row_bytes(int fmt) {
  return fmt == kRawU8 ? 96 : fmt == kRawU16 ? 160 : fmt == kRawRaw10 ? 112 : 128;
}

// ---- Programmatic dependent launch ------------------------------------------

// Lets the grid launched after this one (as a programmatic dependent) start
// before this grid finishes.
__device__ __forceinline__ void griddep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Waits until the grid this one depends on has completed and its memory
// writes are visible; returns at once when there is no such dependency.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---- TMA and mbarrier -----------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Requests a box of `bytes` bytes into dst, completing on bar. (The checked
// build makes no copy whose box would leave dst's region: it arrives on the
// barrier without one, so that the wait still ends.)
__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, Span<uint8_t> dst, uint64_t* bar, int x, int y,
                                            unsigned int bytes) {
#ifdef ISP_CHECKED
  if (span_range(dst, bytes) != span_ptr(dst)) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
    return;
  }
#endif
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_u32(span_ptr(dst))),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Waits for the barrier's phase `parity` to complete; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned int limit = kWaitLimit) {
  for (unsigned int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// A bounded wait gave up: the frame's outputs are not trustworthy. The flag
// stays set until isp_b200_device_status reads and clears it.
__device__ __forceinline__ void report_wait_timeout(Span<Scratch> s) { atomicExch(&s->error, 1); }

__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Copies of 4 or 8 bytes from global to shared memory that bypass the
// registers: a thread's copies are all in flight at once (a fill loop of
// plain loads and stores waits out one L2 round trip per iteration), and
// cp_async_wait_all() returns once this thread's copies have landed.
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
#ifdef ISP_CHECKED
  if (!__isShared(dst)) {  // a refused destination: the check's sink in global memory
    *static_cast<uint32_t*>(dst) = *static_cast<const uint32_t*>(src);
    return;
  }
#endif
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(__cvta_generic_to_global(src))
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
#ifdef ISP_CHECKED
  if (!__isShared(dst)) {
    *static_cast<uint2*>(dst) = *static_cast<const uint2*>(src);
    return;
  }
#endif
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(__cvta_generic_to_global(src))
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The TMA coordinates of the box for a tile at (x0, y0) (x in the tensor's
// elements: bytes, or uint16 samples), 16-byte aligned for any x0 % 64 == 0.
__device__ __forceinline__ int box_x(int fmt, int x0) {
  return fmt == kRawU8 ? x0 - 16 : fmt == kRawU16 ? x0 - 8 : fmt == kRawRaw10 ? 5 * (x0 >> 2) - 16 : 3 * (x0 >> 1) - 16;
}

// ---- Raw unpacking from a box row ----------------------------------------

// Samples x0 - 4 + 4u .. + 3 of a box row (box starting at box_x(fmt, x0)).
__device__ __forceinline__ void unpack4(int fmt, Span<const uint8_t> row, int u, unsigned int s[4]) {
  if (fmt == kRawU8) {
    const unsigned int w = *span_cast<const unsigned int>(row + 12 + 4 * u);
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k] = (w >> (8 * k)) & 0xFFU;
  } else if (fmt == kRawU16) {
    const uint2 w = *span_cast<const uint2>(row + 8 + 8 * u);
    s[0] = w.x & 0xFFFFU;
    s[1] = w.x >> 16;
    s[2] = w.y & 0xFFFFU;
    s[3] = w.y >> 16;
  } else if (fmt == kRawRaw10) {
    // Group g0 - 1 + u at byte 11 + 5u: four high bytes, then the low bits.
    const int b = 11 + 5 * u;
    Span<const unsigned int> w = span_cast<const unsigned int>(row + (b & ~3));
    const unsigned int sh = 8U * static_cast<unsigned int>(b & 3);
    const unsigned int hi4 = __funnelshift_r(w[0], w[1], sh);
    const unsigned int lo = (w[1] >> sh) & 0xFFU;
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k] = (((hi4 >> (8 * k)) & 0xFFU) << 2) | ((lo >> (2 * k)) & 3U);
  } else {
    // Two groups of three bytes at byte 10 + 6u.
    const int b = 10 + 6 * u;
    Span<const unsigned int> w = span_cast<const unsigned int>(row + (b & ~3));
    const unsigned int sh = 8U * static_cast<unsigned int>(b & 3);
    const unsigned int v0 = __funnelshift_r(w[0], w[1], sh);  // a0 a1 a2 b0
    const unsigned int v1 = w[1] >> sh;                        // b1 b2 ..
    const unsigned int a2 = (v0 >> 16) & 0xFFU;
    const unsigned int b2 = (v1 >> 8) & 0xFFU;
    s[0] = ((v0 & 0xFFU) << 4) | (a2 & 15U);
    s[1] = (((v0 >> 8) & 0xFFU) << 4) | (a2 >> 4);
    s[2] = ((v0 >> 24) << 4) | (b2 & 15U);
    s[3] = ((v1 & 0xFFU) << 4) | (b2 >> 4);
  }
}

// One sample at image column mx of a box row (box starting at box_x(fmt, x0)).
__device__ __forceinline__ unsigned int unpack1(int fmt, Span<const uint8_t> row, int mx, int x0) {
  if (fmt == kRawU8) return row[mx - x0 + 16];
  if (fmt == kRawU16) return *span_cast<const uint16_t>(row + 2 * (mx - x0 + 8));
  if (fmt == kRawRaw10) {
    Span<const uint8_t> g = row + 5 * ((mx >> 2) - (x0 >> 2)) + 16;
    const int k = mx & 3;
    return (static_cast<unsigned int>(g[k]) << 2) | ((g[4] >> (2 * k)) & 3U);
  }
  Span<const uint8_t> g = row + 3 * ((mx >> 1) - (x0 >> 1)) + 16;
  const int k = mx & 1;
  return (static_cast<unsigned int>(g[k]) << 4) | ((g[2] >> (4 * k)) & 15U);
}

// ---- Lens shading tables --------------------------------------------------

// Per tile: for every column the grid cell and fraction across, for every
// row the cell and fraction down, and the interpolated "top" rows
//   T[k][parity][i] = g(iy0 + k, ix_i) + (g(iy0 + k, ix_i + 1) - g(iy0 + k, ix_i)) * tx_i
// for the grid rows iy0 .. iy0 + K - 1 the tile's rows use, so that a
// sample's gain is T[k] + (T[k + 1] - T[k]) * ty: the reference's
// top + (bottom - top) * ty (isp_math.hpp:121-140), same operands, same order.
struct LscTile {
  int iy0;
  int rows;  // K; 0 when there is no grid, > kLscTableRows when the table does not fit
};

// Fills the column and row maps (mirrored coordinates, grid cells) and, when
// it fits, the table. Threads 0..ncols-1 do columns, the next nrows do rows.
// kPaired: the table holds float2 pairs {T(s), T(s + kHalf)} for s < kPW
// (the tile pass's paired columns); otherwise one float per column.
// `grid`: the frame's lens shading gains (the frame's own, or a copy in
// shared memory).
template <bool kPaired = false>
__device__ LscTile build_lsc(const FrameDesc& p, Span<const float> grid, int pattern, int x_first, int ncols, int y_first,
                             int nrows,
                             bool mirror_xy, int xclamp, int yclamp, Span<int> col_mx, Span<int> col_ix, Span<float> col_tx,
                             Span<int> row_my, Span<int> row_k, Span<float> row_ty, Span<float> table, int* minmax) {
  const int t = threadIdx.x;
  if (t == 0) {
    minmax[0] = 0x7FFFFFFF;
    minmax[1] = -1;
  }
  int iy_lo = 0x7FFFFFFF;  // this thread's row's grid row, if it has one
  int iy_hi = -1;
  __syncthreads();
  if (t < ncols) {
    int x = x_first + t;
    if (mirror_xy) x = mirror(x < xclamp ? x : xclamp, p.width);
    col_mx[t] = x;
    if (p.lsc != nullptr) {
      const float fx = static_cast<float>(x) * p.lsc_sx;
      int ix = static_cast<int>(fx);
      ix = ix > p.lsc_width - 2 ? p.lsc_width - 2 : ix;
      col_ix[t] = ix;
      col_tx[t] = fx - static_cast<float>(ix);
    }
  } else if (t < ncols + nrows) {
    const int j = t - ncols;
    int y = y_first + j;
    if (mirror_xy) y = mirror(y < yclamp ? y : yclamp, p.height);
    row_my[j] = y;
    if (p.lsc != nullptr) {
      const float fy = static_cast<float>(y) * p.lsc_sy;
      int iy = static_cast<int>(fy);
      iy = iy > p.lsc_height - 2 ? p.lsc_height - 2 : iy;
      row_k[j] = iy;
      row_ty[j] = fy - static_cast<float>(iy);
      iy_lo = iy;
      iy_hi = iy;
    }
  }
  // The rows' grid range: a warp reduction, then one shared atomic per warp
  // (same-address shared atomics from every row thread would serialise).
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
  const auto entry = [&](int k, int par, int i) {
    const int ch = step == 4 ? cfa_of(pattern, (par << 1) | (col_mx[i] & 1)) : 0;
    Span<const float> g = grid + ((lt.iy0 + k) * p.lsc_width + col_ix[i]) * step + ch;
    return g[0] + (g[step] - g[0]) * col_tx[i];
  };
  if constexpr (kPaired) {
    Span<float2> table2 = span_cast<float2>(table);
    for (int e = t; e < lt.rows * planes * kPW; e += kThreads) {
      const int i = e % kPW;
      const int kp = e / kPW;
      const int par = kp % planes;
      const int k = kp / planes;
      table2[(k * 2 + par) * kPW + i] = make_float2(entry(k, par, i), entry(k, par, i + kHalf));
    }
  } else {
    for (int e = t; e < lt.rows * planes * ncols; e += kThreads) {
      const int i = e % ncols;
      const int kp = e / ncols;
      const int par = kp % planes;
      const int k = kp / planes;
      table[(k * 2 + par) * kSW + i] = entry(k, par, i);
    }
  }
  if (t < nrows) row_k[t] -= lt.iy0;
  __syncthreads();
  return lt;
}

// build_lsc<true> for a tile none of whose rows and columns is mirrored:
// the grid rows it spans follow from its first and last rows (a row's grid
// cell never decreases down the frame), so the row maps and the paired table
// are written in one pass behind one block barrier, each table entry working
// out its own column's cell (the same operations as build_lsc's column maps).
// Tiles whose table would not fit take build_lsc<true>. Of the column maps
// only the columns themselves are written (the path of phase A without a TMA
// box reads them); the cells are worked out where the table needs them.
__device__ LscTile build_lsc_inner(const FrameDesc& p, Span<const float> grid, int pattern, int x_first, int y_first,
                                   int nrows, Span<int> col_mx, Span<int> col_ix, Span<float> col_tx, Span<int> row_my, Span<int> row_k,
                                   Span<float> row_ty, Span<float> table, int* minmax) {
  LscTile lt{0, 0};
  const int t = threadIdx.x;
  if (p.lsc == nullptr) {
    if (t < kSW) col_mx[t] = x_first + t;
    if (t < nrows) row_my[t] = y_first + t;
    __syncthreads();
    return lt;
  }
  const auto row_cell = [&](int y) {
    const int iy = static_cast<int>(static_cast<float>(y) * p.lsc_sy);
    return iy > p.lsc_height - 2 ? p.lsc_height - 2 : iy;
  };
  lt.iy0 = row_cell(y_first);
  lt.rows = row_cell(y_first + nrows - 1) - lt.iy0 + 2;
  if (lt.rows > kLscTableRows) {
    return build_lsc<true>(p, grid, pattern, x_first, kSW, y_first, nrows, false, 0, 0, col_mx, col_ix, col_tx, row_my,
                           row_k, row_ty, table, minmax);
  }
  if (t < kSW) col_mx[t] = x_first + t;
  if (t < nrows) {
    const int y = y_first + t;
    row_my[t] = y;
    const float fy = static_cast<float>(y) * p.lsc_sy;
    int iy = static_cast<int>(fy);
    iy = iy > p.lsc_height - 2 ? p.lsc_height - 2 : iy;
    row_k[t] = iy - lt.iy0;
    row_ty[t] = fy - static_cast<float>(iy);
  }
  const int step = p.lsc_channels;
  const int planes = step == 4 ? 2 : 1;
  const auto entry = [&](int k, int par, int i) {
    const int x = x_first + i;
    const float fx = static_cast<float>(x) * p.lsc_sx;
    int ix = static_cast<int>(fx);
    ix = ix > p.lsc_width - 2 ? p.lsc_width - 2 : ix;
    const float tx = fx - static_cast<float>(ix);
    const int ch = step == 4 ? cfa_of(pattern, (par << 1) | (x & 1)) : 0;
    Span<const float> g = grid + ((lt.iy0 + k) * p.lsc_width + ix) * step + ch;
    return g[0] + (g[step] - g[0]) * tx;
  };
  Span<float2> table2 = span_cast<float2>(table);
  for (int e = t; e < lt.rows * planes * kPW; e += kThreads) {
    const int i = e % kPW;
    const int kp = e / kPW;
    const int par = kp % planes;
    const int k = kp / planes;
    table2[(k * 2 + par) * kPW + i] = make_float2(entry(k, par, i), entry(k, par, i + kHalf));
  }
  __syncthreads();
  return lt;
}

__device__ __forceinline__ u64 warp_sum(u64 v) {
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) v += __shfl_down_sync(0xFFFFFFFFU, v, offset);
  return v;
}

// Sum of one u64 per thread over the block; the result in every thread.
__device__ u64 block_sum(u64 v, u64* red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  u64 total = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) total += red[w];
  return total;
}

// Sums of four u64 per thread over the block, in `out` of thread 0; `red`
// holds 4 x kWarps values.
__device__ __forceinline__ void block_sum4(const u64 (&v)[4], u64* red, u64 (&out)[4]) {
  u64 w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) w[k] = warp_sum(v[k]);
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) red[k * kWarps + (threadIdx.x >> 5)] = w[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    u64 total = 0;
#pragma unroll
    for (int i = 0; i < kWarps; ++i) total += red[k * kWarps + i];
    out[k] = total;
  }
}

// Exclusive prefix sum of one u64 per thread over the block.
__device__ u64 block_exclusive_scan(u64 v, u64* red) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  u64 inc = v;
#pragma unroll
  for (int offset = 1; offset < 32; offset <<= 1) {
    const u64 up = __shfl_up_sync(0xFFFFFFFFU, inc, offset);
    if (lane >= offset) inc += up;
  }
  __syncthreads();
  if (lane == 31) red[warp] = inc;
  __syncthreads();
  u64 before = 0;
  for (int w = 0; w < warp; ++w) before += red[w];
  return before + inc - v;
}

// histogram_percentile (isp_math.hpp:336-352) by the whole block: thread t
// owns bins 4t..4t+3; the prefix counts are exact integers, so every
// comparison is the reference's.
__device__ float block_percentile(Span<const unsigned int> hist, float percentile, u64* red, int* first) {
  const int t = threadIdx.x;
  unsigned int h[4];
  u64 mine = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    h[k] = __ldcg(&hist[4 * t + k]);
    mine += h[k];
  }
  const u64 total = block_sum(mine, red);
  if (total == 0) return 0.0F;
  const u64 below0 = block_exclusive_scan(mine, red);
  const double target = static_cast<double>(percentile) * static_cast<double>(total);
  if (t == 0) *first = kAwbBins;
  __syncthreads();
  u64 below = below0;
  int mine_first = kAwbBins;
  u64 mine_below = 0;
  unsigned int mine_count = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (mine_first == kAwbBins && h[k] != 0U && static_cast<double>(below + h[k]) >= target) {
      mine_first = 4 * t + k;
      mine_below = below;
      mine_count = h[k];
    }
    below += h[k];
  }
  if (mine_first < kAwbBins) atomicMin(first, mine_first);
  __syncthreads();
  const int b = *first;
  __shared__ float result;
  if (b == kAwbBins) {
    if (t == 0) result = 1.0F;
  } else if (mine_first == b) {
    const double within = (target - static_cast<double>(mine_below)) / static_cast<double>(mine_count);
    result = static_cast<float>((static_cast<double>(b) + within) / kAwbBins);
  }
  __syncthreads();
  const float r = result;
  __syncthreads();
  return r;
}

// finish_white_balance (isp_math.hpp:357-384) in the statistics pass's last
// CTA; then the sums are cleared for the next frame.
__device__ void awb_finish(const FrameDesc& p, Span<Scratch> s, u64* red, int* first) {
  const u64 nquads = __ldcg(&s->awb_quads);
  float level[3] = {0.0F, 0.0F, 0.0F};
  if (nquads != 0) {
    if (p.awb_mode == kWbGrayWorld) {
      const double q = static_cast<double>(nquads);
      level[0] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[0])) / q);
      level[1] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[1])) / (2.0 * q));
      level[2] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[2])) / q);
    } else {
      for (int k = 0; k < 3; ++k) level[k] = block_percentile(sub_span(s, &s->awb_hist[k][0], kAwbBins), p.awb_percentile, red, first);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && nquads != 0 && level[0] > 0.0F && level[1] > 0.0F && level[2] > 0.0F) {
    const float target[3] = {level[1] / level[0], 1.0F, level[1] / level[2]};
    const bool smooth = s->awb_valid != 0 && p.awb_smoothing < 1.0F;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float t = target[k] < 0.0625F ? 0.0625F : target[k] > 16.0F ? 16.0F : target[k];
      const float g = s->awb_gains[k];
      s->awb_gains[k] = smooth ? g + p.awb_smoothing * (t - g) : t;
    }
    s->awb_valid = 1;
  }
  const Span<unsigned int> bins = sub_span(s, &s->awb_hist[0][0], 3 * kAwbBins);
  for (int i = threadIdx.x; i < 3 * kAwbBins; i += kThreads) bins[i] = 0U;
  if (threadIdx.x < 3) s->awb_sum[threadIdx.x] = 0;
  if (threadIdx.x == 3) s->awb_quads = 0;
  if (threadIdx.x == 4) s->awb_done = 0;
}

// finish_stats (isp_math.hpp:387-425) from the main pass's sums.
__device__ void finish_stats(const FrameDesc& p, const u64 sum[3], u64 saturated, const float gains[3]) {
  const int64_t pixels = static_cast<int64_t>(p.width) * p.height;
  const double n = static_cast<double>(pixels) * static_cast<double>(kFixedOne);
  const double mean[3] = {static_cast<double>(sum[0]) / n, static_cast<double>(sum[1]) / n,
                          static_cast<double>(sum[2]) / n};
  const double luma = 0.2126 * mean[0] + 0.7152 * mean[1] + 0.0722 * mean[2];
  double error = luma > 0.0 ? log2(static_cast<double>(p.ae.target) / luma) : 8.0;
  error = error < -8.0 ? -8.0 : error > 8.0 ? 8.0 : error;
  const double scale = exp2(static_cast<double>(p.ae.damping) * error);
  double next_exposure = 0.0;
  double next_gain = 0.0;
  if (p.exposure_ns > 0) {
    const double gain = p.exposure_gain > 0.0F ? p.exposure_gain : p.ae.min_gain;
    const double wanted = static_cast<double>(p.exposure_ns) * gain * scale;
    next_exposure = wanted / p.ae.min_gain;
    const double low = static_cast<double>(p.ae.min_exposure_ns);
    const double high = static_cast<double>(p.ae.max_exposure_ns);
    next_exposure = next_exposure < low ? low : next_exposure > high ? high : next_exposure;
    next_gain = wanted / next_exposure;
    next_gain = next_gain < p.ae.min_gain ? p.ae.min_gain : next_gain > p.ae.max_gain ? p.ae.max_gain : next_gain;
  }
  Span<float> out = p.stats_out;
  out[0] = static_cast<float>(mean[0]);
  out[1] = static_cast<float>(mean[1]);
  out[2] = static_cast<float>(mean[2]);
  out[3] = static_cast<float>(luma);
  out[4] = static_cast<float>(error);
  out[5] = static_cast<float>(scale);
  out[6] = static_cast<float>(next_exposure);
  out[7] = static_cast<float>(next_gain);
  out[8] = gains[0];
  out[9] = gains[1];
  out[10] = gains[2];
  out[11] = static_cast<float>(static_cast<double>(saturated) / static_cast<double>(pixels));
}

// ---- The fused tile pass --------------------------------------------------

// Per-tile state the phases share.
struct TileCtx {
  int x0, y0;
  Span<const uint8_t> box;
  Span<const int> col_mx;
  Span<const int> row_my;
  Span<const int> row_k;
  Span<const float> row_ty;
  Span<const float2> table;  // paired lens shading table
  Span<const float> grid;     // the frame's lens shading gains
  LscTile lt;
};

}  // namespace
}  // namespace isp_b200
