// isp_kernels.cu - the sm_100a kernels of the B200 ISP, one frame at a time.
//
// A frame is one or two launches on the caller's stream:
//   isp_awb_kernel   (gray world / white patch only) the white balance
//                    statistics over complete 2x2 quads of 64x64-sample
//                    tiles, block-privatised, then, in the last CTA to
//                    finish, the frame's estimate (finish_white_balance);
//   isp_main_kernel  persistent CTAs over 64x64-pixel tiles:
//                    A. the raw tile and its halo arrive in shared memory by
//                       TMA (cp.async.bulk.tensor, prefetched during the
//                       previous tile's phases B and C), are unpacked four
//                       samples at a time and preprocessed (black level,
//                       lens shading from a per-tile table, white balance);
//                    B. (sharpening) RGB of the tile and a one-pixel ring;
//                    C. per 2x4 pixels: sharpen or demosaic, colour matrix,
//                       statistics sums, tone curve, store, histogram codes;
//                    the last CTA writes the histogram and the statistics.
// The reference issues up to five kernels and three memsets per frame
// (modules/isp/src/cuda_pipeline.cu:294-364); these accumulators clear
// themselves, so no memset is needed.
//
// Edges: the reference reflects coordinates about the first and last sample
// (isp_math.hpp:82-91). Tiles touching an edge map every sample position
// through mirror() into the TMA box, which always holds the reflected
// samples a valid output needs; positions no output needs are clamped into
// the box.
#include <cuda.h>
#include <cuda_runtime.h>

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

// The channel (kChR, kChGr, kChGb, kChB) at quad position (y & 1) * 2 + (x & 1).
__host__ __device__ constexpr int cfa_of(int pattern, int pos) {
  constexpr int t[4][4] = {{kChR, kChGr, kChGb, kChB},
                           {kChB, kChGb, kChGr, kChR},
                           {kChGr, kChR, kChB, kChGb},
                           {kChGb, kChB, kChR, kChGr}};
  return t[pattern][pos];
}

template <bool kSharpen>
struct Geom {
  static constexpr int kHalo = kSharpen ? 4 : 2;  // sample rows above and below the tile
  static constexpr int kSH = kTH + 2 * kHalo;
  static constexpr int kCW = 68;  // RGB planes: x0 - 1 .. x0 + 64, padded
  static constexpr int kCH = kTH + 2;
};

// ---- Shared memory layout -------------------------------------------------

struct Layout {
  int raw;      // TMA box: box rows x box bytes
  int samples;  // float [kSH][kSW]
  int rg;       // float2 [kCH][kCW] (sharpening)
  int b;        // float [kCH][kCW] (sharpening)
  int lsc;      // float [kLscTableRows][2][kSW]
  int cols;     // int col_mx[kSW]; int col_ix[kSW]; float col_tx[kSW]
  int rows;     // int row_my[kSH]; int row_k[kSH]; float row_ty[kSH]
  int hist;     // u32 [4][256]
  int lut;      // float2 [tone_size] when in shared memory
  int total;
};

__host__ __device__ constexpr int align128(int v) { return (v + 127) & ~127; }

__host__ __device__ constexpr Layout layout_of(bool sharpen, int box_bytes_row, int lut_entries) {
  const int halo = sharpen ? 4 : 2;
  const int sh = kTH + 2 * halo;
  Layout l{};
  int o = 0;
  l.raw = o;
  o = align128(o + sh * box_bytes_row);
  l.samples = o;
  o = align128(o + sh * kSW * 4);
  l.rg = o;
  if (sharpen) o = align128(o + (kTH + 2) * 68 * 8);
  l.b = o;
  if (sharpen) o = align128(o + (kTH + 2) * 68 * 4);
  l.lsc = o;
  o = align128(o + kLscTableRows * 2 * kSW * 4);
  l.cols = o;
  o = align128(o + 3 * kSW * 4);
  l.rows = o;
  o = align128(o + 3 * sh * 4);
  l.hist = o;
  o = align128(o + kHistChannels * kHistBins * 4);
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

// ---- TMA and mbarrier -----------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, void* dst, uint64_t* bar, int x, int y,
                                            unsigned int bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Waits for the barrier's phase `parity` to complete; false after kWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (unsigned int i = 0; i < kWaitLimit; ++i) {
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

__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// The TMA coordinates of the box for a tile at (x0, y0) (x in the tensor's
// elements: bytes, or uint16 samples), 16-byte aligned for any x0 % 64 == 0.
__device__ __forceinline__ int box_x(int fmt, int x0) {
  return fmt == kRawU8 ? x0 - 16 : fmt == kRawU16 ? x0 - 8 : fmt == kRawRaw10 ? 5 * (x0 >> 2) - 16 : 3 * (x0 >> 1) - 16;
}

// ---- Raw unpacking from a box row ----------------------------------------

// Samples x0 - 4 + 4u .. + 3 of a box row (box starting at box_x(fmt, x0)).
__device__ __forceinline__ void unpack4(int fmt, const uint8_t* row, int u, unsigned int s[4]) {
  if (fmt == kRawU8) {
    const unsigned int w = *reinterpret_cast<const unsigned int*>(row + 12 + 4 * u);
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k] = (w >> (8 * k)) & 0xFFU;
  } else if (fmt == kRawU16) {
    const uint2 w = *reinterpret_cast<const uint2*>(row + 8 + 8 * u);
    s[0] = w.x & 0xFFFFU;
    s[1] = w.x >> 16;
    s[2] = w.y & 0xFFFFU;
    s[3] = w.y >> 16;
  } else if (fmt == kRawRaw10) {
    // Group g0 - 1 + u at byte 11 + 5u: four high bytes, then the low bits.
    const int b = 11 + 5 * u;
    const unsigned int* w = reinterpret_cast<const unsigned int*>(row + (b & ~3));
    const unsigned int sh = 8U * static_cast<unsigned int>(b & 3);
    const unsigned int hi4 = __funnelshift_r(w[0], w[1], sh);
    const unsigned int lo = (w[1] >> sh) & 0xFFU;
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k] = (((hi4 >> (8 * k)) & 0xFFU) << 2) | ((lo >> (2 * k)) & 3U);
  } else {
    // Two groups of three bytes at byte 10 + 6u.
    const int b = 10 + 6 * u;
    const unsigned int* w = reinterpret_cast<const unsigned int*>(row + (b & ~3));
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
__device__ __forceinline__ unsigned int unpack1(int fmt, const uint8_t* row, int mx, int x0) {
  if (fmt == kRawU8) return row[mx - x0 + 16];
  if (fmt == kRawU16) return *reinterpret_cast<const uint16_t*>(row + 2 * (mx - x0 + 8));
  if (fmt == kRawRaw10) {
    const uint8_t* g = row + 5 * ((mx >> 2) - (x0 >> 2)) + 16;
    const int k = mx & 3;
    return (static_cast<unsigned int>(g[k]) << 2) | ((g[4] >> (2 * k)) & 3U);
  }
  const uint8_t* g = row + 3 * ((mx >> 1) - (x0 >> 1)) + 16;
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
__device__ LscTile build_lsc(const FrameDesc& p, int pattern, int x_first, int ncols, int y_first, int nrows,
                             bool mirror_xy, int xclamp, int yclamp, int* col_mx, int* col_ix, float* col_tx,
                             int* row_my, int* row_k, float* row_ty, float* table, int* minmax) {
  const int t = threadIdx.x;
  if (t == 0) {
    minmax[0] = 0x7FFFFFFF;
    minmax[1] = -1;
  }
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
      atomicMin(&minmax[0], iy);
      atomicMax(&minmax[1], iy);
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
  for (int e = t; e < lt.rows * planes * ncols; e += kThreads) {
    const int i = e % ncols;
    const int kp = e / ncols;
    const int par = kp % planes;
    const int k = kp / planes;
    const int ch = step == 4 ? cfa_of(pattern, (par << 1) | (col_mx[i] & 1)) : 0;
    const float* g = p.lsc + ((lt.iy0 + k) * p.lsc_width + col_ix[i]) * step + ch;
    table[(k * 2 + par) * kSW + i] = g[0] + (g[step] - g[0]) * col_tx[i];
  }
  if (t < nrows) row_k[t] -= lt.iy0;
  __syncthreads();
  return lt;
}

// ---- Per-pixel tail: colour matrix, statistics, tone, codes ---------------

struct Tone {
  const float2* table;
  float scale;  // tone_size - 1
};

__device__ __forceinline__ float tone_of(const Tone& t, float x) {
  const float f = fmul(x, t.scale);
  const float m = magic_trunc(f);
  const float2 e = t.table[magic_int(m)];
  return fadd(e.x, fmul(fsub(f, fsub(m, kTwo23)), e.y));
}

// Stores toned RGB of pixels xb..xb+3 of row y (isp_math.hpp:250-276) and
// counts their 8-bit codes (isp_math.hpp:279-305) into the block's
// histogram. `full`: all four pixels are inside the image.
template <int kOut>
__device__ __forceinline__ void store_row4(const FrameDesc& p, int xb, int y, const float (&t)[4][3], bool full,
                                           bool want_hist, unsigned int* hist) {
  uint8_t* row = p.out + static_cast<int64_t>(y) * p.out_pitch;
  unsigned int q[4][3];
  const bool vec = full && p.out_vector;
  if constexpr (kOut == kOutRgb8 || kOut == kOutRgba8) {
#pragma unroll
    for (int dx = 0; dx < 4; ++dx) {
#pragma unroll
      for (int k = 0; k < 3; ++k) q[dx][k] = magic_int(magic_trunc(fadd(fmul(t[dx][k], 255.0F), 0.5F)));
    }
    if constexpr (kOut == kOutRgb8) {
      if (vec) {
        unsigned int* o = reinterpret_cast<unsigned int*>(row + 3 * xb);
        o[0] = q[0][0] | (q[0][1] << 8) | (q[0][2] << 16) | (q[1][0] << 24);
        o[1] = q[1][1] | (q[1][2] << 8) | (q[2][0] << 16) | (q[2][1] << 24);
        o[2] = q[2][2] | (q[3][0] << 8) | (q[3][1] << 16) | (q[3][2] << 24);
      } else {
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) {
          if (!full && xb + dx >= p.width) break;
#pragma unroll
          for (int k = 0; k < 3; ++k) row[3 * (xb + dx) + k] = static_cast<uint8_t>(q[dx][k]);
        }
      }
    } else {
      unsigned int w[4];
#pragma unroll
      for (int dx = 0; dx < 4; ++dx) w[dx] = q[dx][0] | (q[dx][1] << 8) | (q[dx][2] << 16) | 0xFF000000U;
      if (vec) {
        *reinterpret_cast<uint4*>(row + 4 * xb) = make_uint4(w[0], w[1], w[2], w[3]);
      } else {
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) {
          if (!full && xb + dx >= p.width) break;
#pragma unroll
          for (int k = 0; k < 4; ++k) row[4 * (xb + dx) + k] = static_cast<uint8_t>(w[dx] >> (8 * k));
        }
      }
    }
  } else if constexpr (kOut == kOutRgb16) {
    unsigned int v[4][3];
#pragma unroll
    for (int dx = 0; dx < 4; ++dx) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        v[dx][k] = magic_int(magic_trunc(fadd(fmul(t[dx][k], 65535.0F), 0.5F)));
        q[dx][k] = ((v[dx][k] + 128U) * 0xFF01U) >> 24;  // == (v * 255 + 32767) / 65535 for v < 2^16
      }
    }
    if (vec) {
      uint2* o = reinterpret_cast<uint2*>(row + 6 * xb);
      o[0] = make_uint2(v[0][0] | (v[0][1] << 16), v[0][2] | (v[1][0] << 16));
      o[1] = make_uint2(v[1][1] | (v[1][2] << 16), v[2][0] | (v[2][1] << 16));
      o[2] = make_uint2(v[2][2] | (v[3][0] << 16), v[3][1] | (v[3][2] << 16));
    } else {
      uint16_t* o = reinterpret_cast<uint16_t*>(row);
#pragma unroll
      for (int dx = 0; dx < 4; ++dx) {
        if (!full && xb + dx >= p.width) break;
#pragma unroll
        for (int k = 0; k < 3; ++k) o[3 * (xb + dx) + k] = static_cast<uint16_t>(v[dx][k]);
      }
    }
  } else {
#pragma unroll
    for (int dx = 0; dx < 4; ++dx) {
#pragma unroll
      for (int k = 0; k < 3; ++k) q[dx][k] = magic_int(magic_trunc(fadd(fmul(clamp01(t[dx][k]), 255.0F), 0.5F)));
    }
    if (vec) {
      float4* o = reinterpret_cast<float4*>(row + 12 * xb);
      o[0] = make_float4(t[0][0], t[0][1], t[0][2], t[1][0]);
      o[1] = make_float4(t[1][1], t[1][2], t[2][0], t[2][1]);
      o[2] = make_float4(t[2][2], t[3][0], t[3][1], t[3][2]);
    } else {
      float* o = reinterpret_cast<float*>(row);
#pragma unroll
      for (int dx = 0; dx < 4; ++dx) {
        if (!full && xb + dx >= p.width) break;
#pragma unroll
        for (int k = 0; k < 3; ++k) o[3 * (xb + dx) + k] = t[dx][k];
      }
    }
  }
  if (want_hist) {
#pragma unroll
    for (int dx = 0; dx < 4; ++dx) {
      if (!full && xb + dx >= p.width) break;
      const unsigned int luma = (2126U * q[dx][0] + 7152U * q[dx][1] + 722U * q[dx][2] + 5000U) / 10000U;
      atomicAdd(&hist[luma], 1U);
      atomicAdd(&hist[kHistBins + q[dx][0]], 1U);
      atomicAdd(&hist[2 * kHistBins + q[dx][1]], 1U);
      atomicAdd(&hist[3 * kHistBins + q[dx][2]], 1U);
    }
  }
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
__device__ float block_percentile(const unsigned int* hist, float percentile, u64* red, int* first) {
  const int t = threadIdx.x;
  unsigned int h[4];
  u64 mine = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    h[k] = __ldcg(hist + 4 * t + k);
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
__device__ void awb_finish(const FrameDesc& p, Scratch* s, u64* red, int* first) {
  const u64 nquads = __ldcg(&s->awb_quads);
  float level[3] = {0.0F, 0.0F, 0.0F};
  if (nquads != 0) {
    if (p.awb_mode == kWbGrayWorld) {
      const double q = static_cast<double>(nquads);
      level[0] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[0])) / q);
      level[1] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[1])) / (2.0 * q));
      level[2] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[2])) / q);
    } else {
      for (int k = 0; k < 3; ++k) level[k] = block_percentile(s->awb_hist[k], p.awb_percentile, red, first);
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
  for (int i = threadIdx.x; i < 3 * kAwbBins; i += kThreads) (&s->awb_hist[0][0])[i] = 0U;
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
  float* out = p.stats_out;
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

// The main pass's flush: block sums and histogram into the scratch, then the
// last CTA writes the user's histogram and statistics and clears the scratch.
__device__ void main_finish(const FrameDesc& p, Scratch* sc, const u64 (&acc)[4], const float gains[3],
                            bool want_stats, bool want_hist, unsigned int* hist, u64* red, bool* last) {
  const int tid = threadIdx.x;
  if (!want_stats && !want_hist) return;
  if (want_stats) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const u64 total = block_sum(acc[k], red);
      if (tid == 0 && total != 0) atomicAdd(k < 3 ? &sc->sum[k] : &sc->saturated, total);
    }
  }
  if (want_hist) {
    __syncthreads();
    for (int i = tid; i < kHistChannels * kHistBins; i += kThreads) {
      if (hist[i] != 0U) atomicAdd(&sc->hist[i], hist[i]);
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) *last = atomicAdd(&sc->main_done, 1U) == gridDim.x - 1;
  __syncthreads();
  if (!*last) return;
  __threadfence();
  if (want_hist) {
    for (int i = tid; i < kHistChannels * kHistBins; i += kThreads) {
      p.hist_out[i] = __ldcg(&sc->hist[i]);
      sc->hist[i] = 0U;
    }
  }
  if (want_stats && tid == 0) {
    const u64 sum[3] = {__ldcg(&sc->sum[0]), __ldcg(&sc->sum[1]), __ldcg(&sc->sum[2])};
    finish_stats(p, sum, __ldcg(&sc->saturated), gains);
    sc->sum[0] = sc->sum[1] = sc->sum[2] = 0;
    sc->saturated = 0;
  }
  if (tid == 0) sc->main_done = 0;
}

template <bool kMalvar, int kPat>
__device__ __forceinline__ void demosaic_at(const float (&w)[6][8], int dy, int dx, float rgb[3]) {
  float n[5][5];
#pragma unroll
  for (int a = 0; a < 5; ++a) {
#pragma unroll
    for (int b = 0; b < 5; ++b) n[a][b] = w[dy + a][dx + b];
  }
  demosaic<kMalvar>(n, cfa_of(kPat, (dy << 1) | (dx & 1)), rgb);
}

// ---- White balance statistics ----------------------------------------------

template <bool kWhitePatch, int kPat>
__global__ void __launch_bounds__(kThreads) isp_awb_kernel(const __grid_constant__ CUtensorMap map, FrameDesc p,
                                                         int tiles_x, int tiles, int use_tma) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128U - (smem_u32(smem_raw) & 127U)) & 127U);
  constexpr int kBoxRows = 64;
  uint8_t* box = smem;                                                  // [64][box bytes]
  float* table = reinterpret_cast<float*>(smem + 64 * 128);             // [kLscTableRows][2][kSW]
  int* col_mx = reinterpret_cast<int*>(table + kLscTableRows * 2 * kSW);  // [64] x 3
  int* col_ix = col_mx + 64;
  float* col_tx = reinterpret_cast<float*>(col_ix + 64);
  int* row_my = reinterpret_cast<int*>(col_tx + 64);                    // [64] x 3
  int* row_k = row_my + 64;
  float* row_ty = reinterpret_cast<float*>(row_k + 64);
  unsigned int* hist = reinterpret_cast<unsigned int*>(row_ty + 64);    // [3][1024]
  __shared__ uint64_t bar;
  __shared__ u64 red[kWarps];
  __shared__ int minmax[2];
  __shared__ int first;
  __shared__ bool last;
  Scratch* s = p.scratch;
  const int tid = threadIdx.x;
  const int box_bytes = p.raw_format == kRawU8 ? 64 : p.raw_format == kRawU16 ? 128 : p.raw_format == kRawRaw10 ? 80 : 96;
  if constexpr (kWhitePatch) {
    for (int i = tid; i < 3 * kAwbBins; i += kThreads) hist[i] = 0U;
  }
  if (tid == 0 && use_tma) mbar_init(&bar);
  __syncthreads();
  // Per quad position: channel, colour, black, 1 / range.
  float black[4], inv[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    black[k] = p.black[cfa_of(kPat, k)];
    inv[k] = p.inv_range[cfa_of(kPat, k)];
  }
  const int quads_x = p.width / 2;
  const int quads_y = p.height / 2;
  u64 acc[4] = {0, 0, 0, 0};
  uint32_t phase = 0;
  int tile = blockIdx.x;
  auto issue = [&](int t) {
    const int ty = t / tiles_x;
    const int x0 = (t - ty * tiles_x) * 64;
    const int bx = p.raw_format == kRawU8 ? x0 : p.raw_format == kRawU16 ? x0 : p.raw_format == kRawRaw10 ? 5 * (x0 >> 2) : 3 * (x0 >> 1);
    tma_load_2d(&map, box, &bar, bx, ty * 64, static_cast<unsigned int>(kBoxRows * box_bytes));
  };
  if (use_tma && tid == 0 && tile < tiles) issue(tile);
  for (; tile < tiles; tile += gridDim.x) {
    const int ty = tile / tiles_x;
    const int x0 = (tile - ty * tiles_x) * 64;
    const int y0 = ty * 64;
    const LscTile lt = build_lsc(p, kPat, x0, 64, y0, 64, false, 0, 0, col_mx, col_ix, col_tx, row_my, row_k,
                                 row_ty, table, minmax);
    if (use_tma && !mbar_wait(&bar, phase)) {
      if (tid == 0) atomicExch(&s->error, 1);
    }
    phase ^= 1U;
    // 2 quads (4 samples across, 2 rows) per unit; 32 row pairs x 16 units.
    for (int unit = tid; unit < 512; unit += kThreads) {
      const int a = unit >> 4;
      const int u = unit & 15;
      const int qy = (y0 >> 1) + a;
      const int qx0 = (x0 >> 1) + 2 * u;
      if (qy >= quads_y || qx0 >= quads_x) continue;
      unsigned int top[4], bot[4];
      if (use_tma) {
        // Units of 4 samples at x0 + 4u: reuse unpack4 with its x0 - 4 origin.
        const uint8_t* r0 = box + (2 * a) * box_bytes;
        const uint8_t* r1 = r0 + box_bytes;
        if (p.raw_format == kRawU8) {
          const unsigned int w0 = *reinterpret_cast<const unsigned int*>(r0 + 4 * u);
          const unsigned int w1 = *reinterpret_cast<const unsigned int*>(r1 + 4 * u);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            top[k] = (w0 >> (8 * k)) & 0xFFU;
            bot[k] = (w1 >> (8 * k)) & 0xFFU;
          }
        } else if (p.raw_format == kRawU16) {
          const uint2 w0 = *reinterpret_cast<const uint2*>(r0 + 8 * u);
          const uint2 w1 = *reinterpret_cast<const uint2*>(r1 + 8 * u);
          top[0] = w0.x & 0xFFFFU; top[1] = w0.x >> 16; top[2] = w0.y & 0xFFFFU; top[3] = w0.y >> 16;
          bot[0] = w1.x & 0xFFFFU; bot[1] = w1.x >> 16; bot[2] = w1.y & 0xFFFFU; bot[3] = w1.y >> 16;
        } else {
          // unpack4 reads sample x0 - 4 + 4u' from byte 11 + 5u' (RAW10) or
          // 10 + 6u' (RAW12) of a box starting 16 bytes before x0; this box
          // starts at x0, so shift the row pointer back 16 bytes: unit u' = u + 1.
          unpack4(p.raw_format, r0 - 16, u + 1, top);
          unpack4(p.raw_format, r1 - 16, u + 1, bot);
        }
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int x = x0 + 4 * u + k;
          top[k] = x < p.width ? static_cast<unsigned int>(load_raw(p, x, y0 + 2 * a)) : 0U;
          bot[k] = x < p.width ? static_cast<unsigned int>(load_raw(p, x, y0 + 2 * a + 1)) : 0U;
        }
      }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (qx0 + q >= quads_x) break;
        const unsigned int raw[4] = {top[2 * q], top[2 * q + 1], bot[2 * q], bot[2 * q + 1]};
        const bool ok = raw[0] < static_cast<unsigned int>(p.white) && raw[1] < static_cast<unsigned int>(p.white) &&
                        raw[2] < static_cast<unsigned int>(p.white) && raw[3] < static_cast<unsigned int>(p.white);
        if (!ok) continue;  // white_balance_quad, isp_math.hpp:311-319
        unsigned int fixed[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int ci = 4 * u + 2 * q + (k & 1);  // column in the tile
          const int rj = 2 * a + (k >> 1);         // row in the tile
          float v = fmul(fsub(magic_to_float(raw[k] | kTwo23Bits), black[k]), inv[k]);
          v = v > 0.0F ? v : 0.0F;
          if (lt.rows > 0) {
            float gain;
            if (lt.rows <= kLscTableRows) {
              const int kk = row_k[rj];
              const int par = p.lsc_channels == 4 ? (k >> 1) : 0;
              const float t0 = table[(kk * 2 + par) * kSW + ci];
              const float t1 = table[((kk + 1) * 2 + par) * kSW + ci];
              gain = fadd(t0, fmul(fsub(t1, t0), row_ty[rj]));
            } else {
              gain = lens_shading_gain(p, p.lsc, x0 + ci, y0 + rj, cfa_of(kPat, k));
            }
            v = fmul(v, gain);
          }
          v = v < 4.0F ? v : 4.0F;
          fixed[k] = magic_int(magic_trunc(fadd(fmul(v, kFixedOne), 0.5F)));
          if constexpr (kWhitePatch) {
            const unsigned int bin = magic_int(magic_trunc(fmul(v, static_cast<float>(kAwbBins))));
            atomicAdd(&hist[color_of(cfa_of(kPat, k)) * kAwbBins + (bin < kAwbBins - 1 ? bin : kAwbBins - 1)], 1U);
          }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[color_of(cfa_of(kPat, k))] += fixed[k];
        acc[3] += 1;
      }
    }
    __syncthreads();
    if (use_tma && tid == 0) {
      const int next = tile + gridDim.x;
      if (next < tiles) {
        fence_async_shared();
        issue(next);
      }
    }
  }
  // Flush: block sums, then one atomic per sum and per non-empty bin.
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    u64 v = acc[k];
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) v += __shfl_down_sync(0xFFFFFFFFU, v, offset);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
      u64 total = 0;
      for (int w = 0; w < kWarps; ++w) total += red[w];
      if (total != 0) atomicAdd(k < 3 ? &s->awb_sum[k] : &s->awb_quads, total);
    }
    __syncthreads();
  }
  if constexpr (kWhitePatch) {
    for (int i = tid; i < 3 * kAwbBins; i += kThreads) {
      if (hist[i] != 0U) atomicAdd(&s->awb_hist[0][0] + i, hist[i]);
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(&s->awb_done, 1U) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  awb_finish(p, s, red, &first);
}

// ---- The fused tile pass --------------------------------------------------

template <bool kMalvar, bool kSharpen, int kOut, int kPat>
__global__ void __launch_bounds__(kThreads, 2) isp_main_kernel(const __grid_constant__ CUtensorMap map, FrameDesc p,
                                                               int tiles_x, int tiles, int use_tma, int lut_in_smem) {
  using G = Geom<kSharpen>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128U - (smem_u32(smem_raw) & 127U)) & 127U);
  const int box_bytes = box_row_bytes(p.raw_format);
  const Layout L = layout_of(kSharpen, box_bytes, lut_in_smem ? p.tone_size : 0);
  uint8_t* box = smem + L.raw;
  float* S = reinterpret_cast<float*>(smem + L.samples);
  float2* Crg = reinterpret_cast<float2*>(smem + L.rg);
  float* Cb = reinterpret_cast<float*>(smem + L.b);
  float* table = reinterpret_cast<float*>(smem + L.lsc);
  int* col_mx = reinterpret_cast<int*>(smem + L.cols);
  int* col_ix = col_mx + kSW;
  float* col_tx = reinterpret_cast<float*>(col_ix + kSW);
  int* row_my = reinterpret_cast<int*>(smem + L.rows);
  int* row_k = row_my + G::kSH;
  float* row_ty = reinterpret_cast<float*>(row_k + G::kSH);
  unsigned int* hist = reinterpret_cast<unsigned int*>(smem + L.hist);
  float2* lut_s = reinterpret_cast<float2*>(smem + L.lut);
  __shared__ uint64_t bar;
  __shared__ u64 red[kWarps];
  __shared__ int minmax[2];
  __shared__ bool last;

  const int tid = threadIdx.x;
  Scratch* sc = p.scratch;
  const bool want_hist = p.hist_out != nullptr;
  const bool want_stats = p.stats_out != nullptr;
  float gains[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) gains[k] = p.auto_wb ? __ldcg(&sc->awb_gains[k]) : p.wb[k];
  // Per quad position: black level, 1 / range, white balance gain.
  float qblack[4], qinv[4], qgain[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int ch = cfa_of(kPat, k);
    qblack[k] = p.black[ch];
    qinv[k] = p.inv_range[ch];
    qgain[k] = gains[color_of(ch)];
  }
  Tone tone{p.tone, static_cast<float>(p.tone_size - 1)};
  if (lut_in_smem) {
    for (int i = tid; i < p.tone_size; i += kThreads) lut_s[i] = p.tone[i];
    tone.table = lut_s;
  }
  if (want_hist) {
    for (int i = tid; i < kHistChannels * kHistBins; i += kThreads) hist[i] = 0U;
  }
  if (tid == 0 && use_tma) mbar_init(&bar);
  __syncthreads();

  const int fmt = p.raw_format;
  const unsigned int white = static_cast<unsigned int>(p.white);
  u64 acc[4] = {0, 0, 0, 0};  // linear R, G, B in 2^-20 units; saturated samples
  uint32_t phase = 0;
  int tile = blockIdx.x;
  const auto issue = [&](int t) {
    const int ty = t / tiles_x;
    const int x0 = (t - ty * tiles_x) * kTW;
    tma_load_2d(&map, box, &bar, box_x(fmt, x0), ty * kTH - G::kHalo,
                static_cast<unsigned int>(G::kSH * box_bytes));
  };
  if (use_tma && tid == 0 && tile < tiles) issue(tile);

  for (; tile < tiles; tile += gridDim.x) {
    const int ty = tile / tiles_x;
    const int x0 = (tile - ty * tiles_x) * kTW;
    const int y0 = ty * kTH;
    const bool interior = x0 >= 4 && y0 >= G::kHalo && x0 + kSW - 4 <= p.width && y0 + kTH + G::kHalo <= p.height;
    const LscTile lt = build_lsc(p, kPat, x0 - 4, kSW, y0 - G::kHalo, G::kSH, !interior, p.width + 3,
                                 p.height + G::kHalo - 1, col_mx, col_ix, col_tx, row_my, row_k, row_ty, table, minmax);
    if (use_tma && !mbar_wait(&bar, phase)) {
      if (tid == 0) atomicExch(&sc->error, 1);
    }
    phase ^= 1U;

    // A. Samples of the tile and its halo, preprocessed once
    //    (preprocess, isp_math.hpp:151-155), four per unit.
    unsigned int saturated = 0;
    for (int unit = tid; unit < kUnitsRow * G::kSH; unit += kThreads) {
      const int j = unit / kUnitsRow;
      const int u = unit - j * kUnitsRow;
      const int par = j & 1;  // row parity: y0 - halo is even
      unsigned int s[4];
      if (use_tma) {
        const uint8_t* row = box + (row_my[j] - (y0 - G::kHalo)) * box_bytes;
        if (interior) {
          unpack4(fmt, row, u, s);
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) s[k] = unpack1(fmt, row, col_mx[4 * u + k], x0);
        }
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) s[k] = static_cast<unsigned int>(load_raw(p, col_mx[4 * u + k], row_my[j]));
      }
      if (want_stats && j >= G::kHalo && j < G::kHalo + kTH && u >= 1 && u <= kTW / 4 && y0 + j - G::kHalo < p.height) {
#pragma unroll
        for (int k = 0; k < 4; ++k) saturated += (x0 + 4 * (u - 1) + k < p.width && s[k] >= white) ? 1U : 0U;
      }
      // Constants of the row's two quad positions, selected (not indexed) so
      // they stay in registers.
      const float bl0 = par ? qblack[2] : qblack[0];
      const float bl1 = par ? qblack[3] : qblack[1];
      const float iv0 = par ? qinv[2] : qinv[0];
      const float iv1 = par ? qinv[3] : qinv[1];
      const float gn0 = par ? qgain[2] : qgain[0];
      const float gn1 = par ? qgain[3] : qgain[1];
      float v[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float x = fmul(fsub(magic_to_float(s[k] | kTwo23Bits), (k & 1) ? bl1 : bl0), (k & 1) ? iv1 : iv0);
        v[k] = x > 0.0F ? x : 0.0F;
      }
      if (lt.rows > 0) {
        if (lt.rows <= kLscTableRows) {
          const int kk = row_k[j];
          const int pl = p.lsc_channels == 4 ? par : 0;
          const float4 t0 = *reinterpret_cast<const float4*>(table + (kk * 2 + pl) * kSW + 4 * u);
          const float4 t1 = *reinterpret_cast<const float4*>(table + ((kk + 1) * 2 + pl) * kSW + 4 * u);
          const float tyj = row_ty[j];
          v[0] = fmul(v[0], fadd(t0.x, fmul(fsub(t1.x, t0.x), tyj)));
          v[1] = fmul(v[1], fadd(t0.y, fmul(fsub(t1.y, t0.y), tyj)));
          v[2] = fmul(v[2], fadd(t0.z, fmul(fsub(t1.z, t0.z), tyj)));
          v[3] = fmul(v[3], fadd(t0.w, fmul(fsub(t1.w, t0.w), tyj)));
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            v[k] = fmul(v[k], lens_shading_gain(p, p.lsc, col_mx[4 * u + k], row_my[j], cfa_of(kPat, (par << 1) | (k & 1))));
          }
        }
      }
      float4 out;
      out.x = mul_sat(v[0], gn0);
      out.y = mul_sat(v[1], gn1);
      out.z = mul_sat(v[2], gn0);
      out.w = mul_sat(v[3], gn1);
      *reinterpret_cast<float4*>(S + j * kSW + 4 * u) = out;
    }
    acc[3] += saturated;
    __syncthreads();
    // The box is free: prefetch the next tile's raw samples.
    if (use_tma && tid == 0) {
      const int next = tile + gridDim.x;
      if (next < tiles) {
        fence_async_shared();
        issue(next);
      }
    }

    // B. (Sharpening) RGB of the tile and a one-pixel ring, 2x4 pixels a
    //    unit; outside the image these are the reference's virtual pixels
    //    (cpu_pipeline.cpp:22-46).
    if constexpr (kSharpen) {
      constexpr int kUnitsB = 17 * 34;
      for (int unit = tid; unit < kUnitsB; unit += kThreads) {
        const int qr = unit / 17;
        const int qc = unit - qr * 17;
        float w[6][8];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          const float4 a = *reinterpret_cast<const float4*>(S + (2 * qr + r) * kSW + 4 * qc);
          const float4 b = *reinterpret_cast<const float4*>(S + (2 * qr + r) * kSW + 4 * qc + 4);
          w[r][0] = a.x; w[r][1] = a.y; w[r][2] = a.z; w[r][3] = a.w;
          w[r][4] = b.x; w[r][5] = b.y; w[r][6] = b.z; w[r][7] = b.w;
        }
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
          const int cy = 2 * qr + dy - 1;
          if (cy < 0 || cy >= G::kCH) continue;
#pragma unroll
          for (int dx = 0; dx < 4; ++dx) {
            const int cx = 4 * qc + dx - 1;
            if (cx < 0 || cx >= kTW + 2) continue;
            float rgb[3];
            demosaic_at<kMalvar, kPat>(w, dy, dx, rgb);
            Crg[cy * G::kCW + cx] = make_float2(rgb[0], rgb[1]);
            Cb[cy * G::kCW + cx] = rgb[2];
          }
        }
      }
      __syncthreads();
    }

    // C. Output units of 2x4 pixels: 32 unit rows x 16 unit columns. The
    //    statistics sums of a tile fit 32 bits (16 pixels of at most 2^20).
    unsigned int sums[3] = {0U, 0U, 0U};
    for (int unit = tid; unit < 512; unit += kThreads) {
      const int ur = unit >> 4;
      const int uc = unit & 15;
      float rgb[2][4][3];
      if constexpr (kSharpen) {
        // 3x3 neighbourhoods from the RGB planes, window rows 2ur..2ur+3,
        // columns 4uc..4uc+5 (pixel x0 + 4uc + dx at column 4uc + dx + 1).
        float m[4][6][3];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const float2* rg = Crg + (2 * ur + r) * G::kCW + 4 * uc;
          const float4 a = *reinterpret_cast<const float4*>(rg);
          const float4 b = *reinterpret_cast<const float4*>(rg + 2);
          const float4 c = *reinterpret_cast<const float4*>(rg + 4);
          m[r][0][0] = a.x; m[r][0][1] = a.y; m[r][1][0] = a.z; m[r][1][1] = a.w;
          m[r][2][0] = b.x; m[r][2][1] = b.y; m[r][3][0] = b.z; m[r][3][1] = b.w;
          m[r][4][0] = c.x; m[r][4][1] = c.y; m[r][5][0] = c.z; m[r][5][1] = c.w;
          const float* bp = Cb + (2 * ur + r) * G::kCW + 4 * uc;
          const float4 d = *reinterpret_cast<const float4*>(bp);
          const float2 e = *reinterpret_cast<const float2*>(bp + 4);
          m[r][0][2] = d.x; m[r][1][2] = d.y; m[r][2][2] = d.z; m[r][3][2] = d.w;
          m[r][4][2] = e.x; m[r][5][2] = e.y;
        }
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
          for (int dx = 0; dx < 4; ++dx) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              rgb[dy][dx][k] = sharpen_one(m[dy + 1][dx + 1][k], m[dy][dx + 1][k], m[dy + 2][dx + 1][k],
                                           m[dy + 1][dx][k], m[dy + 1][dx + 2][k], m[dy][dx][k], m[dy][dx + 2][k],
                                           m[dy + 2][dx][k], m[dy + 2][dx + 2][k], p.sharpen);
            }
          }
        }
      } else {
        // Samples rows 2ur .. 2ur + 5 (halo 2), columns 4uc + 2 .. 4uc + 9.
        float w[6][8];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          if (!kMalvar && (r == 0 || r == 5)) {
#pragma unroll
            for (int c = 0; c < 8; ++c) w[r][c] = 0.0F;
            continue;
          }
          const float* row = S + (2 * ur + r) * kSW + 4 * uc;
          const float4 a = *reinterpret_cast<const float4*>(row);
          const float4 b = *reinterpret_cast<const float4*>(row + 4);
          const float4 c = *reinterpret_cast<const float4*>(row + 8);
          w[r][0] = a.z; w[r][1] = a.w; w[r][2] = b.x; w[r][3] = b.y;
          w[r][4] = b.z; w[r][5] = b.w; w[r][6] = c.x; w[r][7] = c.y;
        }
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
          for (int dx = 0; dx < 4; ++dx) demosaic_at<kMalvar, kPat>(w, dy, dx, rgb[dy][dx]);
        }
      }
      const int xb = x0 + 4 * uc;
      const bool full = xb + 3 < p.width;
#pragma unroll
      for (int dy = 0; dy < 2; ++dy) {
        const int y = y0 + 2 * ur + dy;
        if (y >= p.height) continue;
        float toned[4][3];
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) {
          const float* c = rgb[dy][dx];
          float lin[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            // clamp01(m0 r + m1 g + m2 b), isp_math.hpp:229-233.
            lin[k] = add_sat(fadd(fmul(p.ccm[3 * k], c[0]), fmul(p.ccm[3 * k + 1], c[1])), fmul(p.ccm[3 * k + 2], c[2]));
          }
          const bool inside = full || xb + dx < p.width;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            if (want_stats && inside) sums[k] += magic_int(magic_trunc(fadd(fmul(lin[k], kFixedOne), 0.5F)));
            toned[dx][k] = tone_of(tone, lin[k]);
          }
        }
        store_row4<kOut>(p, xb, y, toned, full, want_hist, hist);
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] += sums[k];
    __syncthreads();  // the next tile overwrites the tables, S and C
  }
  main_finish(p, sc, acc, gains, want_stats, want_hist, hist, red, &last);
}

template <bool kMalvar, bool kSharpen, int kOut>
const void* main_by_pattern(int pattern) {
  switch (pattern) {
    case 0: return reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, kOut, 0>);
    case 1: return reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, kOut, 1>);
    case 2: return reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, kOut, 2>);
    default: return reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, kOut, 3>);
  }
}

template <bool kMalvar, bool kSharpen>
const void* main_by_out(int out, int pattern) {
  switch (out) {
    case kOutRgb8: return main_by_pattern<kMalvar, kSharpen, kOutRgb8>(pattern);
    case kOutRgba8: return main_by_pattern<kMalvar, kSharpen, kOutRgba8>(pattern);
    case kOutRgb16: return main_by_pattern<kMalvar, kSharpen, kOutRgb16>(pattern);
    default: return main_by_pattern<kMalvar, kSharpen, kOutRgb32f>(pattern);
  }
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

const void* main_kernel(bool malvar, bool sharpen, int out_format, int pattern) {
  if (malvar) return sharpen ? main_by_out<true, true>(out_format, pattern) : main_by_out<true, false>(out_format, pattern);
  return sharpen ? main_by_out<false, true>(out_format, pattern) : main_by_out<false, false>(out_format, pattern);
}

size_t main_kernel_smem(bool sharpen, int raw_format, int lut_entries) {
  return static_cast<size_t>(layout_of(sharpen, box_row_bytes(raw_format), lut_entries).total) + 128U;
}

int main_box_rows(bool sharpen) { return sharpen ? kTH + 8 : kTH + 4; }
int main_box_row_bytes(int raw_format) { return box_row_bytes(raw_format); }

int main_kernel_tiles(int width, int height, int* tiles_x) {
  *tiles_x = (width + kTW - 1) / kTW;
  return *tiles_x * ((height + kTH - 1) / kTH);
}

int kernel_threads() { return kThreads; }

const void* awb_kernel(bool white_patch, int pattern) {
  return white_patch ? awb_by_pattern<true>(pattern) : awb_by_pattern<false>(pattern);
}

size_t awb_kernel_smem() {
  // box 64 x 128, lens shading table, column and row maps, white-patch histogram.
  return 64U * 128U + kLscTableRows * 2U * kSW * 4U + 6U * 64U * 4U + 3U * kAwbBins * 4U + 128U;
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
