// isp_common.cuh - device building blocks shared by the ISP's kernels: tile
// geometry and shared-memory layout, TMA and mbarrier helpers, raw unpacking,
// lens shading tables, stores, block reductions and the last-CTA finishers.
#pragma once

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

// ---- The fused tile pass --------------------------------------------------

// Per-tile state the phases share.
struct TileCtx {
  int x0, y0;
  const uint8_t* box;
  const int* col_mx;
  const int* row_my;
  const int* row_k;
  const float* row_ty;
  const float* table;
  LscTile lt;
};

// A. Samples of the tile and its halo, preprocessed once (preprocess,
//    isp_math.hpp:151-155), four per unit; returns the saturated count of
//    the tile's own samples (raw >= white, isp_math.hpp:316).
template <int kFmt, int kSrc, int kHalo>
__device__ __forceinline__ unsigned int phase_a(const FrameDesc& p, const TileCtx& t, float* S, int box_bytes,
                                                const float (&qblack)[4], const float (&qinv)[4],
                                                const float (&qgain)[4], bool want_stats) {
  // kSrc: 0 interior tile from the TMA box, 1 edge tile from the box
  // (mirrored columns), 2 no box (global loads, mirrored).
  constexpr int kSH = kTH + 2 * kHalo;
  const unsigned int white = static_cast<unsigned int>(p.white);
  unsigned int saturated = 0;
  for (int unit = threadIdx.x; unit < kUnitsRow * kSH; unit += kThreads) {
    const int j = unit / kUnitsRow;
    const int u = unit - j * kUnitsRow;
    const int par = j & 1;  // row parity: y0 - halo is even
    unsigned int s[4];
    if constexpr (kSrc == 0) {
      unpack4(kFmt, t.box + j * box_bytes, u, s);
    } else if constexpr (kSrc == 1) {
      const uint8_t* row = t.box + (t.row_my[j] - (t.y0 - kHalo)) * box_bytes;
#pragma unroll
      for (int k = 0; k < 4; ++k) s[k] = unpack1(kFmt, row, t.col_mx[4 * u + k], t.x0);
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) s[k] = static_cast<unsigned int>(load_raw(p, t.col_mx[4 * u + k], t.row_my[j]));
    }
    if (want_stats && j >= kHalo && j < kHalo + kTH && u >= 1 && u <= kTW / 4) {
      const int y = t.y0 + j - kHalo;
      const int xs = t.x0 + 4 * (u - 1);
      if (y < p.height) {
#pragma unroll
        for (int k = 0; k < 4; ++k) saturated += (xs + k < p.width && s[k] >= white) ? 1U : 0U;
      }
    }
    // The row's two quad positions' constants, selected so they stay in registers.
    const float bl0 = par ? qblack[2] : qblack[0];
    const float bl1 = par ? qblack[3] : qblack[1];
    const float iv0 = par ? qinv[2] : qinv[0];
    const float iv1 = par ? qinv[3] : qinv[1];
    const float gn0 = par ? qgain[2] : qgain[0];
    const float gn1 = par ? qgain[3] : qgain[1];
    float v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      // linearize (isp_math.hpp:144-148): max((raw - black) * inv_range, 0).
      const float x = fmul(fsub(magic_to_float(s[k] | kTwo23Bits), (k & 1) ? bl1 : bl0), (k & 1) ? iv1 : iv0);
      v[k] = fmaxf(x, 0.0F);
    }
    if (t.lt.rows > 0) {
      if (t.lt.rows <= kLscTableRows) {
        const int kk = t.row_k[j];
        const int pl = p.lsc_channels == 4 ? par : 0;
        const float4 t0 = *reinterpret_cast<const float4*>(t.table + (kk * 2 + pl) * kSW + 4 * u);
        const float4 t1 = *reinterpret_cast<const float4*>(t.table + ((kk + 1) * 2 + pl) * kSW + 4 * u);
        const float tyj = t.row_ty[j];
        v[0] = fmul(v[0], fadd(t0.x, fmul(fsub(t1.x, t0.x), tyj)));
        v[1] = fmul(v[1], fadd(t0.y, fmul(fsub(t1.y, t0.y), tyj)));
        v[2] = fmul(v[2], fadd(t0.z, fmul(fsub(t1.z, t0.z), tyj)));
        v[3] = fmul(v[3], fadd(t0.w, fmul(fsub(t1.w, t0.w), tyj)));
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          v[k] = fmul(v[k], lens_shading_gain(p, p.lsc, t.col_mx[4 * u + k], t.row_my[j], p.cfa[(par << 1) | (k & 1)]));
        }
      }
    }
    // White balance and the clip to 1 (v >= 0): the saturating multiply.
    *reinterpret_cast<float4*>(S + j * kSW + 4 * u) =
        make_float4(mul_sat(v[0], gn0), mul_sat(v[1], gn1), mul_sat(v[2], gn0), mul_sat(v[3], gn1));
  }
  return saturated;
}

template <int kSrc, int kHalo>
__device__ __forceinline__ unsigned int phase_a_fmt(const FrameDesc& p, const TileCtx& t, float* S, int box_bytes,
                                                    const float (&qblack)[4], const float (&qinv)[4],
                                                    const float (&qgain)[4], bool want_stats) {
  // Global loads (no TMA box) read the format at run time in load_raw.
  if constexpr (kSrc == 2) return phase_a<kRawU8, kSrc, kHalo>(p, t, S, box_bytes, qblack, qinv, qgain, want_stats);
  switch (p.raw_format) {
    case kRawU8: return phase_a<kRawU8, kSrc, kHalo>(p, t, S, box_bytes, qblack, qinv, qgain, want_stats);
    case kRawU16: return phase_a<kRawU16, kSrc, kHalo>(p, t, S, box_bytes, qblack, qinv, qgain, want_stats);
    case kRawRaw10: return phase_a<kRawRaw10, kSrc, kHalo>(p, t, S, box_bytes, qblack, qinv, qgain, want_stats);
    default: return phase_a<kRawRaw12, kSrc, kHalo>(p, t, S, box_bytes, qblack, qinv, qgain, want_stats);
  }
}

// The tone curve (isp_math.hpp:235-243) from a table of (lut[i], lut[i+1] -
// lut[i]) pairs: f = x (N - 1), i = trunc(f), lut[i] + (f - i) * diff[i].
// The last entry's difference is -0.0, so x = 1 (t = +0) returns lut[N-1]
// exactly, as the reference's branch does, whatever the sign of lut[N-1].
template <bool kLutSmem>
__device__ __forceinline__ float tone_at(const float2* table, float scale, float x) {
  const float f = fmul(x, scale);
  const float m = magic_trunc(f);
  float2 e;
  if constexpr (kLutSmem) {
    // Shared address of entry trunc(f): base + 8 (bits - 2^23 bits), wrapping.
    const uint32_t addr = smem_u32(table) + (__float_as_uint(m) << 3) - (kTwo23Bits << 3);
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(e.x), "=f"(e.y) : "r"(addr));
  } else {
    e = __ldg(table + magic_int(m));
  }
  return fadd(e.x, fmul(fsub(f, fsub(m, kTwo23)), e.y));
}

// C. One 2x4 unit's RGB -> colour matrix, statistics sums, tone, store,
//    histogram codes. `full`: all eight pixels are inside the image.
template <int kOut, bool kLutSmem>
__device__ __forceinline__ void finish_unit(const FrameDesc& p, const float (&rgb)[2][4][3], int xb, int yb,
                                            bool full, const float2* lut, float lut_scale, bool want_stats,
                                            bool want_hist, unsigned int* hist, unsigned int (&sums)[3],
                                            unsigned int& counted) {
#pragma unroll
  for (int dy = 0; dy < 2; ++dy) {
    const int y = yb + dy;
    if (!full && y >= p.height) continue;
    float toned[4][3];
#pragma unroll
    for (int dx = 0; dx < 4; ++dx) {
      const float* c = rgb[dy][dx];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        // clamp01((m0 r + m1 g) + m2 b), isp_math.hpp:229-233.
        const float lin = add_sat(fadd(fmul(p.ccm[3 * k], c[0]), fmul(p.ccm[3 * k + 1], c[1])), fmul(p.ccm[3 * k + 2], c[2]));
        if (want_stats && (full || xb + dx < p.width)) {
          // to_fixed (isp_math.hpp:245-247): trunc(lin 2^20 + 0.5).
          sums[k] += magic_int(magic_trunc(fadd(fmul(lin, kFixedOne), 0.5F)));
        }
        toned[dx][k] = tone_at<kLutSmem>(lut, lut_scale, lin);
      }
    }
    store_row4<kOut>(p, xb, y, toned, full || xb + 3 < p.width, want_hist, hist);
  }
}


// finish_unit for the frame's output format, chosen once per unit.
template <bool kLutSmem>
__device__ __forceinline__ void finish_unit_any(const FrameDesc& p, const float (&rgb)[2][4][3], int xb, int yb,
                                                bool full, const float2* lut, float lut_scale, bool want_stats,
                                                bool want_hist, unsigned int* hist, unsigned int (&sums)[3],
                                                unsigned int& counted) {
  switch (p.out_format) {
    case kOutRgb8:
      finish_unit<kOutRgb8, kLutSmem>(p, rgb, xb, yb, full, lut, lut_scale, want_stats, want_hist, hist, sums, counted);
      break;
    case kOutRgba8:
      finish_unit<kOutRgba8, kLutSmem>(p, rgb, xb, yb, full, lut, lut_scale, want_stats, want_hist, hist, sums, counted);
      break;
    case kOutRgb16:
      finish_unit<kOutRgb16, kLutSmem>(p, rgb, xb, yb, full, lut, lut_scale, want_stats, want_hist, hist, sums, counted);
      break;
    default:
      finish_unit<kOutRgb32f, kLutSmem>(p, rgb, xb, yb, full, lut, lut_scale, want_stats, want_hist, hist, sums, counted);
      break;
  }
}

}  // namespace
}  // namespace isp_b200
