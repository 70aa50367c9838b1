// isp_device.cuh - per-sample and per-pixel arithmetic of the B200 ISP.
//
// Each function computes the same IEEE single (or double) operations, on the
// same operands in the same order, as the holoscan::isp reference
// (modules/isp/src/isp_math.hpp), so that every output matches its CPU
// backend bit for bit. The library is compiled with --fmad=false: a product
// and a sum are never fused into one rounding. Integer sums (statistics) are
// order-free; float expressions are not, and are kept as written.
#pragma once

#include <cstdint>

#include "isp_ops.cuh"
#include "isp_types.cuh"

namespace isp_b200 {

__device__ __forceinline__ int mirror(int v, int n) {
  // Reflection about the first and last sample (isp_math.hpp:82-91): keeps the
  // coordinate's parity and so its colour in the mosaic.
  const int period = 2 * (n - 1);
  v %= period;
  if (v < 0) v += period;
  return v < n ? v : period - v;
}

__device__ __forceinline__ int color_of(int channel) {
  return channel == kChR ? 0 : channel == kChB ? 2 : 1;
}

__device__ __forceinline__ float clamp01(float v) { return v < 0.0F ? 0.0F : v > 1.0F ? 1.0F : v; }

// One sample's raw counts (isp_math.hpp:101-119), read through the read-only path.
__device__ __forceinline__ int load_raw(const FrameDesc& p, int x, int y) {
  Span<const uint8_t> row = p.raw + static_cast<int64_t>(y) * p.raw_pitch;
  switch (p.raw_format) {
    case kRawU8:
      return __ldg(&row[x]);
    case kRawU16:
      return __ldg(&span_cast<const uint16_t>(row)[x]);
    case kRawRaw10: {
      Span<const uint8_t> g = row + 5 * (x >> 2);
      const int k = x & 3;
      return (static_cast<int>(__ldg(&g[k])) << 2) | ((__ldg(&g[4]) >> (2 * k)) & 3);
    }
    default: {
      Span<const uint8_t> g = row + 3 * (x >> 1);
      const int k = x & 1;
      return (static_cast<int>(__ldg(&g[k])) << 4) | ((__ldg(&g[2]) >> (4 * k)) & 15);
    }
  }
}

// Lens shading gain at (x, y) (isp_math.hpp:121-140): bilinear in the grid,
// first across (top and bottom rows of the cell), then down.
__device__ __forceinline__ float lens_shading_gain(const FrameDesc& p, Span<const float> grid, int x, int y,
                                                   int channel) {
  const float fx = static_cast<float>(x) * p.lsc_sx;
  const float fy = static_cast<float>(y) * p.lsc_sy;
  int ix = static_cast<int>(fx);
  int iy = static_cast<int>(fy);
  ix = ix > p.lsc_width - 2 ? p.lsc_width - 2 : ix;
  iy = iy > p.lsc_height - 2 ? p.lsc_height - 2 : iy;
  const float tx = fx - static_cast<float>(ix);
  const float ty = fy - static_cast<float>(iy);
  const int step = p.lsc_channels;
  const int row = p.lsc_width * step;
  Span<const float> g = grid + (iy * p.lsc_width + ix) * step + (step == 4 ? channel : 0);
  const float top = g[0] + (g[step] - g[0]) * tx;
  const float bottom = g[row] + (g[row + step] - g[row]) * tx;
  return top + (bottom - top) * ty;
}

// Black level and lens shading (isp_math.hpp:144-148): 0 at black, 1 at white.
__device__ __forceinline__ float linearize(const FrameDesc& p, Span<const float> grid, int raw, int x, int y,
                                           int channel) {
  float v = (static_cast<float>(raw) - p.black[channel]) * p.inv_range[channel];
  v = v > 0.0F ? v : 0.0F;
  return grid != nullptr ? v * lens_shading_gain(p, grid, x, y, channel) : v * 1.0F;
}

// The Malvar-He-Cutler or bilinear estimates at the centre of a 5x5
// neighbourhood n[dy + 2][dx + 2] (isp_math.hpp:161-215), only the two that
// the centre's channel needs. R and B sites: green and the diagonal colour.
// In the Malvar estimates a product by 2 or 4 is exact, so round(4c + 2 a1)
// is one fused multiply-add whose only rounding is the sum's (the reference
// rounds the exact products, then the sum): exact_scale_add(a1, 2, 4c). The
// products by 5, 6 and 1.5, and by 0.5 and 0.125 (exact only above the
// subnormal range), stay separate roundings. clamp01(x * 0.125) is the
// saturating multiply.
template <bool kMalvar>
__device__ __forceinline__ void estimate_rb_site(const float (&n)[5][5], float& at_green, float& diagonal) {
  if constexpr (!kMalvar) {
    at_green = (n[1][2] + n[3][2] + n[2][1] + n[2][3]) * 0.25F;
    diagonal = (n[1][1] + n[1][3] + n[3][1] + n[3][3]) * 0.25F;
  } else {
    const float c = n[2][2];
    const float axial1 = n[1][2] + n[3][2] + n[2][1] + n[2][3];
    const float axial2 = n[0][2] + n[4][2] + n[2][0] + n[2][4];
    const float diagonal1 = n[1][1] + n[1][3] + n[3][1] + n[3][3];
    // clamp01((4c + 2 axial1 - axial2) * 0.125)
    at_green = mul_sat(fsub(exact_scale_add(axial1, 2.0F, fmul(4.0F, c)), axial2), 0.125F);
    // clamp01((6c + 2 diagonal1 - 1.5 axial2) * 0.125)
    diagonal = mul_sat(fsub(exact_scale_add(diagonal1, 2.0F, fmul(6.0F, c)), fmul(1.5F, axial2)), 0.125F);
  }
}

// Green sites: the colour left and right (across) and above and below (down).
template <bool kMalvar>
__device__ __forceinline__ void estimate_g_site(const float (&n)[5][5], float& across, float& down) {
  if constexpr (!kMalvar) {
    across = (n[2][1] + n[2][3]) * 0.5F;
    down = (n[1][2] + n[3][2]) * 0.5F;
  } else {
    const float c5 = fmul(5.0F, n[2][2]);
    const float diagonal1 = n[1][1] + n[1][3] + n[3][1] + n[3][3];
    const float horizontal2 = n[2][0] + n[2][4];
    const float vertical2 = n[0][2] + n[4][2];
    // clamp01((5c + 4 (n21 + n23) - horizontal2 - diagonal1 + 0.5 vertical2) * 0.125)
    across = mul_sat(fadd(fsub(fsub(exact_scale_add(fadd(n[2][1], n[2][3]), 4.0F, c5), horizontal2), diagonal1),
                          fmul(0.5F, vertical2)),
                     0.125F);
    down = mul_sat(fadd(fsub(fsub(exact_scale_add(fadd(n[1][2], n[3][2]), 4.0F, c5), vertical2), diagonal1),
                        fmul(0.5F, horizontal2)),
                   0.125F);
  }
}

// RGB of a pixel whose channel is `channel` (isp_math.hpp:193-214).
template <bool kMalvar>
__device__ __forceinline__ void demosaic(const float (&n)[5][5], int channel, float rgb[3]) {
  const float c = n[2][2];
  if (channel == kChR || channel == kChB) {
    float g, d;
    estimate_rb_site<kMalvar>(n, g, d);
    rgb[1] = g;
    rgb[0] = channel == kChR ? c : d;
    rgb[2] = channel == kChR ? d : c;
  } else {
    float across, down;
    estimate_g_site<kMalvar>(n, across, down);
    rgb[1] = c;
    rgb[0] = channel == kChGr ? across : down;
    rgb[2] = channel == kChGr ? down : across;
  }
}

// Unsharp mask of one channel's centre c against the 1-2-1 binomial blur of
// its 3x3 neighbourhood (isp_math.hpp:219-227): axial = m01, m21, m10, m12 in
// that order, corners = m00, m02, m20, m22.
__device__ __forceinline__ float sharpen_one(float c, float m01, float m21, float m10, float m12, float m00,
                                             float m02, float m20, float m22, float amount) {
  // (4c + 2 axial + corners) * 0.0625 with round(4c + 2 axial) one fused
  // rounding (both products exact); clamp01(c + amount (c - blur)) saturating.
  const float axial = fadd(fadd(fadd(m01, m21), m10), m12);
  const float corners = fadd(fadd(fadd(m00, m02), m20), m22);
  const float blur = fmul(fadd(exact_scale_add(axial, 2.0F, fmul(4.0F, c)), corners), 0.0625F);
  return add_sat(c, fmul(amount, fsub(c, blur)));
}

// ---- The same estimates on two pixels at once (f32x2 lanes) ----------------
//
// estimate_rb_site, estimate_g_site and sharpen_one with the operations
// two-lane ones: each lane sees exactly the scalar function's operations, in
// the same order (sums left to right as written above). A sum that consumes
// a product runs per lane (isp_ops.cuh: the assembler may fuse two-lane
// products into two-lane sums).

template <bool kMalvar>
__device__ __forceinline__ void estimate_rb_site2(const float2 (&n)[5][5], float2& at_green, float2& diagonal) {
  if constexpr (!kMalvar) {
    at_green = mul2(add2(add2(add2(n[1][2], n[3][2]), n[2][1]), n[2][3]), bc2(0.25F));
    diagonal = mul2(add2(add2(add2(n[1][1], n[1][3]), n[3][1]), n[3][3]), bc2(0.25F));
  } else {
    const float2 c = n[2][2];
    const float2 axial1 = add2(add2(add2(n[1][2], n[3][2]), n[2][1]), n[2][3]);
    const float2 axial2 = add2(add2(add2(n[0][2], n[4][2]), n[2][0]), n[2][4]);
    const float2 diagonal1 = add2(add2(add2(n[1][1], n[1][3]), n[3][1]), n[3][3]);
    at_green = mul_sat2(sub2(exact_scale_add2(axial1, bc2(2.0F), mul2(bc2(4.0F), c)), axial2), bc2(0.125F));
    // 1.5 axial2 is a rounded product: subtracted per lane (isp_ops.cuh).
    diagonal = mul_sat2(sub_lanes(exact_scale_add2(diagonal1, bc2(2.0F), mul2(bc2(6.0F), c)), mul2(bc2(1.5F), axial2)),
                        bc2(0.125F));
  }
}

template <bool kMalvar>
__device__ __forceinline__ void estimate_g_site2(const float2 (&n)[5][5], float2& across, float2& down) {
  if constexpr (!kMalvar) {
    across = mul2(add2(n[2][1], n[2][3]), bc2(0.5F));
    down = mul2(add2(n[1][2], n[3][2]), bc2(0.5F));
  } else {
    const float2 c5 = mul2(bc2(5.0F), n[2][2]);
    const float2 diagonal1 = add2(add2(add2(n[1][1], n[1][3]), n[3][1]), n[3][3]);
    const float2 horizontal2 = add2(n[2][0], n[2][4]);
    const float2 vertical2 = add2(n[0][2], n[4][2]);
    // 0.5 v2 is exact except below the normal range: added per lane all the same.
    across = mul_sat2(add_lanes(sub2(sub2(exact_scale_add2(add2(n[2][1], n[2][3]), bc2(4.0F), c5), horizontal2), diagonal1),
                                mul2(bc2(0.5F), vertical2)),
                      bc2(0.125F));
    down = mul_sat2(add_lanes(sub2(sub2(exact_scale_add2(add2(n[1][2], n[3][2]), bc2(4.0F), c5), vertical2), diagonal1),
                              mul2(bc2(0.5F), horizontal2)),
                    bc2(0.125F));
  }
}

// RGB of two pixels whose channel is `channel` (isp_math.hpp:193-214).
template <bool kMalvar>
__device__ __forceinline__ void demosaic2(const float2 (&n)[5][5], int channel, float2 rgb[3]) {
  const float2 c = n[2][2];
  if (channel == kChR || channel == kChB) {
    float2 g, d;
    estimate_rb_site2<kMalvar>(n, g, d);
    rgb[1] = g;
    rgb[0] = channel == kChR ? c : d;
    rgb[2] = channel == kChR ? d : c;
  } else {
    float2 across, down;
    estimate_g_site2<kMalvar>(n, across, down);
    rgb[1] = c;
    rgb[0] = channel == kChGr ? across : down;
    rgb[2] = channel == kChGr ? down : across;
  }
}

__device__ __forceinline__ float2 sharpen_one2(float2 c, float2 m01, float2 m21, float2 m10, float2 m12, float2 m00,
                                               float2 m02, float2 m20, float2 m22, float2 amount) {
  const float2 axial = add2(add2(add2(m01, m21), m10), m12);
  const float2 corners = add2(add2(add2(m00, m02), m20), m22);
  const float2 blur = mul2(add2(exact_scale_add2(axial, bc2(2.0F), mul2(bc2(4.0F), c)), corners), bc2(0.0625F));
  return add_sat2(c, mul2(amount, sub_lanes(c, blur)));  // blur is a product: per lane
}

// Colour correction (isp_math.hpp:229-233).
__device__ __forceinline__ void correct_color(const float* ccm, const float in[3], float out[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    out[k] = clamp01(ccm[3 * k] * in[0] + ccm[3 * k + 1] * in[1] + ccm[3 * k + 2] * in[2]);
  }
}

// Tone curve (isp_math.hpp:235-243) from the table of (lut[i], lut[i+1] -
// lut[i]) pairs, whose differences the host formed with the same float
// subtraction: lut[i] + t * (lut[i+1] - lut[i]).
__device__ __forceinline__ float tone(Span<const float2> table, int size, float last, float x) {
  const float f = x * static_cast<float>(size - 1);
  const int i = static_cast<int>(f);
  if (i >= size - 1) return last;
  const float t = f - static_cast<float>(i);
  const float2 e = table[i];
  return e.x + t * e.y;
}

__device__ __forceinline__ unsigned int to_fixed(float v) {
  // isp_math.hpp:245-247: units of 2^-20.
  return static_cast<unsigned int>(v * kFixedOne + 0.5F);
}

__device__ __forceinline__ int luma_code(int r, int g, int b) {
  return (2126 * r + 7152 * g + 722 * b + 5000) / 10000;  // isp_math.hpp:303-305
}

}  // namespace isp_b200
