// isp_awb.cuh - the white balance statistics pass as device templates: the
// sums of one 64x64-sample tile, and a frame's flush by a CTA with the
// last-tile finish. The single-frame kernel (isp_awb.cu) and the batch kernel
// (isp_batch.cu) are both built from them.
#pragma once

#include "isp_common.cuh"

namespace isp_b200 {
namespace {

__host__ __device__ constexpr int awb_box_bytes(int fmt) {
  return fmt == kRawU8 ? 64 : fmt == kRawU16 ? 128 : fmt == kRawRaw10 ? 80 : 96;
}

// TMA x coordinate (bytes, or uint16 samples) of the statistics box of a
// tile at column x0 (x0 % 64 == 0): 16-byte aligned.
__device__ __forceinline__ int awb_box_x(int fmt, int x0) {
  return fmt == kRawRaw10 ? 5 * (x0 >> 2) : fmt == kRawRaw12 ? 3 * (x0 >> 1) : x0;
}

// Units of two complete quads (4 samples across, 2 rows) of one tile: the
// white balance sums (white_balance_quad, isp_math.hpp:311-332) into 32-bit
// per-tile sums (at most 8 samples of 2^22 per colour and thread) and, for
// white patch, the block's bins.
template <int kFmt, int kSrc, bool kWhitePatch, int kPat>
__device__ __forceinline__ void awb_tile(const FrameDesc& p, Span<const uint8_t> box, int box_bytes, int x0, int y0,
                                         const LscTile& lt, Span<const int> row_k, Span<const float> row_ty,
                                         Span<const float> table, const float (&black)[4], const float (&inv)[4],
                                         Span<unsigned int> hist, unsigned int (&sum)[3], unsigned int& quads) {
  const int quads_x = p.width / 2;
  const int quads_y = p.height / 2;
  const unsigned int white = static_cast<unsigned int>(p.white);
  unsigned int counted = 0;  // quads summed by this call
  static_assert(512 % kThreads == 0, "a tile's units split evenly over the block");
#pragma unroll
  for (int it = 0; it < 512 / kThreads; ++it) {
    const int unit = static_cast<int>(threadIdx.x) + it * kThreads;
    const int a = unit >> 4;
    const int u = unit & 15;
    const int qy = (y0 >> 1) + a;
    const int qx0 = (x0 >> 1) + 2 * u;
    if (qy >= quads_y || qx0 >= quads_x) continue;
    unsigned int top[4], bot[4];
    if constexpr (kSrc == 0) {
      Span<const uint8_t> r0 = box + (2 * a) * box_bytes;
      Span<const uint8_t> r1 = r0 + box_bytes;
      if constexpr (kFmt == kRawU8) {
        const unsigned int w0 = *span_cast<const unsigned int>(r0 + 4 * u);
        const unsigned int w1 = *span_cast<const unsigned int>(r1 + 4 * u);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          top[k] = (w0 >> (8 * k)) & 0xFFU;
          bot[k] = (w1 >> (8 * k)) & 0xFFU;
        }
      } else if constexpr (kFmt == kRawU16) {
        const uint2 w0 = *span_cast<const uint2>(r0 + 8 * u);
        const uint2 w1 = *span_cast<const uint2>(r1 + 8 * u);
        top[0] = w0.x & 0xFFFFU; top[1] = w0.x >> 16; top[2] = w0.y & 0xFFFFU; top[3] = w0.y >> 16;
        bot[0] = w1.x & 0xFFFFU; bot[1] = w1.x >> 16; bot[2] = w1.y & 0xFFFFU; bot[3] = w1.y >> 16;
      } else {
        // unpack4 reads sample x0 - 4 + 4u' from a box starting 16 bytes
        // before x0; this box starts at x0: step the row back 16 bytes, u' = u + 1.
        unpack4(kFmt, r0 - 16, u + 1, top);
        unpack4(kFmt, r1 - 16, u + 1, bot);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int x = x0 + 4 * u + k;
        top[k] = x < p.width ? static_cast<unsigned int>(load_raw(p, x, y0 + 2 * a)) : 0U;
        bot[k] = x < p.width ? static_cast<unsigned int>(load_raw(p, x, y0 + 2 * a + 1)) : 0U;
      }
    }
    // Linear values before white balance, capped at 4 (isp_math.hpp:320-330).
    // The two quads of the unit run as the two lanes of f32x2 instructions:
    // lane x holds sample j of quad 0, lane y sample j of quad 1 (columns
    // 4u + j and 4u + j + 2, the same Bayer colour). The products feed only a
    // multiply, a clamp, a per-lane sum or an exact power-of-two scale
    // (isp_ops.cuh).
    float2 v[2][2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const unsigned int* s = r == 0 ? top : bot;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int q = (r << 1) | j;
        const float2 lin = mul2(sub2(magic_to_float2(s[j] | kTwo23Bits, s[j + 2] | kTwo23Bits), bc2(black[q])),
                                bc2(inv[q]));
        v[r][j] = make_float2(fmaxf(lin.x, 0.0F), fmaxf(lin.y, 0.0F));
      }
    }
    if (lt.rows > 0) {
      if (lt.rows <= kLscTableRows) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int rj = 2 * a + r;
          const int kk = row_k[rj];
          const float2 tyj = bc2(row_ty[rj]);
          const int pl = p.lsc_channels == 4 ? r : 0;
          const float4 t0 = *span_cast<const float4>(table + (kk * 2 + pl) * kSW + 4 * u);
          const float4 t1 = *span_cast<const float4>(table + ((kk + 1) * 2 + pl) * kSW + 4 * u);
          // gain = t0 + (t1 - t0) ty per column (lens_shading_gain, isp_math.hpp:121-140).
          const float2 a0 = make_float2(t0.x, t0.z), a1 = make_float2(t0.y, t0.w);
          const float2 g0 = add_lanes(a0, mul2(sub2(make_float2(t1.x, t1.z), a0), tyj));
          const float2 g1 = add_lanes(a1, mul2(sub2(make_float2(t1.y, t1.w), a1), tyj));
          v[r][0] = mul2(v[r][0], g0);
          v[r][1] = mul2(v[r][1], g1);
        }
      } else {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int channel = cfa_of(kPat, (r << 1) | j);
            const float gx = lens_shading_gain(p, p.lsc, x0 + 4 * u + j, y0 + 2 * a + r, channel);
            const float gy = lens_shading_gain(p, p.lsc, x0 + 4 * u + j + 2, y0 + 2 * a + r, channel);
            v[r][j] = mul2(v[r][j], make_float2(gx, gy));
          }
        }
      }
    }
    // The quad test per lane: no sample at or above white (isp_math.hpp:316-318).
    const bool ok0 = qx0 < quads_x && top[0] < white && top[1] < white && bot[0] < white && bot[1] < white;
    const bool ok1 = qx0 + 1 < quads_x && top[2] < white && top[3] < white && bot[2] < white && bot[3] < white;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 x = make_float2(fminf(v[k >> 1][k & 1].x, 4.0F), fminf(v[k >> 1][k & 1].y, 4.0F));
      // to_fixed: trunc(x 2^20 + 0.5), the product exact. Summed as 2^23
      // bits + value; the 2^23 bits come off once, after the units.
      const float2 m = magic_trunc2(exact_scale_add2(x, bc2(kFixedOne), bc2(0.5F)));
      sum[color_of(cfa_of(kPat, k))] += (ok0 ? __float_as_uint(m.x) : 0U) + (ok1 ? __float_as_uint(m.y) : 0U);
      if constexpr (kWhitePatch) {
        // trunc(x 1024): an exact product, so its two-lane truncation is safe.
        const float2 b = magic_trunc2(mul2(x, bc2(static_cast<float>(kAwbBins))));
        const unsigned int b0 = magic_int(b.x), b1 = magic_int(b.y);
        Span<unsigned int> h = hist + color_of(cfa_of(kPat, k)) * kAwbBins;
        if (ok0) atomicAdd(&h[b0 < kAwbBins - 1 ? b0 : kAwbBins - 1], 1U);
        if (ok1) atomicAdd(&h[b1 < kAwbBins - 1 ? b1 : kAwbBins - 1], 1U);
      }
    }
    counted += (ok0 ? 1U : 0U) + (ok1 ? 1U : 0U);
  }
  // Every counted quad added one red, two green and one blue sample, each
  // with 2^23 bits on top (sums mod 2^32; the true sums fit 32 bits).
  sum[0] -= counted * kTwo23Bits;
  sum[1] -= 2U * counted * kTwo23Bits;
  sum[2] -= counted * kTwo23Bits;
  quads += counted;
}

template <int kSrc, bool kWhitePatch, int kPat>
__device__ __forceinline__ void awb_tile_fmt(const FrameDesc& p, Span<const uint8_t> box, int box_bytes, int x0, int y0,
                                             const LscTile& lt, Span<const int> row_k, Span<const float> row_ty,
                                             Span<const float> table, const float (&black)[4], const float (&inv)[4],
                                             Span<unsigned int> hist, unsigned int (&sum)[3], unsigned int& quads) {
  if constexpr (kSrc == 1) {
    awb_tile<kRawU8, 1, kWhitePatch, kPat>(p, box, box_bytes, x0, y0, lt, row_k, row_ty, table, black, inv, hist, sum, quads);
  } else {
    switch (p.raw_format) {
      case kRawU8:
        awb_tile<kRawU8, 0, kWhitePatch, kPat>(p, box, box_bytes, x0, y0, lt, row_k, row_ty, table, black, inv, hist, sum, quads);
        break;
      case kRawU16:
        awb_tile<kRawU16, 0, kWhitePatch, kPat>(p, box, box_bytes, x0, y0, lt, row_k, row_ty, table, black, inv, hist, sum, quads);
        break;
      case kRawRaw10:
        awb_tile<kRawRaw10, 0, kWhitePatch, kPat>(p, box, box_bytes, x0, y0, lt, row_k, row_ty, table, black, inv, hist, sum, quads);
        break;
      default:
        awb_tile<kRawRaw12, 0, kWhitePatch, kPat>(p, box, box_bytes, x0, y0, lt, row_k, row_ty, table, black, inv, hist, sum, quads);
        break;
    }
  }
}

// A frame's flush by one CTA after it summed `tiles_done` of the frame's
// `tiles_total` statistics tiles: block sums and bins into the frame's
// scratch; the CTA that completes the count forms the frame's estimate
// (awb_finish). The block's bins are left for the caller to clear.
// With kAfterPrevious, the last CTA first waits (griddepcontrol.wait) for the
// kernel this pass was launched behind: the single-frame pass may begin
// while the previous frame's tile pass finishes, and only the estimate
// (which reads and writes the white balance state that tile pass read) must
// follow it.
template <bool kAfterPrevious = false>
__device__ void awb_flush(const FrameDesc& p, const u64 (&acc)[4], Span<const unsigned int> hist, bool white_patch,
                          u64* red, int* first, bool* last, unsigned int tiles_done, unsigned int tiles_total) {
  Span<Scratch> s = p.scratch;
  const int tid = threadIdx.x;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const u64 total = block_sum(acc[k], red);
    if (tid == 0 && total != 0) atomicAdd(k < 3 ? &s->awb_sum[k] : &s->awb_quads, total);
  }
  if (white_patch) {
    __syncthreads();
    const Span<unsigned int> bins = sub_span(s, &s->awb_hist[0][0], 3 * kAwbBins);
    for (int i = tid; i < 3 * kAwbBins; i += kThreads) {
      if (hist[i] != 0U) atomicAdd(&bins[i], hist[i]);
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) *last = atomicAdd(&s->awb_done, tiles_done) + tiles_done == tiles_total;
  __syncthreads();
  if (*last) {
    if constexpr (kAfterPrevious) griddep_wait();
    __threadfence();
    awb_finish(p, s, red, first);
  }
  __syncthreads();
}

}  // namespace
}  // namespace isp_b200
