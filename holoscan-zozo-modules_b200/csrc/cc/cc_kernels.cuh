// cc_kernels.cuh - the colour converter's kernels.
//
// Direct path (source and content the same size on both axes, which is every
// plain format conversion): whatever the resize mode, each destination pixel
// then reads exactly the one source pixel under it (bilinear and area
// weights are exactly 1 and 0 there), so a thread converts a group of four
// pixels across (two rows of them for a 4:2:0 destination: two whole chroma
// blocks) with both formats known at compile time, and writes each row's
// segment with 32-bit stores where it is aligned.
//
// Resample path: one thread per destination block (a pixel, or the pixels
// sharing a chroma sample), the source format and resize mode known at
// compile time, the destination's stores chosen at run time.
#pragma once

#include "../isp_ops.cuh"
#include "cc_common.cuh"

namespace cc_b200 {

constexpr int kGroupX = 4;     // pixels across per direct-path thread
constexpr int kThreadsX = 32;  // CTA shape for both paths
constexpr int kThreadsY = 8;
// Five 256-thread CTAs of the direct path per SM (at most 48 registers a
// thread): at four, a 4K frame's 2,025 CTAs ran 3.42 waves, the last 42 % full.
constexpr int kDirectBlocksPerSm = 5;

__device__ __forceinline__ bool yuv_dst(int f) { return f <= CC_UYVY; }

// Writes n bytes held little-endian in w to q: whole words where q is
// 4-byte aligned, bytes otherwise.
template <int kWords>
__device__ __forceinline__ void put_segment(uint8_t* q, const uint32_t (&w)[kWords], int n) {
  if ((reinterpret_cast<uintptr_t>(q) & 3U) == 0U && n == 4 * kWords) {
#pragma unroll
    for (int i = 0; i < kWords; ++i) reinterpret_cast<uint32_t*>(q)[i] = w[i];
  } else {
#pragma unroll
    for (int i = 0; i < 4 * kWords; ++i) {
      if (i < n) q[i] = static_cast<uint8_t>(w[i >> 2] >> (8 * (i & 3)));
    }
  }
}

__device__ __forceinline__ void set_byte(uint32_t* w, int i, uint32_t b) { w[i >> 2] |= b << (8 * (i & 3)); }

// One row segment of up to four destination pixels (v[0..n)) of format kDst
// at (x, y); chroma of YCbCr formats is written separately, except for the
// packed 4:2:2 ones, whose row words interleave it (cb/cr per pixel pair).
template <int kDst>
__device__ __forceinline__ void store_row4(const Image& img, int x, int y, const Px (&v)[kGroupX], int n,
                                           const uint32_t (&cb)[2], const uint32_t (&cr)[2]) {
  uint8_t* row = img.data[0] + static_cast<size_t>(y) * img.pitch[0];
  constexpr FormatInfo fi = info_of(kDst);
  constexpr int kBpp = fi.model == kYuv && fi.channels == 2 ? 2 : fi.channels * fi.bytes;
  constexpr int kWords = kBpp;  // 4 pixels x kBpp bytes = kBpp words
  uint32_t w[kWords];
#pragma unroll
  for (int i = 0; i < kWords; ++i) w[i] = 0U;
#pragma unroll
  for (int i = 0; i < kGroupX; ++i) {
    if constexpr (kDst == CC_NV12 || kDst == CC_NV16 || kDst == CC_I420 || kDst == CC_MONO8) {
      set_byte(w, i, code8(v[i].c0));
    } else if constexpr (kDst == CC_YUYV) {
      set_byte(w, 2 * i, code8(v[i].c0));
      set_byte(w, 2 * i + 1, (i & 1) ? cr[i >> 1] : cb[i >> 1]);
    } else if constexpr (kDst == CC_UYVY) {
      set_byte(w, 2 * i + 1, code8(v[i].c0));
      set_byte(w, 2 * i, (i & 1) ? cr[i >> 1] : cb[i >> 1]);
    } else if constexpr (kDst == CC_RGB8 || kDst == CC_BGR8) {
      const bool bgr = kDst == CC_BGR8;
      set_byte(w, 3 * i, code8(bgr ? v[i].c2 : v[i].c0));
      set_byte(w, 3 * i + 1, code8(v[i].c1));
      set_byte(w, 3 * i + 2, code8(bgr ? v[i].c0 : v[i].c2));
    } else if constexpr (kDst == CC_RGBA8 || kDst == CC_BGRA8) {
      const bool bgr = kDst == CC_BGRA8;
      w[i] = code8(bgr ? v[i].c2 : v[i].c0) | (code8(v[i].c1) << 8) | (code8(bgr ? v[i].c0 : v[i].c2) << 16) |
             (code8(v[i].a) << 24);
    } else if constexpr (kDst == CC_MONO16) {
      const uint32_t c = code16(v[i].c0);
      set_byte(w, 2 * i, c & 0xFFU);
      set_byte(w, 2 * i + 1, c >> 8);
    } else {
      const uint32_t r = code16(v[i].c0), g = code16(v[i].c1), b = code16(v[i].c2);
      set_byte(w, 6 * i, r & 0xFFU);
      set_byte(w, 6 * i + 1, r >> 8);
      set_byte(w, 6 * i + 2, g & 0xFFU);
      set_byte(w, 6 * i + 3, g >> 8);
      set_byte(w, 6 * i + 4, b & 0xFFU);
      set_byte(w, 6 * i + 5, b >> 8);
    }
  }
  put_segment<kWords>(row + static_cast<size_t>(x) * kBpp, w, n * kBpp);
}

// The colour map of two pixels at once: the nine products two lanes at a
// time (mul.rn.f32x2, each lane rounded as the scalar product), every sum per
// lane in the definition's order; a two-lane product never feeds a two-lane
// sum, which the assembler could fuse into one rounding.
template <bool kIdentity>
__device__ __forceinline__ void affine_pair(const Plan& p, Px& a, Px& b) {
  if constexpr (!kIdentity) {
    using isp_b200::add_lanes;
    using isp_b200::bc2;
    using isp_b200::mul2;
    const float2 s0 = make_float2(a.c0, b.c0), s1 = make_float2(a.c1, b.c1), s2 = make_float2(a.c2, b.c2);
    float2 out[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float2 t0 = mul2(bc2(p.m[3 * k]), s0);
      const float2 t1 = mul2(bc2(p.m[3 * k + 1]), s1);
      const float2 t2 = mul2(bc2(p.m[3 * k + 2]), s2);
      out[k] = add_lanes(add_lanes(add_lanes(t0, t1), t2), bc2(p.o[k]));
    }
    a.c0 = out[0].x;
    b.c0 = out[0].y;
    a.c1 = out[1].x;
    b.c1 = out[1].y;
    a.c2 = out[2].x;
    b.c2 = out[2].y;
  }
}

// code8_bits of two values: the + 0.5 and the add of 2^23 rounded toward
// zero (equal to rounding down, the value being clamped to [0, 255]) two
// lanes at a time, the clamps per lane. Neither add consumes a product, so
// nothing can be fused into it.
__device__ __forceinline__ uint2 code8_bits2(float a, float b) {
  using isp_b200::add2;
  using isp_b200::add2_rz;
  using isp_b200::bc2;
  const float2 h = add2(make_float2(a, b), bc2(0.5F));
  const float2 c = make_float2(fminf(fmaxf(h.x, 0.0F), 255.0F), fminf(fmaxf(h.y, 0.0F), 255.0F));
  const float2 r = add2_rz(c, bc2(kTwo23));
  return make_uint2(__float_as_uint(r.x), __float_as_uint(r.y));
}

// One four-pixel row segment of format kDst at (x, y) from whole, aligned
// groups: every word of it stored, the row start known to be 4-byte aligned.
// Codes come as their 2^23-biased bits (code8_bits / code16_bits); cb and cr
// are the pair chroma of the packed 4:2:2 formats.
template <int kDst>
__device__ __forceinline__ void store_full4(const Image& img, int x, int y, const Px (&v)[kGroupX],
                                            const uint32_t (&cb)[2], const uint32_t (&cr)[2]) {
  uint8_t* row = img.data[0] + static_cast<size_t>(y) * img.pitch[0];
  if constexpr (kDst == CC_NV12 || kDst == CC_NV16 || kDst == CC_I420 || kDst == CC_MONO8) {
    const uint2 a = code8_bits2(v[0].c0, v[1].c0), b = code8_bits2(v[2].c0, v[3].c0);
    *reinterpret_cast<uint32_t*>(row + x) = pack8(a.x, a.y, b.x, b.y);
  } else if constexpr (kDst == CC_YUYV || kDst == CC_UYVY) {
    uint32_t* q = reinterpret_cast<uint32_t*>(row + 2 * x);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const uint2 yy = code8_bits2(v[2 * k].c0, v[2 * k + 1].c0);
      q[k] = kDst == CC_YUYV ? pack8(yy.x, cb[k], yy.y, cr[k]) : pack8(cb[k], yy.x, cr[k], yy.y);
    }
  } else if constexpr (kDst == CC_RGB8 || kDst == CC_BGR8) {
    const bool bgr = kDst == CC_BGR8;
    uint32_t b[12];
#pragma unroll
    for (int i = 0; i < 4; i += 2) {
      const uint2 r = code8_bits2(bgr ? v[i].c2 : v[i].c0, bgr ? v[i + 1].c2 : v[i + 1].c0);
      const uint2 g = code8_bits2(v[i].c1, v[i + 1].c1);
      const uint2 bl = code8_bits2(bgr ? v[i].c0 : v[i].c2, bgr ? v[i + 1].c0 : v[i + 1].c2);
      b[3 * i] = r.x;
      b[3 * i + 1] = g.x;
      b[3 * i + 2] = bl.x;
      b[3 * i + 3] = r.y;
      b[3 * i + 4] = g.y;
      b[3 * i + 5] = bl.y;
    }
    uint32_t* q = reinterpret_cast<uint32_t*>(row + 3 * x);
#pragma unroll
    for (int k = 0; k < 3; ++k) q[k] = pack8(b[4 * k], b[4 * k + 1], b[4 * k + 2], b[4 * k + 3]);
  } else if constexpr (kDst == CC_RGBA8 || kDst == CC_BGRA8) {
    const bool bgr = kDst == CC_BGRA8;
    uint32_t* q = reinterpret_cast<uint32_t*>(row + 4 * x);
#pragma unroll
    for (int i = 0; i < 4; i += 2) {
      const uint2 r = code8_bits2(bgr ? v[i].c2 : v[i].c0, bgr ? v[i + 1].c2 : v[i + 1].c0);
      const uint2 g = code8_bits2(v[i].c1, v[i + 1].c1);
      const uint2 bl = code8_bits2(bgr ? v[i].c0 : v[i].c2, bgr ? v[i + 1].c0 : v[i + 1].c2);
      const uint2 al = code8_bits2(v[i].a, v[i + 1].a);
      q[i] = pack8(r.x, g.x, bl.x, al.x);
      q[i + 1] = pack8(r.y, g.y, bl.y, al.y);
    }
  } else if constexpr (kDst == CC_MONO16) {
    uint32_t* q = reinterpret_cast<uint32_t*>(row + 2 * x);
    q[0] = pack16(code16_bits(v[0].c0), code16_bits(v[1].c0));
    q[1] = pack16(code16_bits(v[2].c0), code16_bits(v[3].c0));
  } else {
    uint32_t h[12];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      h[3 * i] = code16_bits(v[i].c0);
      h[3 * i + 1] = code16_bits(v[i].c1);
      h[3 * i + 2] = code16_bits(v[i].c2);
    }
    uint32_t* q = reinterpret_cast<uint32_t*>(row + 6 * x);
#pragma unroll
    for (int k = 0; k < 6; ++k) q[k] = pack16(h[2 * k], h[2 * k + 1]);
  }
}

// Four-pixel subgroups a direct-path thread takes across: two for a 4:2:0
// destination (whose thread also takes two rows), four otherwise, so that
// each thread has a few dozen bytes of loads in flight.
__host__ __device__ constexpr int direct_subgroups(int dst) {
  return (dst == CC_NV12 || dst == CC_I420) ? 2 : 4;
}

// Direct path: a warp converts kSub x 32 four-pixel groups of rows
// [gy << bsy, (gy + 1) << bsy); its lane L takes groups g0 + 32 h (h < kSub),
// so that every load and store instruction of the warp covers contiguous
// bytes. All of a thread's whole, aligned source groups are read first
// (fetch4); then each group is converted and stored; pixels outside the
// content take the fill, and groups that are partial or unaligned read pixel
// by pixel. groups_x = ceil(width / 4).
template <int kSrc, int kDst>
__global__ void __launch_bounds__(kThreadsX* kThreadsY, kDirectBlocksPerSm) cc_direct_kernel(const __grid_constant__ Plan p, int groups_x,
                                                                         int groups_y) {
  const int gy = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
  if (gy >= groups_y) return;
  constexpr FormatInfo fi = info_of(kDst);
  constexpr bool kYuvDst = fi.model == kYuv;
  constexpr int kRows = kYuvDst ? (1 << fi.shift_y) : 1;
  constexpr int kSub = direct_subgroups(kDst);
  const int g0 = static_cast<int>(blockIdx.x) * kThreadsX * kSub + static_cast<int>(threadIdx.x);
  if (g0 >= groups_x) return;
  const int y0 = gy * kRows;
  // Source offset of destination pixel (x, y) inside the content.
  const int ox = p.sx0 - p.cx0;
  const int oy = p.sy0 - p.cy0;

  uint32_t raw[kRows][kSub][kRawWords];
  bool ok[kRows][kSub];
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    const int y = y0 + r;
    const bool row_in = (r == 0 || y < p.dst.height) && y >= p.cy0 && y < p.cy1;
#pragma unroll
    for (int h = 0; h < kSub; ++h) {
      const int xs = (g0 + kThreadsX * h) * kGroupX;
      ok[r][h] = row_in && xs + kGroupX <= p.dst.width && xs >= p.cx0 && xs + kGroupX <= p.cx1 &&
                 fetch4<kSrc>(p.src, xs + ox, y + oy, raw[r][h]);
    }
  }

  // Interior fast path: every group fetched (so whole, inside the content
  // and the frame, rows included) and every destination row it writes
  // 4-byte aligned (2-byte for the I420 chroma planes): no per-pixel checks.
  bool full = true;
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
#pragma unroll
    for (int h = 0; h < kSub; ++h) full = full && ok[r][h];
    full = full && aligned4(row_of(p.dst, 0, y0 + r));
  }
  if constexpr (kDst == CC_NV12 || kDst == CC_NV16) {
    full = full && aligned4(row_of(p.dst, 1, y0 >> fi.shift_y));
  } else if constexpr (kDst == CC_I420) {
    full = full && ((reinterpret_cast<uintptr_t>(row_of(p.dst, 1, y0 >> 1)) |
                     reinterpret_cast<uintptr_t>(row_of(p.dst, 2, y0 >> 1))) & 1U) == 0U;
  }
  if (full) {
    constexpr bool kIdentity = info_of(kSrc).model == fi.model;
#pragma unroll
    for (int h = 0; h < kSub; ++h) {
      const int xs = (g0 + kThreadsX * h) * kGroupX;
      float cbs[2] = {0.0F, 0.0F}, crs[2] = {0.0F, 0.0F};
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        Px v[kGroupX];
        decode4<kSrc>(raw[r][h], v);
        affine_pair<kIdentity>(p, v[0], v[1]);
        affine_pair<kIdentity>(p, v[2], v[3]);
#pragma unroll
        for (int i = 0; i < kGroupX; ++i) {
          if constexpr (kYuvDst) {
            cbs[i >> 1] = __fadd_rn(cbs[i >> 1], v[i].c1);
            crs[i >> 1] = __fadd_rn(crs[i >> 1], v[i].c2);
          }
        }
        uint32_t cb[2] = {0U, 0U}, cr[2] = {0U, 0U};
        if constexpr (kDst == CC_YUYV || kDst == CC_UYVY) {
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            cb[b] = code8_bits(__fmul_rn(cbs[b], 0.5F));
            cr[b] = code8_bits(__fmul_rn(crs[b], 0.5F));
          }
        }
        store_full4<kDst>(p.dst, xs, y0 + r, v, cb, cr);
      }
      if constexpr (kDst == CC_NV12 || kDst == CC_NV16 || kDst == CC_I420) {
        constexpr float kInv = kRows == 2 ? 0.25F : 0.5F;  // 2 x kRows pixels a block
        const uint32_t b0 = code8_bits(__fmul_rn(cbs[0], kInv)), r0 = code8_bits(__fmul_rn(crs[0], kInv));
        const uint32_t b1 = code8_bits(__fmul_rn(cbs[1], kInv)), r1 = code8_bits(__fmul_rn(crs[1], kInv));
        const int cy = y0 >> fi.shift_y;
        if constexpr (kDst == CC_I420) {
          *reinterpret_cast<uint16_t*>(p.dst.data[1] + static_cast<size_t>(cy) * p.dst.pitch[1] + (xs >> 1)) =
              static_cast<uint16_t>(__byte_perm(b0, b1, 0x0040U));
          *reinterpret_cast<uint16_t*>(p.dst.data[2] + static_cast<size_t>(cy) * p.dst.pitch[2] + (xs >> 1)) =
              static_cast<uint16_t>(__byte_perm(r0, r1, 0x0040U));
        } else {
          *reinterpret_cast<uint32_t*>(p.dst.data[1] + static_cast<size_t>(cy) * p.dst.pitch[1] + xs) =
              pack8(b0, r0, b1, r1);
        }
      }
    }
    return;
  }

#pragma unroll
  for (int h = 0; h < kSub; ++h) {
    const int xs = (g0 + kThreadsX * h) * kGroupX;
    if (xs >= p.dst.width) break;  // later groups lie further right
    const int n = p.dst.width - xs < kGroupX ? p.dst.width - xs : kGroupX;
    float cbs[2] = {0.0F, 0.0F}, crs[2] = {0.0F, 0.0F};
    int rows = 0;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int y = y0 + r;
      if (r > 0 && y >= p.dst.height) break;
      ++rows;
      Px v[kGroupX];
      if (ok[r][h]) {
        decode4<kSrc>(raw[r][h], v);
#pragma unroll
        for (int i = 0; i < kGroupX; ++i) v[i] = apply_affine(p, v[i]);
      } else {
        const bool row_in = y >= p.cy0 && y < p.cy1;
#pragma unroll
        for (int i = 0; i < kGroupX; ++i) {
          const int x = xs + i;
          if (i < n && row_in && x >= p.cx0 && x < p.cx1) {
            v[i] = apply_affine(p, load_px<kSrc>(p.src, x + ox, y + oy));
          } else {
            v[i] = Px{p.fill[0], p.fill[1], p.fill[2], p.fill[3]};
          }
        }
      }
      if constexpr (kYuvDst) {
#pragma unroll
        for (int i = 0; i < kGroupX; ++i) {
          if (i < n) {
            cbs[i >> 1] = __fadd_rn(cbs[i >> 1], v[i].c1);
            crs[i >> 1] = __fadd_rn(crs[i >> 1], v[i].c2);
          }
        }
      }
      // Chroma means: a block holds 1, 2 or 4 pixels, and a sum of these
      // samples is zero or far above the subnormals, so dividing by the count
      // (as the definition does) is exactly the product by its reciprocal.
      if constexpr (kDst == CC_YUYV || kDst == CC_UYVY) {
        // One row per block: the chroma of each pixel pair is known now.
        uint32_t cb[2], cr[2];
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          const float inv = n - 2 * b >= 2 ? 0.5F : 1.0F;
          cb[b] = code8(__fmul_rn(cbs[b], inv));
          cr[b] = code8(__fmul_rn(crs[b], inv));
        }
        store_row4<kDst>(p.dst, xs, y, v, n, cb, cr);
      } else {
        const uint32_t none[2] = {0U, 0U};
        store_row4<kDst>(p.dst, xs, y, v, n, none, none);
      }
    }
    if constexpr (kDst == CC_NV12 || kDst == CC_NV16 || kDst == CC_I420) {
      const int cx = xs >> 1;
      const int cy = y0 >> fi.shift_y;
      const int nb = (n + 1) >> 1;  // chroma samples in this subgroup: 1 or 2
      uint32_t code[2][2];
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int cnt = (n - 2 * b >= 2 ? 2 : 1) * rows;
        const float inv = cnt == 4 ? 0.25F : (cnt == 2 ? 0.5F : 1.0F);
        code[b][0] = code8(__fmul_rn(cbs[b], inv));
        code[b][1] = code8(__fmul_rn(crs[b], inv));
      }
      if constexpr (kDst == CC_I420) {
        uint8_t* u = p.dst.data[1] + static_cast<size_t>(cy) * p.dst.pitch[1] + cx;
        uint8_t* vv = p.dst.data[2] + static_cast<size_t>(cy) * p.dst.pitch[2] + cx;
        if (nb == 2 && (reinterpret_cast<uintptr_t>(u) & 1U) == 0U && (reinterpret_cast<uintptr_t>(vv) & 1U) == 0U) {
          *reinterpret_cast<uint16_t*>(u) = static_cast<uint16_t>(code[0][0] | (code[1][0] << 8));
          *reinterpret_cast<uint16_t*>(vv) = static_cast<uint16_t>(code[0][1] | (code[1][1] << 8));
        } else {
          u[0] = static_cast<uint8_t>(code[0][0]);
          vv[0] = static_cast<uint8_t>(code[0][1]);
          if (nb == 2) {
            u[1] = static_cast<uint8_t>(code[1][0]);
            vv[1] = static_cast<uint8_t>(code[1][1]);
          }
        }
      } else {
        uint8_t* q = p.dst.data[1] + static_cast<size_t>(cy) * p.dst.pitch[1] + 2 * cx;
        const uint32_t w[1] = {code[0][0] | (code[0][1] << 8) | (code[1][0] << 16) | (code[1][1] << 24)};
        put_segment<1>(q, w, 2 * nb);
      }
    }
  }
}

// Resample path helpers: the destination's stores chosen at run time.
__device__ __forceinline__ void store_any(const Image& img, int x, int y, const Px& v) {
  switch (img.format) {
    case CC_NV12: store_px<CC_NV12>(img, x, y, v); break;
    case CC_NV16: store_px<CC_NV16>(img, x, y, v); break;
    case CC_I420: store_px<CC_I420>(img, x, y, v); break;
    case CC_YUYV: store_px<CC_YUYV>(img, x, y, v); break;
    case CC_UYVY: store_px<CC_UYVY>(img, x, y, v); break;
    case CC_RGB8: store_px<CC_RGB8>(img, x, y, v); break;
    case CC_BGR8: store_px<CC_BGR8>(img, x, y, v); break;
    case CC_RGBA8: store_px<CC_RGBA8>(img, x, y, v); break;
    case CC_BGRA8: store_px<CC_BGRA8>(img, x, y, v); break;
    case CC_MONO8: store_px<CC_MONO8>(img, x, y, v); break;
    case CC_MONO16: store_px<CC_MONO16>(img, x, y, v); break;
    default: store_px<CC_RGB16>(img, x, y, v); break;
  }
}

__device__ __forceinline__ void store_chroma_any(const Image& img, int cx, int cy, float cb, float cr) {
  switch (img.format) {
    case CC_NV12: store_chroma<CC_NV12>(img, cx, cy, cb, cr); break;
    case CC_NV16: store_chroma<CC_NV16>(img, cx, cy, cb, cr); break;
    case CC_I420: store_chroma<CC_I420>(img, cx, cy, cb, cr); break;
    case CC_YUYV: store_chroma<CC_YUYV>(img, cx, cy, cb, cr); break;
    default: store_chroma<CC_UYVY>(img, cx, cy, cb, cr); break;
  }
}

template <int kSrc, int kMode>
__device__ __forceinline__ Px pixel_at(const Plan& p, int x, int y) {
  if (!in_content(p, x, y)) return Px{p.fill[0], p.fill[1], p.fill[2], p.fill[3]};
  return apply_affine(p, sample_px<kSrc, kMode>(p, x, y));
}

// Resample path: thread (bx, by) converts destination block (bx, by)
// (kernel_math.hpp:345-370).
template <int kSrc, int kMode>
__global__ void __launch_bounds__(kThreadsX* kThreadsY) cc_resample_kernel(const __grid_constant__ Plan p, int across,
                                                                           int down) {
  const int bx = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  const int by = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
  if (bx >= across || by >= down) return;
  if (!yuv_dst(p.dst.format)) {
    store_any(p.dst, bx, by, pixel_at<kSrc, kMode>(p, bx, by));
    return;
  }
  const int x0 = bx << p.bsx;
  const int y0 = by << p.bsy;
  const int x1 = min(x0 + (1 << p.bsx), p.dst.width);
  const int y1 = min(y0 + (1 << p.bsy), p.dst.height);
  float cb = 0.0F, cr = 0.0F;
  int n = 0;
  for (int y = y0; y < y1; ++y) {
    for (int x = x0; x < x1; ++x) {
      const Px v = pixel_at<kSrc, kMode>(p, x, y);
      store_any(p.dst, x, y, v);
      cb = __fadd_rn(cb, v.c1);
      cr = __fadd_rn(cr, v.c2);
      ++n;
    }
  }
  const float cnt = static_cast<float>(n);
  store_chroma_any(p.dst, bx, by, __fdiv_rn(cb, cnt), __fdiv_rn(cr, cnt));
}

// Launchers of each source format's direct kernels (cc_direct_*.cu) and of
// the resample kernels (cc_resample.cu): a kernel pointer or null.
const void* direct_kernel(int src, int dst);
const void* direct_kernel_yuv(int src, int dst);
const void* direct_kernel_rgb(int src, int dst);
const void* direct_kernel_gray(int src, int dst);
const void* resample_kernel(int src, int mode);

}  // namespace cc_b200
