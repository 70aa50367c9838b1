// cc_common.cuh - the B200 colour converter's plan and per-pixel arithmetic.
//
// One conversion is defined as in holoscan::color_convert
// (modules/color-convert/include/holoscan/color_convert/conversion.hpp:9-27,
// arithmetic in src/kernel_math.hpp:70-370):
//   1. a source pixel decodes to its format's samples (Y Cb Cr, R G B or
//      luma; chroma from the chroma sample covering the pixel; 16-bit
//      samples divided by 257; alpha 255 unless stored);
//   2. a destination pixel inside the content rectangle samples the source
//      rectangle (nearest, bilinear or area); outside it takes the fill;
//   3. the samples go through one 3x4 affine map to the destination's
//      model (none between equal models), are rounded half up and clamped;
//      a subsampled destination stores the mean chroma of its block.
// Every sum and product below is a separate IEEE single operation, in the
// reference's order (the library is compiled with --fmad=false), so the
// kernels give the reference's bytes.
#pragma once

#include <cstddef>
#include <cstdint>

#include "cc_b200.h"

#if defined(__CUDACC__)
#define CC_HD __host__ __device__ __forceinline__
#else
#define CC_HD inline
#endif

namespace cc_b200 {

enum Model : int { kYuv = 0, kRgb = 1, kGray = 2 };

struct FormatInfo {
  int model, planes, shift_x, shift_y, bytes, channels;
};

// pixel_format.hpp:58-84.
CC_HD constexpr FormatInfo info_of(int f) {
  return f == CC_NV12    ? FormatInfo{kYuv, 2, 1, 1, 1, 1}
         : f == CC_NV16  ? FormatInfo{kYuv, 2, 1, 0, 1, 1}
         : f == CC_I420  ? FormatInfo{kYuv, 3, 1, 1, 1, 1}
         : f == CC_YUYV  ? FormatInfo{kYuv, 1, 1, 0, 1, 2}
         : f == CC_UYVY  ? FormatInfo{kYuv, 1, 1, 0, 1, 2}
         : f == CC_RGB8  ? FormatInfo{kRgb, 1, 0, 0, 1, 3}
         : f == CC_BGR8  ? FormatInfo{kRgb, 1, 0, 0, 1, 3}
         : f == CC_RGBA8 ? FormatInfo{kRgb, 1, 0, 0, 1, 4}
         : f == CC_BGRA8 ? FormatInfo{kRgb, 1, 0, 0, 1, 4}
         : f == CC_MONO8 ? FormatInfo{kGray, 1, 0, 0, 1, 1}
         : f == CC_MONO16 ? FormatInfo{kGray, 1, 0, 0, 2, 1}
                          : FormatInfo{kRgb, 1, 0, 0, 2, 3};
}

struct Image {
  int format, width, height;
  uint8_t* data[3];
  size_t pitch[3];
};

// Everything one conversion needs, by value in the kernel's parameters.
struct Plan {
  Image src, dst;
  int mode;
  int sx0, sy0, sx1, sy1;  // source rectangle, inclusive bounds
  float scale_x, scale_y;  // source pixels per content pixel
  int cx0, cy0, cx1, cy1;  // content rectangle [cx0, cx1) x [cy0, cy1)
  float m[9], o[3];
  int identity;
  float fill[4];  // in the destination's model
  int bsx, bsy;   // log2 of the pixels one destination chroma sample covers
};

struct Px {
  float c0, c1, c2, a;
};

#if defined(__CUDACC__)

// Integers to floats and back without the conversion unit (a quarter of the
// FP32 rate): 2^23 + k has k in its low mantissa bits for 0 <= k < 2^23, so
// a byte b becomes the float b exactly as (2^23 + b) - 2^23, and a float c in
// [0, 2^23) becomes floor(c) as the mantissa of c + 2^23 rounded down.
constexpr uint32_t kTwo23Bits = 0x4B000000U;
constexpr float kTwo23 = 8388608.0F;

__device__ __forceinline__ float byte_f(uint32_t b) { return __fsub_rn(__uint_as_float(kTwo23Bits | b), kTwo23); }

// Byte k (0..3) of w as a float, exactly.
__device__ __forceinline__ float byte_of(uint32_t w, int k) {
  return __fsub_rn(__uint_as_float(__byte_perm(w, kTwo23Bits, 0x7650U | static_cast<uint32_t>(k))), kTwo23);
}

__device__ __forceinline__ uint32_t floor_bits(float c) { return __float_as_uint(__fadd_rd(c, kTwo23)) - kTwo23Bits; }

// code8 and code16 (below) left in the bits of 2^23 + code: the code in the
// low byte (low half-word) for packing with byte permutes.
__device__ __forceinline__ uint32_t code8_bits(float v) {
  return __float_as_uint(__fadd_rd(fminf(fmaxf(__fadd_rn(v, 0.5F), 0.0F), 255.0F), kTwo23));
}
__device__ __forceinline__ uint32_t code16_bits(float v) {
  return __float_as_uint(__fadd_rd(fminf(fmaxf(__fadd_rn(__fmul_rn(v, 257.0F), 0.5F), 0.0F), 65535.0F), kTwo23));
}
// The low bytes of a, b, c, d as one little-endian word.
__device__ __forceinline__ uint32_t pack8(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  return __byte_perm(__byte_perm(a, b, 0x0040U), __byte_perm(c, d, 0x0040U), 0x5410U);
}
// The low half-words of a and b as one little-endian word.
__device__ __forceinline__ uint32_t pack16(uint32_t a, uint32_t b) { return __byte_perm(a, b, 0x5410U); }

// Rounded half up and clamped to 0..255 (kernel_math.hpp:89-92): r =
// floor(v + 0.5) then 0 where r <= 0 and 255 where r >= 255 equals the floor
// of v + 0.5 first clamped to [0, 255].
__device__ __forceinline__ uint32_t code8(float v) {
  return floor_bits(fminf(fmaxf(__fadd_rn(v, 0.5F), 0.0F), 255.0F));
}

// 16-bit codes: the floor of v * 257 + 0.5, clamped to 0..65535 (:94-97).
__device__ __forceinline__ uint32_t code16(float v) {
  return floor_bits(fminf(fmaxf(__fadd_rn(__fmul_rn(v, 257.0F), 0.5F), 0.0F), 65535.0F));
}

// v / 257 correctly rounded for an integer 0 <= v < 2^16, as the IEEE
// division the definition uses (:99-104): the product by r = RN(1/257)
// corrected once by its exact FMA residual (Markstein's correction step),
// which gives the correctly rounded quotient for every one of the 65,536
// inputs (checked exhaustively against exact rational arithmetic, and on the
// GPU against the oracle's division).
__device__ __forceinline__ float div257(uint32_t v) {
  constexpr float kR = 1.0F / 257.0F;
  const float x = byte_f(v);  // exact for v < 2^23
  const float q = __fmul_rn(x, kR);
  const float e = __fmaf_rn(-q, 257.0F, x);
  return __fmaf_rn(e, kR, q);
}

// A 16-bit little-endian sample on the 8-bit scale, read byte-wise since a
// pitched row of 16-bit samples need not be 2-byte aligned.
__device__ __forceinline__ float word_sample(const uint8_t* p) {
  return div257(static_cast<uint32_t>(__ldg(p)) | (static_cast<uint32_t>(__ldg(p + 1)) << 8));
}

__device__ __forceinline__ const uint8_t* row_of(const Image& img, int plane, int y) {
  return img.data[plane] + static_cast<size_t>(y) * img.pitch[plane];
}

// Pixel (x, y) of a source image of format kF, in its own samples (:112-161).
template <int kF>
__device__ __forceinline__ Px load_px(const Image& img, int x, int y) {
  const uint8_t* row = row_of(img, 0, y);
  if constexpr (kF == CC_NV12 || kF == CC_NV16) {
    const uint8_t* uv = row_of(img, 1, kF == CC_NV12 ? (y >> 1) : y) + 2 * (x >> 1);
    return {byte_f(__ldg(row + x)), byte_f(__ldg(uv)), byte_f(__ldg(uv + 1)), 255.0F};
  } else if constexpr (kF == CC_I420) {
    const int cx = x >> 1, cy = y >> 1;
    return {byte_f(__ldg(row + x)), byte_f(__ldg(row_of(img, 1, cy) + cx)), byte_f(__ldg(row_of(img, 2, cy) + cx)),
            255.0F};
  } else if constexpr (kF == CC_YUYV) {
    const uint8_t* pair = row + 4 * (x >> 1);
    return {byte_f(__ldg(pair + 2 * (x & 1))), byte_f(__ldg(pair + 1)), byte_f(__ldg(pair + 3)), 255.0F};
  } else if constexpr (kF == CC_UYVY) {
    const uint8_t* pair = row + 4 * (x >> 1);
    return {byte_f(__ldg(pair + 1 + 2 * (x & 1))), byte_f(__ldg(pair)), byte_f(__ldg(pair + 2)), 255.0F};
  } else if constexpr (kF == CC_RGB8 || kF == CC_BGR8) {
    const uint8_t* p = row + 3 * x;
    const float a = byte_f(__ldg(p)), b = byte_f(__ldg(p + 1)), c = byte_f(__ldg(p + 2));
    return kF == CC_RGB8 ? Px{a, b, c, 255.0F} : Px{c, b, a, 255.0F};
  } else if constexpr (kF == CC_RGBA8 || kF == CC_BGRA8) {
    const uint8_t* p = row + 4 * x;
    const float a = byte_f(__ldg(p)), b = byte_f(__ldg(p + 1)), c = byte_f(__ldg(p + 2));
    const float al = byte_f(__ldg(p + 3));
    return kF == CC_RGBA8 ? Px{a, b, c, al} : Px{c, b, a, al};
  } else if constexpr (kF == CC_MONO8) {
    return {byte_f(__ldg(row + x)), 0.0F, 0.0F, 255.0F};
  } else if constexpr (kF == CC_MONO16) {
    return {word_sample(row + 2 * x), 0.0F, 0.0F, 255.0F};
  } else {
    const uint8_t* p = row + 6 * x;
    return {word_sample(p), word_sample(p + 2), word_sample(p + 4), 255.0F};
  }
}

__device__ __forceinline__ bool aligned4(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 3U) == 0U; }

__device__ __forceinline__ uint32_t ldw(const uint8_t* p) { return __ldg(reinterpret_cast<const uint32_t*>(p)); }

// Source pixels sx .. sx + 3 of row sy in two steps, so that a thread can
// issue all its loads before its arithmetic: fetch4 reads their bytes as
// whole words (false, reading nothing, where the words would not be 4-byte
// aligned), decode4 turns the words into the samples load_px gives.
constexpr int kRawWords = 6;

template <int kF>
__device__ __forceinline__ bool fetch4(const Image& img, int sx, int sy, uint32_t (&w)[kRawWords]) {
  const uint8_t* row = row_of(img, 0, sy);
  if constexpr (kF == CC_RGB8 || kF == CC_BGR8) {
    const uint8_t* p = row + 3 * sx;
    if (!aligned4(p)) return false;
#pragma unroll
    for (int k = 0; k < 3; ++k) w[k] = ldw(p + 4 * k);
  } else if constexpr (kF == CC_RGBA8 || kF == CC_BGRA8) {
    const uint8_t* p = row + 4 * sx;
    if (!aligned4(p)) return false;
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k] = ldw(p + 4 * k);
  } else if constexpr (kF == CC_MONO8) {
    const uint8_t* p = row + sx;
    if (!aligned4(p)) return false;
    w[0] = ldw(p);
  } else if constexpr (kF == CC_MONO16) {
    const uint8_t* p = row + 2 * sx;
    if (!aligned4(p)) return false;
    w[0] = ldw(p);
    w[1] = ldw(p + 4);
  } else if constexpr (kF == CC_RGB16) {
    const uint8_t* p = row + 6 * sx;
    if (!aligned4(p)) return false;
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = ldw(p + 4 * k);
  } else if constexpr (kF == CC_NV12 || kF == CC_NV16) {
    // Four luma bytes and, from an even column, the two chroma pairs covering them.
    const uint8_t* p = row + sx;
    const uint8_t* uv = row_of(img, 1, kF == CC_NV12 ? (sy >> 1) : sy) + sx;
    if ((sx & 1) != 0 || !aligned4(p) || !aligned4(uv)) return false;
    w[0] = ldw(p);
    w[1] = ldw(uv);
  } else if constexpr (kF == CC_I420) {
    const uint8_t* p = row + sx;
    if ((sx & 1) != 0 || !aligned4(p)) return false;
    w[0] = ldw(p);
    const uint8_t* u = row_of(img, 1, sy >> 1) + (sx >> 1);
    const uint8_t* v = row_of(img, 2, sy >> 1) + (sx >> 1);
    // Cb0, Cr0, Cb1, Cr1 as the chroma word of the semi-planar formats.
    w[1] = static_cast<uint32_t>(__ldg(u)) | (static_cast<uint32_t>(__ldg(v)) << 8) |
           (static_cast<uint32_t>(__ldg(u + 1)) << 16) | (static_cast<uint32_t>(__ldg(v + 1)) << 24);
  } else {
    // YUYV / UYVY: two pixel pairs, one word each, from an even column.
    const uint8_t* p = row + 2 * sx;
    if ((sx & 1) != 0 || !aligned4(p)) return false;
    w[0] = ldw(p);
    w[1] = ldw(p + 4);
  }
  return true;
}

// Two bytes (byte ka of wa, byte kb of wb) as the floats of two lanes: the
// 2^23-biased bits of each, less 2^23 two lanes at a time (an exact result).
__device__ __forceinline__ float2 bytes2(uint32_t wa, int ka, uint32_t wb, int kb) {
  const float2 biased = make_float2(__uint_as_float(__byte_perm(wa, kTwo23Bits, 0x7650U | static_cast<uint32_t>(ka))),
                                    __uint_as_float(__byte_perm(wb, kTwo23Bits, 0x7650U | static_cast<uint32_t>(kb))));
  float2 r;
  asm("{ .reg .b64 a, b, d; mov.b64 a, {%2, %3}; mov.b64 b, {%4, %5}; sub.rn.f32x2 d, a, b; mov.b64 {%0, %1}, d; }"
      : "=f"(r.x), "=f"(r.y)
      : "f"(biased.x), "f"(biased.y), "f"(kTwo23), "f"(kTwo23));
  return r;
}

template <int kF>
__device__ __forceinline__ void decode4(const uint32_t (&w)[kRawWords], Px (&s)[4]) {
  if constexpr (kF == CC_RGB8 || kF == CC_BGR8) {
    // Pixels (0, 1) and (2, 3) as lane pairs, channel by channel.
#pragma unroll
    for (int i = 0; i < 4; i += 2) {
      float2 c[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        c[j] = bytes2(w[(3 * i + j) >> 2], (3 * i + j) & 3, w[(3 * (i + 1) + j) >> 2], (3 * (i + 1) + j) & 3);
      }
      s[i] = kF == CC_RGB8 ? Px{c[0].x, c[1].x, c[2].x, 255.0F} : Px{c[2].x, c[1].x, c[0].x, 255.0F};
      s[i + 1] = kF == CC_RGB8 ? Px{c[0].y, c[1].y, c[2].y, 255.0F} : Px{c[2].y, c[1].y, c[0].y, 255.0F};
    }
  } else if constexpr (kF == CC_RGBA8 || kF == CC_BGRA8) {
#pragma unroll
    for (int i = 0; i < 4; i += 2) {
      const float2 a = bytes2(w[i], 0, w[i + 1], 0), b = bytes2(w[i], 1, w[i + 1], 1);
      const float2 c = bytes2(w[i], 2, w[i + 1], 2), al = bytes2(w[i], 3, w[i + 1], 3);
      s[i] = kF == CC_RGBA8 ? Px{a.x, b.x, c.x, al.x} : Px{c.x, b.x, a.x, al.x};
      s[i + 1] = kF == CC_RGBA8 ? Px{a.y, b.y, c.y, al.y} : Px{c.y, b.y, a.y, al.y};
    }
  } else if constexpr (kF == CC_MONO8) {
    const float2 a = bytes2(w[0], 0, w[0], 1), b = bytes2(w[0], 2, w[0], 3);
    s[0] = Px{a.x, 0.0F, 0.0F, 255.0F};
    s[1] = Px{a.y, 0.0F, 0.0F, 255.0F};
    s[2] = Px{b.x, 0.0F, 0.0F, 255.0F};
    s[3] = Px{b.y, 0.0F, 0.0F, 255.0F};
  } else if constexpr (kF == CC_MONO16) {
#pragma unroll
    for (int i = 0; i < 4; ++i) s[i] = Px{div257((w[i >> 1] >> (16 * (i & 1))) & 0xFFFFU), 0.0F, 0.0F, 255.0F};
  } else if constexpr (kF == CC_RGB16) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float c[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) c[j] = div257((w[(3 * i + j) >> 1] >> (16 * ((3 * i + j) & 1))) & 0xFFFFU);
      s[i] = Px{c[0], c[1], c[2], 255.0F};
    }
  } else if constexpr (kF == CC_NV12 || kF == CC_NV16 || kF == CC_I420) {
    // Luma of pixels (0, 1) and (2, 3); the two chroma pairs (Cb, Cr) of the run.
    const float2 y01 = bytes2(w[0], 0, w[0], 1), y23 = bytes2(w[0], 2, w[0], 3);
    const float2 cb = bytes2(w[1], 0, w[1], 2), cr = bytes2(w[1], 1, w[1], 3);
    s[0] = Px{y01.x, cb.x, cr.x, 255.0F};
    s[1] = Px{y01.y, cb.x, cr.x, 255.0F};
    s[2] = Px{y23.x, cb.y, cr.y, 255.0F};
    s[3] = Px{y23.y, cb.y, cr.y, 255.0F};
  } else {
    constexpr int kY = kF == CC_YUYV ? 0 : 1;  // byte of the first luma in a pair
    constexpr int kU = kF == CC_YUYV ? 1 : 0;  // byte of Cb; Cr two later
    const float2 y01 = bytes2(w[0], kY, w[0], kY + 2), y23 = bytes2(w[1], kY, w[1], kY + 2);
    const float2 cb = bytes2(w[0], kU, w[1], kU), cr = bytes2(w[0], kU + 2, w[1], kU + 2);
    s[0] = Px{y01.x, cb.x, cr.x, 255.0F};
    s[1] = Px{y01.y, cb.x, cr.x, 255.0F};
    s[2] = Px{y23.x, cb.y, cr.y, 255.0F};
    s[3] = Px{y23.y, cb.y, cr.y, 255.0F};
  }
}

// c = m s + o on the colour samples, each row summed left to right; alpha
// passes through (:236-244). kKnown: whether the identity is settled at
// compile time (kIdentity then says which), else p.identity decides.
template <bool kKnown = false, bool kIdentity = false>
__device__ __forceinline__ Px apply_affine(const Plan& p, Px s) {
  if constexpr (kKnown) {
    if constexpr (kIdentity) return s;
  } else {
    if (p.identity) return s;
  }
  Px r;
  r.c0 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p.m[0], s.c0), __fmul_rn(p.m[1], s.c1)), __fmul_rn(p.m[2], s.c2)),
                   p.o[0]);
  r.c1 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p.m[3], s.c0), __fmul_rn(p.m[4], s.c1)), __fmul_rn(p.m[5], s.c2)),
                   p.o[1]);
  r.c2 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p.m[6], s.c0), __fmul_rn(p.m[7], s.c1)), __fmul_rn(p.m[8], s.c2)),
                   p.o[2]);
  r.a = s.a;
  return r;
}

__device__ __forceinline__ void put_word(uint8_t* q, uint32_t w) {
  q[0] = static_cast<uint8_t>(w & 0xFFU);
  q[1] = static_cast<uint8_t>(w >> 8);
}

// Everything but chroma of pixel (x, y) of a destination of format kF (the
// luma of a YCbCr one), :256-307.
template <int kF>
__device__ __forceinline__ void store_px(const Image& img, int x, int y, const Px& v) {
  uint8_t* row = img.data[0] + static_cast<size_t>(y) * img.pitch[0];
  if constexpr (kF == CC_NV12 || kF == CC_NV16 || kF == CC_I420 || kF == CC_MONO8) {
    row[x] = static_cast<uint8_t>(code8(v.c0));
  } else if constexpr (kF == CC_YUYV) {
    row[4 * (x >> 1) + 2 * (x & 1)] = static_cast<uint8_t>(code8(v.c0));
  } else if constexpr (kF == CC_UYVY) {
    row[4 * (x >> 1) + 1 + 2 * (x & 1)] = static_cast<uint8_t>(code8(v.c0));
  } else if constexpr (kF == CC_RGB8 || kF == CC_BGR8) {
    uint8_t* q = row + 3 * x;
    const bool bgr = kF == CC_BGR8;
    q[0] = static_cast<uint8_t>(code8(bgr ? v.c2 : v.c0));
    q[1] = static_cast<uint8_t>(code8(v.c1));
    q[2] = static_cast<uint8_t>(code8(bgr ? v.c0 : v.c2));
  } else if constexpr (kF == CC_RGBA8 || kF == CC_BGRA8) {
    const bool bgr = kF == CC_BGRA8;
    const uint32_t w = code8(bgr ? v.c2 : v.c0) | (code8(v.c1) << 8) | (code8(bgr ? v.c0 : v.c2) << 16) |
                       (code8(v.a) << 24);
    uint8_t* q = row + 4 * x;
    if ((reinterpret_cast<uintptr_t>(q) & 3U) == 0U) {
      *reinterpret_cast<uint32_t*>(q) = w;
    } else {
      q[0] = static_cast<uint8_t>(w);
      q[1] = static_cast<uint8_t>(w >> 8);
      q[2] = static_cast<uint8_t>(w >> 16);
      q[3] = static_cast<uint8_t>(w >> 24);
    }
  } else if constexpr (kF == CC_MONO16) {
    put_word(row + 2 * x, code16(v.c0));
  } else {
    uint8_t* q = row + 6 * x;
    put_word(q, code16(v.c0));
    put_word(q + 2, code16(v.c1));
    put_word(q + 4, code16(v.c2));
  }
}

// Chroma sample (cx, cy) of a YCbCr destination (:311-341).
template <int kF>
__device__ __forceinline__ void store_chroma(const Image& img, int cx, int cy, float cb, float cr) {
  if constexpr (kF == CC_NV12 || kF == CC_NV16) {
    uint8_t* q = img.data[1] + static_cast<size_t>(cy) * img.pitch[1] + 2 * cx;
    q[0] = static_cast<uint8_t>(code8(cb));
    q[1] = static_cast<uint8_t>(code8(cr));
  } else if constexpr (kF == CC_I420) {
    img.data[1][static_cast<size_t>(cy) * img.pitch[1] + cx] = static_cast<uint8_t>(code8(cb));
    img.data[2][static_cast<size_t>(cy) * img.pitch[2] + cx] = static_cast<uint8_t>(code8(cr));
  } else if constexpr (kF == CC_YUYV) {
    uint8_t* q = img.data[0] + static_cast<size_t>(cy) * img.pitch[0] + 4 * cx;
    q[1] = static_cast<uint8_t>(code8(cb));
    q[3] = static_cast<uint8_t>(code8(cr));
  } else if constexpr (kF == CC_UYVY) {
    uint8_t* q = img.data[0] + static_cast<size_t>(cy) * img.pitch[0] + 4 * cx;
    q[0] = static_cast<uint8_t>(code8(cb));
    q[2] = static_cast<uint8_t>(code8(cr));
  }
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// sum + s w per sample, product then sum, each rounded (:163-165).
__device__ __forceinline__ Px accumulate(Px sum, const Px& s, float w) {
  return {__fadd_rn(sum.c0, __fmul_rn(s.c0, w)), __fadd_rn(sum.c1, __fmul_rn(s.c1, w)),
          __fadd_rn(sum.c2, __fmul_rn(s.c2, w)), __fadd_rn(sum.a, __fmul_rn(s.a, w))};
}

// Weight of source pixel [i, i + 1) in the footprint [lo, hi) (:168-172).
__device__ __forceinline__ float covered(int i, float lo, float hi) {
  const float fi = static_cast<float>(i);
  const float fj = static_cast<float>(i + 1);
  const float a = fi > lo ? fi : lo;
  const float b = fj < hi ? fj : hi;
  return b > a ? __fsub_rn(b, a) : 0.0F;
}

// The source sampled for content pixel (dx, dy) (:175-233), resize mode kMode.
template <int kSrc, int kMode>
__device__ __forceinline__ Px sample_px(const Plan& p, int dx, int dy) {
  const float rx = static_cast<float>(dx - p.cx0);
  const float ry = static_cast<float>(dy - p.cy0);
  const float x0 = static_cast<float>(p.sx0);
  const float y0 = static_cast<float>(p.sy0);
  if constexpr (kMode == CC_NEAREST) {
    const int sx = clampi(static_cast<int>(floorf(__fadd_rn(x0, __fmul_rn(__fadd_rn(rx, 0.5F), p.scale_x)))), p.sx0, p.sx1);
    const int sy = clampi(static_cast<int>(floorf(__fadd_rn(y0, __fmul_rn(__fadd_rn(ry, 0.5F), p.scale_y)))), p.sy0, p.sy1);
    return load_px<kSrc>(p.src, sx, sy);
  } else if constexpr (kMode == CC_BILINEAR) {
    const float fx = __fsub_rn(__fadd_rn(x0, __fmul_rn(__fadd_rn(rx, 0.5F), p.scale_x)), 0.5F);
    const float fy = __fsub_rn(__fadd_rn(y0, __fmul_rn(__fadd_rn(ry, 0.5F), p.scale_y)), 0.5F);
    const float bx = floorf(fx);
    const float by = floorf(fy);
    const float ax = __fsub_rn(fx, bx);
    const float ay = __fsub_rn(fy, by);
    const int ix = static_cast<int>(bx);
    const int iy = static_cast<int>(by);
    const int xa = clampi(ix, p.sx0, p.sx1);
    const int xb = clampi(ix + 1, p.sx0, p.sx1);
    const int ya = clampi(iy, p.sy0, p.sy1);
    const int yb = clampi(iy + 1, p.sy0, p.sy1);
    const float bx1 = __fsub_rn(1.0F, ax);
    const float by1 = __fsub_rn(1.0F, ay);
    const float w00 = __fmul_rn(bx1, by1);
    const float w10 = __fmul_rn(ax, by1);
    const float w01 = __fmul_rn(bx1, ay);
    const float w11 = __fmul_rn(ax, ay);
    // Taps of zero weight are skipped, as the definition does.
    Px s{0.0F, 0.0F, 0.0F, 0.0F};
    if (w00 != 0.0F) s = accumulate(s, load_px<kSrc>(p.src, xa, ya), w00);
    if (w10 != 0.0F) s = accumulate(s, load_px<kSrc>(p.src, xb, ya), w10);
    if (w01 != 0.0F) s = accumulate(s, load_px<kSrc>(p.src, xa, yb), w01);
    if (w11 != 0.0F) s = accumulate(s, load_px<kSrc>(p.src, xb, yb), w11);
    return s;
  } else {
    // Area: the footprint [lo, hi) on each axis, inside the source rectangle.
    const float lx = __fadd_rn(x0, __fmul_rn(rx, p.scale_x));
    const float ly = __fadd_rn(y0, __fmul_rn(ry, p.scale_y));
    const float right = static_cast<float>(p.sx1 + 1);
    const float bottom = static_cast<float>(p.sy1 + 1);
    const float lxs = __fadd_rn(lx, p.scale_x);
    const float lys = __fadd_rn(ly, p.scale_y);
    const float hx = lxs < right ? lxs : right;
    const float hy = lys < bottom ? lys : bottom;
    const int ix0 = clampi(static_cast<int>(floorf(lx)), p.sx0, p.sx1);
    const int iy0 = clampi(static_cast<int>(floorf(ly)), p.sy0, p.sy1);
    Px s{0.0F, 0.0F, 0.0F, 0.0F};
    float total = 0.0F;
    for (int y = iy0; y <= p.sy1 && static_cast<float>(y) < hy; ++y) {
      const float wy = covered(y, ly, hy);
      for (int x = ix0; x <= p.sx1 && static_cast<float>(x) < hx; ++x) {
        const float w = __fmul_rn(covered(x, lx, hx), wy);
        if (w != 0.0F) {
          s = accumulate(s, load_px<kSrc>(p.src, x, y), w);
          total = __fadd_rn(total, w);
        }
      }
    }
    if (total <= 0.0F) return load_px<kSrc>(p.src, ix0, iy0);
    return {__fdiv_rn(s.c0, total), __fdiv_rn(s.c1, total), __fdiv_rn(s.c2, total), __fdiv_rn(s.a, total)};
  }
}

__device__ __forceinline__ bool in_content(const Plan& p, int x, int y) {
  return x >= p.cx0 && x < p.cx1 && y >= p.cy0 && y < p.cy1;
}

#endif  // __CUDACC__

// Host side (cc_plan.cpp): names, geometry, checks and the plan.
int make_plan(const cc_image_c* src, const cc_image_c* dst, const cc_params_c* params, Plan* plan);
int compute_mapping(int sw, int sh, int w, int h, int dst_format, const cc_params_c* params, cc_mapping_c* out);
int validate(const cc_image_c* src, const cc_image_c* dst, const cc_params_c* params);
bool known_format(int f);

// Kernel launchers (cc_kernels*.cu).
int launch_convert(const Plan& plan, void* stream);
int launch_pattern(uint8_t* data, size_t pitch, int width, int height, uint32_t frame, void* stream);

}  // namespace cc_b200
