// isp_ops.cuh - exact arithmetic building blocks of the sm_100a kernels.
//
// Conversions between float and integer run on a quarter-rate pipe on this
// GPU; the kernels replace each one with a full-rate float add whose result
// is provably the same:
//   - an integer n < 2^23 as a float: the bits 0x4B000000 | n are 2^23 + n,
//     and subtracting 2^23 leaves n exactly;
//   - trunc(x) of 0 <= x < 2^23: x + 2^23 rounded toward zero lands on
//     2^23 + trunc(x) (the floats in [2^23, 2^24) are the integers), so its
//     bits minus 0x4B000000 are trunc(x), and the float minus 2^23 is
//     (float)trunc(x).
// clamp01(v) = min(max(v, 0), 1) is the saturating form of the last multiply
// or add (.sat, which maps the result into [0, 1]); no NaN reaches it.
#pragma once

#include <cstdint>

namespace isp_b200 {

constexpr float kTwo23 = 8388608.0F;
constexpr unsigned int kTwo23Bits = 0x4B000000U;

// (float)n for 0 <= n < 2^23, n already OR-ed with kTwo23Bits.
__device__ __forceinline__ float magic_to_float(unsigned int n_or_bits) {
  return __uint_as_float(n_or_bits) - kTwo23;
}

// 2^23 + trunc(x) as a float, for 0 <= x < 2^23.
__device__ __forceinline__ float magic_trunc(float x) { return __fadd_rz(x, kTwo23); }

// trunc(x) from magic_trunc(x).
__device__ __forceinline__ unsigned int magic_int(float m) { return __float_as_uint(m) - kTwo23Bits; }

// Rounded product clamped to [0, 1]: clamp01(a * b).
__device__ __forceinline__ float mul_sat(float a, float b) {
  float r;
  asm("mul.rn.sat.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// Rounded sum clamped to [0, 1]: clamp01(a + b).
__device__ __forceinline__ float add_sat(float a, float b) {
  float r;
  asm("add.rn.sat.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// Plain rounded operations, spelled out so no contraction can merge them.
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }

// round(k * a + b) where k * a is exact (k a power of two >= 1, no
// overflow): one rounding, as the reference's round(round(k * a) + b).
__device__ __forceinline__ float exact_scale_add(float a, float k, float b) { return __fmaf_rn(a, k, b); }

// ---- Two lanes per instruction ---------------------------------------------
//
// sm_100 executes f32x2 add, multiply and fused multiply-add: one instruction,
// two independent IEEE single operations, each lane rounded exactly as the
// scalar operation is. The tile pass runs two pixels of identical arithmetic
// (columns c and c + 32 of a row) through them. There is no saturating or
// min/max form, so clamps stay per lane.
//
// The assembler may fuse a two-lane product into a two-lane add or subtract
// that consumes it (one rounding instead of two), whatever rounding mode the
// instructions name; measured on this toolchain, about half of such sums
// then differ from the reference in the last bit. Scalar operations with an
// explicit rounding mode are never fused. So in this code a two-lane product
// feeds only a multiply, an operand of a fused multiply-add, a per-lane
// (scalar) add, or a two-lane add when the product is exact (a scale by a
// power of two), where one rounding and two give the same result.
#define ISP_F32X2_BINARY(NAME, OP)                                                                      \
  __device__ __forceinline__ float2 NAME(float2 a, float2 b) {                                          \
    float2 r;                                                                                           \
    asm("{ .reg .b64 a, b, d; mov.b64 a, {%2, %3}; mov.b64 b, {%4, %5}; " OP " d, a, b; "             \
        "mov.b64 {%0, %1}, d; }"                                                                        \
        : "=f"(r.x), "=f"(r.y)                                                                          \
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                                      \
    return r;                                                                                           \
  }
ISP_F32X2_BINARY(add2, "add.rn.f32x2")
ISP_F32X2_BINARY(sub2, "sub.rn.f32x2")
ISP_F32X2_BINARY(mul2, "mul.rn.f32x2")
ISP_F32X2_BINARY(add2_rz, "add.rz.f32x2")
#undef ISP_F32X2_BINARY

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
// exact_scale_add per lane: round(k a + b) with k a exact.
__device__ __forceinline__ float2 exact_scale_add2(float2 a, float2 k, float2 b) {
  float2 r;
  asm("{ .reg .b64 a, k, b, d; mov.b64 a, {%2, %3}; mov.b64 k, {%4, %5}; mov.b64 b, {%6, %7}; "
      "fma.rn.f32x2 d, a, k, b; mov.b64 {%0, %1}, d; }"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(k.x), "f"(k.y), "f"(b.x), "f"(b.y));
  return r;
}
// magic_trunc per lane: 2^23 + trunc(x) for 0 <= x < 2^23 (x not a product).
__device__ __forceinline__ float2 magic_trunc2(float2 x) { return add2_rz(x, bc2(kTwo23)); }
// Per-lane scalar forms, for sums that consume a two-lane product.
__device__ __forceinline__ float2 add_lanes(float2 a, float2 b) { return make_float2(fadd(a.x, b.x), fadd(a.y, b.y)); }
__device__ __forceinline__ float2 sub_lanes(float2 a, float2 b) { return make_float2(fsub(a.x, b.x), fsub(a.y, b.y)); }
__device__ __forceinline__ float2 magic_trunc_lanes(float2 x) { return make_float2(magic_trunc(x.x), magic_trunc(x.y)); }
// (float)n per lane from n OR-ed with kTwo23Bits.
__device__ __forceinline__ float2 magic_to_float2(unsigned int a_bits, unsigned int b_bits) {
  return sub2(make_float2(__uint_as_float(a_bits), __uint_as_float(b_bits)), bc2(kTwo23));
}
__device__ __forceinline__ float2 mul_sat2(float2 a, float2 b) { return make_float2(mul_sat(a.x, b.x), mul_sat(a.y, b.y)); }
__device__ __forceinline__ float2 add_sat2(float2 a, float2 b) { return make_float2(add_sat(a.x, b.x), add_sat(a.y, b.y)); }

}  // namespace isp_b200
