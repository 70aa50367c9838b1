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

}  // namespace isp_b200
