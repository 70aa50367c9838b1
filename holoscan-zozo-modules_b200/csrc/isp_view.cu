// isp_view.cu - the demo's side-by-side view of raw and processed frames
// (applications/isp/src/view_op.cu:35-75), as a headless device image: the
// raw mosaic as square-rooted gray on the left, the ISP's RGB8 image on the
// right. One thread converts a run of sixteen pixels of a row and copies
// the sixteen RGB pixels beside them.
#include <cuda_runtime.h>

#include <string>

#include "isp_host.hpp"
#include "isp_trace.hpp"

namespace isp_b200 {
namespace {

struct ViewArgs {
  const uint8_t* raw;
  size_t raw_pitch;
  int width, height, format;
  float black, scale;
  const uint8_t* rgb;
  size_t rgb_pitch;
  uint8_t* out;
  size_t out_pitch;
};

// One raw sample's counts (view_op.cu:35-51; isp_math.hpp:101-119).
__device__ __forceinline__ int view_sample(const uint8_t* row, int format, int x) {
  switch (format) {
    case ISP_RAW_U8: return __ldg(row + x);
    case ISP_RAW_U16: return __ldg(row + 2 * x) | (__ldg(row + 2 * x + 1) << 8);
    case ISP_RAW_RAW10: {
      const uint8_t* g = row + 5 * (x >> 2);
      return (__ldg(g + (x & 3)) << 2) | ((__ldg(g + 4) >> (2 * (x & 3))) & 3);
    }
    default: {
      const uint8_t* g = row + 3 * (x >> 1);
      return (__ldg(g + (x & 1)) << 4) | ((__ldg(g + 2) >> (4 * (x & 1))) & 15);
    }
  }
}

// The gray code of one sample: (s - black) * scale clamped to [0, 1], its
// square root, times 255, plus 0.5, truncated; every step rounded once.
__device__ __forceinline__ uint32_t view_gray(int s, float black, float scale) {
  float v = __fmul_rn(__fsub_rn(static_cast<float>(s), black), scale);
  v = v < 0.0F ? 0.0F : (v > 1.0F ? 1.0F : v);
  return __float2uint_rz(__fadd_rn(__fmul_rn(__fsqrt_rn(v), 255.0F), 0.5F));
}

// One thread per run of 16 pixels of a row (x0 = 16 g): their 16 gray codes
// and the 16 RGB pixels beside them. Where the rows allow it (16-byte aligned
// RGB and view rows, a whole run inside the frame) the 48-byte runs move as
// three 16-byte words each and the raw samples come as 32-bit words; else
// byte by byte.
__global__ void __launch_bounds__(256) isp_view_kernel(const __grid_constant__ ViewArgs a) {
  constexpr int kRun = 16;
  const int x0 = kRun * static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
  if (x0 >= a.width || y >= a.height) return;
  const int n = a.width - x0 < kRun ? a.width - x0 : kRun;
  const uint8_t* raw = a.raw + static_cast<size_t>(y) * a.raw_pitch;
  const uint8_t* rgb = a.rgb + static_cast<size_t>(y) * a.rgb_pitch + 3 * static_cast<size_t>(x0);
  uint8_t* left = a.out + static_cast<size_t>(y) * a.out_pitch + 3 * static_cast<size_t>(x0);
  uint8_t* right = left + 3 * static_cast<size_t>(a.width);
  const bool vec = n == kRun && ((reinterpret_cast<uintptr_t>(rgb) | reinterpret_cast<uintptr_t>(left) |
                                  reinterpret_cast<uintptr_t>(right)) & 15U) == 0U;
  if (vec) {
    // The RGB run: three 16-byte words, loaded before the arithmetic.
    const uint4 c0 = __ldg(reinterpret_cast<const uint4*>(rgb));
    const uint4 c1 = __ldg(reinterpret_cast<const uint4*>(rgb) + 1);
    const uint4 c2 = __ldg(reinterpret_cast<const uint4*>(rgb) + 2);
    uint32_t g[kRun];
#pragma unroll
    for (int i = 0; i < kRun; ++i) g[i] = view_gray(view_sample(raw, a.format, x0 + i), a.black, a.scale);
    // Gray pixels: bytes g, g, g per pixel, 48 bytes as 12 words.
    uint32_t w[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      uint32_t v = 0U;
#pragma unroll
      for (int b = 0; b < 4; ++b) v |= g[(4 * k + b) / 3] << (8 * b);
      w[k] = v;
    }
    uint4* l = reinterpret_cast<uint4*>(left);
    l[0] = make_uint4(w[0], w[1], w[2], w[3]);
    l[1] = make_uint4(w[4], w[5], w[6], w[7]);
    l[2] = make_uint4(w[8], w[9], w[10], w[11]);
    uint4* r = reinterpret_cast<uint4*>(right);
    r[0] = c0;
    r[1] = c1;
    r[2] = c2;
    return;
  }
  for (int i = 0; i < n; ++i) {
    const uint8_t g = static_cast<uint8_t>(view_gray(view_sample(raw, a.format, x0 + i), a.black, a.scale));
    left[3 * i] = left[3 * i + 1] = left[3 * i + 2] = g;
#pragma unroll
    for (int k = 0; k < 3; ++k) right[3 * i + k] = __ldg(rgb + 3 * i + k);
  }
}

}  // namespace
}  // namespace isp_b200

extern "C" ISP_B200_API int isp_b200_view_compose(const isp_raw_view_c* raw, float black_level, const void* rgb8,
                                                  size_t rgb8_pitch, void* view, size_t view_pitch, void* stream) {
  using namespace isp_b200;
  const TraceRange range("isp.view", kTraceKernel);
  clear_error();
  if (raw == nullptr || raw->data == nullptr || rgb8 == nullptr || view == nullptr) {
    return fail(ISP_EINVAL, "view_compose: a buffer is missing");
  }
  if (raw->width <= 0 || raw->height <= 0) return fail(ISP_EINVAL, "raw image size must be positive");
  if (raw->format < ISP_RAW_U8 || raw->format > ISP_RAW_RAW12) return fail(ISP_EINVAL, "unknown raw format");
  const int max_bits = raw->format == ISP_RAW_U8 ? 8 : raw->format == ISP_RAW_U16 ? 16 : raw->format == ISP_RAW_RAW10 ? 10 : 12;
  if (raw->bit_depth < 1 || raw->bit_depth > max_bits) {
    return fail(ISP_EINVAL, "raw bit depth " + std::to_string(raw->bit_depth) + " does not fit the raw format");
  }
  if (raw->pitch < raw_row_bytes(raw->format, raw->width)) return fail(ISP_EINVAL, "raw pitch is shorter than a row");
  const size_t rgb_row = 3 * static_cast<size_t>(raw->width);
  if (rgb8_pitch < rgb_row) return fail(ISP_EINVAL, "RGB8 pitch is shorter than a row");
  if (view_pitch < 2 * rgb_row) return fail(ISP_EINVAL, "view pitch is shorter than a row of the double-width image");
  // view_op.cu:143-149: white and the scale in single precision on the host.
  const float white = static_cast<float>((1U << static_cast<unsigned>(raw->bit_depth)) - 1U);
  ViewArgs a{static_cast<const uint8_t*>(raw->data), raw->pitch, raw->width, raw->height, raw->format, black_level,
             1.0F / (white - black_level), static_cast<const uint8_t*>(rgb8), rgb8_pitch,
             static_cast<uint8_t*>(view), view_pitch};
  const dim3 block(32, 8);
  const dim3 grid(static_cast<unsigned>((raw->width + 511) / 512), static_cast<unsigned>((raw->height + 7) / 8));
  isp_view_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "view kernel");
  return ISP_OK;
}
