// cc_resample.cu - the colour converter's resample kernels (one per source
// format and resize mode), the synthetic camera pattern kernel, and the
// launcher that picks the direct or the resample path for a plan.
#include <cuda_runtime.h>

#include "cc_kernels.cuh"

namespace cc_b200 {
namespace {

template <int kSrc>
const void* for_mode(int mode) {
  switch (mode) {
    case CC_NEAREST: return reinterpret_cast<const void*>(&cc_resample_kernel<kSrc, CC_NEAREST>);
    case CC_BILINEAR: return reinterpret_cast<const void*>(&cc_resample_kernel<kSrc, CC_BILINEAR>);
    case CC_AREA: return reinterpret_cast<const void*>(&cc_resample_kernel<kSrc, CC_AREA>);
    default: return nullptr;
  }
}

// The synthetic camera's picture (modules/color-convert/include/holoscan/
// color_convert/reference.hpp:34-55): eight full-intensity bars, white,
// yellow, cyan, green, magenta, red, blue, black, over the top two thirds,
// moving right by four pixels a frame; below them a horizontal black-to-white
// ramp mixed with a vertical red-to-blue one. Integer arithmetic only.
__global__ void cc_pattern_kernel(uint8_t* data, size_t pitch, int width, int height, uint32_t frame) {
  const int x = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= width || y >= height) return;
  uint8_t* q = data + static_cast<size_t>(y) * pitch + 3 * static_cast<size_t>(x);
  const int top = (2 * height) / 3;
  if (y < top) {
    const int shift = static_cast<int>((frame * 4U) % static_cast<uint32_t>(width));
    const int bar = (((x + width - shift) % width) * 8) / width;
    // Bar b's colour (bit 2 red, bit 1 green, bit 0 blue) is the nibble at
    // bits 28 - 4b: 7, 6, 3, 2, 5, 4, 1, 0.
    constexpr uint32_t kColours = 0x76325410U;
    const uint32_t c = (kColours >> (4 * (7 - bar))) & 7U;
    q[0] = (c & 4U) ? 255 : 0;
    q[1] = (c & 2U) ? 255 : 0;
    q[2] = (c & 1U) ? 255 : 0;
    return;
  }
  const int below = height - top;
  const int gray = width > 1 ? (x * 255) / (width - 1) : 0;
  const int blue = below > 1 ? ((y - top) * 255) / (below - 1) : 0;
  q[0] = static_cast<uint8_t>((gray + 255 - blue) / 2);
  q[1] = static_cast<uint8_t>(gray);
  q[2] = static_cast<uint8_t>((gray + blue) / 2);
}

}  // namespace

const void* resample_kernel(int src, int mode) {
  switch (src) {
    case CC_NV12: return for_mode<CC_NV12>(mode);
    case CC_NV16: return for_mode<CC_NV16>(mode);
    case CC_I420: return for_mode<CC_I420>(mode);
    case CC_YUYV: return for_mode<CC_YUYV>(mode);
    case CC_UYVY: return for_mode<CC_UYVY>(mode);
    case CC_RGB8: return for_mode<CC_RGB8>(mode);
    case CC_BGR8: return for_mode<CC_BGR8>(mode);
    case CC_RGBA8: return for_mode<CC_RGBA8>(mode);
    case CC_BGRA8: return for_mode<CC_BGRA8>(mode);
    case CC_MONO8: return for_mode<CC_MONO8>(mode);
    case CC_MONO16: return for_mode<CC_MONO16>(mode);
    case CC_RGB16: return for_mode<CC_RGB16>(mode);
    default: return nullptr;
  }
}

const void* direct_kernel(int src, int dst) {
  if (src <= CC_UYVY) return direct_kernel_yuv(src, dst);
  if (src <= CC_BGRA8) return direct_kernel_rgb(src, dst);
  return direct_kernel_gray(src, dst);
}

// Whether every content pixel reads exactly the source pixel under it: the
// source and content rectangles have the same size, so both scales are
// exactly 1, and coordinates stay below 2^22, where the sampling arithmetic
// is exact.
static bool direct_path(const Plan& p) {
  constexpr int kExact = 1 << 22;
  return p.scale_x == 1.0F && p.scale_y == 1.0F && p.sx1 - p.sx0 + 1 == p.cx1 - p.cx0 &&
         p.sy1 - p.sy0 + 1 == p.cy1 - p.cy0 && p.src.width < kExact && p.src.height < kExact &&
         p.dst.width < kExact && p.dst.height < kExact;
}

int launch_convert(const Plan& plan, void* stream) {
  const dim3 block(kThreadsX, kThreadsY);
  Plan p = plan;
  const bool direct = direct_path(p);
  int across, down, per_block_x;
  const void* fn;
  if (direct) {
    // Four-pixel groups across; a block's warp covers kSub x 32 of them.
    const FormatInfo fi = info_of(p.dst.format);
    const int rows = fi.model == kYuv ? (1 << fi.shift_y) : 1;
    across = (p.dst.width + kGroupX - 1) / kGroupX;
    down = (p.dst.height + rows - 1) / rows;
    per_block_x = kThreadsX * direct_subgroups(p.dst.format);
    fn = direct_kernel(p.src.format, p.dst.format);
  } else {
    across = (p.dst.width + (1 << p.bsx) - 1) >> p.bsx;
    down = (p.dst.height + (1 << p.bsy) - 1) >> p.bsy;
    per_block_x = kThreadsX;
    fn = resample_kernel(p.src.format, p.mode);
  }
  if (fn == nullptr || (down + kThreadsY - 1) / kThreadsY > 65535) return static_cast<int>(cudaErrorInvalidValue);
  const dim3 grid(static_cast<unsigned>((across + per_block_x - 1) / per_block_x),
                  static_cast<unsigned>((down + kThreadsY - 1) / kThreadsY));
  void* args[] = {&p, &across, &down};
  return static_cast<int>(cudaLaunchKernel(fn, grid, block, args, 0, static_cast<cudaStream_t>(stream)));
}

int launch_pattern(uint8_t* data, size_t pitch, int width, int height, uint32_t frame, void* stream) {
  const dim3 block(kThreadsX, kThreadsY);
  const dim3 grid(static_cast<unsigned>((width + kThreadsX - 1) / kThreadsX),
                  static_cast<unsigned>((height + kThreadsY - 1) / kThreadsY));
  cc_pattern_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(data, pitch, width, height, frame);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace cc_b200
