// cc_direct_rgb.cu - direct-path kernels (same-size conversions) of the
// 8-bit RGB sources (RGB8, BGR8, RGBA8, BGRA8) into every destination format;
// split from the other source formats so that they compile in parallel.
#include "cc_kernels.cuh"

namespace cc_b200 {
namespace {

template <int kSrc>
const void* for_destination(int dst) {
  switch (dst) {
    case CC_NV12: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_NV12>);
    case CC_NV16: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_NV16>);
    case CC_I420: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_I420>);
    case CC_YUYV: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_YUYV>);
    case CC_UYVY: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_UYVY>);
    case CC_RGB8: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_RGB8>);
    case CC_BGR8: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_BGR8>);
    case CC_RGBA8: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_RGBA8>);
    case CC_BGRA8: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_BGRA8>);
    case CC_MONO8: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_MONO8>);
    case CC_MONO16: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_MONO16>);
    case CC_RGB16: return reinterpret_cast<const void*>(&cc_direct_kernel<kSrc, CC_RGB16>);
    default: return nullptr;
  }
}

}  // namespace

const void* direct_kernel_rgb(int src, int dst) {
  switch (src) {
    case CC_RGB8: return for_destination<CC_RGB8>(dst);
    case CC_BGR8: return for_destination<CC_BGR8>(dst);
    case CC_RGBA8: return for_destination<CC_RGBA8>(dst);
    case CC_BGRA8: return for_destination<CC_BGRA8>(dst);
    default: return nullptr;
  }
}

}  // namespace cc_b200
