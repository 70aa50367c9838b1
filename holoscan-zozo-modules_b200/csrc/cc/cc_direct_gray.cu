// cc_direct_gray.cu - direct-path kernels (same-size conversions) of the
// MONO8, MONO16 and RGB16 sources into every destination format;
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

const void* direct_kernel_gray(int src, int dst) {
  switch (src) {
    case CC_MONO8: return for_destination<CC_MONO8>(dst);
    case CC_MONO16: return for_destination<CC_MONO16>(dst);
    case CC_RGB16: return for_destination<CC_RGB16>(dst);
    default: return nullptr;
  }
}

}  // namespace cc_b200
