// view_ref_shim.cu - test infrastructure: the reference demo's side-by-side
// view kernel (applications/isp/src/view_op.cu:35-73), compiled from that
// source where it lies (the Makefile passes its path as REF_VIEW_OP) against
// view_sdk_stub.hpp, and launched the way ViewOp::compute launches it
// (view_op.cu:147-160): the same parameters, block and grid. It serves as
// the checker of isp_b200_view_compose; nothing of the product loads it.
#include REF_VIEW_OP

extern "C" int ref_view_compose(const void* raw, size_t raw_pitch, int width, int height, int format, int bit_depth,
                                float black_level, const void* rgb8, void* view, void* stream) {
  // view_op.cu:147-153: white from the bit depth, scale 1 / (white - black).
  const float white = static_cast<float>((1U << static_cast<unsigned>(bit_depth)) - 1U);
  const isp_demo::ViewParams p{width, height, format, raw_pitch, black_level, 1.0F / (white - black_level)};
  const dim3 block(32, 8);
  const dim3 grid((2 * width + 31) / 32, (height + 7) / 8);
  isp_demo::view_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      p, static_cast<const unsigned char*>(raw), static_cast<const unsigned char*>(rgb8),
      static_cast<unsigned char*>(view));
  return static_cast<int>(cudaGetLastError());
}
