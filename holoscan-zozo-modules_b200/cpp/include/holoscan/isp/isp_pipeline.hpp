// isp_pipeline.hpp - holoscan::isp::IspPipeline for C++ callers of the B200 ISP.
//
// The reference module's class (include/holoscan/isp/isp_pipeline.hpp:39-73)
// with the same constructor, methods, ownership and exceptions, over
// libisp_b200.so's C ABI: isp_b200_create / isp_b200_process /
// isp_b200_reset / isp_b200_destroy. Views are borrowed; the pipeline owns
// its tone table, lens shading grid, statistics scratch and white balance
// state on the device. Consecutive process() calls run on the GPU in call
// order, whatever their streams. Header-only: link libisp_b200.so and the
// CUDA runtime.
#pragma once

#include <cuda_runtime_api.h>

#include <memory>
#include <stdexcept>

#include "holoscan/isp/isp_params.hpp"

namespace holoscan::isp {

enum class MemoryLocation : std::uint8_t { kHost, kDevice };

// Whether a CUDA device is usable in this process.
[[nodiscard]] inline PlatformFacts probe_platform() noexcept {
  int count = 0;
  const bool usable = cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
  if (!usable) static_cast<void>(cudaGetLastError());
  return PlatformFacts{usable};
}

[[nodiscard]] inline Backend resolve_backend(Backend backend) noexcept {
  return backend == Backend::kAuto ? resolve_auto(probe_platform()) : backend;
}

class IspPipeline {
 public:
  // @throws std::invalid_argument if `params` are not valid, or for
  //         Backend::kCpu (and kAuto without a CUDA device): this build
  //         ships the GPU pipeline only.
  // @throws std::runtime_error if CUDA fails.
  IspPipeline(Backend backend, IspParams params) : params_(std::move(params)) {
    backend_ = resolve_backend(backend);
    validate_params(params_);
    if (backend_ != Backend::kCuda) {
      throw std::invalid_argument("backend cpu is not part of the B200 build: use Backend::kCuda");
    }
    const isp_params_c c = detail::to_c(params_);
    isp_b200_pipeline* p = nullptr;
    detail::check(isp_b200_create(&c, &p));
    handle_.reset(p);
  }
  ~IspPipeline() = default;
  IspPipeline(const IspPipeline&) = delete;
  IspPipeline& operator=(const IspPipeline&) = delete;

  [[nodiscard]] Backend backend() const noexcept { return backend_; }
  [[nodiscard]] MemoryLocation location() const noexcept { return MemoryLocation::kDevice; }
  [[nodiscard]] const IspParams& params() const noexcept { return params_; }

  // Forgets the white balance estimate after the frames already queued.
  // @throws std::runtime_error if CUDA fails.
  void reset() { detail::check(isp_b200_reset(handle_.get())); }

  // Queues one frame on `stream`, all buffers in device memory.
  // @throws std::invalid_argument if a view is not usable (nothing is queued).
  // @throws std::runtime_error if CUDA fails.
  void process(const RawImageView& raw, const RgbImageView& out, const StatsOutput& stats = {},
               const FrameExposure& exposure = {}, cudaStream_t stream = nullptr) {
    const isp_raw_view_c r = detail::to_c(raw);
    const isp_rgb_view_c o = detail::to_c(out);
    const isp_stats_c s{stats.histogram, stats.stats};
    const isp_exposure_c e{exposure.exposure_ns, exposure.gain};
    detail::check(isp_b200_process(handle_.get(), &r, &o, &s, &e, stream));
  }

  // The white balance state after the frames queued so far (waits for them):
  // the gains the next frame starts from, and whether an estimate exists.
  void white_balance_state(float gains[3], bool* valid) {
    int32_t v = 0;
    detail::check(isp_b200_awb_state(handle_.get(), gains, &v));
    *valid = v != 0;
  }

 private:
  struct Destroy {
    void operator()(isp_b200_pipeline* p) const noexcept { isp_b200_destroy(p); }
  };
  IspParams params_;
  Backend backend_{Backend::kCuda};
  std::unique_ptr<isp_b200_pipeline, Destroy> handle_;
};

}  // namespace holoscan::isp
