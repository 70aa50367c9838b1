// converter.hpp - holoscan::color_convert::Converter for C++ callers of the
// B200 converter: the reference module's class and free functions
// (include/holoscan/color_convert/backend.hpp:15-53, converter.hpp:27-80)
// with the same constructor, methods and exceptions, over the C ABI
// (cc_b200_convert, cc_b200_test_pattern). The conversion runs on the B200's
// CUDA kernels; the VIC is Jetson hardware and is not part of this build, so
// Backend::kVic is refused as a build without VPI refuses it and
// Backend::kAuto always chooses kCuda. Header-only: link libisp_b200.so and
// the CUDA runtime.
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>

#include "holoscan/color_convert/conversion.hpp"

namespace holoscan::color_convert {

enum class Backend : std::uint8_t { kCuda, kVic, kAuto };

[[nodiscard]] inline std::string_view backend_name(Backend backend) noexcept {
  switch (backend) {
    case Backend::kCuda: return "cuda";
    case Backend::kVic: return "vic";
    case Backend::kAuto: return "auto";
  }
  return "unknown";
}

[[nodiscard]] inline std::optional<Backend> parse_backend(std::string_view name) noexcept {
  if (name == "cuda") return Backend::kCuda;
  if (name == "vic") return Backend::kVic;
  if (name == "auto") return Backend::kAuto;
  return std::nullopt;
}

struct PlatformFacts {
  bool vpi_compiled{};
  bool has_vic{};
};

[[nodiscard]] constexpr Backend resolve_auto(const PlatformFacts& facts, bool vic_can_convert) noexcept {
  return facts.vpi_compiled && facts.has_vic && vic_can_convert ? Backend::kVic : Backend::kCuda;
}

// This build has no VPI: neither fact holds.
[[nodiscard]] inline PlatformFacts probe_platform() noexcept { return PlatformFacts{}; }

// @throws std::invalid_argument for Backend::kVic, which this build lacks.
inline void check_available(Backend backend) {
  if (backend == Backend::kVic) {
    throw std::invalid_argument("backend vic: this build has no VPI; install VPI 4 and rebuild");
  }
}

// Fills `rgb8`, a device RGB8 view, with the synthetic camera's frame `frame`.
[[nodiscard]] inline cudaError_t launch_test_pattern(const ImageView& rgb8, std::uint32_t frame,
                                                     cudaStream_t stream) {
  const cc_image_c v = detail::to_c(rgb8);
  const int s = cc_b200_test_pattern(&v, frame, stream);
  if (s == ISP_OK) return cudaSuccess;
  if (s == ISP_EINVAL) return cudaErrorInvalidValue;
  return static_cast<cudaError_t>(isp_b200_last_cuda_error());
}

class Converter {
 public:
  // @throws std::invalid_argument for Backend::kVic (check_available()).
  explicit Converter(Backend backend) : backend_(backend) { check_available(backend); }
  Converter(const Converter&) = delete;
  Converter& operator=(const Converter&) = delete;

  // The backend that would convert these images, with why (empty for a
  // configured backend).
  [[nodiscard]] std::pair<Backend, std::string> choose(const ImageView&, const ImageView&,
                                                       const ConversionParams&) const {
    if (backend_ != Backend::kAuto) return {backend_, std::string()};
    return {Backend::kCuda, "this build has no vic backend"};
  }

  // Converts `source` into `destination`, both in CUDA device memory, after
  // the work already queued on `stream`; returns the backend that ran.
  // @throws std::invalid_argument if the images or params are not usable.
  // @throws std::runtime_error on a CUDA failure.
  Backend convert(const ImageView& source, const ImageView& destination, const ConversionParams& params,
                  cudaStream_t stream) {
    const cc_image_c s = detail::to_c(source);
    const cc_image_c d = detail::to_c(destination);
    const cc_params_c c = detail::to_c(params);
    detail::check(cc_b200_convert(&s, &d, &c, stream));
    return Backend::kCuda;
  }

  [[nodiscard]] Backend backend() const noexcept { return backend_; }

 private:
  Backend backend_;
};

}  // namespace holoscan::color_convert
