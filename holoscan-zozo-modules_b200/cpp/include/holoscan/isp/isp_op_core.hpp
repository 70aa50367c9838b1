// isp_op_core.hpp - the Holoscan operator's work, without the Holoscan SDK.
//
// The reference module's IspOp (include/holoscan/isp/isp_op.hpp:33-115,
// src/isp_op.cpp) reads a raw image from its `raw` port, describes it as a
// RawImageView (encoding, element type, shape, strides, packing), stages it
// into device memory when it arrived in host memory, runs IspPipeline, and
// emits an RGB image whose descriptor keeps the input's header, region
// offsets, exposure and gain. Everything but the ports is here, for the CUDA
// backend, on a plain description of the received image (ImageInput) in
// place of holoscan::schema::ImageT and its tensor; an IspOp over the SDK
// fills an ImageInput from the received ImageT, calls IspOpCore::process
// with the output tensors it allocated, and emits. Configuration checks,
// error messages and the wait/copy accounting follow the reference's.
#pragma once

#include <cuda_runtime_api.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <optional>
#include <string>
#include <utility>
#include <vector>

#include "holoscan/isp/isp_pipeline.hpp"

namespace holoscan::isp {

enum class Packing : std::uint8_t { kNone, kMipiRaw10, kMipiRaw12 };

struct IspOpConfig {
  Backend backend{Backend::kCuda};
  IspParams params;
  OutputFormat output_format{OutputFormat::kRgb8};
  std::optional<BayerPattern> pattern;  // for MONO8/MONO16 inputs; must agree with a BAYER_* encoding
  int bit_depth{0};                     // 0: the image's significant bits, else the container's
  Packing packing{Packing::kNone};
  bool stats{false};
  int max_width{3840};
  int max_height{2160};
};

// @throws std::invalid_argument naming the first unusable field.
inline void validate_config(const IspOpConfig& config) {
  validate_params(config.params);
  if (config.max_width < 2 || config.max_height < 2 || config.max_width > 16384 || config.max_height > 16384) {
    throw std::invalid_argument("max_width and max_height must be 2..16384");
  }
  if (config.bit_depth < 0 || config.bit_depth > 16) {
    throw std::invalid_argument("bit_depth must be 0 (from the image) or 1..16");
  }
  if ((config.packing == Packing::kMipiRaw10 && config.bit_depth != 0 && config.bit_depth != 10) ||
      (config.packing == Packing::kMipiRaw12 && config.bit_depth != 0 && config.bit_depth != 12)) {
    throw std::invalid_argument("packed RAW10 and RAW12 samples have 10 and 12 bits");
  }
}

// The image encodings the operator distinguishes.
enum class ImageEncoding : std::uint8_t { kBayerRggb, kBayerBggr, kBayerGrbg, kBayerGbrg, kMono8, kMono16, kOther };
enum class MemoryKind : std::uint8_t { kHost, kPinnedHost, kDevice, kOther };
enum class ElementType : std::uint8_t { kUint8, kUint16, kOther };

// A received raw image: its tensor (data, memory, element type, shape,
// strides in bytes) and its descriptor's fields.
struct ImageInput {
  const void* data{};
  MemoryKind memory{MemoryKind::kDevice};
  ElementType dtype{ElementType::kUint16};
  std::vector<std::int64_t> shape;
  std::vector<std::int64_t> strides;  // bytes
  ImageEncoding encoding{ImageEncoding::kBayerRggb};
  std::string encoding_name;  // for the message about an unsupported encoding
  int width{};                // descriptor; 0 unknown
  int height{};
  unsigned significant_bits{};  // 0 (or kUnknownSignificantBits) unknown
  std::int64_t exposure_time_ns{};
  float gain{};
  // For pinned host memory: keeps the tensor's memory from reuse until the
  // work queued on the stream so far is done (the SDK's
  // Tensor::set_deallocation_stream); false when the tensor cannot. Without
  // it, or when it fails, the operator waits for the stream after the copy.
  std::function<bool(cudaStream_t)> hold_until_done;
};
inline constexpr unsigned kUnknownSignificantBits = 0xFFFFFFFFU;

// The raw view of an input, the bytes its rows span and whether the rows
// follow each other without padding; or why the input cannot be processed.
struct RawDescription {
  RawImageView view;
  std::size_t span{};
  bool contiguous{};
  std::string error;  // "IspOp: ..." when the input is unusable
  explicit operator bool() const noexcept { return error.empty(); }
};

inline RawDescription describe(const ImageInput& in, const IspOpConfig& config) {
  RawDescription f;
  const auto invalid = [&f](const std::string& m) {
    f.error = "IspOp: " + m;
    return f;
  };
  if (in.memory == MemoryKind::kOther) return invalid("raw images must be in host or CUDA memory");
  std::optional<BayerPattern> pattern;
  switch (in.encoding) {
    case ImageEncoding::kBayerRggb: pattern = BayerPattern::kRGGB; break;
    case ImageEncoding::kBayerBggr: pattern = BayerPattern::kBGGR; break;
    case ImageEncoding::kBayerGrbg: pattern = BayerPattern::kGRBG; break;
    case ImageEncoding::kBayerGbrg: pattern = BayerPattern::kGBRG; break;
    default: break;
  }
  const bool mono = in.encoding == ImageEncoding::kMono8 || in.encoding == ImageEncoding::kMono16;
  if (!pattern && !mono) {
    return invalid("unsupported raw encoding " + in.encoding_name +
                   "; use BAYER_RGGB, BAYER_BGGR, BAYER_GRBG, BAYER_GBRG, MONO8 or MONO16");
  }
  if (mono && !config.pattern) return invalid("a MONO8 or MONO16 raw image needs the Bayer pattern in the configuration");
  if (pattern && config.pattern && *pattern != *config.pattern) {
    return invalid("the image's pattern " + std::string(pattern_name(*pattern)) + " disagrees with the configured " +
                   std::string(pattern_name(*config.pattern)));
  }
  RawImageView& v = f.view;
  v.pattern = pattern ? *pattern : *config.pattern;
  v.data = in.data;
  int container_bits = 0;
  std::int64_t row_bytes = 0;
  const auto stride = [&in](std::size_t i) { return i < in.strides.size() ? in.strides[i] : 0; };
  if (config.packing == Packing::kNone) {
    const bool u8 = in.dtype == ElementType::kUint8;
    if (!(u8 || in.dtype == ElementType::kUint16)) return invalid("raw samples must be uint8 or uint16");
    if ((in.encoding == ImageEncoding::kMono8 && !u8) || (in.encoding == ImageEncoding::kMono16 && u8)) {
      return invalid("raw element type disagrees with its encoding");
    }
    if (!(in.shape.size() == 2 || (in.shape.size() == 3 && in.shape[2] == 1))) {
      return invalid("raw tensor must be [H, W] or [H, W, 1]");
    }
    v.height = static_cast<int>(in.shape[0]);
    v.width = static_cast<int>(in.shape[1]);
    v.format = u8 ? RawFormat::kUint8 : RawFormat::kUint16;
    container_bits = u8 ? 8 : 16;
    const std::int64_t element = u8 ? 1 : 2;
    if (v.width > 1 && stride(1) != element) return invalid("raw samples within a row must be packed");
    row_bytes = element * v.width;
    if ((in.width != 0 && in.width != v.width) || (in.height != 0 && in.height != v.height)) {
      return invalid("the descriptor's size disagrees with its tensor");
    }
  } else {
    if (in.dtype != ElementType::kUint8 || in.shape.size() != 2) {
      return invalid("packed raw images must be uint8 [H, row bytes]");
    }
    if (in.shape[1] > 1 && stride(1) != 1) return invalid("packed raw rows must be contiguous");
    v.height = static_cast<int>(in.shape[0]);
    v.width = in.width;
    v.format = config.packing == Packing::kMipiRaw10 ? RawFormat::kRaw10 : RawFormat::kRaw12;
    container_bits = config.packing == Packing::kMipiRaw10 ? 10 : 12;
    row_bytes = in.shape[1];
    if (in.height != 0 && in.height != v.height) return invalid("the descriptor's height disagrees with its tensor");
    if (static_cast<std::size_t>(row_bytes) < raw_row_bytes(v.format, v.width)) {
      return invalid("packed rows of " + std::to_string(row_bytes) + " bytes cannot hold " + std::to_string(v.width) +
                     " samples");
    }
  }
  if (v.width < 2 || v.height < 2 || v.width > config.max_width || v.height > config.max_height) {
    return invalid("raw image " + std::to_string(v.width) + "x" + std::to_string(v.height) +
                   " is outside 2x2 to the configured " + std::to_string(config.max_width) + "x" +
                   std::to_string(config.max_height));
  }
  const std::int64_t pitch = v.height > 1 ? stride(0) : row_bytes;
  if (pitch < row_bytes) return invalid("raw rows overlap");
  v.pitch = static_cast<std::size_t>(pitch);
  f.contiguous = pitch == row_bytes;
  if (v.format == RawFormat::kUint16 &&
      (reinterpret_cast<std::uintptr_t>(v.data) % 2U != 0U || v.pitch % 2U != 0U)) {
    return invalid("uint16 raw data must be aligned to 2 bytes");
  }
  const bool known_bits = in.significant_bits != 0U && in.significant_bits != kUnknownSignificantBits;
  v.bit_depth = config.bit_depth > 0                                 ? config.bit_depth
                : known_bits && config.packing == Packing::kNone ? static_cast<int>(in.significant_bits)
                                                                   : container_bits;
  f.span = v.pitch * static_cast<std::size_t>(v.height - 1) + raw_row_bytes(v.format, v.width);
  return f;
}

// The emitted image's shape and encoding: [H, W, channels] of the output
// format's element type; its descriptor copies the input's header, region
// offsets, exposure time and gain, colour space unspecified.
struct ImageOutput {
  int height{}, width{}, channels{};
  int element_bytes{};
  OutputFormat format{OutputFormat::kRgb8};
};
inline ImageOutput output_of(const RawDescription& raw, OutputFormat format) {
  return ImageOutput{raw.view.height, raw.view.width, output_channels(format), output_channel_bytes(format), format};
}

// Waits of the operator's thread and raw frames copied between host and
// device, over every IspOpCore of the process.
struct IspOpStatistics {
  std::uint64_t host_waits{};
  std::uint64_t copies{};
};
namespace detail {
inline std::atomic<std::uint64_t> g_op_host_waits{0};
inline std::atomic<std::uint64_t> g_op_copies{0};
}  // namespace detail
[[nodiscard]] inline IspOpStatistics isp_op_statistics() noexcept {
  return IspOpStatistics{detail::g_op_host_waits.load(std::memory_order_relaxed),
                         detail::g_op_copies.load(std::memory_order_relaxed)};
}

// The operator's per-frame work on the CUDA backend.
class IspOpCore {
 public:
  // @throws std::invalid_argument if `config` is not valid (or asks for the
  //         CPU backend, which this build does not ship).
  // @throws std::runtime_error if CUDA fails.
  explicit IspOpCore(IspOpConfig config) : config_(std::move(config)) {
    validate_config(config_);
    pipeline_ = std::make_unique<IspPipeline>(config_.backend, config_.params);
  }
  ~IspOpCore() {
    if (staging_ != nullptr) {
      cudaStreamSynchronize(last_stream_);
      cudaFree(staging_);
    }
  }
  IspOpCore(const IspOpCore&) = delete;
  IspOpCore& operator=(const IspOpCore&) = delete;

  [[nodiscard]] const IspOpConfig& config() const noexcept { return config_; }

  // One received frame: described, staged into device memory when it
  // arrived in host memory, and queued through the pipeline on `stream` into
  // `image` (device memory, packed rows) and, with config().stats,
  // `histogram` and `stats`. Staging follows isp_op.cpp:392-441: a pageable
  // frame is waited for (its producer) and its copy returns once staged (a
  // second wait); a pinned frame's copy is queued, and its memory is kept
  // from reuse until the stream has passed the copy, by the input's
  // hold_until_done where it succeeds, else by waiting for the stream (one
  // wait).
  // @throws std::invalid_argument with the operator's message for an unusable input.
  // @throws std::runtime_error if CUDA fails.
  ImageOutput process(const ImageInput& in, void* image, std::uint32_t* histogram, float* stats,
                      cudaStream_t stream) {
    RawDescription f = describe(in, config_);
    if (!f) throw std::invalid_argument(f.error);
    if (in.memory != MemoryKind::kDevice) {
      // A pageable input: its producer has finished writing it (the SDK's
      // synchronize_for_host), a wait of this thread.
      if (in.memory == MemoryKind::kHost) count_wait();
      if (staging_bytes_ < f.span) {
        if (staging_ != nullptr) {
          count_wait();
          check(cudaStreamSynchronize(last_stream_), "cudaStreamSynchronize");
          check(cudaFree(staging_), "cudaFree");
          staging_ = nullptr;
          staging_bytes_ = 0;
        }
        check(cudaMalloc(&staging_, f.span), "cudaMalloc");
        staging_bytes_ = f.span;
      }
      check(cudaMemcpyAsync(staging_, f.view.data, f.span, cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync");
      detail::g_op_copies.fetch_add(1, std::memory_order_relaxed);
      if (in.memory == MemoryKind::kHost) {
        count_wait();  // a pageable copy returns once staged
      } else if (!in.hold_until_done || !in.hold_until_done(stream)) {
        // The producer must not reuse pinned memory while the copy reads it.
        count_wait();
        check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
      }
      f.view.data = staging_;
    }
    last_stream_ = stream;
    const ImageOutput out = output_of(f, config_.output_format);
    const RgbImageView view{image, static_cast<std::size_t>(out.width) * out.channels * out.element_bytes,
                            config_.output_format};
    const StatsOutput so{config_.stats ? histogram : nullptr, config_.stats ? stats : nullptr};
    pipeline_->process(f.view, view, so, FrameExposure{in.exposure_time_ns, in.gain}, stream);
    return out;
  }

 private:
  static void count_wait() noexcept { detail::g_op_host_waits.fetch_add(1, std::memory_order_relaxed); }
  static void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("IspOp: ") + what + ": " + cudaGetErrorString(e));
  }

  IspOpConfig config_;
  std::unique_ptr<IspPipeline> pipeline_;
  void* staging_{};
  std::size_t staging_bytes_{};
  cudaStream_t last_stream_{};
};

}  // namespace holoscan::isp
