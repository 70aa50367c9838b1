// Exercises holoscan::isp's C++ interface of the B200 build (the headers in
// holoscan-zozo-modules_b200/cpp/include) and prints one JSON object per
// check for tests/test_cpp_facade.py.
//
//   facade_check host           settings checks, tables, names; no GPU needed
//   facade_check gpu OUT_FILE   two frames through IspPipeline(kCuda); writes
//                               the images, histograms and statistics
#include <cstdio>
#include <cstring>
#include <exception>
#include <functional>
#include <string>
#include <vector>

#include "holoscan/isp/isp_pipeline.hpp"

using namespace holoscan::isp;

namespace {

std::string escape(const std::string& s) {
  std::string o;
  for (char c : s) o += (c == '"' || c == '\\') ? std::string("\\") + c : std::string(1, c);
  return o;
}

// Runs f and reports which exception it threw ("none", "invalid_argument",
// "runtime_error", "other") and its message.
void report(const char* name, const std::function<void()>& f) {
  std::string kind = "none", what;
  try {
    f();
  } catch (const std::invalid_argument& e) {
    kind = "invalid_argument";
    what = e.what();
  } catch (const std::runtime_error& e) {
    kind = "runtime_error";
    what = e.what();
  } catch (const std::exception& e) {
    kind = "other";
    what = e.what();
  }
  std::printf("{\"check\": \"%s\", \"throws\": \"%s\", \"what\": \"%s\"}\n", name, kind.c_str(), escape(what).c_str());
}

// The deterministic frame of the GPU check: xorshift32 counts below 2^10,
// MIPI RAW10 packed (four samples in five bytes).
std::vector<unsigned char> raw10_frame(int width, int height, unsigned seed) {
  const std::size_t row = raw_row_bytes(RawFormat::kRaw10, width);
  std::vector<unsigned char> data(row * static_cast<std::size_t>(height), 0);
  unsigned s = seed;
  for (int y = 0; y < height; ++y) {
    for (int x = 0; x < width; ++x) {
      s ^= s << 13;
      s ^= s >> 17;
      s ^= s << 5;
      const unsigned v = s & 1023U;
      unsigned char* g = data.data() + y * row + 5 * (x / 4);
      g[x % 4] = static_cast<unsigned char>(v >> 2);
      g[4] = static_cast<unsigned char>(g[4] | ((v & 3U) << (2 * (x % 4))));
    }
  }
  return data;
}

IspParams gpu_params() {
  IspParams p;
  p.black_level = 64.0F;
  p.white_balance = WhiteBalanceMode::kGrayWorld;
  p.demosaic = DemosaicMethod::kMalvar;
  p.sharpen = 0.5F;
  p.ccm = {1.6F, -0.3F, -0.3F, -0.3F, 1.6F, -0.3F, -0.3F, -0.3F, 1.6F};
  LensShading l;
  l.width = 5;
  l.height = 4;
  l.channels = 4;
  for (int i = 0; i < l.width * l.height * l.channels; ++i) l.gains.push_back(1.0F + static_cast<float>(i % 7) * 0.125F);
  p.lens_shading = l;
  return p;
}

int host_checks() {
  IspParams ok;
  report("valid_params", [&] { validate_params(ok); });
  IspParams bad_sharpen;
  bad_sharpen.sharpen = 5.0F;
  report("bad_sharpen", [&] { validate_params(bad_sharpen); });
  IspParams bad_gain;
  bad_gain.wb_gains = {0.0F, 1.0F, 1.0F};
  report("bad_wb_gain", [&] { validate_params(bad_gain); });
  IspParams bad_lut;
  bad_lut.tone_curve = ToneCurve::kLut;
  bad_lut.lut = {0.5F};
  report("bad_lut", [&] { validate_params(bad_lut); });
  IspParams bad_grid = gpu_params();
  bad_grid.lens_shading->gains.pop_back();
  report("bad_grid", [&] { validate_params(bad_grid); });
  RawImageView narrow{reinterpret_cast<const void*>(0x100), 1, 4, 8, RawFormat::kUint16, 12, BayerPattern::kRGGB};
  report("bad_raw_width", [&] { validate_raw(narrow, ok); });
  RawImageView deep{reinterpret_cast<const void*>(0x100), 4, 4, 8, RawFormat::kUint16, 17, BayerPattern::kRGGB};
  report("bad_bit_depth", [&] { validate_raw(deep, ok); });
  report("cpu_backend", [&] { IspPipeline pipe(Backend::kCpu, ok); });
  report("bad_params_before_cuda", [&] { IspPipeline pipe(Backend::kCuda, bad_sharpen); });
  // Tables and sizes.
  IspParams gamma;
  gamma.tone_curve = ToneCurve::kGamma;
  gamma.gamma = 2.4F;
  const std::vector<float> t = tone_lut(gamma);
  double checksum = 0.0;
  for (float v : t) checksum += v;
  std::printf("{\"check\": \"tone_gamma\", \"size\": %zu, \"first\": %.9g, \"mid\": %.9g, \"last\": %.9g, \"sum\": %.17g}\n",
              t.size(), t.front(), t[t.size() / 2], t.back(), checksum);
  std::printf("{\"check\": \"row_bytes\", \"u8\": %zu, \"u16\": %zu, \"raw10\": %zu, \"raw12\": %zu}\n",
              raw_row_bytes(RawFormat::kUint8, 3839), raw_row_bytes(RawFormat::kUint16, 3839),
              raw_row_bytes(RawFormat::kRaw10, 3839), raw_row_bytes(RawFormat::kRaw12, 3839));
  std::printf("{\"check\": \"names\", \"pattern\": \"%s\", \"parsed\": %d, \"wb\": \"%s\", \"backend\": %d, \"unknown\": %d}\n",
              std::string(pattern_name(BayerPattern::kGBRG)).c_str(), static_cast<int>(*parse_pattern("GRBG")),
              std::string(white_balance_name(WhiteBalanceMode::kWhitePatch)).c_str(),
              static_cast<int>(*parse_backend("cuda")), parse_demosaic("nearest").has_value() ? 1 : 0);
  std::printf("{\"check\": \"channels\", \"rgba8\": %d, \"rgb16_bytes\": %d, \"resolve_no_gpu\": %d}\n",
              output_channels(OutputFormat::kRgba8), output_channel_bytes(OutputFormat::kRgb16),
              static_cast<int>(resolve_auto(PlatformFacts{false})));
  return 0;
}

int gpu_check(const char* path) {
  const int width = 200, height = 120;
  const IspParams params = gpu_params();
  IspPipeline pipe(Backend::kCuda, params);
  const std::size_t row = raw_row_bytes(RawFormat::kRaw10, width);
  const std::size_t out_pitch = static_cast<std::size_t>(width) * 6;  // RGB16
  void *d_raw = nullptr, *d_out = nullptr, *d_hist = nullptr, *d_stats = nullptr;
  if (cudaMalloc(&d_raw, row * height) != cudaSuccess || cudaMalloc(&d_out, out_pitch * height) != cudaSuccess ||
      cudaMalloc(&d_hist, kHistogramChannels * kHistogramBins * 4) != cudaSuccess ||
      cudaMalloc(&d_stats, stats::kStatsSize * 4) != cudaSuccess) {
    std::printf("{\"check\": \"gpu\", \"error\": \"cudaMalloc\"}\n");
    return 1;
  }
  std::FILE* f = std::fopen(path, "wb");
  if (f == nullptr) return 1;
  for (unsigned frame = 0; frame < 2; ++frame) {
    const std::vector<unsigned char> raw = raw10_frame(width, height, 12345U + frame);
    cudaMemcpy(d_raw, raw.data(), raw.size(), cudaMemcpyHostToDevice);
    const RawImageView rv{d_raw, width, height, row, RawFormat::kRaw10, 10, BayerPattern::kGRBG};
    const RgbImageView ov{d_out, out_pitch, OutputFormat::kRgb16};
    const StatsOutput so{static_cast<std::uint32_t*>(d_hist), static_cast<float*>(d_stats)};
    pipe.process(rv, ov, so, FrameExposure{8'000'000, 1.5F});
    std::vector<unsigned char> image(out_pitch * height);
    std::vector<std::uint32_t> hist(kHistogramChannels * kHistogramBins);
    std::vector<float> st(stats::kStatsSize);
    cudaMemcpy(image.data(), d_out, image.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(hist.data(), d_hist, hist.size() * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(st.data(), d_stats, st.size() * 4, cudaMemcpyDeviceToHost);
    std::fwrite(image.data(), 1, image.size(), f);
    std::fwrite(hist.data(), 4, hist.size(), f);
    std::fwrite(st.data(), 4, st.size(), f);
  }
  std::fclose(f);
  std::printf("{\"check\": \"gpu\", \"error\": \"%s\"}\n", cudaGetErrorString(cudaDeviceSynchronize()));
  cudaFree(d_raw);
  cudaFree(d_out);
  cudaFree(d_hist);
  cudaFree(d_stats);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc >= 2 && std::strcmp(argv[1], "host") == 0) return host_checks();
  if (argc >= 3 && std::strcmp(argv[1], "gpu") == 0) return gpu_check(argv[2]);
  std::fprintf(stderr, "usage: facade_check host | gpu OUT_FILE\n");
  return 2;
}
