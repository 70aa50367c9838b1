// cc_facade_check.cpp - compiled use of holoscan::color_convert's C++
// interface in the B200 build (holoscan-zozo-modules_b200/cpp/include/
// holoscan/color_convert/), run by tests/test_cc_facade.py.
//
//   cc_facade_check host        names, sizes, geometry and exceptions (no GPU)
//   cc_facade_check gpu <file>  the synthetic camera's 1920x1080 frame 3 into
//                               NV12 (BT.709, nearest), then that into a
//                               letterboxed 640x640 RGB8 (bilinear); both
//                               outputs written to <file>
// Host results print as one JSON object per line.
#include <cuda_runtime_api.h>

#include <cstdio>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include <holoscan/color_convert/converter.hpp>

namespace cc = holoscan::color_convert;

namespace {

template <class F>
void expect_throw(const char* name, F&& f) {
  std::string kind = "none", what;
  try {
    f();
  } catch (const std::invalid_argument& e) {
    kind = "invalid_argument";
    what = e.what();
  } catch (const std::exception& e) {
    kind = "other";
    what = e.what();
  }
  std::printf("{\"check\": \"%s\", \"throws\": \"%s\", \"what\": \"%s\"}\n", name, kind.c_str(), what.c_str());
}

int host() {
  std::printf("{\"check\": \"names\", \"nv12\": \"%s\", \"rgb16\": \"%s\", \"parsed_uyvy\": %d, \"bt2020\": \"%s\", "
              "\"full\": \"%s\", \"area\": \"%s\", \"bad\": %d, \"auto\": \"%s\"}\n",
              std::string(cc::format_name(cc::PixelFormat::kNv12)).c_str(),
              std::string(cc::format_name(cc::PixelFormat::kRgb16)).c_str(),
              static_cast<int>(*cc::parse_format("uyvy")), std::string(cc::matrix_name(cc::ColorMatrix::kBt2020)).c_str(),
              std::string(cc::range_name(cc::ColorRange::kFull)).c_str(),
              std::string(cc::resize_mode_name(cc::ResizeMode::kArea)).c_str(), cc::parse_format("nv21") ? 1 : 0,
              std::string(cc::backend_name(cc::Backend::kAuto)).c_str());
  std::printf("{\"check\": \"sizes\", \"nv12_5x3\": %zu, \"i420_5x3\": %zu, \"nv16_5x3\": %zu, \"yuyv_even\": %d, "
              "\"alpha\": %d, \"planar\": %d}\n",
              cc::packed_size(cc::PixelFormat::kNv12, 5, 3), cc::packed_size(cc::PixelFormat::kI420, 5, 3),
              cc::packed_size(cc::PixelFormat::kNv16, 5, 3), cc::needs_even_width(cc::PixelFormat::kYuyv) ? 1 : 0,
              cc::has_alpha(cc::PixelFormat::kBgra8) ? 1 : 0, cc::is_planar(cc::PixelFormat::kI420) ? 1 : 0);
  cc::ConversionParams box;
  box.letterbox = true;
  const cc::Mapping m = cc::compute_mapping(1920, 1080, 640, 640, cc::PixelFormat::kRgb8, box);
  std::printf("{\"check\": \"letterbox\", \"content\": [%d, %d, %d, %d], \"source\": [%d, %d, %d, %d]}\n",
              m.content.x, m.content.y, m.content.width, m.content.height, m.source.x, m.source.y, m.source.width,
              m.source.height);
  expect_throw("bad_crop", [] {
    cc::ConversionParams p;
    p.crop = cc::Rect{90, 0, 20, 10};
    (void)cc::compute_mapping(100, 100, 10, 10, cc::PixelFormat::kRgb8, p);
  });
  std::vector<std::uint8_t> buf(4096);
  expect_throw("odd_yuyv", [&] {
    cc::ImageView odd = cc::packed_view(buf.data(), cc::PixelFormat::kYuyv, 4, 2, cc::MemoryLocation::kDevice);
    odd.width = 3;
    const cc::ImageView rgb = cc::packed_view(buf.data(), cc::PixelFormat::kRgb8, 3, 2, cc::MemoryLocation::kDevice);
    cc::validate_conversion(odd, rgb, {});
  });
  expect_throw("host_images", [&] {
    cc::Converter c(cc::Backend::kCuda);
    const cc::ImageView h = cc::packed_view(buf.data(), cc::PixelFormat::kRgb8, 8, 8, cc::MemoryLocation::kHost);
    c.convert(h, h, {}, nullptr);
  });
  expect_throw("vic_backend", [] { cc::Converter c(cc::Backend::kVic); });
  cc::Converter autoc(cc::Backend::kAuto);
  const cc::ImageView v = cc::packed_view(buf.data(), cc::PixelFormat::kRgb8, 8, 8, cc::MemoryLocation::kDevice);
  const auto chosen = autoc.choose(v, v, {});
  std::printf("{\"check\": \"auto\", \"chosen\": \"%s\", \"why\": \"%s\"}\n",
              std::string(cc::backend_name(chosen.first)).c_str(), chosen.second.c_str());
  return 0;
}

int gpu(const char* path) {
  const int w = 1920, h = 1080;
  std::uint8_t *rgb = nullptr, *nv12 = nullptr, *box = nullptr;
  const std::size_t n_rgb = cc::packed_size(cc::PixelFormat::kRgb8, w, h);
  const std::size_t n_nv12 = cc::packed_size(cc::PixelFormat::kNv12, w, h);
  const std::size_t n_box = cc::packed_size(cc::PixelFormat::kRgb8, 640, 640);
  if (cudaMalloc(reinterpret_cast<void**>(&rgb), n_rgb) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&nv12), n_nv12) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&box), n_box) != cudaSuccess) {
    return 2;
  }
  const cc::ImageView v_rgb = cc::packed_view(rgb, cc::PixelFormat::kRgb8, w, h, cc::MemoryLocation::kDevice);
  const cc::ImageView v_nv12 = cc::packed_view(nv12, cc::PixelFormat::kNv12, w, h, cc::MemoryLocation::kDevice);
  const cc::ImageView v_box = cc::packed_view(box, cc::PixelFormat::kRgb8, 640, 640, cc::MemoryLocation::kDevice);
  if (cc::launch_test_pattern(v_rgb, 3, nullptr) != cudaSuccess) return 3;
  cc::Converter conv(cc::Backend::kCuda);
  cc::ConversionParams p;
  p.matrix = cc::ColorMatrix::kBt709;
  p.mode = cc::ResizeMode::kNearest;
  conv.convert(v_rgb, v_nv12, p, nullptr);
  cc::ConversionParams q;
  q.matrix = cc::ColorMatrix::kBt709;
  q.letterbox = true;
  q.fill_rgb = {200, 30, 90};
  conv.convert(v_nv12, v_box, q, nullptr);
  std::vector<std::uint8_t> out(n_nv12 + n_box);
  if (cudaMemcpy(out.data(), nv12, n_nv12, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(out.data() + n_nv12, box, n_box, cudaMemcpyDeviceToHost) != cudaSuccess) {
    return 4;
  }
  FILE* f = std::fopen(path, "wb");
  if (f == nullptr || std::fwrite(out.data(), 1, out.size(), f) != out.size()) return 5;
  std::fclose(f);
  cudaFree(rgb);
  cudaFree(nv12);
  cudaFree(box);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const std::string mode = argc > 1 ? argv[1] : "host";
  if (mode == "gpu" && argc > 2) return gpu(argv[2]);
  return host();
}
