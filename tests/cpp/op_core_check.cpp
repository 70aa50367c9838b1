// Exercises the operator core of the B200 build (holoscan/isp/isp_op_core.hpp)
// and prints one JSON object per check for tests/test_cpp_facade.py.
//
//   op_core_check host   configuration checks and input descriptions; no GPU
//   op_core_check gpu    frames from pageable, pinned and device memory
#include <cstdio>
#include <cstring>
#include <exception>
#include <functional>
#include <string>
#include <vector>

#include "holoscan/isp/isp_op_core.hpp"

using namespace holoscan::isp;

namespace {

std::string escape(const std::string& s) {
  std::string o;
  for (char c : s) o += (c == '"' || c == '\\') ? std::string("\\") + c : std::string(1, c);
  return o;
}

void config_check(const char* name, const IspOpConfig& c) {
  std::string what;
  try {
    validate_config(c);
  } catch (const std::invalid_argument& e) {
    what = e.what();
  }
  std::printf("{\"check\": \"%s\", \"error\": \"%s\"}\n", name, escape(what).c_str());
}

void describe_check(const char* name, const ImageInput& in, const IspOpConfig& c) {
  const RawDescription f = describe(in, c);
  std::printf("{\"check\": \"%s\", \"error\": \"%s\", \"width\": %d, \"height\": %d, \"pitch\": %zu, \"format\": %d, "
              "\"bits\": %d, \"pattern\": %d, \"span\": %zu, \"contiguous\": %d}\n",
              name, escape(f.error).c_str(), f.view.width, f.view.height, f.view.pitch,
              static_cast<int>(f.view.format), f.view.bit_depth, static_cast<int>(f.view.pattern), f.span,
              f.contiguous ? 1 : 0);
}

ImageInput u16_input(int w, int h, std::int64_t pitch) {
  ImageInput in;
  in.data = reinterpret_cast<const void*>(0x1000);
  in.memory = MemoryKind::kDevice;
  in.dtype = ElementType::kUint16;
  in.shape = {h, w};
  in.strides = {pitch, 2};
  in.encoding = ImageEncoding::kBayerGrbg;
  in.width = w;
  in.height = h;
  in.significant_bits = 12;
  return in;
}

int host_checks() {
  IspOpConfig ok;
  config_check("config_ok", ok);
  IspOpConfig big = ok;
  big.max_width = 20000;
  config_check("config_max_size", big);
  IspOpConfig bits = ok;
  bits.bit_depth = 17;
  config_check("config_bit_depth", bits);
  IspOpConfig packed_bits = ok;
  packed_bits.packing = Packing::kMipiRaw10;
  packed_bits.bit_depth = 12;
  config_check("config_packed_bits", packed_bits);
  IspOpConfig sharp = ok;
  sharp.params.sharpen = 9.0F;
  config_check("config_params", sharp);

  describe_check("u16_padded", u16_input(64, 32, 160), ok);
  describe_check("u16_contiguous", u16_input(64, 32, 128), ok);
  ImageInput other = u16_input(64, 32, 128);
  other.encoding = ImageEncoding::kOther;
  other.encoding_name = "RGB8";
  describe_check("bad_encoding", other, ok);
  ImageInput mono = u16_input(64, 32, 128);
  mono.encoding = ImageEncoding::kMono16;
  describe_check("mono_without_pattern", mono, ok);
  IspOpConfig with_pattern = ok;
  with_pattern.pattern = BayerPattern::kBGGR;
  describe_check("mono_with_pattern", mono, with_pattern);
  describe_check("pattern_disagrees", u16_input(64, 32, 128), with_pattern);
  ImageInput mono8 = mono;
  mono8.encoding = ImageEncoding::kMono8;
  describe_check("element_vs_encoding", mono8, with_pattern);
  ImageInput strided = u16_input(64, 32, 256);
  strided.strides = {256, 4};
  describe_check("strided_row", strided, ok);
  describe_check("overlap", u16_input(64, 32, 64), ok);
  describe_check("too_large", u16_input(4000, 32, 8000), ok);
  ImageInput odd = u16_input(64, 32, 129);
  describe_check("misaligned", odd, ok);
  ImageInput unknown_bits = u16_input(64, 32, 128);
  unknown_bits.significant_bits = kUnknownSignificantBits;
  describe_check("unknown_bits", unknown_bits, ok);
  IspOpConfig raw10 = ok;
  raw10.packing = Packing::kMipiRaw10;
  ImageInput packed;
  packed.data = reinterpret_cast<const void*>(0x1000);
  packed.dtype = ElementType::kUint8;
  packed.shape = {32, 100};
  packed.strides = {112, 1};
  packed.encoding = ImageEncoding::kBayerRggb;
  packed.width = 80;
  describe_check("raw10", packed, raw10);
  packed.width = 81;
  describe_check("raw10_short_rows", packed, raw10);
  ImageInput elsewhere = u16_input(64, 32, 128);
  elsewhere.memory = MemoryKind::kOther;
  describe_check("elsewhere", elsewhere, ok);
  return 0;
}

int gpu_checks() {
  const int w = 96, h = 64;
  IspOpConfig c;
  c.params.demosaic = DemosaicMethod::kMalvar;
  c.params.black_level = 256.0F;
  c.output_format = OutputFormat::kRgb16;
  c.stats = true;
  std::vector<std::uint16_t> host(w * h);
  for (int i = 0; i < w * h; ++i) host[i] = static_cast<std::uint16_t>(256 + (i * 2654435761U >> 20) % 3800);
  const std::size_t bytes = host.size() * 2, out_bytes = static_cast<std::size_t>(w) * h * 6;
  void *d_raw = nullptr, *pinned = nullptr, *outs[4] = {};
  std::uint32_t* hist = nullptr;
  float* st = nullptr;
  cudaMalloc(&d_raw, bytes);
  cudaMallocHost(&pinned, bytes);
  for (auto& o : outs) cudaMalloc(&o, out_bytes);
  cudaMalloc(reinterpret_cast<void**>(&hist), 4096);
  cudaMalloc(reinterpret_cast<void**>(&st), 48);
  cudaMemcpy(d_raw, host.data(), bytes, cudaMemcpyHostToDevice);
  std::memcpy(pinned, host.data(), bytes);
  IspOpCore core(c);
  IspPipeline direct(Backend::kCuda, c.params);
  ImageInput in = u16_input(w, h, w * 2);
  const IspOpStatistics s0 = isp_op_statistics();
  in.memory = MemoryKind::kHost;
  in.data = host.data();
  core.process(in, outs[0], hist, st, nullptr);
  const IspOpStatistics s1 = isp_op_statistics();
  in.memory = MemoryKind::kPinnedHost;
  in.data = pinned;
  core.process(in, outs[1], hist, st, nullptr);
  const IspOpStatistics s2 = isp_op_statistics();
  // Pinned again, with a tensor that holds its memory until the stream has
  // passed the copy (the SDK's set_deallocation_stream): no wait.
  int holds = 0;
  cudaStream_t held_on = reinterpret_cast<cudaStream_t>(1);
  in.hold_until_done = [&](cudaStream_t s) {
    ++holds;
    held_on = s;
    return true;
  };
  core.process(in, outs[1], hist, st, nullptr);
  in.hold_until_done = nullptr;
  const IspOpStatistics s2h = isp_op_statistics();
  in.memory = MemoryKind::kDevice;
  in.data = d_raw;
  core.process(in, outs[2], hist, st, nullptr);
  const IspOpStatistics s3 = isp_op_statistics();
  // The same three frames straight through a pipeline of the same settings.
  const RawImageView rv{d_raw, w, h, static_cast<std::size_t>(w) * 2, RawFormat::kUint16, 12, BayerPattern::kGRBG};
  const RgbImageView ov{outs[3], static_cast<std::size_t>(w) * 6, OutputFormat::kRgb16};
  std::vector<unsigned char> a(out_bytes), b(out_bytes);
  int same = 1;
  for (int k = 0; k < 3; ++k) {
    direct.process(rv, ov, {}, {}, nullptr);
    cudaMemcpy(a.data(), outs[k], out_bytes, cudaMemcpyDeviceToHost);
    cudaMemcpy(b.data(), outs[3], out_bytes, cudaMemcpyDeviceToHost);
    same = same && std::memcmp(a.data(), b.data(), out_bytes) == 0;
  }
  std::printf("{\"check\": \"gpu\", \"error\": \"%s\", \"same\": %d, \"pageable_waits\": %llu, \"pageable_copies\": %llu, "
              "\"pinned_waits\": %llu, \"pinned_copies\": %llu, \"held_waits\": %llu, \"held_copies\": %llu, "
              "\"holds\": %d, \"held_on_stream\": %d, \"device_waits\": %llu, \"device_copies\": %llu}\n",
              cudaGetErrorString(cudaDeviceSynchronize()), same,
              static_cast<unsigned long long>(s1.host_waits - s0.host_waits),
              static_cast<unsigned long long>(s1.copies - s0.copies),
              static_cast<unsigned long long>(s2.host_waits - s1.host_waits),
              static_cast<unsigned long long>(s2.copies - s1.copies),
              static_cast<unsigned long long>(s2h.host_waits - s2.host_waits),
              static_cast<unsigned long long>(s2h.copies - s2.copies), holds, held_on == nullptr ? 1 : 0,
              static_cast<unsigned long long>(s3.host_waits - s2h.host_waits),
              static_cast<unsigned long long>(s3.copies - s2h.copies));
  for (auto& o : outs) cudaFree(o);
  cudaFree(d_raw);
  cudaFreeHost(pinned);
  cudaFree(hist);
  cudaFree(st);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc >= 2 && std::strcmp(argv[1], "host") == 0) return host_checks();
  if (argc >= 2 && std::strcmp(argv[1], "gpu") == 0) return gpu_checks();
  std::fprintf(stderr, "usage: op_core_check host | gpu\n");
  return 2;
}
