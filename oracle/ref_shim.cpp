// ref_shim.cpp - TEST INFRASTRUCTURE ONLY. A C ABI over the reference's own
// CPU backend, compiled together with the reference's unmodified sources
// (modules/isp/src/cpu_pipeline.cpp, isp_params.cpp, synthetic_raw.cpp) into
// oracle/_ref/libisp_ref.so by oracle/Makefile. It lets the tests pin the C
// oracle to the reference's outputs, generate tests/golden/, and lets the
// benchmark time the reference's CPU path on the host cores.
//
// The per-frame call reproduces IspPipeline(Backend::kCpu)::process
// (modules/isp/src/isp_pipeline.cpp:65-84): validate_raw, the output view
// checks, make_frame_params and cpu_process, with the pipeline's tone table,
// white balance state and scratch kept in a handle.

#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "cpu_pipeline.hpp"
#include "holoscan/isp/isp_params.hpp"
#ifdef ISP_REF_CUDA
#include <cuda_runtime_api.h>

#include "holoscan/isp/isp_pipeline.hpp"
#endif
#include "holoscan/isp/synthetic_raw.hpp"
#include "isp_b200.h"

namespace isp = holoscan::isp;

namespace {

thread_local std::string g_error;

isp::IspParams to_params(const isp_params_c& c) {
  isp::IspParams p;
  p.black_level = c.black_level;
  if (c.has_channel_black_levels) {
    p.channel_black_levels = std::array<float, 4>{c.channel_black_levels[0], c.channel_black_levels[1],
                                                  c.channel_black_levels[2], c.channel_black_levels[3]};
  }
  p.white_level = c.white_level;
  if (c.has_lens_shading) {
    isp::LensShading s;
    s.width = c.lsc_width;
    s.height = c.lsc_height;
    s.channels = c.lsc_channels;
    if (c.lsc_gains != nullptr) s.gains.assign(c.lsc_gains, c.lsc_gains + c.lsc_gains_count);
    p.lens_shading = std::move(s);
  }
  p.white_balance = static_cast<isp::WhiteBalanceMode>(c.white_balance);
  for (int k = 0; k < 3; ++k) p.wb_gains[k] = c.wb_gains[k];
  p.awb_smoothing = c.awb_smoothing;
  p.white_patch_percentile = c.white_patch_percentile;
  p.demosaic = static_cast<isp::DemosaicMethod>(c.demosaic);
  for (int k = 0; k < 9; ++k) p.ccm[k] = c.ccm[k];
  p.tone_curve = static_cast<isp::ToneCurve>(c.tone_curve);
  p.gamma = c.gamma;
  if (c.lut != nullptr) p.lut.assign(c.lut, c.lut + c.lut_size);
  p.sharpen = c.sharpen;
  p.auto_exposure.target = c.auto_exposure.target;
  p.auto_exposure.damping = c.auto_exposure.damping;
  p.auto_exposure.min_exposure_ns = c.auto_exposure.min_exposure_ns;
  p.auto_exposure.max_exposure_ns = c.auto_exposure.max_exposure_ns;
  p.auto_exposure.min_gain = c.auto_exposure.min_gain;
  p.auto_exposure.max_gain = c.auto_exposure.max_gain;
  return p;
}

isp::RawImageView to_raw(const isp_raw_view_c& r) {
  return isp::RawImageView{r.data,
                           r.width,
                           r.height,
                           r.pitch,
                           static_cast<isp::RawFormat>(r.format),
                           r.bit_depth,
                           static_cast<isp::BayerPattern>(r.pattern)};
}

struct RefPipeline {
  isp::IspParams params;
  std::vector<float> lut;
  isp::detail::AwbState awb{};
  isp::detail::CpuScratch scratch;
};

// The synthetic camera's settings (synthetic_raw.hpp:40-59), as plain C.
struct ref_synthetic_config {
  int32_t width, height, pattern, format, bit_depth;
  float black_levels[4];
  float wb_gains[3];
  float ccm[9];
  float vignetting;
  int32_t kind;
  float exposure;
  uint32_t frame;
};

isp::SyntheticRawConfig to_config(const ref_synthetic_config& c) {
  isp::SyntheticRawConfig s;
  s.width = c.width;
  s.height = c.height;
  s.pattern = static_cast<isp::BayerPattern>(c.pattern);
  s.format = static_cast<isp::RawFormat>(c.format);
  s.bit_depth = c.bit_depth;
  for (int k = 0; k < 4; ++k) s.black_levels[k] = c.black_levels[k];
  for (int k = 0; k < 3; ++k) s.wb_gains[k] = c.wb_gains[k];
  for (int k = 0; k < 9; ++k) s.ccm[k] = c.ccm[k];
  s.vignetting = c.vignetting;
  s.kind = static_cast<isp::SceneKind>(c.kind);
  s.exposure = c.exposure;
  s.frame = c.frame;
  return s;
}

template <typename F>
int guarded(F&& body) {
  try {
    body();
    g_error.clear();
    return ISP_OK;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return ISP_EINVAL;
  } catch (const std::exception& e) {
    g_error = e.what();
    return ISP_ESTATE;
  }
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

size_t ref_raw_row_bytes(int32_t format, int32_t width) {
  return isp::raw_row_bytes(static_cast<isp::RawFormat>(format), width);
}

int ref_validate_params(const isp_params_c* params) {
  return guarded([&] { isp::validate_params(to_params(*params)); });
}

int ref_validate_raw(const isp_raw_view_c* raw, const isp_params_c* params) {
  return guarded([&] { isp::validate_raw(to_raw(*raw), to_params(*params)); });
}

size_t ref_tone_lut(const isp_params_c* params, float* out, size_t cap) {
  const std::vector<float> lut = isp::tone_lut(to_params(*params));
  for (size_t i = 0; i < lut.size() && i < cap; ++i) out[i] = lut[i];
  return lut.size();
}

void* ref_pipeline_create(const isp_params_c* params) {
  RefPipeline* p = nullptr;
  const int status = guarded([&] {
    isp::IspParams ip = to_params(*params);
    isp::validate_params(ip);
    p = new RefPipeline;
    p->lut = isp::tone_lut(ip);
    p->awb = isp::detail::initial_white_balance(ip);
    p->params = std::move(ip);
  });
  return status == ISP_OK ? p : nullptr;
}

void ref_pipeline_destroy(void* handle) { delete static_cast<RefPipeline*>(handle); }

void ref_pipeline_reset(void* handle) {
  auto* p = static_cast<RefPipeline*>(handle);
  p->awb = isp::detail::initial_white_balance(p->params);
}

void ref_pipeline_awb(void* handle, float gains[3], int32_t* valid) {
  auto* p = static_cast<RefPipeline*>(handle);
  for (int k = 0; k < 3; ++k) gains[k] = p->awb.gains[k];
  *valid = p->awb.valid;
}

int ref_pipeline_process(void* handle, const isp_raw_view_c* raw, const isp_rgb_view_c* out,
                         const isp_stats_c* stats, const isp_exposure_c* exposure) {
  auto* p = static_cast<RefPipeline*>(handle);
  return guarded([&] {
    const isp::RawImageView view = to_raw(*raw);
    isp::validate_raw(view, p->params);
    const isp::RgbImageView rgb{out->data, out->pitch, static_cast<isp::OutputFormat>(out->format)};
    if (rgb.data == nullptr) throw std::invalid_argument("output image has no data");
    const std::size_t row = static_cast<std::size_t>(view.width) * isp::output_channels(rgb.format) *
                            isp::output_channel_bytes(rgb.format);
    if (rgb.pitch < row ||
        rgb.pitch % static_cast<std::size_t>(isp::output_channel_bytes(rgb.format))) {
      throw std::invalid_argument("output image pitch is shorter than a row or misaligned");
    }
    const isp::detail::FrameParams fp = isp::detail::make_frame_params(
        p->params, view, rgb, p->lut.data(), static_cast<int>(p->lut.size()),
        p->params.lens_shading ? p->params.lens_shading->gains.data() : nullptr);
    isp::StatsOutput so{};
    if (stats != nullptr) so = isp::StatsOutput{stats->histogram, stats->stats};
    isp::FrameExposure fe{};
    if (exposure != nullptr) fe = isp::FrameExposure{exposure->exposure_ns, exposure->gain};
    isp::detail::cpu_process(fp, p->params, so, fe, p->awb, p->scratch);
  });
}

// The white balance sums of one frame from the reference's per-quad function
// (isp_math.hpp:311-332), summed as cpu_process sums them (cpu_pipeline.cpp:101-119).
int ref_awb_stats(const isp_params_c* params, const isp_raw_view_c* raw, uint64_t sum[3],
                  uint64_t* quads, uint32_t* hist /* [3][1024] */) {
  return guarded([&] {
    const isp::IspParams ip = to_params(*params);
    const isp::RawImageView view = to_raw(*raw);
    const isp::detail::FrameParams p = isp::detail::make_frame_params(
        ip, view, isp::RgbImageView{}, nullptr, 0,
        ip.lens_shading ? ip.lens_shading->gains.data() : nullptr);
    for (int k = 0; k < 3; ++k) sum[k] = 0;
    *quads = 0;
    std::memset(hist, 0, sizeof(uint32_t) * 3 * isp::detail::kAwbBins);
    for (int qy = 0; qy < p.height / 2; ++qy) {
      for (int qx = 0; qx < p.width / 2; ++qx) {
        int color[4];
        unsigned int fixed[4];
        int bin[4];
        if (!isp::detail::white_balance_quad(p, qx, qy, color, fixed, bin)) continue;
        for (int k = 0; k < 4; ++k) {
          sum[color[k]] += fixed[k];
          ++hist[color[k] * isp::detail::kAwbBins + bin[k]];
        }
        ++*quads;
      }
    }
  });
}

// The reference's synthetic camera (synthetic_raw.hpp, synthetic_raw.cpp).
int ref_render_synthetic(const ref_synthetic_config* config, void* data, size_t pitch) {
  return guarded([&] { isp::render_synthetic_raw(isp::make_synthetic_scene(to_config(*config)), data, pitch); });
}

// synthetic_isp_params (synthetic_raw.cpp:102-133) flattened: the scalar
// settings into *out, the lens shading gains into lsc (capacity cap); out's
// lsc_gains pointer is set to lsc.
int ref_synthetic_params(const ref_synthetic_config* config, int grid, isp_params_c* out, float* lsc,
                         size_t cap) {
  return guarded([&] {
    const isp::IspParams p = isp::synthetic_isp_params(to_config(*config), grid);
    std::memset(out, 0, sizeof *out);
    out->black_level = p.black_level;
    out->has_channel_black_levels = p.channel_black_levels.has_value();
    if (p.channel_black_levels) {
      for (int k = 0; k < 4; ++k) out->channel_black_levels[k] = (*p.channel_black_levels)[k];
    }
    out->white_level = p.white_level;
    out->has_lens_shading = p.lens_shading.has_value();
    if (p.lens_shading) {
      const isp::LensShading& s = *p.lens_shading;
      if (s.gains.size() > cap) throw std::invalid_argument("lens shading buffer too small");
      out->lsc_width = s.width;
      out->lsc_height = s.height;
      out->lsc_channels = s.channels;
      std::memcpy(lsc, s.gains.data(), s.gains.size() * sizeof(float));
      out->lsc_gains = lsc;
      out->lsc_gains_count = s.gains.size();
    }
    out->white_balance = static_cast<int32_t>(p.white_balance);
    for (int k = 0; k < 3; ++k) out->wb_gains[k] = p.wb_gains[k];
    out->awb_smoothing = p.awb_smoothing;
    out->white_patch_percentile = p.white_patch_percentile;
    out->demosaic = static_cast<int32_t>(p.demosaic);
    for (int k = 0; k < 9; ++k) out->ccm[k] = p.ccm[k];
    out->tone_curve = static_cast<int32_t>(p.tone_curve);
    out->gamma = p.gamma;
    out->sharpen = p.sharpen;
    out->auto_exposure.target = p.auto_exposure.target;
    out->auto_exposure.damping = p.auto_exposure.damping;
    out->auto_exposure.min_exposure_ns = p.auto_exposure.min_exposure_ns;
    out->auto_exposure.max_exposure_ns = p.auto_exposure.max_exposure_ns;
    out->auto_exposure.min_gain = p.auto_exposure.min_gain;
    out->auto_exposure.max_gain = p.auto_exposure.max_gain;
  });
}


#ifdef ISP_REF_CUDA
// The reference's own CUDA backend, IspPipeline(Backend::kCuda)
// (modules/isp/src/isp_pipeline.cpp, cuda_pipeline.cu), built for sm_100a
// into oracle/_ref/libisp_ref_cuda.so: the GPU bar the B200 build is timed
// against. Device buffers; frames queued on `stream`.
__attribute__((visibility("default"))) void* ref_cuda_pipeline_create(const isp_params_c* params) {
  void* handle = nullptr;
  const int status = guarded([&] { handle = new isp::IspPipeline(isp::Backend::kCuda, to_params(*params)); });
  return status == 0 ? handle : nullptr;
}

__attribute__((visibility("default"))) void ref_cuda_pipeline_destroy(void* handle) {
  delete static_cast<isp::IspPipeline*>(handle);
}

__attribute__((visibility("default"))) int ref_cuda_pipeline_process(void* handle, const isp_raw_view_c* raw,
                                                                    const isp_rgb_view_c* out, const isp_stats_c* stats,
                                                                    const isp_exposure_c* exposure, void* stream) {
  auto* p = static_cast<isp::IspPipeline*>(handle);
  return guarded([&] {
    const isp::RgbImageView rgb{out->data, out->pitch, static_cast<isp::OutputFormat>(out->format)};
    isp::StatsOutput so{};
    if (stats != nullptr) so = isp::StatsOutput{stats->histogram, stats->stats};
    isp::FrameExposure fe{};
    if (exposure != nullptr) fe = isp::FrameExposure{exposure->exposure_ns, exposure->gain};
    p->process(to_raw(*raw), rgb, so, fe, static_cast<cudaStream_t>(stream));
  });
}
#endif

}  // extern "C"
