// isp_synth.cu - seeded synthetic raw frames rendered on the device
// (isp_b200_synthetic_raw, include/isp_b200.h).
//
// The benchmark workloads' scene: linear RGB in [0, 1] made of a base level
// plus a linear gradient, 8 Gaussian blobs (sigma 50..300 pixels) and 64
// axis-aligned rectangles of uniform colour painted in order, clipped to
// [0, 1], times a cos^4 vignette whose corner gain is `vignette_edge`; then
// mosaicked in the Bayer pattern, scaled to [black, 2^bits - 1], given
// Poisson shot noise (gain counts per electron) and Gaussian read noise,
// rounded, clipped and packed in the raw format. It plays the part of the
// reference module's synthetic camera (its render kernel) for the
// throughput workloads, which need fresh frames at rate. The scene's
// random choices come from the seed on the host; the noise from a
// counter-based hash of (seed, pixel) on the device, so a frame is a pure
// function of its seed and settings.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>

#include "isp_b200.h"
#include "isp_host.hpp"

namespace isp_b200 {
namespace {

constexpr int kBlobs = 8;
constexpr int kRects = 64;

struct SynthScene {
  float base[3];
  float gx[3];  // per pixel across
  float gy[3];  // per pixel down
  float blob_x[kBlobs], blob_y[kBlobs], blob_k[kBlobs];  // k = -1 / (2 sigma^2)
  float blob_amp[kBlobs][3];
  int rect[kRects][4];  // x0, y0, x1, y1 (exclusive)
  float rect_rgb[kRects][3];
  int channel_of[4];    // colour (0 R, 1 G, 2 B) at quad position (y & 1) * 2 + (x & 1)
  int width, height, format, white;
  float black, span;    // counts = black + sig * span
  float inv_gain, gain, read_noise;
  float cx, cy, inv_rc, tan_edge;
  unsigned long long seed;
};

// SplitMix64 (Steele, Lea and Flood 2014): a 64-bit counter mixed into a
// well-distributed 64-bit value.
__host__ __device__ inline unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Uniform in [0, 1) from the top 24 bits.
__host__ __device__ inline float unit(unsigned long long h) { return static_cast<float>(h >> 40) * 5.9604645e-8F; }

// The scene's random choices, drawn in a fixed order from the seed.
struct HostDraw {
  unsigned long long state;
  float uniform(float lo, float hi) {
    state = mix64(state);
    return lo + (hi - lo) * unit(state);
  }
};

__device__ inline float normal(unsigned long long key) {
  // Box-Muller on two uniforms of the key's hash; u1 in (0, 1].
  const unsigned long long h = mix64(key);
  const float u1 = 1.0F - unit(h);
  const float u2 = static_cast<float>(h & 0xFFFFFFULL) * 5.9604645e-8F;
  return sqrtf(-2.0F * logf(u1)) * cospif(2.0F * u2);
}

// Poisson(lambda): multiplication of uniforms below 16, else the normal
// approximation rounded to an integer (shot noise of bright pixels).
__device__ inline float poisson(float lambda, unsigned long long key) {
  if (!(lambda > 0.0F)) return 0.0F;
  if (lambda < 16.0F) {
    const float limit = expf(-lambda);
    float prod = 1.0F;
    int k = 0;
    unsigned long long h = key;
    for (; k < 64; ++k) {  // bounded: P(k >= 64 | lambda < 16) is below 1e-16
      h = mix64(h);
      prod *= unit(h);
      if (prod <= limit) break;
    }
    return static_cast<float>(k);
  }
  return fmaxf(0.0F, rintf(lambda + sqrtf(lambda) * normal(key)));
}

__device__ inline int sample(const SynthScene& s, int x, int y) {
  if (x >= s.width) return 0;  // packing padding
  const int c = s.channel_of[((y & 1) << 1) | (x & 1)];
  const float fx = static_cast<float>(x);
  const float fy = static_cast<float>(y);
  float v = s.base[c] + s.gx[c] * fx + s.gy[c] * fy;
#pragma unroll
  for (int b = 0; b < kBlobs; ++b) {
    const float dx = fx - s.blob_x[b];
    const float dy = fy - s.blob_y[b];
    v += s.blob_amp[b][c] * expf((dx * dx + dy * dy) * s.blob_k[b]);
  }
  for (int r = kRects - 1; r >= 0; --r) {  // the last painted rectangle covering (x, y) wins
    if (x >= s.rect[r][0] && y >= s.rect[r][1] && x < s.rect[r][2] && y < s.rect[r][3]) {
      v = s.rect_rgb[r][c];
      break;
    }
  }
  v = fminf(fmaxf(v, 0.0F), 1.0F);
  // cos^4(atan(r tan(theta_edge))) = 1 / (1 + (r tan(theta_edge))^2)^2.
  const float dxc = (fx - s.cx) * s.inv_rc;
  const float dyc = (fy - s.cy) * s.inv_rc;
  const float u2 = (dxc * dxc + dyc * dyc) * s.tan_edge * s.tan_edge;
  const float vig = 1.0F / ((1.0F + u2) * (1.0F + u2));
  float dn = v * vig * s.span;
  const unsigned long long key = s.seed ^ (static_cast<unsigned long long>(y) << 32 | static_cast<unsigned int>(x));
  if (s.gain > 0.0F) dn = poisson(dn * s.inv_gain, mix64(key)) * s.gain;
  if (s.read_noise > 0.0F) dn += s.read_noise * normal(mix64(key ^ 0x5EED5EEDULL));
  const float counts = rintf(s.black + dn);
  return static_cast<int>(fminf(fmaxf(counts, 0.0F), static_cast<float>(s.white)));
}

// One packing group per thread: 4 samples (u8, RAW10) or 2 (u16, RAW12).
__global__ void isp_synth_kernel(const __grid_constant__ SynthScene s, uint8_t* raw, size_t pitch, int groups) {
  const int g = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = static_cast<int>(blockIdx.y);
  if (g >= groups) return;
  uint8_t* row = raw + static_cast<size_t>(y) * pitch;
  switch (s.format) {
    case ISP_RAW_U8:
      for (int k = 0; k < 4; ++k) {
        const int x = 4 * g + k;
        if (x < s.width) row[x] = static_cast<uint8_t>(sample(s, x, y));
      }
      break;
    case ISP_RAW_U16:
      for (int k = 0; k < 2; ++k) {
        const int x = 2 * g + k;
        if (x < s.width) {
          const int v = sample(s, x, y);
          row[2 * x] = static_cast<uint8_t>(v & 0xFF);
          row[2 * x + 1] = static_cast<uint8_t>(v >> 8);
        }
      }
      break;
    case ISP_RAW_RAW10: {
      int v[4];
      for (int k = 0; k < 4; ++k) v[k] = sample(s, 4 * g + k, y);
      uint8_t* o = row + 5 * g;
      for (int k = 0; k < 4; ++k) o[k] = static_cast<uint8_t>(v[k] >> 2);
      o[4] = static_cast<uint8_t>((v[0] & 3) | ((v[1] & 3) << 2) | ((v[2] & 3) << 4) | ((v[3] & 3) << 6));
      break;
    }
    default: {
      const int a = sample(s, 2 * g, y);
      const int b = sample(s, 2 * g + 1, y);
      uint8_t* o = row + 3 * g;
      o[0] = static_cast<uint8_t>(a >> 4);
      o[1] = static_cast<uint8_t>(b >> 4);
      o[2] = static_cast<uint8_t>((a & 15) | ((b & 15) << 4));
      break;
    }
  }
}

}  // namespace
}  // namespace isp_b200

using namespace isp_b200;

extern "C" void isp_b200_synth_default(isp_synth_c* c) {
  if (c == nullptr) return;
  *c = isp_synth_c{};
  c->width = 1920;
  c->height = 1080;
  c->format = ISP_RAW_U16;
  c->bit_depth = 12;
  c->pattern = ISP_BAYER_RGGB;
  c->black = 256.0F;
  c->gain = 0.5F;
  c->read_noise = 3.0F;
  c->vignette_edge = 0.5F;
}

extern "C" int isp_b200_synthetic_raw(const isp_synth_c* cfg, uint64_t seed, void* raw, size_t pitch, void* stream) {
  if (cfg == nullptr || raw == nullptr) return fail(ISP_EINVAL, "synthetic frame: config or raw is null");
  isp_params_c probe_params{};
  isp_b200_params_default(&probe_params);
  probe_params.black_level = 0.0F;
  const isp_raw_view_c view{raw, cfg->width, cfg->height, pitch, cfg->format, cfg->bit_depth, cfg->pattern};
  if (const std::string why = validate_raw(view, probe_params); !why.empty()) return fail(ISP_EINVAL, why);
  const int white = (1 << cfg->bit_depth) - 1;
  if (!(cfg->black >= 0.0F && cfg->black < static_cast<float>(white)) || !(cfg->gain >= 0.0F) ||
      !(cfg->read_noise >= 0.0F) || !(cfg->vignette_edge > 0.0F && cfg->vignette_edge <= 1.0F)) {
    return fail(ISP_EINVAL, "synthetic frame: black in [0, white), gain and read noise >= 0, vignette edge in (0, 1]");
  }
  SynthScene s{};
  HostDraw d{seed};
  const float w = static_cast<float>(cfg->width), h = static_cast<float>(cfg->height);
  for (int c = 0; c < 3; ++c) s.base[c] = d.uniform(0.05F, 0.35F);
  for (int c = 0; c < 3; ++c) s.gx[c] = d.uniform(-0.25F, 0.25F) / std::fmax(w - 1.0F, 1.0F);
  for (int c = 0; c < 3; ++c) s.gy[c] = d.uniform(-0.25F, 0.25F) / std::fmax(h - 1.0F, 1.0F);
  for (int b = 0; b < kBlobs; ++b) {
    s.blob_x[b] = d.uniform(0.0F, w);
    s.blob_y[b] = d.uniform(0.0F, h);
    const float sigma = d.uniform(50.0F, 300.0F);
    s.blob_k[b] = -1.0F / (2.0F * sigma * sigma);
    for (int c = 0; c < 3; ++c) s.blob_amp[b][c] = d.uniform(0.05F, 0.5F);
  }
  for (int r = 0; r < kRects; ++r) {
    const int rw = static_cast<int>(d.uniform(0.02F, 0.2F) * w) + 1;
    const int rh = static_cast<int>(d.uniform(0.02F, 0.2F) * h) + 1;
    const int x0 = static_cast<int>(d.uniform(0.0F, std::fmax(w - static_cast<float>(rw), 1.0F)));
    const int y0 = static_cast<int>(d.uniform(0.0F, std::fmax(h - static_cast<float>(rh), 1.0F)));
    s.rect[r][0] = x0;
    s.rect[r][1] = y0;
    s.rect[r][2] = x0 + rw;
    s.rect[r][3] = y0 + rh;
    for (int c = 0; c < 3; ++c) s.rect_rgb[r][c] = d.uniform(0.0F, 1.0F);
  }
  static constexpr int kColour[4][4] = {{0, 1, 1, 2}, {2, 1, 1, 0}, {1, 0, 2, 1}, {1, 2, 0, 1}};
  for (int q = 0; q < 4; ++q) s.channel_of[q] = kColour[cfg->pattern][q];
  s.width = cfg->width;
  s.height = cfg->height;
  s.format = cfg->format;
  s.white = white;
  s.black = cfg->black;
  s.span = static_cast<float>(white) - cfg->black;
  s.gain = cfg->gain;
  s.inv_gain = cfg->gain > 0.0F ? 1.0F / cfg->gain : 0.0F;
  s.read_noise = cfg->read_noise;
  s.cx = (w - 1.0F) / 2.0F;
  s.cy = (h - 1.0F) / 2.0F;
  const float rc = std::hypot(s.cx, s.cy);
  s.inv_rc = rc > 0.0F ? 1.0F / rc : 1.0F;
  // cos^4(theta_edge) = vignette_edge at the corners (r = 1).
  s.tan_edge = std::tan(std::acos(std::pow(cfg->vignette_edge, 0.25F)));
  s.seed = mix64(seed ^ 0xA5A5A5A5DEADBEEFULL);
  const int per_group = cfg->format == ISP_RAW_U8 || cfg->format == ISP_RAW_RAW10 ? 4 : 2;
  const int groups = (cfg->width + per_group - 1) / per_group;
  const dim3 grid(static_cast<unsigned int>((groups + 127) / 128), static_cast<unsigned int>(cfg->height));
  static_cast<void>(cudaGetLastError());
  isp_synth_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(s, static_cast<uint8_t*>(raw), pitch, groups);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_synthetic_raw");
  clear_error();
  return ISP_OK;
}
