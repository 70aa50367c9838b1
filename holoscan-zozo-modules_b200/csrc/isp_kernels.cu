// isp_kernels.cu - the sm_100a kernels of the B200 ISP, one frame at a time.
//
// A frame is one or two launches on the caller's stream:
//   isp_awb_kernel   (gray world / white patch only) the white balance
//                    statistics over complete 2x2 quads, block-privatised,
//                    then, in the last CTA to finish, the new estimate;
//   isp_main_kernel  persistent CTAs over 64x32-pixel tiles: the tile and
//                    its halo preprocessed into shared memory, demosaic,
//                    sharpen, colour matrix, tone curve, store, and the
//                    statistics sums and output histogram from registers;
//                    the last CTA writes the histogram and the statistics.
// The reference issues up to five kernels and three memsets per frame
// (modules/isp/src/cuda_pipeline.cu:294-364); the accumulators here clear
// themselves, so no memset is needed.
#include <cuda_runtime.h>

#include <cstdint>

#include "isp_device.cuh"
#include "isp_kernels.cuh"

namespace isp_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTileW = 64;
constexpr int kTileH = 32;

template <bool kSharpen>
struct Geom {
  // Sample halo: 2 covers the Malvar 5x5 (and the bilinear 3x3); with the
  // sharpening's extra ring of RGB, 4. Even, so the tile's samples keep the
  // mosaic's quad alignment.
  static constexpr int kHalo = kSharpen ? 4 : 2;
  static constexpr int kSW = kTileW + 2 * kHalo;
  static constexpr int kSH = kTileH + 2 * kHalo;
  static constexpr int kSamples = kSW * kSH;
  // RGB of the tile plus a one-pixel ring, origin (x0 - 1, y0 - 1), planar.
  static constexpr int kCW = kTileW + 2;
  static constexpr int kCH = kTileH + 2;
  static constexpr int kColors = kSharpen ? 3 * kCW * kCH : 0;
};

// Picks v[i] for a small runtime i without indexing a local array.
__device__ __forceinline__ float pick3(const float (&v)[3], int i) {
  return i == 0 ? v[0] : i == 1 ? v[1] : v[2];
}

__device__ __forceinline__ u64 warp_sum(u64 v) {
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) v += __shfl_down_sync(0xFFFFFFFFU, v, offset);
  return v;
}

// Sum of one u64 per thread over the block; the result in every thread.
__device__ u64 block_sum(u64 v, u64* red /* kWarps */) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  u64 total = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) total += red[w];
  return total;
}

// Exclusive prefix sum of one u64 per thread over the block.
__device__ u64 block_exclusive_scan(u64 v, u64* red /* kWarps */) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  u64 inc = v;
#pragma unroll
  for (int offset = 1; offset < 32; offset <<= 1) {
    const u64 up = __shfl_up_sync(0xFFFFFFFFU, inc, offset);
    if (lane >= offset) inc += up;
  }
  __syncthreads();
  if (lane == 31) red[warp] = inc;
  __syncthreads();
  u64 before = 0;
  for (int w = 0; w < warp; ++w) before += red[w];
  return before + inc - v;
}

// The value at `percentile` of a 1024-bin white-patch histogram, 0..1,
// interpolated within its bin; 0 for an empty histogram (isp_math.hpp:336-352).
// The whole block takes part: thread t owns bins 4t..4t+3; the prefix counts
// are exact integers, so the comparisons are the reference's.
__device__ float block_percentile(const unsigned int* hist, float percentile, u64* red, int* first) {
  const int t = threadIdx.x;
  unsigned int h[4];
  u64 mine = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    h[k] = __ldcg(hist + 4 * t + k);
    mine += h[k];
  }
  const u64 total = block_sum(mine, red);
  if (total == 0) return 0.0F;
  const u64 below0 = block_exclusive_scan(mine, red);
  const double target = static_cast<double>(percentile) * static_cast<double>(total);
  if (t == 0) *first = kAwbBins;
  __syncthreads();
  u64 below = below0;
  int mine_first = kAwbBins;
  u64 mine_below = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (mine_first == kAwbBins && h[k] != 0U && static_cast<double>(below + h[k]) >= target) {
      mine_first = 4 * t + k;
      mine_below = below;
    }
    below += h[k];
  }
  if (mine_first < kAwbBins) atomicMin(first, mine_first);
  __syncthreads();
  const int b = *first;
  __shared__ float result;
  if (b == kAwbBins) {
    if (t == 0) result = 1.0F;
  } else if (mine_first == b) {
    const double within = (target - static_cast<double>(mine_below)) / static_cast<double>(h[b & 3]);
    result = static_cast<float>((static_cast<double>(b) + within) / kAwbBins);
  }
  __syncthreads();
  const float r = result;
  __syncthreads();
  return r;
}

// ---- White balance statistics --------------------------------------------

template <bool kWhitePatch>
__global__ void __launch_bounds__(kThreads) isp_awb_kernel(FrameDesc p, const float* lsc) {
  __shared__ unsigned int hist[kWhitePatch ? 3 * kAwbBins : 1];
  __shared__ u64 red[kWarps];
  __shared__ int first;
  __shared__ bool last;
  Scratch* s = p.scratch;
  if constexpr (kWhitePatch) {
    for (int i = threadIdx.x; i < 3 * kAwbBins; i += kThreads) hist[i] = 0;
    __syncthreads();
  }
  const int quads_x = p.width / 2;
  const int64_t quads = static_cast<int64_t>(quads_x) * (p.height / 2);
  u64 acc[4] = {0, 0, 0, 0};
  for (int64_t i = blockIdx.x * static_cast<int64_t>(kThreads) + threadIdx.x; i < quads;
       i += static_cast<int64_t>(gridDim.x) * kThreads) {
    const int qy = static_cast<int>(i / quads_x);
    const int qx = static_cast<int>(i - static_cast<int64_t>(qy) * quads_x);
    int raw[4];
    bool saturated = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      raw[k] = load_raw(p, 2 * qx + (k & 1), 2 * qy + (k >> 1));
      saturated = saturated || raw[k] >= p.white;
    }
    if (saturated) continue;  // white_balance_quad, isp_math.hpp:311-319
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int x = 2 * qx + (k & 1);
      const int y = 2 * qy + (k >> 1);
      const int channel = p.cfa[k];
      float v = linearize(p, lsc, raw[k], x, y, channel);
      v = v < 4.0F ? v : 4.0F;
      const int color = color_of(channel);
      const unsigned int fixed = to_fixed(v);
      acc[0] += color == 0 ? fixed : 0U;
      acc[1] += color == 1 ? fixed : 0U;
      acc[2] += color == 2 ? fixed : 0U;
      if constexpr (kWhitePatch) {
        const int b = static_cast<int>(v * static_cast<float>(kAwbBins));
        atomicAdd(&hist[color * kAwbBins + (b < kAwbBins - 1 ? b : kAwbBins - 1)], 1U);
      }
    }
    acc[3] += 1;
  }
  // Flush: block sums, then one atomic per sum and per non-empty bin.
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const u64 total = block_sum(acc[k], red);
    if (threadIdx.x == 0 && total != 0) atomicAdd(k < 3 ? &s->awb_sum[k] : &s->awb_quads, total);
  }
  if constexpr (kWhitePatch) {
    for (int i = threadIdx.x; i < 3 * kAwbBins; i += kThreads) {
      if (hist[i] != 0U) atomicAdd(&s->awb_hist[0][0] + i, hist[i]);
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&s->awb_done, 1U) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();

  // finish_white_balance (isp_math.hpp:357-384), in the last CTA.
  const u64 nquads = __ldcg(&s->awb_quads);
  float level[3] = {0.0F, 0.0F, 0.0F};
  if (nquads != 0) {
    if (p.awb_mode == kWbGrayWorld) {
      const double q = static_cast<double>(nquads);
      level[0] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[0])) / q);
      level[1] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[1])) / (2.0 * q));
      level[2] = static_cast<float>(static_cast<double>(__ldcg(&s->awb_sum[2])) / q);
    } else {
      for (int k = 0; k < 3; ++k) level[k] = block_percentile(s->awb_hist[k], p.awb_percentile, red, &first);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && nquads != 0 && level[0] > 0.0F && level[1] > 0.0F && level[2] > 0.0F) {
    float target[3] = {level[1] / level[0], 1.0F, level[1] / level[2]};
    const bool smooth = s->awb_valid != 0 && p.awb_smoothing < 1.0F;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float t = target[k] < 0.0625F ? 0.0625F : target[k] > 16.0F ? 16.0F : target[k];
      const float g = s->awb_gains[k];
      s->awb_gains[k] = smooth ? g + p.awb_smoothing * (t - g) : t;
    }
    s->awb_valid = 1;
  }
  // Clear the sums for the next frame.
  for (int i = threadIdx.x; i < 3 * kAwbBins; i += kThreads) (&s->awb_hist[0][0])[i] = 0U;
  if (threadIdx.x < 3) s->awb_sum[threadIdx.x] = 0;
  if (threadIdx.x == 3) s->awb_quads = 0;
  if (threadIdx.x == 4) s->awb_done = 0;
}

// ---- The fused tile pass --------------------------------------------------

// finish_stats (isp_math.hpp:387-425) from the main pass's sums.
__device__ void finish_stats(const FrameDesc& p, const u64 sum[3], u64 saturated, const float gains[3]) {
  const int64_t pixels = static_cast<int64_t>(p.width) * p.height;
  const double n = static_cast<double>(pixels) * static_cast<double>(kFixedOne);
  const double mean[3] = {static_cast<double>(sum[0]) / n, static_cast<double>(sum[1]) / n,
                          static_cast<double>(sum[2]) / n};
  const double luma = 0.2126 * mean[0] + 0.7152 * mean[1] + 0.0722 * mean[2];
  double error = luma > 0.0 ? log2(static_cast<double>(p.ae.target) / luma) : 8.0;
  error = error < -8.0 ? -8.0 : error > 8.0 ? 8.0 : error;
  const double scale = exp2(static_cast<double>(p.ae.damping) * error);
  double next_exposure = 0.0;
  double next_gain = 0.0;
  if (p.exposure_ns > 0) {
    const double gain = p.exposure_gain > 0.0F ? p.exposure_gain : p.ae.min_gain;
    const double wanted = static_cast<double>(p.exposure_ns) * gain * scale;
    next_exposure = wanted / p.ae.min_gain;
    const double low = static_cast<double>(p.ae.min_exposure_ns);
    const double high = static_cast<double>(p.ae.max_exposure_ns);
    next_exposure = next_exposure < low ? low : next_exposure > high ? high : next_exposure;
    next_gain = wanted / next_exposure;
    next_gain = next_gain < p.ae.min_gain ? p.ae.min_gain : next_gain > p.ae.max_gain ? p.ae.max_gain : next_gain;
  }
  float* out = p.stats_out;
  out[0] = static_cast<float>(mean[0]);
  out[1] = static_cast<float>(mean[1]);
  out[2] = static_cast<float>(mean[2]);
  out[3] = static_cast<float>(luma);
  out[4] = static_cast<float>(error);
  out[5] = static_cast<float>(scale);
  out[6] = static_cast<float>(next_exposure);
  out[7] = static_cast<float>(next_gain);
  out[8] = gains[0];
  out[9] = gains[1];
  out[10] = gains[2];
  out[11] = static_cast<float>(static_cast<double>(saturated) / static_cast<double>(pixels));
}

// The 8-bit code of a toned value as the output stores it (isp_math.hpp:250-301),
// and the stored value itself.
template <int kOut>
__device__ __forceinline__ int code_of(float t) {
  if constexpr (kOut == kOutRgb8 || kOut == kOutRgba8) {
    return static_cast<unsigned char>(t * 255.0F + 0.5F);
  } else if constexpr (kOut == kOutRgb16) {
    const unsigned int v = static_cast<uint16_t>(t * 65535.0F + 0.5F);
    return static_cast<int>((v * 255U + 32767U) / 65535U);
  } else {
    return static_cast<int>(clamp01(t) * 255.0F + 0.5F);
  }
}

template <int kOut>
__device__ __forceinline__ void store_pixel(const FrameDesc& p, int x, int y, const float t[3]) {
  uint8_t* row = p.out + static_cast<int64_t>(y) * p.out_pitch;
  if constexpr (kOut == kOutRgb8) {
#pragma unroll
    for (int k = 0; k < 3; ++k) row[3 * x + k] = static_cast<unsigned char>(t[k] * 255.0F + 0.5F);
  } else if constexpr (kOut == kOutRgba8) {
    const unsigned int v = static_cast<unsigned char>(t[0] * 255.0F + 0.5F) |
                           (static_cast<unsigned int>(static_cast<unsigned char>(t[1] * 255.0F + 0.5F)) << 8) |
                           (static_cast<unsigned int>(static_cast<unsigned char>(t[2] * 255.0F + 0.5F)) << 16) |
                           0xFF000000U;
    if (p.out_vector) {
      *reinterpret_cast<unsigned int*>(row + 4 * x) = v;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) row[4 * x + k] = static_cast<unsigned char>(v >> (8 * k));
    }
  } else if constexpr (kOut == kOutRgb16) {
    uint16_t* r = reinterpret_cast<uint16_t*>(row);
#pragma unroll
    for (int k = 0; k < 3; ++k) r[3 * x + k] = static_cast<uint16_t>(t[k] * 65535.0F + 0.5F);
  } else {
    float* r = reinterpret_cast<float*>(row);
#pragma unroll
    for (int k = 0; k < 3; ++k) r[3 * x + k] = t[k];
  }
}

template <bool kMalvar, bool kSharpen, int kOut>
__global__ void __launch_bounds__(kThreads) isp_main_kernel(FrameDesc p, int tiles_x, int tiles) {
  using G = Geom<kSharpen>;
  extern __shared__ __align__(16) unsigned char smem[];
  float* S = reinterpret_cast<float*>(smem);          // preprocessed samples [kSH][kSW]
  float* Cc = S + G::kSamples;                        // RGB planes [3][kCH][kCW]
  unsigned int* hist = reinterpret_cast<unsigned int*>(Cc + G::kColors);  // [4][256]
  float2* lut_s = reinterpret_cast<float2*>(hist + kHistChannels * kHistBins);
  __shared__ u64 red[kWarps];
  __shared__ bool last;

  const int tid = threadIdx.x;
  Scratch* sc = p.scratch;
  const bool want_hist = p.hist_out != nullptr;
  const bool want_stats = p.stats_out != nullptr;
  float gains[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) gains[k] = p.auto_wb ? __ldcg(&sc->awb_gains[k]) : p.wb[k];
  // Per quad position: the channel, and its white balance gain.
  float qgain[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) qgain[k] = pick3(gains, color_of(p.cfa[k]));

  // The tone table in shared memory when it fits (the built-in tables and
  // tables up to 4097 entries); the lens shading grid is read through L1.
  const float2* lut = p.tone;
  if (p.tone_size <= kLutSmemEntries) {
    for (int i = tid; i < p.tone_size; i += kThreads) lut_s[i] = p.tone[i];
    lut = lut_s;
  }
  if (want_hist) {
    for (int i = tid; i < kHistChannels * kHistBins; i += kThreads) hist[i] = 0U;
  }
  __syncthreads();

  u64 acc[4] = {0, 0, 0, 0};  // linear R, G, B in 2^-20 units; saturated samples
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int ty = tile / tiles_x;
    const int x0 = (tile - ty * tiles_x) * kTileW;
    const int y0 = ty * kTileH;
    const bool interior = x0 >= G::kHalo && y0 >= G::kHalo && x0 + kTileW + G::kHalo <= p.width &&
                          y0 + kTileH + G::kHalo <= p.height;

    // 1. Samples of the tile and its halo, reflected at the image's edges,
    //    preprocessed once (cuda_pipeline.cu:39-45): pairs of horizontal
    //    neighbours, which share a row parity.
    constexpr int kPairsRow = G::kSW / 2;
    for (int i = tid; i < kPairsRow * G::kSH; i += kThreads) {
      const int r = i / kPairsRow;
      const int c2 = 2 * (i - r * kPairsRow);
      const int vy = y0 - G::kHalo + r;
      const int vx = x0 - G::kHalo + c2;
      int my = vy, mx0 = vx, mx1 = vx + 1;
      if (!interior) {
        my = mirror(vy, p.height);
        mx0 = mirror(vx, p.width);
        mx1 = mirror(vx + 1, p.width);
      }
      const int raw0 = load_raw(p, mx0, my);
      const int raw1 = load_raw(p, mx1, my);
      const int q = (vy & 1) << 1;
      const int ch0 = p.cfa[q];
      const int ch1 = p.cfa[q | 1];
      const float g0 = q ? qgain[2] : qgain[0];
      const float g1 = q ? qgain[3] : qgain[1];
      float v0 = linearize(p, p.lsc, raw0, mx0, my, ch0) * g0;
      float v1 = linearize(p, p.lsc, raw1, mx1, my, ch1) * g1;
      v0 = v0 < 1.0F ? v0 : 1.0F;
      v1 = v1 < 1.0F ? v1 : 1.0F;
      *reinterpret_cast<float2*>(S + r * G::kSW + c2) = make_float2(v0, v1);
      if (want_stats && r >= G::kHalo && r < G::kHalo + kTileH && c2 >= G::kHalo && c2 < G::kHalo + kTileW &&
          vy < p.height) {
        acc[3] += (vx < p.width && raw0 >= p.white ? 1U : 0U) + (vx + 1 < p.width && raw1 >= p.white ? 1U : 0U);
      }
    }
    __syncthreads();

    // 2. (Sharpening) RGB of the tile and a one-pixel ring, quad by quad.
    //    The ring's pixels outside the image are the reference's virtual
    //    pixels (cpu_pipeline.cpp:22-46): their neighbourhoods are reflected
    //    samples, as the tile holds them.
    if constexpr (kSharpen) {
      constexpr int kQW = (kTileW + 4) / 2;
      constexpr int kQH = (kTileH + 4) / 2;
      for (int i = tid; i < kQW * kQH; i += kThreads) {
        const int qy = i / kQW;
        const int qx = i - qy * kQW;
        // Window of 6x6 samples whose top-left is S[2qy][2qx]; the quad's
        // pixels sit at window (2..3, 2..3).
        float w[6][6];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
#pragma unroll
          for (int c = 0; c < 6; c += 2) {
            const float2 v = *reinterpret_cast<const float2*>(S + (2 * qy + r) * G::kSW + 2 * qx + c);
            w[r][c] = v.x;
            w[r][c + 1] = v.y;
          }
        }
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
          for (int dx = 0; dx < 2; ++dx) {
            const int cy = 2 * qy + dy - 1;
            const int cx = 2 * qx + dx - 1;
            float n[5][5];
#pragma unroll
            for (int a = 0; a < 5; ++a) {
#pragma unroll
              for (int b = 0; b < 5; ++b) n[a][b] = w[dy + a][dx + b];
            }
            float rgb[3];
            demosaic<kMalvar>(n, p.cfa[dy * 2 + dx], rgb);
            if (cy >= 0 && cy < G::kCH && cx >= 0 && cx < G::kCW) {
#pragma unroll
              for (int k = 0; k < 3; ++k) Cc[(k * G::kCH + cy) * G::kCW + cx] = rgb[k];
            }
          }
        }
      }
      __syncthreads();
    }

    // 3. Output quads: sharpen (or demosaic), colour matrix, tone, store,
    //    statistics sums and histogram codes from registers.
    constexpr int kQW = kTileW / 2;
    constexpr int kQH = kTileH / 2;
    for (int i = tid; i < kQW * kQH; i += kThreads) {
      const int qy = i / kQW;
      const int qx = i - qy * kQW;
      float rgb[2][2][3];
      if constexpr (kSharpen) {
        // 4x4 RGB window per channel, top-left C[2qy][2qx] (pixel x0+2qx-1).
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          float m[4][4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
#pragma unroll
            for (int c = 0; c < 4; c += 2) {
              const float2 v =
                  *reinterpret_cast<const float2*>(Cc + (k * G::kCH + 2 * qy + r) * G::kCW + 2 * qx + c);
              m[r][c] = v.x;
              m[r][c + 1] = v.y;
            }
          }
#pragma unroll
          for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
              rgb[dy][dx][k] = sharpen_one(m[dy + 1][dx + 1], m[dy][dx + 1], m[dy + 2][dx + 1], m[dy + 1][dx],
                                           m[dy + 1][dx + 2], m[dy][dx], m[dy][dx + 2], m[dy + 2][dx],
                                           m[dy + 2][dx + 2], p.sharpen);
            }
          }
        }
      } else {
        // 6x6 samples, top-left S[2qy][2qx] (halo 2): pixel (dy, dx) at (2+dy, 2+dx).
        float w[6][6];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
#pragma unroll
          for (int c = 0; c < 6; c += 2) {
            if (!kMalvar && (r == 0 || r == 5)) {
              w[r][c] = 0.0F;
              w[r][c + 1] = 0.0F;
              continue;
            }
            const float2 v = *reinterpret_cast<const float2*>(S + (2 * qy + r) * G::kSW + 2 * qx + c);
            w[r][c] = v.x;
            w[r][c + 1] = v.y;
          }
        }
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
          for (int dx = 0; dx < 2; ++dx) {
            float n[5][5];
#pragma unroll
            for (int a = 0; a < 5; ++a) {
#pragma unroll
              for (int b = 0; b < 5; ++b) n[a][b] = w[dy + a][dx + b];
            }
            demosaic<kMalvar>(n, p.cfa[dy * 2 + dx], rgb[dy][dx]);
          }
        }
      }
#pragma unroll
      for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) {
          const int x = x0 + 2 * qx + dx;
          const int y = y0 + 2 * qy + dy;
          if (x >= p.width || y >= p.height) continue;
          float linear[3];
          correct_color(p.ccm, rgb[dy][dx], linear);
          if (want_stats) {
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[k] += to_fixed(linear[k]);
          }
          float toned[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) toned[k] = tone(lut, p.tone_size, p.tone_last, linear[k]);
          store_pixel<kOut>(p, x, y, toned);
          if (want_hist) {
            const int r8 = code_of<kOut>(toned[0]);
            const int g8 = code_of<kOut>(toned[1]);
            const int b8 = code_of<kOut>(toned[2]);
            atomicAdd(&hist[luma_code(r8, g8, b8)], 1U);
            atomicAdd(&hist[kHistBins + r8], 1U);
            atomicAdd(&hist[2 * kHistBins + g8], 1U);
            atomicAdd(&hist[3 * kHistBins + b8], 1U);
          }
        }
      }
    }
    __syncthreads();  // the next tile overwrites S and C
  }

  if (!want_stats && !want_hist) return;
  if (want_stats) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const u64 total = block_sum(acc[k], red);
      if (tid == 0 && total != 0) atomicAdd(k < 3 ? &sc->sum[k] : &sc->saturated, total);
    }
  }
  if (want_hist) {
    __syncthreads();
    for (int i = tid; i < kHistChannels * kHistBins; i += kThreads) {
      if (hist[i] != 0U) atomicAdd(&sc->hist[i], hist[i]);
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(&sc->main_done, 1U) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (want_hist) {
    for (int i = tid; i < kHistChannels * kHistBins; i += kThreads) {
      p.hist_out[i] = __ldcg(&sc->hist[i]);
      sc->hist[i] = 0U;
    }
  }
  if (want_stats && tid == 0) {
    const u64 sum[3] = {__ldcg(&sc->sum[0]), __ldcg(&sc->sum[1]), __ldcg(&sc->sum[2])};
    finish_stats(p, sum, __ldcg(&sc->saturated), gains);
    sc->sum[0] = sc->sum[1] = sc->sum[2] = 0;
    sc->saturated = 0;
  }
  if (tid == 0) sc->main_done = 0;
}

template <bool kMalvar, bool kSharpen, int kOut>
const void* main_kernel_ptr() {
  return reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, kOut>);
}

template <bool kMalvar, bool kSharpen>
const void* main_kernel_by_out(int out) {
  switch (out) {
    case kOutRgb8: return main_kernel_ptr<kMalvar, kSharpen, kOutRgb8>();
    case kOutRgba8: return main_kernel_ptr<kMalvar, kSharpen, kOutRgba8>();
    case kOutRgb16: return main_kernel_ptr<kMalvar, kSharpen, kOutRgb16>();
    default: return main_kernel_ptr<kMalvar, kSharpen, kOutRgb32f>();
  }
}

}  // namespace

const void* main_kernel(bool malvar, bool sharpen, int out) {
  if (malvar) return sharpen ? main_kernel_by_out<true, true>(out) : main_kernel_by_out<true, false>(out);
  return sharpen ? main_kernel_by_out<false, true>(out) : main_kernel_by_out<false, false>(out);
}

size_t main_kernel_smem(bool sharpen, int tone_size) {
  const size_t samples = sharpen ? Geom<true>::kSamples : Geom<false>::kSamples;
  const size_t colors = sharpen ? Geom<true>::kColors : 0;
  const size_t lut = tone_size <= kLutSmemEntries ? static_cast<size_t>(tone_size) * sizeof(float2) : 0;
  return (samples + colors) * sizeof(float) + kHistChannels * kHistBins * sizeof(unsigned int) + lut;
}

int main_kernel_tiles(int width, int height, int* tiles_x) {
  *tiles_x = (width + kTileW - 1) / kTileW;
  return *tiles_x * ((height + kTileH - 1) / kTileH);
}

int kernel_threads() { return kThreads; }

const void* awb_kernel(bool white_patch) {
  return white_patch ? reinterpret_cast<const void*>(&isp_awb_kernel<true>)
                     : reinterpret_cast<const void*>(&isp_awb_kernel<false>);
}

}  // namespace isp_b200
