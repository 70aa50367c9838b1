// isp_types.cuh - the device-side descriptors of the B200 ISP.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "isp_checked.cuh"

namespace isp_b200 {

// Channels of the mosaic (isp_params.hpp:65-68) and sample/output formats.
enum : int { kChR = 0, kChGr = 1, kChGb = 2, kChB = 3 };
enum : int { kRawU8 = 0, kRawU16 = 1, kRawRaw10 = 2, kRawRaw12 = 3 };
enum : int { kOutRgb8 = 0, kOutRgba8 = 1, kOutRgb16 = 2, kOutRgb32f = 3 };
enum : int { kWbManual = 0, kWbGrayWorld = 1, kWbWhitePatch = 2 };

constexpr float kFixedOne = 1048576.0F;  // statistics' fixed point: 2^-20 units
constexpr int kAwbBins = 1024;           // white-patch histogram bins
constexpr int kAwbBandRows = 1024;       // most rows of one statistics band (16 tiles of 64)
constexpr int kHistBins = 256;
constexpr int kHistChannels = 4;
constexpr int kStatsSize = 12;

using u64 = unsigned long long;

// The accumulators a frame's kernels sum into, in device memory. Every field
// is zero between frames: the kernel that consumes them (the last CTA to
// finish) clears them, so a frame needs no memset.
struct Scratch {
  // White balance statistics (isp_math.hpp:64-68).
  u64 awb_sum[3];
  u64 awb_quads;
  unsigned int awb_hist[3][kAwbBins];
  unsigned int awb_done;  // tiles of the statistics pass flushed so far
  // The white balance state carried from frame to frame (isp_math.hpp:71-74).
  float awb_gains[3];
  int awb_valid;
  // Main pass sums (isp_math.hpp:77-80) and the output histogram.
  u64 sum[3];
  u64 saturated;
  unsigned int hist[kHistChannels * kHistBins];
  unsigned int main_done;  // tiles of the main pass flushed so far
  int error;  // a bounded wait in a kernel gave up (1)
  unsigned int tile_next;  // the single-frame tile pass's tiles claimed beyond the first one per CTA
  unsigned int pad;
#ifdef ISP_CHECKED
  CheckRecord check;  // out-of-bounds accesses refused by the checked build
#endif
};

struct AutoExposure {
  float target;
  float damping;
  int64_t min_exposure_ns;
  int64_t max_exposure_ns;
  float min_gain;
  float max_gain;
};

// Everything a frame's kernels read, passed by value (FrameParams of
// isp_math.hpp:35-60 plus this build's outputs and scratch).
struct FrameDesc {
  int width;
  int height;
  Span<const uint8_t> raw;
  int64_t raw_pitch;
  int raw_format;
  int pattern;
  int cfa[4];  // channel at quad position (y & 1) * 2 + (x & 1)
  float black[4];
  float inv_range[4];
  int white;
  float wb[3];
  int auto_wb;  // gains from scratch->awb_gains
  Span<const float> lsc;  // lens shading grid in device memory, or null
  int lsc_width;
  int lsc_height;
  int lsc_channels;
  float lsc_sx;
  float lsc_sy;
  float ccm[9];
  Span<const float2> tone;  // (lut[i], lut[i+1] - lut[i]) pairs in device memory
  int tone_size;
  float tone_last;
  float sharpen;
  Span<uint8_t> out;
  int64_t out_pitch;
  int out_format;
  int out_vector;  // out and out_pitch allow the kernels' vector stores
  Span<uint32_t> hist_out;  // user histogram [4][256], or null
  Span<float> stats_out;    // user statistics [12], or null
  Span<Scratch> scratch;
  AutoExposure ae;
  int64_t exposure_ns;
  float exposure_gain;
  int awb_mode;
  float awb_percentile;
  float awb_smoothing;
};

// One frame of a batch, in device memory: its TMA descriptors, its
// FrameDesc, and where its tiles sit in the two passes' work lists (items of
// a frame are consecutive; frames in order).
struct alignas(64) BatchFrame {
  CUtensorMap main_map;  // box of the tile pass, when use_tma
  CUtensorMap awb_map;   // box of the statistics pass, when use_tma
  FrameDesc desc;
  int tiles_x;       // tile pass: tiles across
  int tiles;         // tile pass: tiles of the frame
  int tile_begin;    // tile pass: first work item
  int awb_tiles_x;   // statistics pass: tiles across
  int awb_tiles;     // statistics pass: tiles (0: manual white balance)
  int awb_begin;     // statistics pass: first work item
  int variant;       // bit 0 Malvar, bit 1 sharpening, bit 2 GRBG/GBRG layout
  int use_tma;
};

}  // namespace isp_b200
