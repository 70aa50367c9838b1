// isp_host.hpp - host-side pieces shared by the C ABI's translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "isp_b200.h"
#include "isp_types.cuh"

namespace isp_b200 {

void params_default(isp_params_c* p);
// nullptr when valid, else the message of the first unusable field.
const char* validate_params(const isp_params_c& p);
size_t raw_row_bytes(int32_t format, int32_t width);
float white_level_of(const isp_params_c& p, int bit_depth);
// Empty when usable, else the message.
std::string validate_raw(const isp_raw_view_c& raw, const isp_params_c& p);
std::string validate_out(const isp_raw_view_c& raw, const isp_rgb_view_c& out);
std::vector<float> tone_lut(const isp_params_c& p);
// tone_lut into `out` (room for the user table's size, or ISP_TONE_LUT_SIZE);
// returns the entry count. Allocates nothing.
size_t tone_table(const isp_params_c& p, float* out);

// Thread-local error reporting behind isp_b200_last_error().
int fail(int status, const std::string& message);
int fail_cuda(cudaError_t error, const char* what);
void clear_error();

// A deep copy of isp_params_c: its borrowed arrays owned.
struct OwnedParams {
  isp_params_c c{};
  std::vector<float> lsc;
  std::vector<float> lut;
  void assign(const isp_params_c& p) {
    c = p;
    lsc.assign(p.has_lens_shading && p.lsc_gains ? p.lsc_gains : nullptr,
               p.has_lens_shading && p.lsc_gains ? p.lsc_gains + p.lsc_gains_count : nullptr);
    lut.assign(p.lut ? p.lut : nullptr, p.lut ? p.lut + p.lut_size : nullptr);
    c.lsc_gains = lsc.empty() ? nullptr : lsc.data();
    c.lut = lut.empty() ? nullptr : lut.data();
  }
};

// The per-camera resident state on the device: the tone table as
// (value, next - value) pairs, the lens shading grid, and the scratch
// accumulators with the white balance state.
struct DeviceState {
  float2* tone = nullptr;
  int tone_size = 0;
  float tone_last = 0.0F;
  float* lsc = nullptr;
  Scratch* scratch = nullptr;
};

// Builds `state` on the current device from validated params.
cudaError_t device_state_create(const isp_params_c& p, DeviceState* state);
void device_state_free(DeviceState* state);
// The initial white balance state (cpu_pipeline.cpp:90-95) written on `stream`.
cudaError_t device_state_reset_awb(const isp_params_c& p, DeviceState* state, cudaStream_t stream);

// The FrameDesc of a frame (make_frame_params, cpu_pipeline.cpp:50-88).
FrameDesc make_desc(const isp_params_c& p, const DeviceState& state, const isp_raw_view_c& raw,
                    const isp_rgb_view_c& out, const isp_stats_c* stats, const isp_exposure_c* exposure);

// Launch shapes, per device, cached.
struct LaunchShapes {
  int sm_count = 0;
  std::set<const void*> configured;                         // kernels whose smem attribute is set
  std::map<std::pair<const void*, size_t>, int> occupancy;  // (kernel, dynamic smem) -> CTAs per SM
};

// CTAs per SM of `kernel` at `smem` bytes of dynamic shared memory; on first
// use sets the kernel's limit to `smem_max`. Thread-safe.
cudaError_t blocks_per_sm(LaunchShapes& shapes, const void* kernel, size_t smem_max, size_t smem, int* blocks);

// Dynamic shared memory that still lets two CTAs of the fused kernel share an
// SM (228 KB per SM, 1 KB reserved per CTA, static shared memory).
constexpr size_t kSmemPerTwoCtas = 112U * 1024U;

// A 2-D TMA descriptor over the raw frame: bytes (uint16 samples for
// ISP_RAW_U16) across, rows down, boxes of box_row_bytes x box_rows. False
// (and a zeroed map) when the frame's base or pitch is not 16-byte aligned.
bool encode_raw_map(const FrameDesc& d, int box_row_bytes, int box_rows, CUtensorMap* map);

// The launch shapes of the current device (SM count, occupancy cache).
LaunchShapes& shapes_for_current_device(cudaError_t* error);

// Queues one frame's kernels on `stream` (no host synchronisation).
// before_main / after_main (may be null) are recorded around the fused tile kernel.
// `step` names the call that failed.
cudaError_t launch_frame(const FrameDesc& d, const isp_params_c& p, LaunchShapes& shapes, cudaStream_t stream,
                         cudaEvent_t before_main, cudaEvent_t after_main, const char** step, bool after_previous = false,
                         int tile_rows = 64);

}  // namespace isp_b200

// One camera's pipeline behind the C ABI (isp_b200_create).
struct isp_b200_pipeline {
  isp_b200::OwnedParams params;
  isp_b200::DeviceState state;
  int device = 0;
  cudaEvent_t done = nullptr;
  bool queued = false;
  cudaStream_t last_stream = nullptr;  // the stream of the last queued frame
  bool frame_overlap = true;           // isp_b200_set_frame_overlap
  int tile_rows = 0;                   // isp_b200_set_tile_rows: 0 = per shape (isp_b200_autotune), else 64 / 32
  struct ShapePick {
    int32_t format, width, height, rows;
  };
  ShapePick picks[8] = {};  // isp_b200_autotune's choices, oldest replaced first
  int npicks = 0;
  // The tile height for a frame: the forced one, the shape's pick, else 64.
  int rows_for(const isp_raw_view_c& raw) const {
    if (tile_rows != 0) return tile_rows;
    for (int i = 0; i < npicks && i < 8; ++i) {
      const ShapePick& k = picks[i];
      if (k.format == raw.format && k.width == raw.width && k.height == raw.height) return k.rows;
    }
    return 64;
  }
  // Staging for isp_b200_process_host, grown on demand.
  cudaStream_t host_stream = nullptr;
  void* d_raw = nullptr;
  size_t d_raw_cap = 0;
  void* d_out = nullptr;
  size_t d_out_cap = 0;
  void* d_stats = nullptr;  // histogram then statistics
  // Profiling events around the fused tile kernel (isp_b200_set_kernel_events).
  cudaEvent_t before_main = nullptr;
  cudaEvent_t after_main = nullptr;
};

