// isp_noalloc.cu - one frame through the ISP without allocating any memory.
//
// Some callers cannot allocate device memory: code running where
// cudaMalloc is forbidden or unsafe (a real-time loop whose allocator must
// not be touched, a plugin host that owns every allocation).
// isp_b200_process_noalloc serves
// them: the caller passes the raw frame and the outputs (device memory it
// already owns), and everything the kernels need besides - the tone table,
// the lens shading grid, the statistics sums and the white balance state -
// lives in one file-scope device array of kNoAllocBytes, which every GPU that
// loads this library holds until the process exits.
//
// Host code cannot use that array's name as a device address (it is a host
// stand-in); the first call on each device, with that device current, takes
// the real address with cudaGetSymbolAddress, sets the kernels' shared-memory
// limits and keeps both for that device's context (a device reset makes a new
// context, and the next call sets up again). That first call should therefore
// come before any stream capture. Every call stages its tables from host
// memory that the next call reuses, so while its stream is capturing it
// refuses (ISP_EINVAL) and queues nothing. Every call writes its tables and
// clears its sums in the array on the caller's stream before its kernels, so
// consecutive calls on one stream are ordered and each sees only its own
// frame; calls that may overlap on the GPU (other streams, other threads)
// race on the shared array and must not be issued.
//
// The frame is processed as the first frame of a fresh pipeline: an auto
// white balance takes the frame's own estimate, unsmoothed. No cudaMalloc,
// cudaFree or other allocating routine is called, on the device or the host.
// isp_b200_noalloc_status reads (and clears) the array's flag that a bounded
// wait gave up, after the stream's work is done and before the next call,
// which clears it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "isp_b200.h"
#include "isp_host.hpp"
#include "isp_kernels.cuh"
#include "isp_trace.hpp"

namespace isp_b200 {
namespace {

// The array: scratch sums and state, then the tone table pairs, then the grid.
constexpr size_t kNoAllocBytes = 160U * 1024U;
constexpr size_t kScratchOffset = 0;
constexpr size_t kToneOffset = (sizeof(Scratch) + 255U) & ~size_t{255};
constexpr size_t kMaxToneEntries = 4097;
constexpr size_t kLscOffset = (kToneOffset + kMaxToneEntries * sizeof(float2) + 255U) & ~size_t{255};
constexpr size_t kMaxLscGains = (kNoAllocBytes - kLscOffset) / sizeof(float);
static_assert(kLscOffset < kNoAllocBytes, "no-alloc layout");
static_assert(kMaxLscGains >= 17 * 13 * 4, "a 17x13 four-channel grid fits");

static __device__ __align__(256) unsigned char g_noalloc[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
// Per device: the array's address in the context it was looked up in, that
// context's id (a device reset makes a new context, and the lookup is
// redone) and the SM count; the kernels' shared-memory limits are set then.
struct DeviceSetup {
  unsigned long long context = 0;
  unsigned char* address = nullptr;
  int sm_count = 0;
};
DeviceSetup g_setup[kMaxDevices];

// Host-side staging of the tables (no heap): filled under g_mutex, copied to
// the device before the lock is released (a copy from pageable memory
// returns once the bytes are staged).
float g_lut[kMaxToneEntries];
float2 g_pairs[kMaxToneEntries];

using CtxGetCurrent = CUresult (*)(CUcontext*);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long*);

void* driver_entry(const char* name) {
  void* f = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPoint(name, &f, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) {
    return nullptr;
  }
  return f;
}

// The id of the context current on this thread, 0 when there is none yet.
unsigned long long current_context_id() {
  static const auto get_current = reinterpret_cast<CtxGetCurrent>(driver_entry("cuCtxGetCurrent"));
  static const auto get_id = reinterpret_cast<CtxGetId>(driver_entry("cuCtxGetId"));
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current == nullptr || get_id == nullptr || get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr ||
      get_id(ctx, &id) != CUDA_SUCCESS) {
    return 0;
  }
  return id;
}

// Set-up on the current device: the array's device address (in host code its
// name is only a stand-in), the SM count and every kernel's shared-memory
// limit. Redone when the device's context changed since (after a reset).
cudaError_t noalloc_setup(DeviceSetup** out) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  DeviceSetup& d = g_setup[device];
  const unsigned long long ctx = current_context_id();
  if (d.address == nullptr || ctx == 0 || ctx != d.context) {
    void* address = nullptr;
    e = cudaGetSymbolAddress(&address, g_noalloc);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, device);
    for (int wp = 0; wp < 2 && e == cudaSuccess; ++wp) {
      for (int pattern = 0; pattern < 4 && e == cudaSuccess; ++pattern) {
        e = cudaFuncSetAttribute(awb_kernel(wp != 0, pattern), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(awb_kernel_smem()));
      }
    }
    for (int k = 0; k < 64 && e == cudaSuccess; ++k) {
      const bool malvar = (k & 1) != 0, sharpen = (k & 2) != 0, lut = (k & 8) != 0;
      const int pattern = (k & 4) != 0 ? 2 : 0;
      const int fmt = k >> 4;
      const size_t most = main_kernel_smem(sharpen, kRawU16, lut ? kLutSmemEntries : 0);
      e = cudaFuncSetAttribute(main_kernel(malvar, sharpen, pattern, lut, fmt),
                               cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(most));
    }
    if (e != cudaSuccess) return e;
    d.address = static_cast<unsigned char*>(address);
    d.context = current_context_id();
  }
  *out = &d;
  return cudaSuccess;
}

cudaError_t launch_noalloc(const FrameDesc& d, const isp_params_c& p, int sm_count, cudaStream_t stream) {
  const int threads = kernel_threads();
  if (d.auto_wb) {
    const bool white_patch = p.white_balance == ISP_WB_WHITE_PATCH;
    const void* k = awb_kernel(white_patch, d.pattern);
    const size_t smem = awb_kernel_smem();
    int bpsm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k, threads, smem);
    if (e != cudaSuccess) return e;
    alignas(64) CUtensorMap map;
    int use_tma = encode_raw_map(d, awb_box_row_bytes(d.raw_format), 64, &map) ? 1 : 0;
    int strips = 0, tiles_y = 0, band_tiles = 0;
    const int blocks = awb_kernel_bands(d.width, d.height, sm_count * std::max(bpsm, 1), &strips, &tiles_y,
                                        &band_tiles);
    FrameDesc desc = d;
    void* args[] = {&map, &desc, &strips, &tiles_y, &band_tiles, &use_tma};
    e = cudaLaunchKernel(k, dim3(blocks), dim3(threads), args, smem, stream);
    if (e != cudaSuccess) return e;
  }
  const bool sharpen = p.sharpen > 0.0F;
  const size_t with_lut = main_kernel_smem(sharpen, d.raw_format, d.tone_size);
  int lut_in_smem = d.tone_size <= kLutSmemEntries && with_lut <= kSmemPerTwoCtas ? 1 : 0;
  const size_t need = lut_in_smem ? with_lut : main_kernel_smem(sharpen, d.raw_format, 0);
  const void* k = main_kernel(p.demosaic == ISP_DEMOSAIC_MALVAR, sharpen, d.pattern, lut_in_smem != 0, d.out_format);
  int bpsm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k, threads, need);
  if (e != cudaSuccess) return e;
  alignas(64) CUtensorMap map;
  int use_tma = encode_raw_map(d, main_box_row_bytes(d.raw_format), main_box_rows(sharpen), &map) ? 1 : 0;
  int tiles_x = 0;
  int tiles = main_kernel_tiles(d.width, d.height, &tiles_x);
  const int blocks = std::max(1, std::min(tiles, sm_count * std::max(bpsm, 1)));
  FrameDesc desc = d;
  void* args[] = {&map, &desc, &tiles_x, &tiles, &use_tma, &lut_in_smem};
  return cudaLaunchKernel(k, dim3(blocks), dim3(threads), args, need, stream);
}

}  // namespace
}  // namespace isp_b200

using namespace isp_b200;

extern "C" int isp_b200_process_noalloc(const isp_params_c* params, const isp_raw_view_c* raw,
                                        const isp_rgb_view_c* out, const isp_stats_c* stats,
                                        const isp_exposure_c* exposure, void* stream_ptr) {
  if (params == nullptr || raw == nullptr || out == nullptr) return fail(ISP_EINVAL, "params, raw or out is null");
  const TraceRange range("isp.process_noalloc");
  if (const char* why = validate_params(*params)) return fail(ISP_EINVAL, why);
  if (params->tone_curve == ISP_TONE_LUT && params->lut_size > kMaxToneEntries) {
    return fail(ISP_EINVAL, "isp_b200_process_noalloc: a tone table holds at most 4097 entries here");
  }
  if (params->has_lens_shading && params->lsc_gains_count > kMaxLscGains) {
    return fail(ISP_EINVAL, "isp_b200_process_noalloc: the lens shading grid holds at most " +
                                std::to_string(kMaxLscGains) + " gains here");
  }
  if (const std::string why = validate_raw(*raw, *params); !why.empty()) return fail(ISP_EINVAL, why);
  if (const std::string why = validate_out(*raw, *out); !why.empty()) return fail(ISP_EINVAL, why);
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  // Every call stages its tables from host memory that the next call reuses:
  // a stream capture would record copies of memory that changes under it.
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(stream, &capturing);
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_process_noalloc: cudaStreamIsCapturing");
  if (capturing != cudaStreamCaptureStatusNone) {
    return fail(ISP_EINVAL, "isp_b200_process_noalloc: the stream is capturing; the call stages its tables from host "
                            "memory that the next call reuses, so it queues nothing while capturing");
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceSetup* setup = nullptr;
  e = noalloc_setup(&setup);
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_process_noalloc: set-up");
  unsigned char* base = setup->address;
  const int sm_count = setup->sm_count;
  // The tables, as isp_b200_create keeps them (isp_capi.cu device_state_create).
  const size_t n = tone_table(*params, g_lut);
  for (size_t i = 0; i + 1 < n; ++i) g_pairs[i] = make_float2(g_lut[i], g_lut[i + 1] - g_lut[i]);
  g_pairs[n - 1] = make_float2(g_lut[n - 1], 0.0F);
  DeviceState state;
  state.tone = reinterpret_cast<float2*>(base + kToneOffset);
  state.tone_size = static_cast<int>(n);
  state.tone_last = g_lut[n - 1];
  state.lsc = params->has_lens_shading ? reinterpret_cast<float*>(base + kLscOffset) : nullptr;
  state.scratch = reinterpret_cast<Scratch*>(base + kScratchOffset);
  // Sums start at zero; the white balance state is the configured gains, no estimate.
  struct {
    float gains[3];
    int valid;
  } init = {{params->wb_gains[0], params->wb_gains[1], params->wb_gains[2]}, 0};
  static_cast<void>(cudaGetLastError());
  e = cudaMemsetAsync(state.scratch, 0, sizeof(Scratch), stream);
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(&state.scratch->awb_gains[0], &init, sizeof(init), cudaMemcpyHostToDevice, stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(state.tone, g_pairs, n * sizeof(float2), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && state.lsc != nullptr) {
    e = cudaMemcpyAsync(state.lsc, params->lsc_gains, params->lsc_gains_count * sizeof(float), cudaMemcpyHostToDevice,
                        stream);
  }
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_process_noalloc: table upload");
  const FrameDesc d = make_desc(*params, state, *raw, *out, stats, exposure);
  e = launch_noalloc(d, *params, sm_count, stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_process_noalloc");
  clear_error();
  return ISP_OK;
}

extern "C" int isp_b200_noalloc_status(void* stream_ptr, int32_t* status) {
  if (status == nullptr) return fail(ISP_EINVAL, "status is null");
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceSetup* setup = nullptr;
  cudaError_t e = noalloc_setup(&setup);
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_noalloc_status: set-up");
  int* error = &reinterpret_cast<Scratch*>(setup->address + kScratchOffset)->error;
  int value = 0;
  const int zero = 0;
  e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess) e = cudaMemcpy(&value, error, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(error, &zero, sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_noalloc_status");
  *status = value;
  clear_error();
  return ISP_OK;
}
