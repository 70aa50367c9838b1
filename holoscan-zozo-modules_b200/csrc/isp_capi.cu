// isp_capi.cu - the C ABI of the B200 ISP (include/isp_b200.h): one
// pipeline per camera, its resident device state, and frame submission.
//
// Mirrors holoscan::isp::IspPipeline with the CUDA backend
// (modules/isp/src/isp_pipeline.cpp:37-90, cuda_pipeline.cu:226-364): the
// same validation and errors, frames of one pipeline ordered on the GPU by an
// event even across streams, all work asynchronous on the caller's stream.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "isp_b200.h"
#include "isp_host.hpp"
#include "isp_kernels.cuh"
#include "isp_trace.hpp"

namespace isp_b200 {

namespace {

thread_local std::string t_error;
thread_local int t_cuda_error = 0;

// The channel at quad position (y & 1) * 2 + (x & 1) per pattern (cpu_pipeline.cpp:15-20).
constexpr int kCfa[4][4] = {
    {kChR, kChGr, kChGb, kChB},
    {kChB, kChGb, kChGr, kChR},
    {kChGr, kChR, kChB, kChGb},
    {kChGb, kChB, kChR, kChGr},
};

std::mutex g_shapes_mutex;
std::deque<LaunchShapes> g_shapes;  // per device; growing keeps references valid

}  // namespace

int fail(int status, const std::string& message) {
  t_error = message;
  t_cuda_error = 0;
  return status;
}

int fail_cuda(cudaError_t error, const char* what) {
  t_error = std::string(what) + ": " + cudaGetErrorString(error);
  t_cuda_error = static_cast<int>(error);
  return ISP_ECUDA;
}

void clear_error() {
  t_error.clear();
  t_cuda_error = 0;
}

namespace {

// Copies on a stream of their own, waited for: the caller's streams (blocking
// or not) neither wait for these nor are waited for (cuda_pipeline.cu:281-292).
struct PrivateStream {
  cudaStream_t s = nullptr;
  cudaError_t error = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  ~PrivateStream() {
    if (s != nullptr) cudaStreamDestroy(s);
  }
  cudaError_t copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    if (error == cudaSuccess) error = cudaMemcpyAsync(dst, src, bytes, kind, s);
    return error;
  }
  cudaError_t zero(void* dst, size_t bytes) {
    if (error == cudaSuccess) error = cudaMemsetAsync(dst, 0, bytes, s);
    return error;
  }
  cudaError_t finish() {
    if (error == cudaSuccess) error = cudaStreamSynchronize(s);
    return error;
  }
};

}  // namespace

cudaError_t device_state_create(const isp_params_c& p, DeviceState* s) {
  const std::vector<float> lut = tone_lut(p);
  const int n = static_cast<int>(lut.size());
  std::vector<float2> pairs(static_cast<size_t>(n));
  for (int i = 0; i + 1 < n; ++i) pairs[static_cast<size_t>(i)] = make_float2(lut[i], lut[i + 1] - lut[i]);
  pairs[static_cast<size_t>(n - 1)] = make_float2(lut[n - 1], 0.0F);
  s->tone_size = n;
  s->tone_last = lut[static_cast<size_t>(n - 1)];
  PrivateStream ps;
  cudaError_t e = ps.error;
  if (e == cudaSuccess) e = cudaMalloc(&s->tone, pairs.size() * sizeof(float2));
  if (e == cudaSuccess) e = ps.copy(s->tone, pairs.data(), pairs.size() * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && p.has_lens_shading) {
    e = cudaMalloc(&s->lsc, p.lsc_gains_count * sizeof(float));
    if (e == cudaSuccess) e = ps.copy(s->lsc, p.lsc_gains, p.lsc_gains_count * sizeof(float), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc(&s->scratch, sizeof(Scratch));
  if (e == cudaSuccess) e = ps.zero(s->scratch, sizeof(Scratch));
  if (e == cudaSuccess) e = ps.finish();
  if (e == cudaSuccess) e = device_state_reset_awb(p, s, nullptr);
  if (e != cudaSuccess) device_state_free(s);
  return e;
}

void device_state_free(DeviceState* s) {
  cudaFree(s->tone);
  cudaFree(s->lsc);
  cudaFree(s->scratch);
  *s = DeviceState{};
}

cudaError_t device_state_reset_awb(const isp_params_c& p, DeviceState* s, cudaStream_t stream) {
  struct {
    float gains[3];
    int valid;
  } init = {{p.wb_gains[0], p.wb_gains[1], p.wb_gains[2]}, 0};
  static_assert(sizeof(init) == sizeof(float) * 3 + sizeof(int), "AwbState layout");
  if (stream != nullptr) {
    const cudaError_t e = cudaMemcpyAsync(&s->scratch->awb_gains[0], &init, sizeof(init), cudaMemcpyHostToDevice, stream);
    return e == cudaSuccess ? cudaStreamSynchronize(stream) : e;
  }
  PrivateStream ps;
  ps.copy(&s->scratch->awb_gains[0], &init, sizeof(init), cudaMemcpyHostToDevice);
  return ps.finish();
}

FrameDesc make_desc(const isp_params_c& p, const DeviceState& s, const isp_raw_view_c& raw,
                    const isp_rgb_view_c& out, const isp_stats_c* stats, const isp_exposure_c* exposure) {
  FrameDesc d{};
  // Each buffer's extent, which the bounds-checked build holds its accesses
  // to (the regular build keeps plain pointers).
#ifdef ISP_CHECKED
  CheckRecord* rec = &s.scratch->check;
#else
  CheckRecord* rec = nullptr;
#endif
  const size_t rows_before_last = static_cast<size_t>(raw.height - 1);
  const size_t out_row = static_cast<size_t>(raw.width) * (out.format == ISP_OUT_RGBA8 ? 4U : 3U) *
                         (out.format == ISP_OUT_RGB16 ? 2U : out.format == ISP_OUT_RGB32F ? 4U : 1U);
  d.width = raw.width;
  d.height = raw.height;
  d.raw = make_span(static_cast<const uint8_t*>(raw.data),
                    raw.pitch * rows_before_last + raw_row_bytes(raw.format, raw.width), rec);
  d.raw_pitch = static_cast<int64_t>(raw.pitch);
  d.raw_format = raw.format;
  d.pattern = raw.pattern;
  for (int k = 0; k < 4; ++k) d.cfa[k] = kCfa[raw.pattern][k];
  const float white = white_level_of(p, raw.bit_depth);
  for (int k = 0; k < 4; ++k) {
    d.black[k] = p.has_channel_black_levels ? p.channel_black_levels[k] : p.black_level;
    d.inv_range[k] = 1.0F / (white - d.black[k]);
  }
  d.white = static_cast<int>(std::ceil(white));
  for (int k = 0; k < 3; ++k) d.wb[k] = p.wb_gains[k];
  d.auto_wb = p.white_balance != ISP_WB_MANUAL;
  if (p.has_lens_shading) {
    d.lsc = make_span(static_cast<const float*>(s.lsc),
                      static_cast<size_t>(p.lsc_width) * p.lsc_height * p.lsc_channels, rec);
    d.lsc_width = p.lsc_width;
    d.lsc_height = p.lsc_height;
    d.lsc_channels = p.lsc_channels;
    d.lsc_sx = static_cast<float>(p.lsc_width - 1) / static_cast<float>(raw.width - 1);
    d.lsc_sy = static_cast<float>(p.lsc_height - 1) / static_cast<float>(raw.height - 1);
  }
  for (int k = 0; k < 9; ++k) d.ccm[k] = p.ccm[k];
  d.tone = make_span(static_cast<const float2*>(s.tone), static_cast<size_t>(s.tone_size), rec);
  d.tone_size = s.tone_size;
  d.tone_last = s.tone_last;
  d.sharpen = p.sharpen;
  size_t out_bytes = out.pitch * rows_before_last + out_row;
#ifdef ISP_CHECKED
  // Test hook of the checked build: ISP_CHECKED_SHRINK_OUTPUT=n declares the
  // output n bytes shorter than it is, so that a frame's last stores are
  // refused and counted (they fall inside the real buffer either way).
  if (const char* shrink = std::getenv("ISP_CHECKED_SHRINK_OUTPUT")) {
    out_bytes -= std::min(out_bytes, static_cast<size_t>(std::strtoull(shrink, nullptr, 10)));
  }
#endif
  d.out = make_span(static_cast<uint8_t*>(out.data), out_bytes, rec);
  d.out_pitch = static_cast<int64_t>(out.pitch);
  d.out_format = out.format;
  d.out_vector = (reinterpret_cast<uintptr_t>(out.data) % 16U == 0U) && (out.pitch % 16U == 0U);
  d.hist_out = make_span(stats != nullptr ? stats->histogram : nullptr,
                         static_cast<size_t>(ISP_HISTOGRAM_CHANNELS) * ISP_HISTOGRAM_BINS, rec);
  d.stats_out = make_span(stats != nullptr ? stats->stats : nullptr, static_cast<size_t>(ISP_STATS_SIZE), rec);
  d.scratch = make_span(s.scratch, 1, rec);
  d.ae.target = p.auto_exposure.target;
  d.ae.damping = p.auto_exposure.damping;
  d.ae.min_exposure_ns = p.auto_exposure.min_exposure_ns;
  d.ae.max_exposure_ns = p.auto_exposure.max_exposure_ns;
  d.ae.min_gain = p.auto_exposure.min_gain;
  d.ae.max_gain = p.auto_exposure.max_gain;
  d.exposure_ns = exposure != nullptr ? exposure->exposure_ns : 0;
  d.exposure_gain = exposure != nullptr ? exposure->gain : 0.0F;
  d.awb_mode = p.white_balance;
  d.awb_percentile = p.white_patch_percentile;
  d.awb_smoothing = p.awb_smoothing;
  return d;
}

LaunchShapes& shapes_for_current_device(cudaError_t* error) {
  int device = 0;
  *error = cudaGetDevice(&device);
  std::lock_guard<std::mutex> lock(g_shapes_mutex);
  if (g_shapes.size() <= static_cast<size_t>(device)) g_shapes.resize(static_cast<size_t>(device) + 1);
  LaunchShapes& s = g_shapes[static_cast<size_t>(device)];
  if (s.sm_count == 0 && *error == cudaSuccess) {
    *error = cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, device);
  }
  return s;
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      f = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

}  // namespace

bool encode_raw_map(const FrameDesc& d, int box_row_bytes, int box_rows, CUtensorMap* map) {
  std::memset(map, 0, sizeof(*map));
  const auto base = reinterpret_cast<uintptr_t>(span_ptr(d.raw));
  if (base % 16U != 0U || d.raw_pitch % 16 != 0 || d.raw_pitch >= (int64_t{1} << 40)) return false;
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (encode == nullptr) return false;
  const bool u16 = d.raw_format == kRawU16;
  const cuuint64_t dims[2] = {u16 ? static_cast<cuuint64_t>(d.width) : raw_row_bytes(d.raw_format, d.width),
                              static_cast<cuuint64_t>(d.height)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(d.raw_pitch)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(u16 ? box_row_bytes / 2 : box_row_bytes),
                             static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = encode(map, u16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 2,
                            const_cast<uint8_t*>(span_ptr(d.raw)), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    std::memset(map, 0, sizeof(*map));
    return false;
  }
  return true;
}

cudaError_t blocks_per_sm(LaunchShapes& shapes, const void* kernel, size_t smem_max, size_t smem, int* blocks) {
  std::lock_guard<std::mutex> lock(g_shapes_mutex);
  if (shapes.configured.count(kernel) == 0) {
    const cudaError_t e =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_max));
    if (e != cudaSuccess) return e;
    shapes.configured.insert(kernel);
  }
  const auto key = std::make_pair(kernel, smem);
  auto it = shapes.occupancy.find(key);
  if (it == shapes.occupancy.end()) {
    int n = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kernel_threads(), smem);
    if (e != cudaSuccess) return e;
    it = shapes.occupancy.emplace(key, n > 0 ? n : 1).first;
  }
  *blocks = it->second;
  return cudaSuccess;
}

cudaError_t launch_frame(const FrameDesc& d, const isp_params_c& p, LaunchShapes& shapes, cudaStream_t stream,
                         cudaEvent_t before_main, cudaEvent_t after_main, const char** step, bool after_previous,
                         int tile_rows) {
  *step = "launch";
  const int threads = kernel_threads();
  const int pattern = d.pattern;
  if (d.auto_wb) {
    const bool white_patch = p.white_balance == ISP_WB_WHITE_PATCH;
    const void* k = awb_kernel(white_patch, pattern);
    const size_t smem = awb_kernel_smem();
    int bpsm = 0;
    *step = "white balance kernel attributes";
    const cudaError_t e = blocks_per_sm(shapes, k, smem, smem, &bpsm);
    if (e != cudaSuccess) return e;
    alignas(64) CUtensorMap map;
    int use_tma = encode_raw_map(d, awb_box_row_bytes(d.raw_format), 64, &map) ? 1 : 0;
    int strips = 0, tiles_y = 0, band_tiles = 0;
    const int blocks = awb_kernel_bands(d.width, d.height, shapes.sm_count * std::max(bpsm, 1), &strips, &tiles_y,
                                        &band_tiles);
    FrameDesc desc = d;
    void* args[] = {&map, &desc, &strips, &tiles_y, &band_tiles, &use_tma};
    *step = "white balance kernel launch";
    const TraceRange range("isp.statistics_pass", kTraceKernel);
    // With after_previous, as a programmatic dependent of the kernel queued
    // just before it (the previous frame's tile pass, when frames follow each
    // other on one stream): its CTAs sum this frame's raw samples on the SMs
    // that pass leaves as it finishes, and its estimate waits in the kernel
    // for that pass to complete. A kernel that does not signal its dependents
    // early (griddepcontrol.launch_dependents) is waited for in full, as is
    // any copy, event or other operation queued in between.
    cudaLaunchConfig_t acfg{};
    acfg.gridDim = dim3(blocks);
    acfg.blockDim = dim3(threads);
    acfg.dynamicSmemBytes = smem;
    acfg.stream = stream;
    cudaLaunchAttribute aattr[1];
    aattr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    aattr[0].val.programmaticStreamSerializationAllowed = 1;
    acfg.attrs = aattr;
    acfg.numAttrs = after_previous ? 1 : 0;
    const cudaError_t e2 = cudaLaunchKernelExC(&acfg, k, args);
    if (e2 != cudaSuccess) return e2;
  }
  const bool malvar = p.demosaic == ISP_DEMOSAIC_MALVAR;
  const bool sharpen = p.sharpen > 0.0F;
  // The tone table goes to shared memory when that still lets two CTAs share an SM.
  const size_t without_lut = main_kernel_smem(sharpen, d.raw_format, 0, tile_rows);
  const size_t with_lut = main_kernel_smem(sharpen, d.raw_format, d.tone_size, tile_rows);
  int lut_in_smem = d.tone_size <= kLutSmemEntries && with_lut <= kSmemPerTwoCtas ? 1 : 0;
  const size_t need = lut_in_smem ? with_lut : without_lut;
  const void* k = main_kernel(malvar, sharpen, pattern, lut_in_smem != 0, d.out_format, tile_rows);
  // The instance's attribute covers its largest footprint (uint16 boxes, a
  // full shared tone table), so frames of any format can share it.
  const size_t most = main_kernel_smem(sharpen, kRawU16, lut_in_smem ? kLutSmemEntries : 0, tile_rows);
  int bpsm = 0;
  *step = "tile kernel attributes";
  if (const cudaError_t e = blocks_per_sm(shapes, k, most, need, &bpsm); e != cudaSuccess) return e;
  alignas(64) CUtensorMap map;
  int use_tma = encode_raw_map(d, main_box_row_bytes(d.raw_format), main_box_rows(sharpen, tile_rows), &map) ? 1 : 0;
  int tiles_x = 0;
  int tiles = main_kernel_tiles(d.width, d.height, &tiles_x, tile_rows);
  const int blocks = std::min(tiles, shapes.sm_count * bpsm);
  FrameDesc desc = d;
  void* args[] = {&map, &desc, &tiles_x, &tiles, &use_tma, &lut_in_smem};
  if (before_main != nullptr) {
    const cudaError_t e = cudaEventRecord(before_main, stream);
    if (e != cudaSuccess) return e;
  }
  *step = "tile kernel launch";
  const TraceRange range("isp.tile_pass", kTraceKernel);
  // After the statistics pass, as its programmatic dependent: the tile pass
  // becomes resident on the SMs the statistics pass leaves and waits in the
  // kernel (griddepcontrol.wait) for its completion before anything else. An
  // event recorded in between (before_main) keeps the two kernels apart.
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = need;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = d.auto_wb ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelExC(&cfg, k, args);
  if (e != cudaSuccess || after_main == nullptr) return e;
  return cudaEventRecord(after_main, stream);
}

}  // namespace isp_b200

using namespace isp_b200;


extern "C" {

int isp_b200_abi_version(void) { return ISP_B200_ABI_VERSION; }

const char* isp_b200_last_error(void) { return t_error.c_str(); }

int isp_b200_last_cuda_error(void) { return t_cuda_error; }

void isp_b200_params_default(isp_params_c* params) {
  if (params != nullptr) params_default(params);
}

int isp_b200_validate_params(const isp_params_c* params) {
  if (params == nullptr) return fail(ISP_EINVAL, "params is null");
  if (const char* why = validate_params(*params)) return fail(ISP_EINVAL, why);
  clear_error();
  return ISP_OK;
}

int isp_b200_validate_raw(const isp_raw_view_c* raw, const isp_params_c* params) {
  if (raw == nullptr || params == nullptr) return fail(ISP_EINVAL, "raw view or params is null");
  const std::string why = validate_raw(*raw, *params);
  if (!why.empty()) return fail(ISP_EINVAL, why);
  clear_error();
  return ISP_OK;
}

size_t isp_b200_raw_row_bytes(int32_t format, int32_t width) { return raw_row_bytes(format, width); }

int isp_b200_tone_lut(const isp_params_c* params, float* out, size_t capacity, size_t* size) {
  if (params == nullptr) return fail(ISP_EINVAL, "params is null");
  if (const char* why = validate_params(*params)) return fail(ISP_EINVAL, why);
  const std::vector<float> lut = tone_lut(*params);
  if (out != nullptr) std::memcpy(out, lut.data(), std::min(capacity, lut.size()) * sizeof(float));
  if (size != nullptr) *size = lut.size();
  clear_error();
  return ISP_OK;
}

int isp_b200_create(const isp_params_c* params, isp_b200_pipeline** out) {
  if (out == nullptr) return fail(ISP_EINVAL, "out is null");
  *out = nullptr;
  if (params == nullptr) return fail(ISP_EINVAL, "params is null");
  if (const char* why = validate_params(*params)) return fail(ISP_EINVAL, why);
  auto* pl = new isp_b200_pipeline;
  pl->params.assign(*params);
  cudaError_t e = cudaGetDevice(&pl->device);
  if (e == cudaSuccess) e = device_state_create(pl->params.c, &pl->state);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pl->done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    device_state_free(&pl->state);
    delete pl;
    return fail_cuda(e, "IspPipeline (cuda)");
  }
  *out = pl;
  clear_error();
  return ISP_OK;
}

void isp_b200_destroy(isp_b200_pipeline* pl) {
  if (pl == nullptr) return;
  if (pl->queued) cudaEventSynchronize(pl->done);
  if (pl->host_stream != nullptr) cudaStreamSynchronize(pl->host_stream);
  device_state_free(&pl->state);
  cudaFree(pl->d_raw);
  cudaFree(pl->d_out);
  cudaFree(pl->d_stats);
  if (pl->host_stream != nullptr) cudaStreamDestroy(pl->host_stream);
  if (pl->done != nullptr) cudaEventDestroy(pl->done);
  delete pl;
}

int isp_b200_reset(isp_b200_pipeline* pl) {
  if (pl == nullptr) return fail(ISP_EINVAL, "pipeline is null");
  if (pl->queued) {
    const cudaError_t e = cudaEventSynchronize(pl->done);
    if (e != cudaSuccess) return fail_cuda(e, "cudaEventSynchronize");
  }
  const cudaError_t e = device_state_reset_awb(pl->params.c, &pl->state, nullptr);
  if (e != cudaSuccess) return fail_cuda(e, "reset");
  clear_error();
  return ISP_OK;
}

int isp_b200_awb_state(isp_b200_pipeline* pl, float gains[3], int32_t* valid) {
  if (pl == nullptr) return fail(ISP_EINVAL, "pipeline is null");
  if (pl->queued) {
    const cudaError_t e = cudaEventSynchronize(pl->done);
    if (e != cudaSuccess) return fail_cuda(e, "cudaEventSynchronize");
  }
  struct {
    float g[3];
    int v;
  } st{};
  PrivateStream ps;
  ps.copy(&st, &pl->state.scratch->awb_gains[0], sizeof(st), cudaMemcpyDeviceToHost);
  const cudaError_t e = ps.finish();
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync");
  if (gains != nullptr) {
    for (int k = 0; k < 3; ++k) gains[k] = st.g[k];
  }
  if (valid != nullptr) *valid = st.v;
  clear_error();
  return ISP_OK;
}

int isp_b200_process(isp_b200_pipeline* pl, const isp_raw_view_c* raw, const isp_rgb_view_c* out,
                     const isp_stats_c* stats, const isp_exposure_c* exposure, void* stream_ptr) {
  if (pl == nullptr || raw == nullptr || out == nullptr) return fail(ISP_EINVAL, "pipeline, raw or out is null");
  const TraceRange range("isp.process");
  std::string why = validate_raw(*raw, pl->params.c);
  if (why.empty()) why = validate_out(*raw, *out);
  if (!why.empty()) return fail(ISP_EINVAL, why);
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  cudaError_t error = cudaSuccess;
  LaunchShapes& shapes = shapes_for_current_device(&error);
  if (error != cudaSuccess) return fail_cuda(error, "cudaGetDevice");
  const FrameDesc d = make_desc(pl->params.c, pl->state, *raw, *out, stats, exposure);
  // Clear an error an earlier, unrelated call left (cuda_pipeline.cu:301-303).
  static_cast<void>(cudaGetLastError());
  // Frames share the scratch and white balance state: the GPU waits for the
  // previous frame first (cuda_pipeline.cu:304-310). On the same stream the
  // next frame's statistics pass may still overlap this one's end
  // (frame_overlap): it follows the tile pass as its programmatic dependent.
  const bool same_stream = pl->queued && stream == pl->last_stream;
  if (pl->queued) {
    error = cudaStreamWaitEvent(stream, pl->done, 0);
    if (error != cudaSuccess) return fail_cuda(error, "cudaStreamWaitEvent");
  }
  const char* step = "launch";
  error = launch_frame(d, pl->params.c, shapes, stream, pl->before_main, pl->after_main, &step,
                       same_stream && pl->frame_overlap, pl->rows_for(*raw));
  if (error == cudaSuccess) error = cudaGetLastError();
  if (error != cudaSuccess) return fail_cuda(error, (std::string("IspPipeline (cuda) ") + step).c_str());
  error = cudaEventRecord(pl->done, stream);
  if (error != cudaSuccess) return fail_cuda(error, "cudaEventRecord");
  pl->queued = true;
  pl->last_stream = stream;
  clear_error();
  return ISP_OK;
}

int isp_b200_set_frame_overlap(isp_b200_pipeline* pl, int32_t enable) {
  if (pl == nullptr) return fail(ISP_EINVAL, "pipeline is null");
  pl->frame_overlap = enable != 0;
  clear_error();
  return ISP_OK;
}

int isp_b200_set_tile_rows(isp_b200_pipeline* pl, int32_t tile_rows) {
  if (pl == nullptr) return fail(ISP_EINVAL, "pipeline is null");
  if (tile_rows != 0 && tile_rows_valid(tile_rows) == 0) return fail(ISP_EINVAL, "tile_rows must be 0, 64 or 32");
  pl->tile_rows = tile_rows;
  clear_error();
  return ISP_OK;
}

int isp_b200_autotune(isp_b200_pipeline* pl, const isp_raw_view_c* raw, const isp_rgb_view_c* out,
                      const isp_stats_c* stats, const isp_exposure_c* exposure, void* stream_ptr, int32_t* tile_rows) {
  if (pl == nullptr || raw == nullptr || out == nullptr) return fail(ISP_EINVAL, "pipeline, raw or out is null");
  const TraceRange range("isp.autotune");
  std::string why = validate_raw(*raw, pl->params.c);
  if (why.empty()) why = validate_out(*raw, *out);
  if (!why.empty()) return fail(ISP_EINVAL, why);
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  cudaError_t e = pl->queued ? cudaEventSynchronize(pl->done) : cudaSuccess;
  // The white balance state, kept aside: the timed frames must leave no trace.
  struct {
    float g[3];
    int v;
  } saved{};
  if (e == cudaSuccess) {
    PrivateStream ps;
    ps.copy(&saved, &pl->state.scratch->awb_gains[0], sizeof(saved), cudaMemcpyDeviceToHost);
    e = ps.finish();
  }
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&t0);
  if (e == cudaSuccess) e = cudaEventCreate(&t1);
  const int forced = pl->tile_rows;
  int best_rows = 64;
  float best_ms = 1e30F;
  int status = ISP_OK;
  for (const int rows : {64, 32}) {
    pl->tile_rows = rows;
    float fastest = 1e30F;
    for (int rep = 0; rep < 4 && e == cudaSuccess && status == ISP_OK; ++rep) {
      e = cudaEventRecord(t0, stream);
      if (e == cudaSuccess) status = isp_b200_process(pl, raw, out, stats, exposure, stream_ptr);
      if (e == cudaSuccess && status == ISP_OK) e = cudaEventRecord(t1, stream);
      if (e == cudaSuccess && status == ISP_OK) e = cudaEventSynchronize(t1);
      float ms = 0.0F;
      if (e == cudaSuccess && status == ISP_OK) e = cudaEventElapsedTime(&ms, t0, t1);
      if (rep > 0) fastest = std::min(fastest, ms);  // the first run warms up
    }
    if (fastest < best_ms) {
      best_ms = fastest;
      best_rows = rows;
    }
  }
  pl->tile_rows = forced;
  if (e == cudaSuccess && status == ISP_OK) {
    e = cudaStreamSynchronize(stream);
    PrivateStream ps;
    ps.copy(&pl->state.scratch->awb_gains[0], &saved, sizeof(saved), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = ps.finish();
  }
  if (t0 != nullptr) cudaEventDestroy(t0);
  if (t1 != nullptr) cudaEventDestroy(t1);
  if (status != ISP_OK) return status;
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_autotune");
  int slot = -1;
  for (int i = 0; i < pl->npicks && i < 8; ++i) {
    const auto& k = pl->picks[i];
    if (k.format == raw->format && k.width == raw->width && k.height == raw->height) slot = i;
  }
  if (slot < 0) slot = pl->npicks++ % 8;
  pl->picks[slot] = {raw->format, raw->width, raw->height, best_rows};
  if (tile_rows != nullptr) *tile_rows = best_rows;
  clear_error();
  return ISP_OK;
}

int isp_b200_device_status(isp_b200_pipeline* pl, int32_t* status) {
  if (pl == nullptr || status == nullptr) return fail(ISP_EINVAL, "pipeline or status is null");
  if (pl->queued) {
    const cudaError_t e = cudaEventSynchronize(pl->done);
    if (e != cudaSuccess) return fail_cuda(e, "cudaEventSynchronize");
  }
  int value = 0;
  const int zero = 0;
  PrivateStream ps;
  ps.copy(&value, &pl->state.scratch->error, sizeof(int), cudaMemcpyDeviceToHost);
  ps.copy(&pl->state.scratch->error, &zero, sizeof(int), cudaMemcpyHostToDevice);
  const cudaError_t e = ps.finish();
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync");
  *status = value;
  clear_error();
  return ISP_OK;
}

int isp_b200_checked_violations(isp_b200_pipeline* pl, uint32_t* count, uint64_t* first_address) {
  if (pl == nullptr || count == nullptr || first_address == nullptr) {
    return fail(ISP_EINVAL, "pipeline, count or first_address is null");
  }
#ifdef ISP_CHECKED
  if (pl->queued) {
    const cudaError_t e = cudaEventSynchronize(pl->done);
    if (e != cudaSuccess) return fail_cuda(e, "cudaEventSynchronize");
  }
  CheckRecord record{};
  const CheckRecord zero{};
  PrivateStream ps;
  ps.copy(&record, &pl->state.scratch->check, sizeof(CheckRecord), cudaMemcpyDeviceToHost);
  ps.copy(&pl->state.scratch->check, &zero, sizeof(CheckRecord), cudaMemcpyHostToDevice);
  const cudaError_t e = ps.finish();
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync");
  *count = record.count;
  *first_address = record.count != 0U ? record.address : 0U;
  clear_error();
  return ISP_OK;
#else
  *count = 0;
  *first_address = 0;
  return fail(ISP_EINVAL, "isp_b200_checked_violations: this is not the bounds-checked build (libisp_b200_checked.so)");
#endif
}

int isp_b200_check_bounded_wait(isp_b200_pipeline* pl, uint32_t polls, void* stream_ptr) {
  if (pl == nullptr) return fail(ISP_EINVAL, "pipeline is null");
  if (polls == 0U || polls > (1U << 20)) return fail(ISP_EINVAL, "polls must be 1..1048576");
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  static_cast<void>(cudaGetLastError());
  cudaError_t error = cudaSuccess;
  if (pl->queued) error = cudaStreamWaitEvent(stream, pl->done, 0);
  if (error == cudaSuccess) {
    Scratch* scratch = pl->state.scratch;
    unsigned int n = polls;
    void* args[] = {&scratch, &n};
    error = cudaLaunchKernel(wait_check_kernel(), dim3(1), dim3(32), args, 0, stream);
  }
  if (error == cudaSuccess) error = cudaEventRecord(pl->done, stream);
  if (error != cudaSuccess) return fail_cuda(error, "isp_b200_check_bounded_wait");
  pl->queued = true;
  pl->last_stream = stream;
  clear_error();
  return ISP_OK;
}

int isp_b200_set_kernel_events(isp_b200_pipeline* pl, void* before, void* after) {
  if (pl == nullptr) return fail(ISP_EINVAL, "pipeline is null");
  pl->before_main = static_cast<cudaEvent_t>(before);
  pl->after_main = static_cast<cudaEvent_t>(after);
  clear_error();
  return ISP_OK;
}

int isp_b200_process_host(isp_b200_pipeline* pl, const isp_raw_view_c* raw, const isp_rgb_view_c* out,
                          const isp_stats_c* stats, const isp_exposure_c* exposure) {
  if (pl == nullptr || raw == nullptr || out == nullptr) return fail(ISP_EINVAL, "pipeline, raw or out is null");
  const TraceRange range("isp.process_host");
  std::string why = validate_raw(*raw, pl->params.c);
  if (why.empty()) why = validate_out(*raw, *out);
  if (!why.empty()) return fail(ISP_EINVAL, why);
  cudaError_t e = cudaSuccess;
  if (pl->host_stream == nullptr) {
    e = cudaStreamCreateWithFlags(&pl->host_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamCreate");
  }
  // Device copies: raw rows packed to a 16-byte pitch, output rows packed.
  const size_t row = raw_row_bytes(raw->format, raw->width);
  const size_t raw_pitch = (row + 15U) & ~size_t{15};
  const size_t raw_bytes = raw_pitch * static_cast<size_t>(raw->height);
  const size_t cb = out->format == ISP_OUT_RGB16 ? 2U : out->format == ISP_OUT_RGB32F ? 4U : 1U;
  const size_t out_row = static_cast<size_t>(raw->width) * (out->format == ISP_OUT_RGBA8 ? 4U : 3U) * cb;
  const size_t out_bytes = out_row * static_cast<size_t>(raw->height);
  const auto grow = [&](void** buffer, size_t* cap, size_t bytes) -> cudaError_t {
    if (*cap >= bytes) return cudaSuccess;
    cudaStreamSynchronize(pl->host_stream);
    cudaFree(*buffer);
    *buffer = nullptr;
    *cap = 0;
    const cudaError_t err = cudaMalloc(buffer, bytes);
    if (err == cudaSuccess) *cap = bytes;
    return err;
  };
  e = grow(&pl->d_raw, &pl->d_raw_cap, raw_bytes);
  if (e == cudaSuccess) e = grow(&pl->d_out, &pl->d_out_cap, out_bytes);
  if (e == cudaSuccess && pl->d_stats == nullptr) {
    e = cudaMalloc(&pl->d_stats, (ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS + ISP_STATS_SIZE) * 4U);
  }
  if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc");
  cudaStream_t s = pl->host_stream;
  {
    const TraceRange upload("isp.upload", kTraceCopy);
    e = cudaMemcpy2DAsync(pl->d_raw, raw_pitch, raw->data, raw->pitch, row, static_cast<size_t>(raw->height),
                          cudaMemcpyHostToDevice, s);
  }
  if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpy2DAsync");
  isp_raw_view_c draw = *raw;
  draw.data = pl->d_raw;
  draw.pitch = raw_pitch;
  const isp_rgb_view_c dout{pl->d_out, out_row, out->format};
  auto* d_hist = static_cast<uint32_t*>(pl->d_stats);
  float* d_st = reinterpret_cast<float*>(d_hist + ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS);
  const isp_stats_c dstats{stats != nullptr && stats->histogram != nullptr ? d_hist : nullptr,
                           stats != nullptr && stats->stats != nullptr ? d_st : nullptr};
  const int status = isp_b200_process(pl, &draw, &dout, &dstats, exposure, s);
  if (status != ISP_OK) return status;
  const TraceRange download("isp.download", kTraceCopy);
  e = cudaMemcpy2DAsync(out->data, out->pitch, pl->d_out, out_row, out_row, static_cast<size_t>(raw->height),
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && dstats.histogram != nullptr) {
    e = cudaMemcpyAsync(stats->histogram, d_hist, ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS * 4U,
                        cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess && dstats.stats != nullptr) {
    e = cudaMemcpyAsync(stats->stats, d_st, ISP_STATS_SIZE * 4U, cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_cuda(e, "IspPipeline (cuda) host staging");
  clear_error();
  return ISP_OK;
}

}  // extern "C"
