// isp_batch_host.cu - the batch C ABI (include/isp_b200.h): frames of many
// cameras, each with its own resident state, through one launch per pass
// (isp_batch.cuh), directly or as a CUDA graph that is replayed while the
// batch keeps its shape.
//
// A launch writes the frames' descriptors (FrameDesc, TMA maps, work-list
// positions) and the per-CTA work ranges into one of four pinned staging
// slots, has a staging kernel copy them to the device (SM reads of the
// pinned slot, so that they never queue behind frame transfers on the copy
// engines) on the launch stream, then runs the
// statistics pass (when a frame estimates its white balance) and the tile
// pass. Work ranges are contiguous and of even estimated cost: each tile is
// weighted by its variant's measured cost (isp_b200_batch_autotune) or a
// default. Each camera's previous frames finish first and its later frames
// wait for this batch (the pipeline's event), as with isp_b200_process.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "isp_b200.h"
#include "isp_host.hpp"
#include "isp_kernels.cuh"
#include "isp_trace.hpp"

using namespace isp_b200;

namespace {

// Default relative cost of one tile per variant (bit 0 Malvar, bit 1
// sharpening; the layout bit costs nothing), replaced by measurements.
constexpr float kDefaultWeights[4] = {1.0F, 1.25F, 1.9F, 2.1F};

struct Entry {
  isp_b200_pipeline* camera;
  isp_raw_view_c raw;
  isp_rgb_view_c out;
  isp_stats_c stats;
  isp_exposure_c exposure;
};

struct Slot {
  BatchFrame* frames = nullptr;  // pinned
  int2* ranges = nullptr;        // pinned: tile pass then statistics pass
  const uint4* frames_dev = nullptr;  // the same memory as the device reads it
  const uint4* ranges_dev = nullptr;
  cudaEvent_t consumed = nullptr;
  bool pending = false;
};

// What a captured graph depends on besides the descriptors' contents.
struct Shape {
  int nframes = 0;
  int main_ctas = 0;
  int awb_ctas = 0;
  bool lut_smem = false;
  int tile_rows = 64;
  bool operator==(const Shape& o) const {
    return nframes == o.nframes && main_ctas == o.main_ctas && awb_ctas == o.awb_ctas && lut_smem == o.lut_smem &&
           tile_rows == o.tile_rows;
  }
};

}  // namespace

// Pinned descriptor slots: up to this many launches may be queued before
// a launch waits for the oldest one's descriptors to be consumed.
constexpr int kStagingSlots = 4;

struct isp_b200_batch {
  int capacity = 0;
  std::vector<Entry> entries;
  BatchFrame* d_frames = nullptr;
  int2* d_ranges = nullptr;
  int max_ctas = 0;
  Slot slots[kStagingSlots];
  int next_slot = 0;
  float weights[4] = {kDefaultWeights[0], kDefaultWeights[1], kDefaultWeights[2], kDefaultWeights[3]};
  int ctas_per_sm = 0;  // 0: as many as fit
  int tile_rows = 64;   // the tile pass's tile height: 64 or 32
  bool tuned = false;
  // The graph of the last shape, its nodes, and the slot its copies read.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphNode_t stage = nullptr;
  Shape graph_shape;
  int replays = 0;
};

namespace {

cudaError_t build(isp_b200_batch* b, const Slot& slot, Shape* shape) {
  cudaError_t error = cudaSuccess;
  LaunchShapes& dev = shapes_for_current_device(&error);
  if (error != cudaSuccess) return error;
  const int n = static_cast<int>(b->entries.size());
  bool lut_smem = true;
  for (const Entry& e : b->entries) lut_smem = lut_smem && e.camera->state.tone_size <= kBatchLutEntries;
  std::vector<float> tile_cost;
  int tiles = 0;
  int awb_tiles = 0;
  for (int i = 0; i < n; ++i) {
    const Entry& e = b->entries[static_cast<size_t>(i)];
    const isp_params_c& p = e.camera->params.c;
    BatchFrame& f = slot.frames[i];
    std::memset(static_cast<void*>(&f), 0, sizeof(f));
    f.desc = make_desc(p, e.camera->state, e.raw, e.out, &e.stats, &e.exposure);
    const bool malvar = p.demosaic == ISP_DEMOSAIC_MALVAR;
    const bool sharpen = p.sharpen > 0.0F;
    f.variant = (malvar ? 1 : 0) | (sharpen ? 2 : 0) | ((e.raw.pattern >> 1) << 2);
    f.tiles = main_kernel_tiles(e.raw.width, e.raw.height, &f.tiles_x, b->tile_rows);
    f.tile_begin = tiles;
    tiles += f.tiles;
    const bool tma_main = encode_raw_map(f.desc, main_box_row_bytes(e.raw.format), main_box_rows(sharpen, b->tile_rows),
                                         &f.main_map);
    bool tma_awb = true;
    if (f.desc.auto_wb) {
      f.awb_tiles = awb_kernel_tiles(e.raw.width, e.raw.height, &f.awb_tiles_x);
      tma_awb = encode_raw_map(f.desc, awb_box_row_bytes(e.raw.format), 64, &f.awb_map);
    }
    f.awb_begin = awb_tiles;
    awb_tiles += f.awb_tiles;
    f.use_tma = tma_main && tma_awb ? 1 : 0;
    tile_cost.insert(tile_cost.end(), static_cast<size_t>(f.tiles), b->weights[f.variant & 3]);
  }
  // CTAs: as many as fit (or the tuned count) per SM, never more than items.
  int bpsm = 0;
  const size_t smem = batch_kernel_smem(lut_smem, b->tile_rows);
  error = blocks_per_sm(dev, batch_kernel(lut_smem, b->tile_rows), smem, smem, &bpsm);
  if (error != cudaSuccess) return error;
  if (b->ctas_per_sm > 0) bpsm = std::min(bpsm, b->ctas_per_sm);
  const int main_ctas = std::max(1, std::min({tiles, dev.sm_count * bpsm, b->max_ctas}));
  int awb_bpsm = 0;
  error = blocks_per_sm(dev, awb_batch_kernel(), awb_kernel_smem(), awb_kernel_smem(), &awb_bpsm);
  if (error != cudaSuccess) return error;
  const int awb_ctas = awb_tiles == 0 ? 0 : std::max(1, std::min({awb_tiles, dev.sm_count * awb_bpsm, b->max_ctas}));
  // Contiguous ranges of even cost.
  double total = 0.0;
  for (const float c : tile_cost) total += c;
  int item = 0;
  double acc = 0.0;
  for (int k = 0; k < main_ctas; ++k) {
    const int begin = item;
    const double goal = total * (k + 1) / main_ctas;
    while (item < tiles && (acc + tile_cost[static_cast<size_t>(item)] * 0.5 <= goal || k == main_ctas - 1)) {
      acc += tile_cost[static_cast<size_t>(item)];
      ++item;
    }
    slot.ranges[k] = make_int2(begin, item);
  }
  for (int k = 0; k < awb_ctas; ++k) {
    slot.ranges[b->max_ctas + k] =
        make_int2(static_cast<int>(static_cast<int64_t>(awb_tiles) * k / awb_ctas),
                  static_cast<int>(static_cast<int64_t>(awb_tiles) * (k + 1) / awb_ctas));
  }
  shape->nframes = n;
  shape->main_ctas = main_ctas;
  shape->awb_ctas = awb_ctas;
  shape->lut_smem = lut_smem;
  shape->tile_rows = b->tile_rows;
  return cudaSuccess;
}

// The staging kernel's arguments for a slot (kernel arguments are copied at launch).
struct StageArgs {
  const uint4* frames_src;
  uint4* frames_dst;
  int frame_words;
  const uint4* ranges_src;
  uint4* ranges_dst;
  int range_words;
  void* args[6];
  dim3 grid;

  StageArgs(const isp_b200_batch* b, const Slot& slot, const Shape& s)
      : frames_src(slot.frames_dev),
        frames_dst(reinterpret_cast<uint4*>(b->d_frames)),
        frame_words(static_cast<int>(sizeof(BatchFrame) / sizeof(uint4)) * s.nframes),
        ranges_src(slot.ranges_dev),
        ranges_dst(reinterpret_cast<uint4*>(b->d_ranges)),
        range_words(b->max_ctas),  // 2 x max_ctas int2
        args{&frames_src, &frames_dst, &frame_words, &ranges_src, &ranges_dst, &range_words},
        grid((frame_words + range_words + kStageThreads - 1) / kStageThreads) {}
  StageArgs(const StageArgs&) = delete;
  StageArgs& operator=(const StageArgs&) = delete;

  cudaKernelNodeParams node() {
    cudaKernelNodeParams kp{};
    kp.func = const_cast<void*>(batch_stage_kernel());
    kp.gridDim = grid;
    kp.blockDim = dim3(kStageThreads);
    kp.kernelParams = args;
    return kp;
  }
};
static_assert(sizeof(BatchFrame) % sizeof(uint4) == 0, "descriptors are copied in 16-byte words");

// Queues the descriptor staging and the two passes on `stream` (direct launch).
cudaError_t enqueue(isp_b200_batch* b, const Slot& slot, const Shape& s, cudaStream_t stream) {
  StageArgs stage(b, slot, s);
  cudaError_t e = cudaLaunchKernel(batch_stage_kernel(), stage.grid, dim3(kStageThreads), stage.args, 0, stream);
  if (e != cudaSuccess) return e;
  int nframes = s.nframes;
  const int2* awb_ranges = b->d_ranges + b->max_ctas;
  if (s.awb_ctas > 0) {
    void* args[] = {&b->d_frames, &nframes, &awb_ranges};
    e = cudaLaunchKernel(awb_batch_kernel(), dim3(s.awb_ctas), dim3(kernel_threads()), args, awb_kernel_smem(), stream);
    if (e != cudaSuccess) return e;
  }
  void* args[] = {&b->d_frames, &nframes, &b->d_ranges};
  // After the statistics batch, as its programmatic dependent (the tile
  // batch waits for it in the kernel).
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(s.main_ctas);
  cfg.blockDim = dim3(kernel_threads());
  cfg.dynamicSmemBytes = batch_kernel_smem(s.lut_smem, s.tile_rows);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = s.awb_ctas > 0 ? 1 : 0;
  return cudaLaunchKernelExC(&cfg, batch_kernel(s.lut_smem, s.tile_rows), args);
}

// Builds the graph of a shape: the descriptor staging, then the passes.
cudaError_t make_graph(isp_b200_batch* b, const Slot& slot, const Shape& s) {
  if (b->exec != nullptr) cudaGraphExecDestroy(b->exec);
  if (b->graph != nullptr) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  cudaError_t e = cudaGraphCreate(&b->graph, 0);
  if (e != cudaSuccess) return e;
  StageArgs stage(b, slot, s);
  cudaKernelNodeParams sp = stage.node();
  e = cudaGraphAddKernelNode(&b->stage, b->graph, nullptr, 0, &sp);
  if (e != cudaSuccess) return e;
  int nframes = s.nframes;  // kernel node arguments are copied when the node is made
  const int2* awb_ranges = b->d_ranges + b->max_ctas;
  cudaGraphNode_t awb = nullptr;
  if (s.awb_ctas > 0) {
    void* args[] = {&b->d_frames, &nframes, &awb_ranges};
    cudaKernelNodeParams kp{};
    kp.func = const_cast<void*>(awb_batch_kernel());
    kp.gridDim = dim3(s.awb_ctas);
    kp.blockDim = dim3(kernel_threads());
    kp.sharedMemBytes = static_cast<unsigned int>(awb_kernel_smem());
    kp.kernelParams = args;
    e = cudaGraphAddKernelNode(&awb, b->graph, &b->stage, 1, &kp);
    if (e != cudaSuccess) return e;
  }
  void* args[] = {&b->d_frames, &nframes, &b->d_ranges};
  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(batch_kernel(s.lut_smem, s.tile_rows));
  kp.gridDim = dim3(s.main_ctas);
  kp.blockDim = dim3(kernel_threads());
  kp.sharedMemBytes = static_cast<unsigned int>(batch_kernel_smem(s.lut_smem, s.tile_rows));
  kp.kernelParams = args;
  cudaGraphNode_t main = nullptr;
  if (awb != nullptr) {
    // A programmatic edge from the statistics node, as the direct launch's
    // attribute: the tile node waits for it in the kernel.
    e = cudaGraphAddKernelNode(&main, b->graph, nullptr, 0, &kp);
    if (e != cudaSuccess) return e;
    cudaGraphEdgeData edge{};
    edge.from_port = cudaGraphKernelNodePortProgrammatic;
    edge.type = cudaGraphDependencyTypeProgrammatic;
    e = cudaGraphAddDependencies_v2(b->graph, &awb, &main, &edge, 1);
  } else {
    e = cudaGraphAddKernelNode(&main, b->graph, &b->stage, 1, &kp);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e == cudaSuccess) b->graph_shape = s;
  return e;
}

int check_entry(const isp_b200_batch* b, isp_b200_pipeline* camera, const isp_raw_view_c* raw,
                const isp_rgb_view_c* out) {
  if (b == nullptr || camera == nullptr || raw == nullptr || out == nullptr) {
    return fail(ISP_EINVAL, "batch, camera, raw or out is null");
  }
  if (static_cast<int>(b->entries.size()) >= b->capacity) return fail(ISP_EBUSY, "batch is full");
  for (const Entry& e : b->entries) {
    if (e.camera == camera) {
      return fail(ISP_EINVAL, "a camera appears once per batch: its white balance state is sequential");
    }
  }
  std::string why = validate_raw(*raw, camera->params.c);
  if (why.empty()) why = validate_out(*raw, *out);
  if (!why.empty()) return fail(ISP_EINVAL, why);
  return ISP_OK;
}

}  // namespace

extern "C" {

int isp_b200_batch_create(int32_t capacity, isp_b200_batch** out) {
  if (out == nullptr || capacity < 1 || capacity > 4096) return fail(ISP_EINVAL, "batch capacity must be 1..4096");
  *out = nullptr;
  auto* b = new isp_b200_batch;
  b->capacity = capacity;
  cudaError_t e = cudaSuccess;
  LaunchShapes& dev = shapes_for_current_device(&e);
  if (e == cudaSuccess) {
    b->max_ctas = dev.sm_count * 4;
    e = cudaMalloc(&b->d_frames, sizeof(BatchFrame) * static_cast<size_t>(capacity));
  }
  if (e == cudaSuccess) e = cudaMalloc(&b->d_ranges, sizeof(int2) * 2 * static_cast<size_t>(b->max_ctas));
  for (Slot& s : b->slots) {
    if (e == cudaSuccess) e = cudaMallocHost(&s.frames, sizeof(BatchFrame) * static_cast<size_t>(capacity));
    if (e == cudaSuccess) e = cudaMallocHost(&s.ranges, sizeof(int2) * 2 * static_cast<size_t>(b->max_ctas));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.consumed, cudaEventDisableTiming);
    void* dev = nullptr;
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&dev, s.frames, 0);
    s.frames_dev = static_cast<const uint4*>(dev);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&dev, s.ranges, 0);
    s.ranges_dev = static_cast<const uint4*>(dev);
  }
  if (e != cudaSuccess) {
    isp_b200_batch_destroy(b);
    return fail_cuda(e, "isp_b200_batch_create");
  }
  *out = b;
  clear_error();
  return ISP_OK;
}

void isp_b200_batch_destroy(isp_b200_batch* b) {
  if (b == nullptr) return;
  for (Slot& s : b->slots) {
    if (s.consumed != nullptr) {
      cudaEventSynchronize(s.consumed);
      cudaEventDestroy(s.consumed);
    }
    cudaFreeHost(s.frames);
    cudaFreeHost(s.ranges);
  }
  if (b->exec != nullptr) cudaGraphExecDestroy(b->exec);
  if (b->graph != nullptr) cudaGraphDestroy(b->graph);
  cudaFree(b->d_frames);
  cudaFree(b->d_ranges);
  delete b;
}

int isp_b200_batch_clear(isp_b200_batch* b) {
  if (b == nullptr) return fail(ISP_EINVAL, "batch is null");
  b->entries.clear();
  clear_error();
  return ISP_OK;
}

int isp_b200_batch_size(const isp_b200_batch* b) { return b == nullptr ? 0 : static_cast<int>(b->entries.size()); }

int isp_b200_batch_add(isp_b200_batch* b, isp_b200_pipeline* camera, const isp_raw_view_c* raw,
                       const isp_rgb_view_c* out, const isp_stats_c* stats, const isp_exposure_c* exposure) {
  if (const int status = check_entry(b, camera, raw, out); status != ISP_OK) return status;
  Entry e{camera, *raw, *out, {nullptr, nullptr}, {0, 0.0F}};
  if (stats != nullptr) e.stats = *stats;
  if (exposure != nullptr) e.exposure = *exposure;
  b->entries.push_back(e);
  clear_error();
  return ISP_OK;
}

int isp_b200_batch_launch(isp_b200_batch* b, void* stream_ptr, int32_t use_graph) {
  if (b == nullptr) return fail(ISP_EINVAL, "batch is null");
  if (b->entries.empty()) {
    clear_error();
    return ISP_OK;
  }
  const TraceRange range("isp.batch.launch");
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  Slot& slot = b->slots[b->next_slot];
  // The slot's previous contents must have reached the device.
  if (slot.pending) {
    const cudaError_t e = cudaEventSynchronize(slot.consumed);
    if (e != cudaSuccess) return fail_cuda(e, "cudaEventSynchronize");
    slot.pending = false;
  }
  static_cast<void>(cudaGetLastError());
  Shape shape;
  cudaError_t e = cudaSuccess;
  {
    const TraceRange build_range("isp.batch.build", kTraceCopy);
    e = build(b, slot, &shape);
  }
  if (e != cudaSuccess) return fail_cuda(e, "batch build");
  for (const Entry& en : b->entries) {
    if (en.camera->queued) {
      e = cudaStreamWaitEvent(stream, en.camera->done, 0);
      if (e != cudaSuccess) return fail_cuda(e, "cudaStreamWaitEvent");
    }
  }
  // The device descriptor buffers are shared by all launches: the previous
  // launch's kernels finish reading them first (whatever its stream).
  const Slot& previous = b->slots[(b->next_slot + kStagingSlots - 1) % kStagingSlots];
  if (previous.pending) {
    e = cudaStreamWaitEvent(stream, previous.consumed, 0);
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamWaitEvent");
  }
  if (use_graph) {
    if (b->exec == nullptr || !(b->graph_shape == shape)) {
      e = make_graph(b, slot, shape);
      if (e != cudaSuccess) return fail_cuda(e, "batch graph");
    }
    // The staging reads this launch's slot.
    const TraceRange replay("isp.batch.replay", kTraceKernel);
    StageArgs stage(b, slot, shape);
    cudaKernelNodeParams sp = stage.node();
    e = cudaGraphExecKernelNodeSetParams(b->exec, b->stage, &sp);
    if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, stream);
    if (e == cudaSuccess) ++b->replays;
  } else {
    const TraceRange kernels("isp.batch.enqueue", kTraceKernel);
    e = enqueue(b, slot, shape, stream);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e, "batch launch");
  e = cudaEventRecord(slot.consumed, stream);
  if (e != cudaSuccess) return fail_cuda(e, "cudaEventRecord");
  slot.pending = true;
  b->next_slot = (b->next_slot + 1) % kStagingSlots;
  for (const Entry& en : b->entries) {
    e = cudaEventRecord(en.camera->done, stream);
    if (e != cudaSuccess) return fail_cuda(e, "cudaEventRecord");
    en.camera->queued = true;
  }
  clear_error();
  return ISP_OK;
}

int isp_b200_batch_autotune(isp_b200_batch* b, void* stream_ptr) {
  if (b == nullptr) return fail(ISP_EINVAL, "batch is null");
  const TraceRange range("isp.batch.autotune");
  if (b->entries.empty()) return fail(ISP_EINVAL, "batch is empty");
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  const int n = static_cast<int>(b->entries.size());
  // The cameras' white balance states (gains, valid: 16 bytes each), kept
  // aside and put back around every measured launch.
  void* saved = nullptr;
  cudaEvent_t t0 = nullptr;
  cudaEvent_t t1 = nullptr;
  cudaError_t e = cudaMalloc(&saved, 16U * static_cast<size_t>(n));
  if (e == cudaSuccess) e = cudaEventCreate(&t0);
  if (e == cudaSuccess) e = cudaEventCreate(&t1);
  const auto save = [&](bool restore) {
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
      void* state = &b->entries[static_cast<size_t>(i)].camera->state.scratch->awb_gains[0];
      char* copy = static_cast<char*>(saved) + 16 * i;
      e = restore ? cudaMemcpyAsync(state, copy, 16, cudaMemcpyDeviceToDevice, stream)
                  : cudaMemcpyAsync(copy, state, 16, cudaMemcpyDeviceToDevice, stream);
    }
  };
  const auto elapsed = [&]() -> float {
    float ms = 0.0F;
    if (e == cudaSuccess) e = cudaEventSynchronize(t1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
    return ms;
  };
  save(false);
  // 1. Cost of a tile per variant: the largest frame of each variant alone.
  float cost[4] = {0.0F, 0.0F, 0.0F, 0.0F};
  for (int v = 0; v < 4 && e == cudaSuccess; ++v) {
    int best = -1;
    int best_tiles = 0;
    for (int i = 0; i < n; ++i) {
      const Entry& en = b->entries[static_cast<size_t>(i)];
      const isp_params_c& p = en.camera->params.c;
      const int variant = (p.demosaic == ISP_DEMOSAIC_MALVAR ? 1 : 0) | (p.sharpen > 0.0F ? 2 : 0);
      int tx = 0;
      const int tiles = main_kernel_tiles(en.raw.width, en.raw.height, &tx);
      if (variant == v && tiles > best_tiles) {
        best = i;
        best_tiles = tiles;
      }
    }
    if (best < 0) continue;
    const Entry& en = b->entries[static_cast<size_t>(best)];
    float best_ms = 1e30F;
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
      if (e == cudaSuccess) e = cudaEventRecord(t0, stream);
      if (e == cudaSuccess && isp_b200_process(en.camera, &en.raw, &en.out, &en.stats, &en.exposure, stream) != ISP_OK) {
        e = cudaErrorUnknown;
      }
      if (e == cudaSuccess) e = cudaEventRecord(t1, stream);
      const float ms = elapsed();
      if (rep > 0) best_ms = std::min(best_ms, ms);  // the first run warms up
    }
    cost[v] = best_ms / static_cast<float>(best_tiles);
    save(true);
  }
  float lowest = 1e30F;
  for (const float c : cost) {
    if (c > 0.0F) lowest = std::min(lowest, c);
  }
  for (int v = 0; v < 4; ++v) b->weights[v] = cost[v] > 0.0F ? cost[v] / lowest : kDefaultWeights[v];
  // 2. Tile height (64 or 32 rows) and CTAs per SM for the whole batch.
  int best_cps = 0;
  int best_rows = 64;
  float best_ms = 1e30F;
  for (const int rows : {64, 32}) {
    for (const int cps : {1, 2, 3, 0}) {
      b->tile_rows = rows;
      b->ctas_per_sm = cps;
      float fastest = 1e30F;
      for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
        save(true);
        if (e == cudaSuccess) e = cudaEventRecord(t0, stream);
        if (e == cudaSuccess && isp_b200_batch_launch(b, stream, 0) != ISP_OK) e = cudaErrorUnknown;
        if (e == cudaSuccess) e = cudaEventRecord(t1, stream);
        fastest = std::min(fastest, elapsed());
      }
      if (fastest < best_ms) {
        best_ms = fastest;
        best_cps = cps;
        best_rows = rows;
      }
    }
  }
  b->tile_rows = best_rows;
  b->ctas_per_sm = best_cps;
  save(true);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  cudaFree(saved);
  if (t0 != nullptr) cudaEventDestroy(t0);
  if (t1 != nullptr) cudaEventDestroy(t1);
  if (e != cudaSuccess) return fail_cuda(e, "isp_b200_batch_autotune");
  b->tuned = true;
  clear_error();
  return ISP_OK;
}

int isp_b200_batch_info(const isp_b200_batch* b, isp_batch_info_c* info) {
  if (b == nullptr || info == nullptr) return fail(ISP_EINVAL, "batch or info is null");
  std::memset(info, 0, sizeof(*info));
  info->frames = static_cast<int32_t>(b->entries.size());
  for (int k = 0; k < 4; ++k) info->weights[k] = b->weights[k];
  info->ctas_per_sm = b->ctas_per_sm;
  info->tuned = b->tuned ? 1 : 0;
  info->graph_replays = b->replays;
  info->graph_main_ctas = b->graph_shape.main_ctas;
  info->graph_awb_ctas = b->graph_shape.awb_ctas;
  info->tile_rows = b->tile_rows;
  info->block_threads = kernel_threads();
  clear_error();
  return ISP_OK;
}

int isp_b200_batch_set_tuning(isp_b200_batch* b, const float weights[4], int32_t ctas_per_sm) {
  if (b == nullptr || weights == nullptr || ctas_per_sm < 0) return fail(ISP_EINVAL, "bad tuning");
  for (int k = 0; k < 4; ++k) {
    if (!(weights[k] > 0.0F)) return fail(ISP_EINVAL, "weights must be positive");
    b->weights[k] = weights[k];
  }
  b->ctas_per_sm = ctas_per_sm;
  b->tuned = true;
  clear_error();
  return ISP_OK;
}

int isp_b200_batch_set_tile_rows(isp_b200_batch* b, int32_t tile_rows) {
  if (b == nullptr) return fail(ISP_EINVAL, "batch is null");
  if (tile_rows_valid(tile_rows) == 0) return fail(ISP_EINVAL, "tile_rows must be 64 or 32");
  b->tile_rows = tile_rows;
  clear_error();
  return ISP_OK;
}

}  // extern "C"
