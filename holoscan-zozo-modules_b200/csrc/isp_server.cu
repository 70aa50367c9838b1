// isp_server.cu - serving many camera streams with continuous batching
// (include/isp_b200.h, isp_b200_server_*).
//
// Each stream is a camera: a pipeline whose state (tone table, lens shading
// grid, white balance and scratch) stays on the device, device slots for its
// frames in flight, and a host queue of frames that arrived and wait. A
// worker thread runs the loop:
//   1. reap: batches whose done event has completed free their frames' slots
//      and budget bytes; their results become pollable, stamped with the
//      time the worker saw the event complete;
//   2. admit: waiting frames, oldest arrival first, take a free slot of their
//      stream while the bytes of the admitted frames stay within the memory
//      budget, and their host->device copy is issued at once, on one of
//      three copy streams by frame size (below kSmallCopy, below kLargeCopy,
//      larger), so that a small frame does not queue behind a large one;
//   3. launch: while fewer than max_inflight batches are on the GPU, the
//      frames whose copies have completed (at most one per stream, its
//      oldest) form a batch: one statistics pass and one tile pass over all
//      of them (or one isp_b200_process each, with per_frame), then result
//      copies on a readback stream where asked, then the batch's done event;
//   4. with work on the GPU or copies in flight, poll again after a yield
//      (the worker keeps a core busy while anything is pending); with
//      nothing pending, sleep until a frame arrives.
// Continuous batching: frames that arrive while batches run are copied in
// while the GPU computes and join the next batch as soon as a batch slot
// frees. A frame's latency is its arrival to its batch's done event (its
// outputs are then in device memory; with result copies, in host memory).
// Frames of one stream run in arrival order, one per batch (the pipeline's
// event orders its batches).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "isp_b200.h"
#include "isp_host.hpp"
#include "isp_trace.hpp"

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Copy lanes by raw frame size: below kSmallCopy, below kLargeCopy, larger.
constexpr size_t kSmallCopy = size_t{1} << 20;
constexpr size_t kLargeCopy = size_t{8} << 20;
constexpr int kCopyLanes = 3;

struct Request {
  uint64_t ticket;
  uint64_t frame;
  int64_t arrival_ns;
  const void* host_raw;  // pinned memory the frame is copied from (device memory when on_device)
  size_t host_pitch;
  void* host_out;  // optional result copies
  uint32_t* host_hist;
  float* host_stats;
  int staging;     // index of the stream's staging buffer holding the raw, or -1 (borrowed)
  bool on_device;  // host_raw is device memory, read in place
};

// How a submitted frame's raw bytes reach the GPU.
enum class Source { kCopy, kBorrowHost, kDevice };

struct DeviceSlot {
  void* raw = nullptr;
  void* out = nullptr;
  uint32_t* hist = nullptr;
  float* stats = nullptr;
  cudaEvent_t copied = nullptr;  // the host->device copy of the slot's frame
  bool busy = false;
  // Pinned host mirrors the results are copied to (streams with copy_back).
  void* host_out = nullptr;
  uint32_t* host_hist = nullptr;
  float* host_stats = nullptr;
};

// A frame that holds a slot and whose raw is on its way to the device.
struct Admitted {
  Request req;
  int slot;
  bool ready;  // its raw is in device memory
};

struct Stream {
  isp_b200_pipeline* camera = nullptr;
  isp_server_stream_c shape{};
  size_t raw_row = 0;
  size_t raw_pitch = 0;  // device slots: rows at a 16-byte pitch
  size_t out_row = 0;
  size_t frame_bytes = 0;  // raw + image: what a frame in flight holds
  std::vector<DeviceSlot> slots;
  std::vector<void*> staging;  // pinned host copies of submitted frames
  std::vector<bool> staging_busy;
  std::deque<Request> queue;      // arrived, waiting for a slot
  std::deque<Admitted> admitted;  // holding a slot, waiting for a batch
  uint64_t next_frame = 0;
  std::vector<void*> sources;  // frames the synthetic drivers submit, in turn
  bool sources_on_device = false;
  size_t next_source = 0;
};

struct InFlight {
  int stream;
  int slot;
  Request req;
};

struct Batch {
  std::vector<InFlight> frames;
  cudaEvent_t done = nullptr;
  int64_t launch_ns = 0;
  bool failed = false;
};

}  // namespace

struct isp_b200_server {
  isp_server_config_c config{};
  int device = 0;
  std::vector<std::unique_ptr<Stream>> streams;
  isp_b200_batch* batch_builder = nullptr;
  cudaStream_t compute = nullptr;
  cudaStream_t copy[kCopyLanes] = {};  // raw frames host -> device, by size
  cudaStream_t readback = nullptr;  // results device -> host, off the compute stream
  std::mutex mutex;                 // everything below
  std::condition_variable wake;
  std::thread worker;
  bool running = false;
  bool started = false;
  std::deque<std::unique_ptr<Batch>> inflight;
  std::vector<cudaEvent_t> spare_events;
  int64_t inflight_bytes = 0;  // bytes of admitted frames
  int64_t staged = 0;          // admitted frames not yet in a batch
  int64_t queued = 0;          // arrived frames not yet admitted
  int next_stream = 0;         // round-robin start of batch formation
  uint64_t next_ticket = 1;
  std::deque<isp_server_result_c> results;
  std::vector<double> latencies_ms;
  std::vector<double> waits_ms;  // arrival to batch launch
  int64_t submitted = 0;
  int64_t refused = 0;
  int64_t admitted = 0;
  int64_t completed = 0;
  int64_t completed_pixels = 0;
  int64_t batches = 0;
  int64_t batch_frames = 0;
  int64_t first_arrival_ns = 0;
  int64_t last_done_ns = 0;
  std::string worker_error;
};

namespace {

using namespace isp_b200;

void release_stream(Stream* s) {
  for (DeviceSlot& d : s->slots) {
    cudaFree(d.raw);
    cudaFree(d.out);
    cudaFree(d.hist);
    cudaFree(d.stats);
    if (d.copied != nullptr) cudaEventDestroy(d.copied);
    cudaFreeHost(d.host_out);
    cudaFreeHost(d.host_hist);
    cudaFreeHost(d.host_stats);
  }
  for (void* h : s->staging) cudaFreeHost(h);
  for (void* h : s->sources) {
    if (s->sources_on_device) {
      cudaFree(h);
    } else {
      cudaFreeHost(h);
    }
  }
  isp_b200_destroy(s->camera);
}

void worker_fail(isp_b200_server* sv, const std::string& what, cudaError_t e) {
  if (sv->worker_error.empty()) sv->worker_error = what + ": " + cudaGetErrorString(e);
}

// Retires finished batches, oldest first. Caller holds the mutex.
bool reap(isp_b200_server* sv) {
  bool any = false;
  while (!sv->inflight.empty()) {
    Batch& b = *sv->inflight.front();
    if (!b.failed) {
      const cudaError_t q = cudaEventQuery(b.done);
      if (q == cudaErrorNotReady) break;
      if (q != cudaSuccess) worker_fail(sv, "batch", q);
    }
    const TraceRange range("isp.server.retire", kTraceServe);
    const int64_t t = now_ns();
    for (const InFlight& f : b.frames) {
      Stream& s = *sv->streams[static_cast<size_t>(f.stream)];
      DeviceSlot& slot = s.slots[static_cast<size_t>(f.slot)];
      slot.busy = false;
      if (f.req.staging >= 0) s.staging_busy[static_cast<size_t>(f.req.staging)] = false;
      sv->inflight_bytes -= static_cast<int64_t>(s.frame_bytes);
      isp_server_result_c r{};
      r.ticket = f.req.ticket;
      r.stream = f.stream;
      r.frame = f.req.frame;
      r.arrival_ns = f.req.arrival_ns;
      r.launch_ns = b.launch_ns;
      r.done_ns = t;
      r.image = slot.out;
      r.histogram = slot.hist;
      r.stats = slot.stats;
      sv->results.push_back(r);
      sv->latencies_ms.push_back(static_cast<double>(t - f.req.arrival_ns) * 1e-6);
      sv->waits_ms.push_back(static_cast<double>(b.launch_ns - f.req.arrival_ns) * 1e-6);
      ++sv->completed;
      sv->completed_pixels += static_cast<int64_t>(s.shape.width) * s.shape.height;
    }
    sv->last_done_ns = std::max(sv->last_done_ns, t);
    if (b.done != nullptr) sv->spare_events.push_back(b.done);
    sv->inflight.pop_front();
    any = true;
  }
  return any;
}

// Gives waiting frames slots, oldest arrival first, and issues their copies.
// Caller holds the mutex.
bool admit(isp_b200_server* sv) {
  bool any = false;
  while (sv->queued > 0) {
    int pick = -1;
    int pick_slot = -1;
    int64_t oldest = 0;
    for (size_t i = 0; i < sv->streams.size(); ++i) {
      Stream& s = *sv->streams[i];
      if (s.queue.empty()) continue;
      if (pick >= 0 && s.queue.front().arrival_ns >= oldest) continue;
      if (sv->inflight_bytes + static_cast<int64_t>(s.frame_bytes) > sv->config.memory_budget) continue;
      for (size_t d = 0; d < s.slots.size(); ++d) {
        if (!s.slots[d].busy) {
          pick = static_cast<int>(i);
          pick_slot = static_cast<int>(d);
          oldest = s.queue.front().arrival_ns;
          break;
        }
      }
    }
    if (pick < 0) break;
    const TraceRange range("isp.server.admit", kTraceServe);
    Stream& s = *sv->streams[static_cast<size_t>(pick)];
    DeviceSlot& slot = s.slots[static_cast<size_t>(pick_slot)];
    Admitted a{s.queue.front(), pick_slot, false};
    s.queue.pop_front();
    --sv->queued;
    slot.busy = true;
    sv->inflight_bytes += static_cast<int64_t>(s.frame_bytes);
    if (a.req.on_device) {
      a.ready = true;
    } else {
      const size_t bytes = s.raw_row * static_cast<size_t>(s.shape.height);
      cudaStream_t cs = sv->copy[bytes < kSmallCopy ? 0 : bytes < kLargeCopy ? 1 : 2];
      cudaError_t e = cudaMemcpy2DAsync(slot.raw, s.raw_pitch, a.req.host_raw, a.req.host_pitch, s.raw_row,
                                        static_cast<size_t>(s.shape.height), cudaMemcpyHostToDevice, cs);
      if (e == cudaSuccess) e = cudaEventRecord(slot.copied, cs);
      if (e != cudaSuccess) {
        worker_fail(sv, "frame copy", e);
        a.ready = true;  // let it fail through its batch
      }
    }
    s.admitted.push_back(a);
    ++sv->staged;
    ++sv->admitted;
    any = true;
  }
  return any;
}

// Forms and launches one batch from the admitted frames whose raw is on the
// device. Caller holds the mutex (released around the CUDA calls); returns
// false when no frame is ready.
bool launch_ready(isp_b200_server* sv, std::unique_lock<std::mutex>& lock) {
  if (sv->staged == 0) return false;
  const int n = static_cast<int>(sv->streams.size());
  auto b = std::make_unique<Batch>();
  for (int k = 0; k < n && static_cast<int>(b->frames.size()) < sv->config.max_batch; ++k) {
    const int si = (sv->next_stream + k) % n;
    Stream& s = *sv->streams[static_cast<size_t>(si)];
    if (s.admitted.empty()) continue;
    Admitted& a = s.admitted.front();
    if (!a.ready) {
      const cudaError_t q = cudaEventQuery(s.slots[static_cast<size_t>(a.slot)].copied);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) worker_fail(sv, "frame copy", q);
      a.ready = true;
    }
    b->frames.push_back(InFlight{si, a.slot, a.req});
    s.admitted.pop_front();
    --sv->staged;
  }
  if (b->frames.empty()) return false;
  sv->next_stream = (sv->next_stream + 1) % n;
  if (!sv->spare_events.empty()) {
    b->done = sv->spare_events.back();
    sv->spare_events.pop_back();
  }
  Batch* batch = b.get();
  sv->inflight.push_back(std::move(b));
  ++sv->batches;
  sv->batch_frames += static_cast<int64_t>(batch->frames.size());
  lock.unlock();
  const TraceRange range("isp.server.launch", kTraceServe);
  // CUDA work outside the lock: submitters only touch the queues, and only
  // the worker touches slots, admitted frames and in-flight batches.
  cudaError_t e = cudaSuccess;
  if (batch->done == nullptr) e = cudaEventCreateWithFlags(&batch->done, cudaEventDisableTiming);
  const bool per_frame = sv->config.per_frame != 0;
  if (!per_frame) isp_b200_batch_clear(sv->batch_builder);
  const char* step = "batch";
  batch->launch_ns = now_ns();
  for (const InFlight& f : batch->frames) {
    if (e != cudaSuccess) break;
    Stream& s = *sv->streams[static_cast<size_t>(f.stream)];
    DeviceSlot& slot = s.slots[static_cast<size_t>(f.slot)];
    isp_raw_view_c raw{f.req.host_raw, s.shape.width, s.shape.height, f.req.host_pitch, s.shape.format,
                       s.shape.bit_depth, s.shape.pattern};
    if (!f.req.on_device) {
      raw.data = slot.raw;
      raw.pitch = s.raw_pitch;
    }
    const isp_rgb_view_c out{slot.out, s.out_row, s.shape.out_format};
    const isp_stats_c st{s.shape.with_histogram ? slot.hist : nullptr, s.shape.with_stats ? slot.stats : nullptr};
    const isp_exposure_c ex{0, 0.0F};
    const int status = per_frame ? isp_b200_process(s.camera, &raw, &out, &st, &ex, sv->compute)
                                 : isp_b200_batch_add(sv->batch_builder, s.camera, &raw, &out, &st, &ex);
    if (status != ISP_OK) {
      e = cudaErrorLaunchFailure;
      step = isp_b200_last_error();
    }
  }
  if (e == cudaSuccess && !per_frame &&
      isp_b200_batch_launch(sv->batch_builder, sv->compute, sv->config.use_graph) != ISP_OK) {
    e = cudaErrorLaunchFailure;
    step = isp_b200_last_error();
  }
  // Result copies, where asked, on the readback stream so that the next
  // batch's kernels do not queue behind them.
  bool readback = false;
  for (const InFlight& f : batch->frames) {
    const Stream& s = *sv->streams[static_cast<size_t>(f.stream)];
    readback = readback || f.req.host_out != nullptr || f.req.host_hist != nullptr || f.req.host_stats != nullptr ||
               s.shape.copy_back != 0;
  }
  cudaStream_t last = sv->compute;
  if (readback && e == cudaSuccess) {
    e = cudaEventRecord(batch->done, sv->compute);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sv->readback, batch->done, 0);
    last = sv->readback;
  }
  for (const InFlight& f : batch->frames) {
    if (e != cudaSuccess || !readback) break;
    Stream& s = *sv->streams[static_cast<size_t>(f.stream)];
    DeviceSlot& slot = s.slots[static_cast<size_t>(f.slot)];
    const bool mirror = s.shape.copy_back != 0 && f.req.host_out == nullptr && f.req.host_hist == nullptr &&
                        f.req.host_stats == nullptr;
    void* host_out = mirror ? slot.host_out : f.req.host_out;
    uint32_t* host_hist = mirror ? slot.host_hist : f.req.host_hist;
    float* host_stats = mirror ? slot.host_stats : f.req.host_stats;
    if (host_out != nullptr) {
      e = cudaMemcpyAsync(host_out, slot.out, s.out_row * static_cast<size_t>(s.shape.height), cudaMemcpyDeviceToHost,
                          sv->readback);
    }
    if (e == cudaSuccess && host_hist != nullptr && s.shape.with_histogram) {
      e = cudaMemcpyAsync(host_hist, slot.hist, ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS * 4U,
                          cudaMemcpyDeviceToHost, sv->readback);
    }
    if (e == cudaSuccess && host_stats != nullptr && s.shape.with_stats) {
      e = cudaMemcpyAsync(host_stats, slot.stats, ISP_STATS_SIZE * 4U, cudaMemcpyDeviceToHost, sv->readback);
    }
  }
  if (e == cudaSuccess) e = cudaEventRecord(batch->done, last);
  lock.lock();
  if (e != cudaSuccess) {
    worker_fail(sv, std::string("batch launch (") + step + ")", e);
    batch->failed = true;
  }
  return true;
}

bool launchable(const isp_b200_server* sv) {
  return static_cast<int>(sv->inflight.size()) < sv->config.max_inflight;
}

void worker_loop(isp_b200_server* sv) {
  cudaSetDevice(sv->device);
  std::unique_lock<std::mutex> lock(sv->mutex);
  for (;;) {
    const bool pending = !sv->inflight.empty() || sv->staged > 0;
    if (!sv->running && !pending) break;
    bool progress = reap(sv);
    if (sv->running) progress = admit(sv) || progress;
    while (launchable(sv) && launch_ready(sv, lock)) progress = true;
    if (progress) continue;
    if (pending) {
      lock.unlock();
      std::this_thread::yield();
      lock.lock();
    } else {
      sv->wake.wait_for(lock, std::chrono::milliseconds(2));
    }
  }
}

int add_frame(isp_b200_server* sv, int32_t stream, const void* host_raw, size_t pitch, void* host_out,
              uint32_t* host_hist, float* host_stats, int64_t arrival_ns, Source source, uint64_t* ticket) {
  std::unique_lock<std::mutex> lock(sv->mutex);
  if (!sv->running) return fail(ISP_ESTATE, "server is not running");
  if (stream < 0 || stream >= static_cast<int32_t>(sv->streams.size())) return fail(ISP_EINVAL, "unknown stream");
  Stream& s = *sv->streams[static_cast<size_t>(stream)];
  ++sv->submitted;
  if (static_cast<int>(s.queue.size() + s.admitted.size()) >= sv->config.queue_depth) {
    ++sv->refused;
    return fail(ISP_EBUSY, "stream queue full");
  }
  Request r{};
  r.ticket = sv->next_ticket++;
  r.frame = s.next_frame++;
  r.arrival_ns = arrival_ns > 0 ? arrival_ns : now_ns();
  r.host_out = host_out;
  r.host_hist = host_hist;
  r.host_stats = host_stats;
  r.staging = -1;
  r.on_device = source == Source::kDevice;
  if (source != Source::kCopy) {
    r.host_raw = host_raw;
    r.host_pitch = pitch;
  } else {
    int free_slot = -1;
    for (size_t i = 0; i < s.staging_busy.size(); ++i) {
      if (!s.staging_busy[i]) {
        free_slot = static_cast<int>(i);
        break;
      }
    }
    if (free_slot < 0) {
      ++sv->refused;
      return fail(ISP_EBUSY, "stream staging full");
    }
    s.staging_busy[static_cast<size_t>(free_slot)] = true;
    void* dst = s.staging[static_cast<size_t>(free_slot)];
    lock.unlock();
    for (int y = 0; y < s.shape.height; ++y) {
      std::memcpy(static_cast<char*>(dst) + static_cast<size_t>(y) * s.raw_row,
                  static_cast<const char*>(host_raw) + static_cast<size_t>(y) * pitch, s.raw_row);
    }
    lock.lock();
    r.host_raw = dst;
    r.host_pitch = s.raw_row;
    r.staging = free_slot;
  }
  if (sv->first_arrival_ns == 0 || r.arrival_ns < sv->first_arrival_ns) sv->first_arrival_ns = r.arrival_ns;
  s.queue.push_back(r);
  ++sv->queued;
  if (ticket != nullptr) *ticket = r.ticket;
  lock.unlock();
  sv->wake.notify_one();
  return ISP_OK;
}

// The stream's next synthetic source frame, submitted now (or at arrival_ns).
int submit_source(isp_b200_server* sv, int i, int64_t arrival_ns) {
  Stream& s = *sv->streams[static_cast<size_t>(i)];
  const void* src = s.sources[s.next_source];
  const int status = add_frame(sv, i, src, s.raw_pitch, nullptr, nullptr, nullptr, arrival_ns,
                               s.sources_on_device ? Source::kDevice : Source::kBorrowHost, nullptr);
  if (status == ISP_OK) s.next_source = (s.next_source + 1) % s.sources.size();
  return status;
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * static_cast<double>(v.size() - 1);
  const size_t i = static_cast<size_t>(pos);
  const double f = pos - static_cast<double>(i);
  return i + 1 < v.size() ? v[i] + f * (v[i + 1] - v[i]) : v[i];
}

}  // namespace

extern "C" {

void isp_b200_server_config_default(isp_server_config_c* c) {
  if (c == nullptr) return;
  *c = isp_server_config_c{};
  c->max_batch = 64;
  c->memory_budget = int64_t{8} << 30;
  c->max_inflight = 2;
  c->queue_depth = 4;
  c->slots_per_stream = 2;
  c->use_graph = 0;
  c->per_frame = 0;
}

int isp_b200_server_create(const isp_server_config_c* config, isp_b200_server** out) {
  if (out == nullptr || config == nullptr) return fail(ISP_EINVAL, "config or out is null");
  *out = nullptr;
  if (config->max_batch < 1 || config->max_batch > 4096 || config->max_inflight < 1 || config->max_inflight > 8 ||
      config->queue_depth < 1 || config->slots_per_stream < 1 || config->memory_budget <= 0) {
    return fail(ISP_EINVAL, "server config out of range");
  }
  auto* sv = new isp_b200_server;
  sv->config = *config;
  cudaError_t e = cudaGetDevice(&sv->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->compute, cudaStreamNonBlocking);
  for (cudaStream_t& cs : sv->copy) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->readback, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    isp_b200_server_destroy(sv);
    return fail_cuda(e, "isp_b200_server_create");
  }
  if (const int status = isp_b200_batch_create(config->max_batch, &sv->batch_builder); status != ISP_OK) {
    isp_b200_server_destroy(sv);
    return status;
  }
  *out = sv;
  clear_error();
  return ISP_OK;
}

int isp_b200_server_add_stream(isp_b200_server* sv, const isp_params_c* params, const isp_server_stream_c* shape,
                               int32_t* id) {
  if (sv == nullptr || params == nullptr || shape == nullptr) return fail(ISP_EINVAL, "server, params or shape is null");
  if (sv->started) return fail(ISP_ESTATE, "streams are added before the server starts");
  auto s = std::make_unique<Stream>();
  s->shape = *shape;
  // The frame shape must be a valid raw view for these settings.
  isp_raw_view_c probe{reinterpret_cast<const void*>(uintptr_t{256}), shape->width, shape->height,
                       raw_row_bytes(shape->format, shape->width), shape->format, shape->bit_depth, shape->pattern};
  if (const std::string why = validate_raw(probe, *params); !why.empty()) return fail(ISP_EINVAL, why);
  if (shape->out_format < ISP_OUT_RGB8 || shape->out_format > ISP_OUT_RGB32F) return fail(ISP_EINVAL, "output format unknown");
  s->raw_row = raw_row_bytes(shape->format, shape->width);
  s->raw_pitch = (s->raw_row + 15U) & ~size_t{15};
  const size_t cb = shape->out_format == ISP_OUT_RGB16 ? 2U : shape->out_format == ISP_OUT_RGB32F ? 4U : 1U;
  s->out_row = static_cast<size_t>(shape->width) * (shape->out_format == ISP_OUT_RGBA8 ? 4U : 3U) * cb;
  s->frame_bytes = s->raw_pitch * static_cast<size_t>(shape->height) + s->out_row * static_cast<size_t>(shape->height);
  if (static_cast<int64_t>(s->frame_bytes) > sv->config.memory_budget) {
    return fail(ISP_EINVAL, "a frame of this stream is larger than the memory budget");
  }
  if (const int status = isp_b200_create(params, &s->camera); status != ISP_OK) return status;
  cudaError_t e = cudaSuccess;
  s->slots.resize(static_cast<size_t>(sv->config.slots_per_stream));
  for (DeviceSlot& d : s->slots) {
    if (e == cudaSuccess) e = cudaMalloc(&d.raw, s->raw_pitch * static_cast<size_t>(shape->height));
    if (e == cudaSuccess) e = cudaMalloc(&d.out, s->out_row * static_cast<size_t>(shape->height));
    if (e == cudaSuccess) e = cudaMalloc(&d.hist, ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS * 4U);
    if (e == cudaSuccess) e = cudaMalloc(&d.stats, ISP_STATS_SIZE * 4U);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d.copied, cudaEventDisableTiming);
    if (shape->copy_back != 0) {
      if (e == cudaSuccess) e = cudaMallocHost(&d.host_out, s->out_row * static_cast<size_t>(shape->height));
      if (e == cudaSuccess) e = cudaMallocHost(&d.host_hist, ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS * 4U);
      if (e == cudaSuccess) e = cudaMallocHost(&d.host_stats, ISP_STATS_SIZE * 4U);
    }
  }
  s->staging.resize(static_cast<size_t>(sv->config.queue_depth), nullptr);
  s->staging_busy.assign(static_cast<size_t>(sv->config.queue_depth), false);
  for (void*& h : s->staging) {
    if (e == cudaSuccess) e = cudaMallocHost(&h, s->raw_row * static_cast<size_t>(shape->height));
  }
  if (e != cudaSuccess) {
    release_stream(s.get());
    return fail_cuda(e, "isp_b200_server_add_stream");
  }
  *id = static_cast<int32_t>(sv->streams.size());
  sv->streams.push_back(std::move(s));
  clear_error();
  return ISP_OK;
}

int isp_b200_server_start(isp_b200_server* sv) {
  if (sv == nullptr) return fail(ISP_EINVAL, "server is null");
  if (sv->started) return fail(ISP_ESTATE, "server already started");
  if (sv->streams.empty()) return fail(ISP_EINVAL, "server has no streams");
  sv->started = true;
  sv->running = true;
  sv->worker = std::thread(worker_loop, sv);
  clear_error();
  return ISP_OK;
}

int isp_b200_server_submit(isp_b200_server* sv, int32_t stream, const void* host_raw, size_t pitch, void* host_out,
                           uint32_t* host_histogram, float* host_stats, int64_t arrival_ns, uint64_t* ticket) {
  if (sv == nullptr || host_raw == nullptr) return fail(ISP_EINVAL, "server or raw is null");
  const int status =
      add_frame(sv, stream, host_raw, pitch, host_out, host_histogram, host_stats, arrival_ns, Source::kCopy, ticket);
  if (status == ISP_OK) clear_error();
  return status;
}

int isp_b200_server_submit_device(isp_b200_server* sv, int32_t stream, const void* device_raw, size_t pitch,
                                  void* host_out, uint32_t* host_histogram, float* host_stats, int64_t arrival_ns,
                                  uint64_t* ticket) {
  if (sv == nullptr || device_raw == nullptr) return fail(ISP_EINVAL, "server or raw is null");
  if (stream >= 0 && stream < static_cast<int32_t>(sv->streams.size()) &&
      pitch < sv->streams[static_cast<size_t>(stream)]->raw_row) {
    return fail(ISP_EINVAL, "raw pitch is smaller than a row");
  }
  const int status =
      add_frame(sv, stream, device_raw, pitch, host_out, host_histogram, host_stats, arrival_ns, Source::kDevice, ticket);
  if (status == ISP_OK) clear_error();
  return status;
}

int isp_b200_server_poll(isp_b200_server* sv, isp_server_result_c* out, int32_t capacity, int32_t* count) {
  if (sv == nullptr || count == nullptr) return fail(ISP_EINVAL, "server or count is null");
  std::lock_guard<std::mutex> lock(sv->mutex);
  int32_t n = 0;
  while (n < capacity && !sv->results.empty()) {
    out[n++] = sv->results.front();
    sv->results.pop_front();
  }
  *count = n;
  clear_error();
  return ISP_OK;
}

int isp_b200_server_drain(isp_b200_server* sv, int64_t timeout_ns) {
  if (sv == nullptr) return fail(ISP_EINVAL, "server is null");
  const int64_t deadline = now_ns() + timeout_ns;
  for (;;) {
    {
      std::lock_guard<std::mutex> lock(sv->mutex);
      if (sv->inflight.empty() && sv->staged == 0 && sv->queued == 0) break;
      if (!sv->worker_error.empty()) return fail(ISP_ECUDA, sv->worker_error);
    }
    if (now_ns() > deadline) return fail(ISP_ETIMEOUT, "server drain timed out");
    sv->wake.notify_one();
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
  std::lock_guard<std::mutex> lock(sv->mutex);
  if (!sv->worker_error.empty()) return fail(ISP_ECUDA, sv->worker_error);
  clear_error();
  return ISP_OK;
}

int isp_b200_server_stats(isp_b200_server* sv, isp_server_stats_c* st) {
  if (sv == nullptr || st == nullptr) return fail(ISP_EINVAL, "server or stats is null");
  std::lock_guard<std::mutex> lock(sv->mutex);
  std::memset(st, 0, sizeof(*st));
  st->submitted = sv->submitted;
  st->refused = sv->refused;
  st->admitted = sv->admitted;
  st->completed = sv->completed;
  st->batches = sv->batches;
  st->mean_batch_frames = sv->batches > 0 ? static_cast<double>(sv->batch_frames) / sv->batches : 0.0;
  st->p50_ms = percentile(sv->latencies_ms, 0.50);
  st->p99_ms = percentile(sv->latencies_ms, 0.99);
  st->p999_ms = percentile(sv->latencies_ms, 0.999);
  st->max_ms = sv->latencies_ms.empty() ? 0.0 : *std::max_element(sv->latencies_ms.begin(), sv->latencies_ms.end());
  const double span = static_cast<double>(sv->last_done_ns - sv->first_arrival_ns) * 1e-9;
  st->gpix_per_s = span > 0.0 ? static_cast<double>(sv->completed_pixels) / span * 1e-9 : 0.0;
  st->completed_pixels = sv->completed_pixels;
  st->error = sv->worker_error.empty() ? 0 : 1;
  st->p50_wait_ms = percentile(sv->waits_ms, 0.50);
  st->p99_wait_ms = percentile(sv->waits_ms, 0.99);
  clear_error();
  return ISP_OK;
}

int isp_b200_server_reset_stats(isp_b200_server* sv) {
  if (sv == nullptr) return fail(ISP_EINVAL, "server is null");
  std::lock_guard<std::mutex> lock(sv->mutex);
  sv->latencies_ms.clear();
  sv->waits_ms.clear();
  sv->submitted = sv->refused = sv->admitted = sv->completed = sv->completed_pixels = 0;
  sv->batches = sv->batch_frames = 0;
  sv->first_arrival_ns = sv->last_done_ns = 0;
  sv->results.clear();
  clear_error();
  return ISP_OK;
}

int isp_b200_server_add_source(isp_b200_server* sv, int32_t stream, const void* host_raw, size_t pitch,
                               int32_t on_device) {
  if (sv == nullptr || host_raw == nullptr) return fail(ISP_EINVAL, "server or raw is null");
  if (stream < 0 || stream >= static_cast<int32_t>(sv->streams.size())) return fail(ISP_EINVAL, "unknown stream");
  Stream& s = *sv->streams[static_cast<size_t>(stream)];
  if (pitch < s.raw_row) return fail(ISP_EINVAL, "raw pitch is smaller than a row");
  if (!s.sources.empty() && s.sources_on_device != (on_device != 0)) {
    return fail(ISP_EINVAL, "a stream's sources are all on the host or all on the device");
  }
  std::lock_guard<std::mutex> lock(sv->mutex);
  const size_t bytes = s.raw_pitch * static_cast<size_t>(s.shape.height);
  void* dst = nullptr;
  cudaError_t e = on_device != 0 ? cudaMalloc(&dst, bytes) : cudaMallocHost(&dst, bytes);
  if (e != cudaSuccess) return fail_cuda(e, on_device != 0 ? "cudaMalloc" : "cudaMallocHost");
  if (on_device != 0) {
    e = cudaMemcpy2D(dst, s.raw_pitch, host_raw, pitch, s.raw_row, static_cast<size_t>(s.shape.height),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(dst);
      return fail_cuda(e, "isp_b200_server_add_source");
    }
  } else {
    for (int y = 0; y < s.shape.height; ++y) {
      std::memcpy(static_cast<char*>(dst) + static_cast<size_t>(y) * s.raw_pitch,
                  static_cast<const char*>(host_raw) + static_cast<size_t>(y) * pitch, s.raw_row);
    }
  }
  s.sources.push_back(dst);
  s.sources_on_device = on_device != 0;
  clear_error();
  return ISP_OK;
}

int isp_b200_server_run_poisson(isp_b200_server* sv, const double* fps, double seconds, uint64_t seed) {
  if (sv == nullptr || fps == nullptr || !(seconds > 0.0)) return fail(ISP_EINVAL, "server, fps or seconds invalid");
  const int n = static_cast<int>(sv->streams.size());
  for (int i = 0; i < n; ++i) {
    if (sv->streams[static_cast<size_t>(i)]->sources.empty()) return fail(ISP_EINVAL, "a stream has no source frame");
    if (!(fps[i] > 0.0)) return fail(ISP_EINVAL, "frame rates must be positive");
  }
  std::mt19937_64 rng(seed);
  const int64_t start = now_ns();
  const int64_t end = start + static_cast<int64_t>(seconds * 1e9);
  std::vector<int64_t> next(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) {
    std::exponential_distribution<double> gap(fps[i]);
    next[static_cast<size_t>(i)] = start + static_cast<int64_t>(gap(rng) * 1e9);
  }
  for (;;) {
    const auto it = std::min_element(next.begin(), next.end());
    const int i = static_cast<int>(it - next.begin());
    const int64_t t = *it;
    if (t >= end) break;
    // Sleep to within 100 us of the arrival, then spin to it.
    int64_t now = now_ns();
    if (t - now > 150000) std::this_thread::sleep_for(std::chrono::nanoseconds(t - now - 100000));
    while ((now = now_ns()) < t) {
    }
    const int status = submit_source(sv, i, t);
    if (status != ISP_OK && status != ISP_EBUSY) return status;
    std::exponential_distribution<double> gap(fps[i]);
    *it = t + static_cast<int64_t>(gap(rng) * 1e9);
  }
  clear_error();
  return ISP_OK;
}

int isp_b200_server_run_closed(isp_b200_server* sv, double seconds) {
  if (sv == nullptr || !(seconds > 0.0)) return fail(ISP_EINVAL, "server or seconds invalid");
  const int n = static_cast<int>(sv->streams.size());
  for (int i = 0; i < n; ++i) {
    if (sv->streams[static_cast<size_t>(i)]->sources.empty()) return fail(ISP_EINVAL, "a stream has no source frame");
  }
  const int64_t end = now_ns() + static_cast<int64_t>(seconds * 1e9);
  while (now_ns() < end) {
    for (int i = 0; i < n; ++i) {
      for (;;) {
        {
          std::lock_guard<std::mutex> lock(sv->mutex);
          if (!sv->worker_error.empty()) return fail(ISP_ECUDA, sv->worker_error);
          const Stream& s = *sv->streams[static_cast<size_t>(i)];
          if (static_cast<int>(s.queue.size() + s.admitted.size()) >= sv->config.queue_depth) break;
        }
        const int status = submit_source(sv, i, 0);
        if (status != ISP_OK) return status;
      }
    }
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  clear_error();
  return ISP_OK;
}

void isp_b200_server_destroy(isp_b200_server* sv) {
  if (sv == nullptr) return;
  {
    std::lock_guard<std::mutex> lock(sv->mutex);
    sv->running = false;
  }
  sv->wake.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  for (cudaStream_t s : {sv->compute, sv->copy[0], sv->copy[1], sv->copy[2], sv->readback}) {
    if (s != nullptr) cudaStreamSynchronize(s);
  }
  for (auto& b : sv->inflight) {
    if (b->done != nullptr) cudaEventDestroy(b->done);
  }
  for (cudaEvent_t ev : sv->spare_events) cudaEventDestroy(ev);
  for (auto& s : sv->streams) release_stream(s.get());
  isp_b200_batch_destroy(sv->batch_builder);
  for (cudaStream_t s : {sv->compute, sv->copy[0], sv->copy[1], sv->copy[2], sv->readback}) {
    if (s != nullptr) cudaStreamDestroy(s);
  }
  delete sv;
}

}  // extern "C"
