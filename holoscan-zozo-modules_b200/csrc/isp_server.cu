// isp_server.cu - serving many camera streams with continuous batching
// (include/isp_b200.h, isp_b200_server_*).
//
// Each stream is a camera: a pipeline whose state (tone table, lens shading
// grid, white balance and scratch) stays on the device, a ring of device
// slots for its frames in flight, and a host queue of frames that arrived
// and wait for the GPU. A worker thread runs the loop:
//   1. reap batches whose completion the GPU has signalled: their frames'
//      slots and budget bytes free up, their results (with the time the GPU
//      finished them) become pollable;
//   2. while fewer than max_inflight batches are on the GPU and frames wait,
//      form a batch from whatever is queued - the oldest waiting frame of
//      each stream, streams taken round robin, a frame admitted only while
//      the bytes of the frames in flight stay within the memory budget and
//      its stream has a free slot - copy each admitted frame from pinned
//      host memory to its slot (copy stream), and launch the batch (compute
//      stream, one statistics pass and one tile pass) followed by a host
//      function that stamps the batch's completion time;
//   3. otherwise sleep until a frame arrives or a batch may have finished.
// Requests that arrive while batches run join the next batch as soon as a
// batch slot frees: the GPU always has the next batch queued behind the
// running one. A frame's latency is its arrival time to the completion of
// its batch's tile pass (its image, histogram and statistics are then in
// device memory; with result copies requested, to the end of those copies).
// Frames of one stream run in arrival order (its pipeline's event orders
// its batches), one per batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
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

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  uint64_t ticket;
  uint64_t frame;
  int64_t arrival_ns;
  const void* host_raw;  // pinned memory the frame is copied from
  size_t host_pitch;
  void* host_out;  // optional result copies
  uint32_t* host_hist;
  float* host_stats;
  int staging;  // index of the stream's staging buffer holding the raw, or -1 (borrowed)
};

struct DeviceSlot {
  void* raw = nullptr;
  void* out = nullptr;
  uint32_t* hist = nullptr;
  float* stats = nullptr;
  bool busy = false;
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
  std::deque<Request> queue;
  uint64_t next_frame = 0;
  void* source = nullptr;  // pinned frame the synthetic driver submits
  size_t source_pitch = 0;
};

struct InFlight {
  int stream;
  int slot;
  Request req;
};

struct Batch {
  std::vector<InFlight> frames;
  cudaEvent_t done = nullptr;
  int64_t done_ns = 0;  // stamped by the host function when the GPU reaches it
  std::atomic<int> finished{0};
  int64_t pixels = 0;
};

void CUDART_CB stamp(void* data) {
  auto* b = static_cast<Batch*>(data);
  b->done_ns = now_ns();
  b->finished.store(1, std::memory_order_release);
}

}  // namespace

struct isp_b200_server {
  isp_server_config_c config{};
  int device = 0;
  std::vector<std::unique_ptr<Stream>> streams;
  isp_b200_batch* batch_builder = nullptr;
  cudaStream_t compute = nullptr;
  cudaStream_t copy = nullptr;
  std::mutex mutex;  // streams' queues, results, counters
  std::condition_variable wake;
  std::thread worker;
  bool running = false;
  bool started = false;
  std::deque<std::unique_ptr<Batch>> inflight;
  std::vector<cudaEvent_t> copied;  // per batch position: the H2D copies of a batch
  int64_t inflight_bytes = 0;
  int next_stream = 0;  // round-robin start
  uint64_t next_ticket = 1;
  std::deque<isp_server_result_c> results;
  std::vector<double> latencies_ms;
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
  }
  for (void* h : s->staging) cudaFreeHost(h);
  cudaFreeHost(s->source);
  isp_b200_destroy(s->camera);
}

// Reaps finished batches (oldest first). Caller holds the mutex.
void reap(isp_b200_server* sv) {
  while (!sv->inflight.empty() && sv->inflight.front()->finished.load(std::memory_order_acquire) != 0) {
    std::unique_ptr<Batch> b = std::move(sv->inflight.front());
    sv->inflight.pop_front();
    for (const InFlight& f : b->frames) {
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
      r.done_ns = b->done_ns;
      r.image = slot.out;
      r.histogram = slot.hist;
      r.stats = slot.stats;
      sv->results.push_back(r);
      sv->latencies_ms.push_back(static_cast<double>(b->done_ns - f.req.arrival_ns) * 1e-6);
      ++sv->completed;
      sv->completed_pixels += static_cast<int64_t>(s.shape.width) * s.shape.height;
      sv->last_done_ns = std::max(sv->last_done_ns, b->done_ns);
    }
    cudaEventDestroy(b->done);
  }
}

// Forms and launches one batch from the queues. Caller holds the mutex;
// returns false when nothing could be admitted.
bool launch_next(isp_b200_server* sv, std::unique_lock<std::mutex>& lock) {
  const int n = static_cast<int>(sv->streams.size());
  auto b = std::make_unique<Batch>();
  for (int k = 0; k < n && static_cast<int>(b->frames.size()) < sv->config.max_batch; ++k) {
    const int si = (sv->next_stream + k) % n;
    Stream& s = *sv->streams[static_cast<size_t>(si)];
    if (s.queue.empty()) continue;
    if (sv->inflight_bytes + static_cast<int64_t>(s.frame_bytes) > sv->config.memory_budget) continue;
    int slot = -1;
    for (size_t d = 0; d < s.slots.size(); ++d) {
      if (!s.slots[d].busy) {
        slot = static_cast<int>(d);
        break;
      }
    }
    if (slot < 0) continue;
    s.slots[static_cast<size_t>(slot)].busy = true;
    sv->inflight_bytes += static_cast<int64_t>(s.frame_bytes);
    b->frames.push_back(InFlight{si, slot, s.queue.front()});
    s.queue.pop_front();
    b->pixels += static_cast<int64_t>(s.shape.width) * s.shape.height;
  }
  if (b->frames.empty()) return false;
  sv->next_stream = (sv->next_stream + 1) % n;
  sv->admitted += static_cast<int64_t>(b->frames.size());
  Batch* raw_batch = b.get();
  sv->inflight.push_back(std::move(b));
  lock.unlock();
  // CUDA work outside the lock: submitters only touch the queues.
  cudaError_t e = cudaSuccess;
  isp_b200_batch_clear(sv->batch_builder);
  for (const InFlight& f : raw_batch->frames) {
    Stream& s = *sv->streams[static_cast<size_t>(f.stream)];
    DeviceSlot& slot = s.slots[static_cast<size_t>(f.slot)];
    if (e == cudaSuccess) {
      e = cudaMemcpy2DAsync(slot.raw, s.raw_pitch, f.req.host_raw, f.req.host_pitch, s.raw_row,
                            static_cast<size_t>(s.shape.height), cudaMemcpyHostToDevice, sv->copy);
    }
    const isp_raw_view_c raw{slot.raw, s.shape.width, s.shape.height, s.raw_pitch, s.shape.format,
                             s.shape.bit_depth, s.shape.pattern};
    const isp_rgb_view_c out{slot.out, s.out_row, s.shape.out_format};
    const isp_stats_c st{s.shape.with_histogram ? slot.hist : nullptr, s.shape.with_stats ? slot.stats : nullptr};
    const isp_exposure_c ex{0, 0.0F};
    if (e == cudaSuccess && isp_b200_batch_add(sv->batch_builder, s.camera, &raw, &out, &st, &ex) != ISP_OK) {
      e = cudaErrorInvalidValue;
    }
  }
  cudaEvent_t copied = nullptr;
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&copied, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(copied, sv->copy);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(sv->compute, copied, 0);
  if (e == cudaSuccess && isp_b200_batch_launch(sv->batch_builder, sv->compute, sv->config.use_graph) != ISP_OK) {
    e = cudaErrorLaunchFailure;
  }
  // Result copies, when the frames asked for them.
  for (const InFlight& f : raw_batch->frames) {
    if (e != cudaSuccess) break;
    Stream& s = *sv->streams[static_cast<size_t>(f.stream)];
    DeviceSlot& slot = s.slots[static_cast<size_t>(f.slot)];
    if (f.req.host_out != nullptr) {
      e = cudaMemcpyAsync(f.req.host_out, slot.out, s.out_row * static_cast<size_t>(s.shape.height),
                          cudaMemcpyDeviceToHost, sv->compute);
    }
    if (e == cudaSuccess && f.req.host_hist != nullptr && s.shape.with_histogram) {
      e = cudaMemcpyAsync(f.req.host_hist, slot.hist, ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS * 4U,
                          cudaMemcpyDeviceToHost, sv->compute);
    }
    if (e == cudaSuccess && f.req.host_stats != nullptr && s.shape.with_stats) {
      e = cudaMemcpyAsync(f.req.host_stats, slot.stats, ISP_STATS_SIZE * 4U, cudaMemcpyDeviceToHost, sv->compute);
    }
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&raw_batch->done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(raw_batch->done, sv->compute);
  if (e == cudaSuccess) e = cudaLaunchHostFunc(sv->compute, stamp, raw_batch);
  if (copied != nullptr) cudaEventDestroy(copied);  // destruction waits for the recorded work
  lock.lock();
  if (e != cudaSuccess) {
    sv->worker_error = std::string("batch launch: ") + cudaGetErrorString(e) + " " + isp_b200_last_error();
    raw_batch->done_ns = now_ns();
    raw_batch->finished.store(1);
  }
  ++sv->batches;
  sv->batch_frames += static_cast<int64_t>(raw_batch->frames.size());
  return true;
}

void worker_loop(isp_b200_server* sv) {
  cudaSetDevice(sv->device);
  std::unique_lock<std::mutex> lock(sv->mutex);
  while (sv->running || !sv->inflight.empty()) {
    reap(sv);
    bool launched = false;
    while (sv->running && static_cast<int>(sv->inflight.size()) < sv->config.max_inflight) {
      if (!launch_next(sv, lock)) break;
      launched = true;
    }
    if (launched) continue;
    // Nothing to launch now: wait for an arrival, or briefly for a batch.
    sv->wake.wait_for(lock, std::chrono::microseconds(sv->inflight.empty() ? 2000 : 50));
  }
}

int add_frame(isp_b200_server* sv, int32_t stream, const void* host_raw, size_t pitch, void* host_out,
              uint32_t* host_hist, float* host_stats, int64_t arrival_ns, bool borrow, uint64_t* ticket) {
  std::unique_lock<std::mutex> lock(sv->mutex);
  if (!sv->running) return fail(ISP_ESTATE, "server is not running");
  if (stream < 0 || stream >= static_cast<int32_t>(sv->streams.size())) return fail(ISP_EINVAL, "unknown stream");
  Stream& s = *sv->streams[static_cast<size_t>(stream)];
  ++sv->submitted;
  if (static_cast<int>(s.queue.size()) >= sv->config.queue_depth) {
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
  if (borrow) {
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
  if (ticket != nullptr) *ticket = r.ticket;
  lock.unlock();
  sv->wake.notify_one();
  return ISP_OK;
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
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->copy, cudaStreamNonBlocking);
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
  if (const int status = isp_b200_create(params, &s->camera); status != ISP_OK) return status;
  s->raw_row = raw_row_bytes(shape->format, shape->width);
  s->raw_pitch = (s->raw_row + 15U) & ~size_t{15};
  const size_t cb = shape->out_format == ISP_OUT_RGB16 ? 2U : shape->out_format == ISP_OUT_RGB32F ? 4U : 1U;
  s->out_row = static_cast<size_t>(shape->width) * (shape->out_format == ISP_OUT_RGBA8 ? 4U : 3U) * cb;
  s->frame_bytes = s->raw_pitch * static_cast<size_t>(shape->height) + s->out_row * static_cast<size_t>(shape->height);
  cudaError_t e = cudaSuccess;
  s->slots.resize(static_cast<size_t>(sv->config.slots_per_stream));
  for (DeviceSlot& d : s->slots) {
    if (e == cudaSuccess) e = cudaMalloc(&d.raw, s->raw_pitch * static_cast<size_t>(shape->height));
    if (e == cudaSuccess) e = cudaMalloc(&d.out, s->out_row * static_cast<size_t>(shape->height));
    if (e == cudaSuccess) e = cudaMalloc(&d.hist, ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS * 4U);
    if (e == cudaSuccess) e = cudaMalloc(&d.stats, ISP_STATS_SIZE * 4U);
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
  const int status = add_frame(sv, stream, host_raw, pitch, host_out, host_histogram, host_stats, arrival_ns, false, ticket);
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
      bool idle = sv->inflight.empty();
      for (const auto& s : sv->streams) idle = idle && s->queue.empty();
      if (idle) break;
      if (!sv->worker_error.empty()) return fail(ISP_ECUDA, sv->worker_error);
    }
    if (now_ns() > deadline) return fail(ISP_ETIMEOUT, "server drain timed out");
    sv->wake.notify_one();
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
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
  clear_error();
  return ISP_OK;
}

int isp_b200_server_reset_stats(isp_b200_server* sv) {
  if (sv == nullptr) return fail(ISP_EINVAL, "server is null");
  std::lock_guard<std::mutex> lock(sv->mutex);
  sv->latencies_ms.clear();
  sv->submitted = sv->refused = sv->admitted = sv->completed = sv->completed_pixels = 0;
  sv->batches = sv->batch_frames = 0;
  sv->first_arrival_ns = sv->last_done_ns = 0;
  sv->results.clear();
  clear_error();
  return ISP_OK;
}

int isp_b200_server_set_source(isp_b200_server* sv, int32_t stream, const void* host_raw, size_t pitch) {
  if (sv == nullptr || host_raw == nullptr) return fail(ISP_EINVAL, "server or raw is null");
  if (stream < 0 || stream >= static_cast<int32_t>(sv->streams.size())) return fail(ISP_EINVAL, "unknown stream");
  Stream& s = *sv->streams[static_cast<size_t>(stream)];
  if (s.source == nullptr) {
    const cudaError_t e = cudaMallocHost(&s.source, s.raw_row * static_cast<size_t>(s.shape.height));
    if (e != cudaSuccess) return fail_cuda(e, "cudaMallocHost");
  }
  for (int y = 0; y < s.shape.height; ++y) {
    std::memcpy(static_cast<char*>(s.source) + static_cast<size_t>(y) * s.raw_row,
                static_cast<const char*>(host_raw) + static_cast<size_t>(y) * pitch, s.raw_row);
  }
  s.source_pitch = s.raw_row;
  clear_error();
  return ISP_OK;
}

int isp_b200_server_run_poisson(isp_b200_server* sv, const double* fps, double seconds, uint64_t seed) {
  if (sv == nullptr || fps == nullptr || !(seconds > 0.0)) return fail(ISP_EINVAL, "server, fps or seconds invalid");
  const int n = static_cast<int>(sv->streams.size());
  for (int i = 0; i < n; ++i) {
    if (sv->streams[static_cast<size_t>(i)]->source == nullptr) return fail(ISP_EINVAL, "a stream has no source frame");
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
    Stream& s = *sv->streams[static_cast<size_t>(i)];
    const int status = add_frame(sv, i, s.source, s.source_pitch, nullptr, nullptr, nullptr, t, true, nullptr);
    if (status != ISP_OK && status != ISP_EBUSY) return status;
    std::exponential_distribution<double> gap(fps[i]);
    *it = t + static_cast<int64_t>(gap(rng) * 1e9);
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
  if (sv->compute != nullptr) cudaStreamSynchronize(sv->compute);
  if (sv->copy != nullptr) cudaStreamSynchronize(sv->copy);
  for (auto& s : sv->streams) release_stream(s.get());
  isp_b200_batch_destroy(sv->batch_builder);
  if (sv->compute != nullptr) cudaStreamDestroy(sv->compute);
  if (sv->copy != nullptr) cudaStreamDestroy(sv->copy);
  delete sv;
}

}  // extern "C"
