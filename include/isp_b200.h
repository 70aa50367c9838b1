/*
 * isp_b200.h - the C ABI of the B200 image signal processor.
 *
 * A raw Bayer mosaic in, RGB out, with optional histograms and statistics,
 * computed by sm_100a kernels bit for bit as the holoscan::isp CPU backend
 * computes them. Plain C: pointers, sizes and PODs, no CUDA or C++ types, so
 * that any language with a C FFI (ctypes, cgo, JNI, N-API) can bind it.
 *
 * Every entry point returns an isp_status (0 on success). On failure the
 * message of the calling thread's last error is in isp_b200_last_error().
 *
 * Reference interfaces replaced (paths inside the holoscan-zozo-modules tree):
 *   modules/isp/include/holoscan/isp/isp_params.hpp:21-198   enums, IspParams, views, layouts
 *   modules/isp/include/holoscan/isp/isp_pipeline.hpp:39-74  class IspPipeline
 *   modules/isp/src/isp_params.cpp:85-237                     validate_params, tone_lut,
 *                                                             raw_row_bytes, validate_raw
 */
#ifndef ISP_B200_H_
#define ISP_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ISP_B200_API __attribute__((visibility("default")))
#else
#define ISP_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ISP_B200_ABI_VERSION 1

/* Status codes. ISP_EINVAL is std::invalid_argument in the reference façade
 * (isp_pipeline.hpp:41-44), ISP_ECUDA its std::runtime_error from a CUDA failure. */
typedef enum isp_status {
  ISP_OK = 0,
  ISP_EINVAL = 1,   /* A setting or a view is not usable. */
  ISP_ECUDA = 2,    /* A CUDA call failed; isp_b200_last_cuda_error() has its code. */
  ISP_ETIMEOUT = 3, /* A bounded wait ran out (device spin or host poll). */
  ISP_EBUSY = 4,    /* Admission refused: the memory budget or the queue is full. */
  ISP_ESTATE = 5    /* The call does not fit the object's state (e.g. closed server). */
} isp_status;

/* Enumerations, with the reference's numbering (isp_params.hpp:21-61). */
enum { ISP_BAYER_RGGB = 0, ISP_BAYER_BGGR = 1, ISP_BAYER_GRBG = 2, ISP_BAYER_GBRG = 3 };
enum { ISP_RAW_U8 = 0, ISP_RAW_U16 = 1, ISP_RAW_RAW10 = 2, ISP_RAW_RAW12 = 3 };
enum { ISP_DEMOSAIC_BILINEAR = 0, ISP_DEMOSAIC_MALVAR = 1 };
enum { ISP_WB_MANUAL = 0, ISP_WB_GRAY_WORLD = 1, ISP_WB_WHITE_PATCH = 2 };
enum { ISP_TONE_SRGB = 0, ISP_TONE_GAMMA = 1, ISP_TONE_LINEAR = 2, ISP_TONE_LUT = 3 };
enum { ISP_OUT_RGB8 = 0, ISP_OUT_RGBA8 = 1, ISP_OUT_RGB16 = 2, ISP_OUT_RGB32F = 3 };

/* Layouts of the outputs (isp_params.hpp:166-198): histogram rows luma, R, G, B of
 * 256 bins each; a 12-float statistics vector, layout version 1. */
#define ISP_HISTOGRAM_BINS 256
#define ISP_HISTOGRAM_CHANNELS 4
#define ISP_STATS_SIZE 12
#define ISP_STATS_LAYOUT_VERSION 1
#define ISP_TONE_LUT_SIZE 4097

/* AutoExposureParams (isp_params.hpp:82-93). */
typedef struct isp_auto_exposure_c {
  float target;
  float damping;
  int64_t min_exposure_ns;
  int64_t max_exposure_ns;
  float min_gain;
  float max_gain;
} isp_auto_exposure_c;

/* IspParams (isp_params.hpp:95-121). The optionals carry a has_ flag; the
 * vectors are borrowed pointers with counts, read only during the call that
 * takes them (create copies what it keeps). */
typedef struct isp_params_c {
  float black_level;
  int32_t has_channel_black_levels;
  float channel_black_levels[4];
  float white_level;
  int32_t has_lens_shading;
  int32_t lsc_width;      /* grid points across, 2..256 */
  int32_t lsc_height;     /* grid points down, 2..256 */
  int32_t lsc_channels;   /* 1 or 4 */
  const float* lsc_gains; /* [height][width][channels] */
  size_t lsc_gains_count;
  int32_t white_balance;
  float wb_gains[3];
  float awb_smoothing;
  float white_patch_percentile;
  int32_t demosaic;
  float ccm[9];
  int32_t tone_curve;
  float gamma;
  const float* lut; /* ISP_TONE_LUT: 2..65536 entries */
  size_t lut_size;
  float sharpen;
  isp_auto_exposure_c auto_exposure;
} isp_params_c;

/* RawImageView (isp_params.hpp:132-140). pitch is the row stride in bytes. */
typedef struct isp_raw_view_c {
  const void* data;
  int32_t width;
  int32_t height;
  size_t pitch;
  int32_t format;
  int32_t bit_depth;
  int32_t pattern;
} isp_raw_view_c;

/* RgbImageView (isp_params.hpp:143-147). */
typedef struct isp_rgb_view_c {
  void* data;
  size_t pitch;
  int32_t format;
} isp_rgb_view_c;

/* StatsOutput (isp_params.hpp:151-154); either pointer may be null. */
typedef struct isp_stats_c {
  uint32_t* histogram; /* ISP_HISTOGRAM_CHANNELS x ISP_HISTOGRAM_BINS */
  float* stats;        /* ISP_STATS_SIZE */
} isp_stats_c;

/* FrameExposure (isp_params.hpp:157-160); 0 is unknown. */
typedef struct isp_exposure_c {
  int64_t exposure_ns;
  float gain;
} isp_exposure_c;

typedef struct isp_b200_pipeline isp_b200_pipeline;

/* ---- Library ---------------------------------------------------------- */

/* ISP_B200_ABI_VERSION of the loaded library. No reference counterpart. */
ISP_B200_API int isp_b200_abi_version(void);

/* The calling thread's last error message ("" after success). */
ISP_B200_API const char* isp_b200_last_error(void);

/* The cudaError_t of the calling thread's last ISP_ECUDA, else 0. */
ISP_B200_API int isp_b200_last_cuda_error(void);

/* ---- Settings (isp_params.cpp) ------------------------------------------ */

/* IspParams{} defaults (isp_params.hpp:95-121). */
ISP_B200_API void isp_b200_params_default(isp_params_c* params);

/* validate_params (isp_params.cpp:85-164): ISP_EINVAL naming the first unusable field. */
ISP_B200_API int isp_b200_validate_params(const isp_params_c* params);

/* validate_raw (isp_params.cpp:199-237). */
ISP_B200_API int isp_b200_validate_raw(const isp_raw_view_c* raw, const isp_params_c* params);

/* raw_row_bytes (isp_params.cpp:184-197). */
ISP_B200_API size_t isp_b200_raw_row_bytes(int32_t format, int32_t width);

/* tone_lut (isp_params.cpp:166-182): the table the pipeline interpolates.
 * Writes min(size, capacity) entries to out (may be null) and the size to *size. */
ISP_B200_API int isp_b200_tone_lut(const isp_params_c* params, float* out, size_t capacity, size_t* size);

/* ---- One pipeline, one camera (isp_pipeline.hpp:39-74) ----------------- */

/* IspPipeline(Backend::kCuda, params) (isp_pipeline.cpp:43-52, cuda_pipeline.cu:226-251):
 * validates, builds the tone table, and keeps it, the lens shading grid, the
 * white balance state and the scratch sums resident on the current device. */
ISP_B200_API int isp_b200_create(const isp_params_c* params, isp_b200_pipeline** out);

/* ~IspPipeline: waits for the pipeline's queued work, then frees it. Null is a no-op. */
ISP_B200_API void isp_b200_destroy(isp_b200_pipeline* pipeline);

/* IspPipeline::reset (isp_pipeline.cpp:58-63): forgets the white balance
 * estimate after the queued frames finish. */
ISP_B200_API int isp_b200_reset(isp_b200_pipeline* pipeline);

/* IspPipeline::process with device memory (isp_pipeline.cpp:65-90,
 * cuda_pipeline.cu:294-364): raw, out, histogram and stats are device
 * pointers; the work is queued on `stream` (a cudaStream_t, null for the
 * legacy default stream). Consecutive calls run on the GPU in call order, even
 * across streams. stats and exposure may be null. */
ISP_B200_API int isp_b200_process(isp_b200_pipeline* pipeline, const isp_raw_view_c* raw,
                     const isp_rgb_view_c* out, const isp_stats_c* stats,
                     const isp_exposure_c* exposure, void* stream);

/* IspPipeline(Backend::kCpu)::process's contract with the GPU behind it
 * (isp_pipeline.cpp:82-84): raw, out, histogram and stats are HOST pointers and
 * the results are there when the call returns. The pipeline stages through its
 * own pinned and device buffers, grown on demand. */
ISP_B200_API int isp_b200_process_host(isp_b200_pipeline* pipeline, const isp_raw_view_c* raw,
                          const isp_rgb_view_c* out, const isp_stats_c* stats,
                          const isp_exposure_c* exposure);

/* The white balance gains (R, G, B) and validity the next frame starts from:
 * AwbState (isp_math.hpp:71-74). Waits for the queued frames. */
ISP_B200_API int isp_b200_awb_state(isp_b200_pipeline* pipeline, float gains[3], int32_t* valid);

/* ---- Batches: many cameras' frames, one launch per pass ----------------
 * No reference counterpart: the reference processes one frame per
 * IspPipeline::process call. A batch holds frames of different cameras
 * (pipelines), sizes, formats, Bayer patterns and settings; a launch runs
 * the white balance statistics of the frames that estimate it, then every
 * frame's tiles, each pass one persistent kernel over a work list, directly
 * or as a CUDA graph replayed while the batch keeps its shape (frame count
 * and work split). Each frame's results are those of isp_b200_process. */
typedef struct isp_b200_batch isp_b200_batch;

typedef struct isp_batch_info_c {
  int32_t frames;
  float weights[4];   /* relative cost of a tile: bilinear, Malvar, +sharpening */
  int32_t ctas_per_sm; /* 0: as many as fit */
  int32_t tuned;
  int32_t graph_replays;
  int32_t graph_main_ctas;
  int32_t graph_awb_ctas;
  int32_t tile_rows;     /* the tile pass's tile height: 64 or 32 */
  int32_t block_threads; /* threads per CTA of both passes */
} isp_batch_info_c;

/* A batch of up to `capacity` frames on the current device. */
ISP_B200_API int isp_b200_batch_create(int32_t capacity, isp_b200_batch** out);
ISP_B200_API void isp_b200_batch_destroy(isp_b200_batch* batch);
/* Forgets the frames (the tuning and the graph stay). */
ISP_B200_API int isp_b200_batch_clear(isp_b200_batch* batch);
ISP_B200_API int isp_b200_batch_size(const isp_b200_batch* batch);
/* Adds a frame of `camera` (device buffers, as isp_b200_process takes them);
 * a camera appears at most once per batch. ISP_EBUSY when full. */
ISP_B200_API int isp_b200_batch_add(isp_b200_batch* batch, isp_b200_pipeline* camera, const isp_raw_view_c* raw,
                       const isp_rgb_view_c* out, const isp_stats_c* stats,
                       const isp_exposure_c* exposure);
/* Queues the batch on `stream`; use_graph != 0 replays (or first builds) the
 * batch's CUDA graph. Each camera's earlier frames run first. */
ISP_B200_API int isp_b200_batch_launch(isp_b200_batch* batch, void* stream, int32_t use_graph);
/* Measures the batch's per-variant tile costs and the best CTAs per SM on
 * this GPU (the frames are processed a few times; the cameras' white balance
 * states are restored) and keeps them for later launches. */
ISP_B200_API int isp_b200_batch_autotune(isp_b200_batch* batch, void* stream);
/* Sets the tuning by hand: weights per variant, CTAs per SM (0: all that fit). */
ISP_B200_API int isp_b200_batch_set_tuning(isp_b200_batch* batch, const float weights[4], int32_t ctas_per_sm);
ISP_B200_API int isp_b200_batch_info(const isp_b200_batch* batch, isp_batch_info_c* info);
/* The tile pass's tile height for later launches: 64 (two CTAs per SM) or
 * 32 rows (three CTAs per SM, more and smaller work items); the autotuner
 * picks it by timing both. ISP_EINVAL for any other value. */
ISP_B200_API int isp_b200_batch_set_tile_rows(isp_b200_batch* batch, int32_t tile_rows);

/* ---- Serving: many camera streams, continuous batching -----------------
 * No reference counterpart (the reference's operator runs one camera on one
 * worker). A server keeps each stream's pipeline state on the device, takes
 * frames as they arrive, admits them against a device-memory budget, and
 * batches whatever is queued into batch launches (isp_b200_batch_*), up to
 * max_inflight batches on the GPU while newer arrivals queue for the next.
 * A frame's latency is its arrival to the completion of its batch. */
typedef struct isp_b200_server isp_b200_server;

typedef struct isp_server_config_c {
  int32_t max_batch;        /* frames per batch launch */
  int32_t max_inflight;     /* batches on the GPU at once, 1..8 */
  int32_t queue_depth;      /* frames a stream may hold waiting for the GPU */
  int32_t slots_per_stream; /* device buffers per stream for its frames in flight */
  int64_t memory_budget;    /* bytes the frames in flight may hold on the device */
  int32_t use_graph;        /* replay a batch's CUDA graph while its shape repeats */
  int32_t per_frame;        /* launch each admitted frame alone (isp_b200_process) instead of
                               one batch launch: the plain per-frame path, for comparison */
} isp_server_config_c;

/* A stream's frame shape and outputs. */
typedef struct isp_server_stream_c {
  int32_t width;
  int32_t height;
  int32_t format;
  int32_t bit_depth;
  int32_t pattern;
  int32_t out_format;
  int32_t with_histogram;
  int32_t with_stats;
  int32_t copy_back; /* frames submitted without host result buffers (the synthetic
                        drivers') copy image, histogram and statistics back to
                        pinned host memory the server keeps per device slot */
} isp_server_stream_c;

/* A completed frame: its outputs stay in the stream's device slot until the
 * slot serves a later frame (slots_per_stream frames later). */
typedef struct isp_server_result_c {
  uint64_t ticket;
  int32_t stream;
  uint64_t frame;      /* sequence number within the stream */
  int64_t arrival_ns;  /* steady clock */
  int64_t launch_ns;   /* when the frame's batch was launched */
  int64_t done_ns;     /* when the server saw the frame's batch complete */
  const void* image;
  const uint32_t* histogram;
  const float* stats;
} isp_server_result_c;

typedef struct isp_server_stats_c {
  int64_t submitted;
  int64_t refused; /* queue full */
  int64_t admitted;
  int64_t completed;
  int64_t batches;
  int64_t completed_pixels;
  double mean_batch_frames;
  double p50_ms;
  double p99_ms;
  double p999_ms;
  double max_ms;
  double gpix_per_s; /* completed pixels over first arrival to last completion */
  int32_t error;
  double p50_wait_ms; /* arrival to the launch of the frame's batch (copy and queueing) */
  double p99_wait_ms;
} isp_server_stats_c;

ISP_B200_API void isp_b200_server_config_default(isp_server_config_c* config);
ISP_B200_API int isp_b200_server_create(const isp_server_config_c* config, isp_b200_server** out);
/* Adds a camera stream (before start): its pipeline, device slots and pinned staging. */
ISP_B200_API int isp_b200_server_add_stream(isp_b200_server* server, const isp_params_c* params,
                               const isp_server_stream_c* shape, int32_t* id);
ISP_B200_API int isp_b200_server_start(isp_b200_server* server);
/* A frame of `stream` arrived (host memory, copied to pinned staging before
 * the call returns; arrival_ns 0 for now). host_out/histogram/stats, when not
 * null, receive copies of the results. ISP_EBUSY when the stream's queue is full. */
ISP_B200_API int isp_b200_server_submit(isp_b200_server* server, int32_t stream, const void* host_raw, size_t pitch,
                           void* host_out, uint32_t* host_histogram, float* host_stats, int64_t arrival_ns,
                           uint64_t* ticket);
/* A frame of `stream` arrived in device memory (written there by a capture
 * device, for instance): it is read in place, without a copy, and must stay
 * unchanged until the frame completes. Otherwise as isp_b200_server_submit. */
ISP_B200_API int isp_b200_server_submit_device(isp_b200_server* server, int32_t stream, const void* device_raw,
                                  size_t pitch, void* host_out, uint32_t* host_histogram, float* host_stats,
                                  int64_t arrival_ns, uint64_t* ticket);
/* Completed frames since the last poll, oldest first. */
ISP_B200_API int isp_b200_server_poll(isp_b200_server* server, isp_server_result_c* out, int32_t capacity,
                         int32_t* count);
/* Waits until every submitted frame completed; ISP_ETIMEOUT after timeout_ns. */
ISP_B200_API int isp_b200_server_drain(isp_b200_server* server, int64_t timeout_ns);
ISP_B200_API int isp_b200_server_stats(isp_b200_server* server, isp_server_stats_c* stats);
ISP_B200_API int isp_b200_server_reset_stats(isp_b200_server* server);
/* Adds a frame (host memory) to the ring of frames the synthetic arrival
 * drivers submit for `stream`, in turn; call it before the drivers run. The
 * server keeps a copy: pinned host memory (submitted like
 * isp_b200_server_submit frames, copied to the device per frame), or device
 * memory when on_device is set (submitted like isp_b200_server_submit_device
 * frames: already in HBM on arrival). A stream's sources are all on the
 * host or all on the device. */
ISP_B200_API int isp_b200_server_add_source(isp_b200_server* server, int32_t stream, const void* host_raw, size_t pitch,
                               int32_t on_device);
/* Synthetic arrivals: each stream's next source frame submitted at Poisson
 * times of rate fps[stream] for `seconds`, from the calling thread. An
 * arrival that finds its stream's queue full is refused (counted). */
ISP_B200_API int isp_b200_server_run_poisson(isp_b200_server* server, const double* fps, double seconds, uint64_t seed);
/* Saturation: for `seconds`, every stream's queue is kept full with its next
 * source frames (closed loop), from the calling thread. */
ISP_B200_API int isp_b200_server_run_closed(isp_b200_server* server, double seconds);
/* Finishes the frames in flight, then frees everything. */
ISP_B200_API void isp_b200_server_destroy(isp_b200_server* server);

/* ---- Synthetic frames ------------------------------------------------------
 *
 * Seeded raw frames rendered on the device, for throughput workloads that
 * need fresh frames at rate; they play the part of the reference module's
 * synthetic camera (modules/isp/src/synthetic_raw.cu, its render kernel),
 * with the benchmark's scene instead of its test chart: a base level and
 * gradient, 8 Gaussian blobs (sigma 50..300 px), 64 uniform rectangles, a
 * cos^4 vignette (corner gain vignette_edge), mosaicked in `pattern`, scaled
 * to [black, 2^bit_depth - 1], Poisson shot noise (gain counts per
 * electron, 0: none) and Gaussian read noise (read_noise counts), rounded,
 * clipped and packed in `format`. A frame is a pure function of its seed and
 * settings. */
typedef struct isp_synth_c {
  int32_t width;
  int32_t height;
  int32_t format;
  int32_t bit_depth;
  int32_t pattern;
  float black;
  float gain;
  float read_noise;
  float vignette_edge;
} isp_synth_c;

ISP_B200_API void isp_b200_synth_default(isp_synth_c* config);
/* Renders the frame of `seed` into `raw` (device memory, row stride `pitch`)
 * on `stream`. ISP_EINVAL for settings that do not make a valid raw view. */
ISP_B200_API int isp_b200_synthetic_raw(const isp_synth_c* config, uint64_t seed, void* raw, size_t pitch,
                           void* stream);

/* The demo's side-by-side view (applications/isp/src/view_op.cu:35-75 and
 * :143-150), as a headless device image: `view` (RGB8, 2 * raw->width pixels
 * wide, raw->height rows, row stride view_pitch) gets on its left the raw
 * mosaic as gray, g = (uint8)(sqrtf(clamp((s - black_level) * scale, 0, 1))
 * * 255 + 0.5) with scale = 1 / (2^bit_depth - 1 - black_level), each step a
 * single-precision operation as the demo's kernel does it, and on its right
 * the ISP's RGB8 image `rgb8` (row stride rgb8_pitch). Device buffers, queued
 * on stream. ISP_EINVAL for an unusable raw view (as validate_raw: sizes,
 * format, bit depth, pitch), a missing buffer or a pitch shorter than its row. */
ISP_B200_API int isp_b200_view_compose(const isp_raw_view_c* raw, float black_level, const void* rgb8,
                                       size_t rgb8_pitch, void* view, size_t view_pitch, void* stream);

/* One frame without allocating memory. No reference counterpart: for callers
 * that cannot allocate device memory (cudaMalloc forbidden or unsafe where
 * they run, e.g. a host that owns every allocation or a real-time loop that
 * must not touch the allocator). The caller passes raw, out, histogram and
 * stats in device memory and params on the host; the tone table (at most
 * 4097 entries), lens shading grid (at most 28544 gains), statistics sums and
 * white balance state live in one 160 KB device array inside this library,
 * which every GPU that loads it holds until exit; larger tables are refused
 * with ISP_EINVAL. The frame is processed as the first frame of a fresh
 * pipeline (auto white balance: its own estimate, unsmoothed). The first call
 * on a device, with that device current, looks up the array's address and
 * sets the kernels' limits (again after a device reset); make it before any
 * stream capture. Each call stages its tables from host memory that the next
 * call reuses, so it returns ISP_EINVAL and queues nothing while `stream` is
 * capturing. Calls share the array: consecutive calls on one stream are
 * ordered, calls that overlap on the GPU race. No cudaMalloc, cudaFree or
 * other allocating routine is called. */
ISP_B200_API int isp_b200_process_noalloc(const isp_params_c* params, const isp_raw_view_c* raw,
                             const isp_rgb_view_c* out, const isp_stats_c* stats,
                             const isp_exposure_c* exposure, void* stream);

/* Companion of isp_b200_process_noalloc, no reference counterpart, also
 * allocating nothing: waits for `stream`, then reports (and clears) whether a
 * kernel of the last no-alloc frame on the current device gave up a bounded
 * wait (*status 1: that frame's outputs are not trustworthy), else 0. Call it
 * before the next no-alloc call, which clears the flag. */
ISP_B200_API int isp_b200_noalloc_status(void* stream, int32_t* status);

/* Tile height of the fused tile pass, no reference counterpart (the
 * reference's CUDA backend uses one 32x16 block shape, cuda_pipeline.cu:17-19).
 * The pass is compiled for 64-row tiles (two CTAs per SM) and 32-row tiles
 * (three CTAs per SM: a frame of few tiles spreads over more SMs). 0 (the
 * default) uses the height isp_b200_autotune picked for the frame's raw
 * format and size, else 64; 64 or 32 force it for every frame. Outputs are
 * bit-identical either way. ISP_EINVAL for any other value. */
ISP_B200_API int isp_b200_set_tile_rows(isp_b200_pipeline* pipeline, int32_t tile_rows);

/* Tunes the tile height for one frame shape, no reference counterpart:
 * processes `raw` into `out` (device buffers, as isp_b200_process) a few
 * times with each tile height, keeps the faster for this raw format, width
 * and height (up to 8 shapes per pipeline) and writes it to *tile_rows. The
 * pipeline's white balance state is put back afterwards, so the frames it ran
 * leave no trace; waits for `stream`. */
ISP_B200_API int isp_b200_autotune(isp_b200_pipeline* pipeline, const isp_raw_view_c* raw, const isp_rgb_view_c* out,
                                   const isp_stats_c* stats, const isp_exposure_c* exposure, void* stream,
                                   int32_t* tile_rows);

/* Frame overlap, no reference counterpart (on by default): when frames of
 * one pipeline follow each other on one stream, the next frame's white
 * balance statistics pass may begin while the previous frame's tile pass
 * finishes (a programmatic dependent launch); its estimate still waits for
 * that pass, so every output is the one the frames give alone. The pass reads
 * its raw frame before that wait, so a kernel queued just before the call
 * that writes the raw frame must not signal its dependents early
 * (griddepcontrol.launch_dependents / cudaTriggerProgrammaticLaunchCompletion);
 * ordinary kernels, copies and events are waited for in full. 0 turns it off. */
ISP_B200_API int isp_b200_set_frame_overlap(isp_b200_pipeline* pipeline, int32_t enable);

/* Device-side status, no reference counterpart: waits for the pipeline's
 * queued frames, then reports (and clears) whether a kernel gave up a bounded
 * wait while processing them (*status 1: that frame's output is not
 * trustworthy), else 0. */
ISP_B200_API int isp_b200_device_status(isp_b200_pipeline* pipeline, int32_t* status);

/* Check of the bounded device waits, no reference counterpart: queues on
 * `stream`, ordered after the pipeline's frames, one kernel that waits on a
 * barrier no copy ever completes, gives up after `polls` polls (1..2^20) and
 * flags the pipeline as a tile or statistics pass that gave up a wait flags
 * it; isp_b200_device_status then reports 1 once. Nothing is left in flight
 * and the pipeline's next frame is unaffected. */
ISP_B200_API int isp_b200_check_bounded_wait(isp_b200_pipeline* pipeline, uint32_t polls, void* stream);

/* Out-of-bounds report of the bounds-checked build, no reference counterpart
 * (the reference runs its tests under compute-sanitizer instead,
 * modules/isp/tests/CMakeLists.txt:34-50). libisp_b200_checked.so is this
 * library compiled with every shared- and global-memory access of the ISP
 * kernels checked against the extent of the array it indexes; an access
 * outside it is not made and is counted instead. This call waits for the
 * pipeline's queued frames, then reports (and clears) how many accesses were
 * refused since the last call and the address of the first (0 when none).
 * The regular library returns ISP_EINVAL: it makes no checks. */
ISP_B200_API int isp_b200_checked_violations(isp_b200_pipeline* pipeline, uint32_t* count, uint64_t* first_address);

/* Profiling hook, no reference counterpart: events (cudaEvent_t, may be null)
 * that every following process call records on its stream right before and
 * right after the fused tile kernel, so a caller can time that kernel alone. */
ISP_B200_API int isp_b200_set_kernel_events(isp_b200_pipeline* pipeline, void* before, void* after);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* ISP_B200_H_ */
