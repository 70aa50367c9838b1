/*
 * isp_oracle.h - TEST INFRASTRUCTURE ONLY. The CPU oracle of the B200 ISP.
 *
 * A plain-C restatement of the holoscan::isp CPU backend
 * (modules/isp/src/cpu_pipeline.cpp, isp_math.hpp, isp_params.cpp), pinned
 * against the reference itself: tests/golden/ holds outputs of the reference
 * sources compiled unmodified (oracle/_ref, recipe in oracle/Makefile), and
 * the not-gpu tests check this oracle against them byte for byte.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker or the CPU timing baseline: the
 * product (libisp_b200.so) never links or calls it.
 */
#ifndef ISP_ORACLE_H_
#define ISP_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#include "../include/isp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The white balance state carried from frame to frame (isp_math.hpp:71-74). */
typedef struct oracle_awb_state {
  float gains[3];
  int32_t valid;
} oracle_awb_state;

/* A frame's white balance sums (isp_math.hpp:64-68), exposed for the tests of
 * the statistics pass. */
typedef struct oracle_awb_accum {
  uint64_t sum[3];
  uint64_t quads;
  uint32_t hist[3][1024];
} oracle_awb_accum;

size_t oracle_raw_row_bytes(int32_t format, int32_t width);
/* 0 or ISP_EINVAL; the message in `message` (capacity `cap`) when not null. */
int oracle_validate_params(const isp_params_c* params, char* message, size_t cap);
int oracle_validate_raw(const isp_raw_view_c* raw, const isp_params_c* params, char* message,
                        size_t cap);
/* Writes min(size, cap) entries; returns the size. */
size_t oracle_tone_lut(const isp_params_c* params, float* out, size_t cap);
/* initial_white_balance (cpu_pipeline.cpp:90-95). */
void oracle_awb_init(const isp_params_c* params, oracle_awb_state* state);
/* The white balance statistics of one frame (cpu_pipeline.cpp:101-119). */
void oracle_awb_stats(const isp_params_c* params, const isp_raw_view_c* raw,
                      oracle_awb_accum* accum);
/* IspPipeline(kCpu).process (isp_pipeline.cpp:65-84 -> cpu_pipeline.cpp:97-191),
 * validation included: 0 or ISP_EINVAL. All buffers in host memory. */
int oracle_process(const isp_params_c* params, const isp_raw_view_c* raw,
                   const isp_rgb_view_c* out, const isp_stats_c* stats,
                   const isp_exposure_c* exposure, oracle_awb_state* state);

/* The demo's side-by-side view of raw and RGB8 (host buffers). */
void oracle_view_compose(const isp_raw_view_c* raw, float black, const uint8_t* rgb, size_t rgb_pitch, uint8_t* out,
                         size_t out_pitch);

#ifdef __cplusplus
}
#endif

#endif /* ISP_ORACLE_H_ */
