/*
 * isp_oracle.c - TEST INFRASTRUCTURE ONLY: the CPU oracle of the B200 ISP.
 *
 * A plain-C restatement of the holoscan::isp CPU backend. Every float
 * expression keeps the reference's operands and their order, and the file is
 * compiled without contraction (-ffp-contract=off), as the reference is
 * (modules/isp/CMakeLists.txt:64-70), so that it reproduces the reference bit
 * for bit. Parity is pinned by tests/test_oracle_golden.py against outputs of
 * the unmodified reference sources (oracle/_ref). Citations are paths inside
 * the holoscan-zozo-modules tree.
 */
#include "isp_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* Channels of the mosaic (isp_params.hpp:65-68). */
enum { CH_R = 0, CH_GR = 1, CH_GB = 2, CH_B = 3 };
#define FIXED_ONE 1048576.0F /* isp_math.hpp:30 */
#define AWB_BINS 1024        /* isp_math.hpp:32 */

/* The channel at quad position (y & 1) * 2 + (x & 1), per pattern (cpu_pipeline.cpp:15-20). */
static const int kCfa[4][4] = {
    {CH_R, CH_GR, CH_GB, CH_B},  /* RGGB */
    {CH_B, CH_GB, CH_GR, CH_R},  /* BGGR */
    {CH_GR, CH_R, CH_B, CH_GB},  /* GRBG */
    {CH_GB, CH_B, CH_R, CH_GR},  /* GBRG */
};

/* FrameParams (isp_math.hpp:35-60), as make_frame_params fills it (cpu_pipeline.cpp:50-88). */
typedef struct frame {
  int width, height;
  const unsigned char* raw;
  size_t raw_pitch;
  int raw_format;
  int cfa[4];
  float black[4];
  float inv_range[4];
  int white;
  float wb[3];
  const float* lsc;
  int lsc_width, lsc_height, lsc_channels;
  float lsc_sx, lsc_sy;
  float ccm[9];
  const float* lut;
  int lut_size;
  float sharpen;
  unsigned char* out;
  size_t out_pitch;
  int out_format;
} frame;

static void set_message(char* message, size_t cap, const char* text) {
  if (message != NULL && cap > 0) {
    snprintf(message, cap, "%s", text);
  }
}

static int finite_in(float v, float lo, float hi) { return isfinite(v) && v >= lo && v <= hi; }

/* raw_row_bytes (isp_params.cpp:184-197). */
size_t oracle_raw_row_bytes(int32_t format, int32_t width) {
  const size_t w = (size_t)(width < 0 ? 0 : width);
  switch (format) {
    case ISP_RAW_U8: return w;
    case ISP_RAW_U16: return 2U * w;
    case ISP_RAW_RAW10: return 5U * ((w + 3U) / 4U);
    case ISP_RAW_RAW12: return 3U * ((w + 1U) / 2U);
    default: return 0;
  }
}

/* validate_params (isp_params.cpp:85-164), same checks in the same order. */
int oracle_validate_params(const isp_params_c* p, char* message, size_t cap) {
#define REJECT(text)                   \
  do {                                 \
    set_message(message, cap, (text)); \
    return ISP_EINVAL;                 \
  } while (0)
  if (!finite_in(p->black_level, 0.0F, 65535.0F)) REJECT("black_level must be 0..65535");
  if (p->has_channel_black_levels) {
    for (int k = 0; k < 4; ++k) {
      if (!finite_in(p->channel_black_levels[k], 0.0F, 65535.0F)) {
        REJECT("channel_black_levels must be 0..65535");
      }
    }
  }
  if (!finite_in(p->white_level, 0.0F, 65535.0F)) {
    REJECT("white_level must be 0 (from the bit depth) or up to 65535");
  }
  if (p->has_lens_shading) {
    if (p->lsc_width < 2 || p->lsc_height < 2 || p->lsc_width > 256 || p->lsc_height > 256) {
      REJECT("lens_shading grid must be 2x2 to 256x256 points");
    }
    if (p->lsc_channels != 1 && p->lsc_channels != 4) REJECT("lens_shading channels must be 1 or 4");
    if (p->lsc_gains_count != (size_t)p->lsc_width * p->lsc_height * p->lsc_channels ||
        (p->lsc_gains_count > 0 && p->lsc_gains == NULL)) {
      REJECT("lens_shading gains must hold width x height x channels values");
    }
    for (size_t i = 0; i < p->lsc_gains_count; ++i) {
      const float g = p->lsc_gains[i];
      if (!(isfinite(g) && g > 0.0F && g <= 16.0F)) REJECT("lens_shading gains must be in (0, 16]");
    }
  }
  for (int k = 0; k < 3; ++k) {
    const float g = p->wb_gains[k];
    if (!(isfinite(g) && g > 0.0F && g <= 64.0F)) REJECT("wb_gains must be in (0, 64]");
  }
  if (!(isfinite(p->awb_smoothing) && p->awb_smoothing > 0.0F && p->awb_smoothing <= 1.0F)) {
    REJECT("awb_smoothing must be in (0, 1]");
  }
  if (!(isfinite(p->white_patch_percentile) && p->white_patch_percentile >= 0.5F &&
        p->white_patch_percentile < 1.0F)) {
    REJECT("white_patch_percentile must be in [0.5, 1)");
  }
  for (int k = 0; k < 9; ++k) {
    if (!finite_in(p->ccm[k], -16.0F, 16.0F)) REJECT("ccm entries must be finite, -16..16");
  }
  if (p->tone_curve == ISP_TONE_GAMMA && !finite_in(p->gamma, 0.1F, 10.0F)) {
    REJECT("gamma must be 0.1..10");
  }
  if (p->tone_curve == ISP_TONE_LUT) {
    if (p->lut_size < 2 || p->lut_size > 65536 || p->lut == NULL) REJECT("lut must have 2..65536 entries");
    for (size_t i = 0; i < p->lut_size; ++i) {
      if (!finite_in(p->lut[i], 0.0F, 1.0F)) REJECT("lut entries must be 0..1");
    }
  }
  if (!finite_in(p->sharpen, 0.0F, 4.0F)) REJECT("sharpen must be 0..4");
  const isp_auto_exposure_c* ae = &p->auto_exposure;
  if (!(isfinite(ae->target) && ae->target > 0.0F && ae->target < 1.0F)) {
    REJECT("auto_exposure.target must be in (0, 1)");
  }
  if (!finite_in(ae->damping, 0.0F, 1.0F)) REJECT("auto_exposure.damping must be 0..1");
  if (ae->min_exposure_ns <= 0 || ae->max_exposure_ns < ae->min_exposure_ns) {
    REJECT("auto_exposure needs 0 < min_exposure_ns <= max_exposure_ns");
  }
  if (!(isfinite(ae->min_gain) && isfinite(ae->max_gain) && ae->min_gain > 0.0F &&
        ae->max_gain >= ae->min_gain)) {
    REJECT("auto_exposure needs 0 < min_gain <= max_gain");
  }
  return ISP_OK;
}

static float white_of(const isp_params_c* p, int bit_depth) {
  return p->white_level > 0.0F ? p->white_level
                               : (float)((1U << (unsigned)bit_depth) - 1U);
}

/* validate_raw (isp_params.cpp:199-237). */
int oracle_validate_raw(const isp_raw_view_c* raw, const isp_params_c* p, char* message,
                        size_t cap) {
  if (raw->data == NULL) REJECT("raw image has no data");
  if (raw->width < 2 || raw->height < 2 || raw->width > 16384 || raw->height > 16384) {
    REJECT("raw image must be 2x2 to 16384x16384");
  }
  if (raw->format < ISP_RAW_U8 || raw->format > ISP_RAW_RAW12 || raw->pattern < 0 ||
      raw->pattern > 3) {
    REJECT("raw image format or pattern unknown");
  }
  if (raw->pitch < oracle_raw_row_bytes(raw->format, raw->width)) {
    REJECT("raw image pitch is shorter than a row");
  }
  if (raw->format == ISP_RAW_U16 && (raw->pitch % 2U != 0U || ((uintptr_t)raw->data) % 2U != 0U)) {
    REJECT("uint16 raw samples must be aligned to 2 bytes, rows too");
  }
  const int max_bits = raw->format == ISP_RAW_U8      ? 8
                       : raw->format == ISP_RAW_RAW10 ? 10
                       : raw->format == ISP_RAW_RAW12 ? 12
                                                      : 16;
  const int packed = raw->format == ISP_RAW_RAW10 || raw->format == ISP_RAW_RAW12;
  if (raw->bit_depth < 1 || raw->bit_depth > max_bits || (packed && raw->bit_depth != max_bits)) {
    char text[96];
    snprintf(text, sizeof text, "raw bit depth %d does not fit its sample format", raw->bit_depth);
    REJECT(text);
  }
  const float white = white_of(p, raw->bit_depth);
  if (white > (float)((1U << (unsigned)raw->bit_depth) - 1U)) {
    REJECT("white_level exceeds the raw bit depth");
  }
  for (int k = 0; k < 4; ++k) {
    const float level = p->has_channel_black_levels ? p->channel_black_levels[k] : p->black_level;
    if (!(level < white)) REJECT("black levels must be below the white level");
  }
  return ISP_OK;
#undef REJECT
}

/* tone_lut (isp_params.cpp:166-182): double evaluation, rounded to float. */
size_t oracle_tone_lut(const isp_params_c* p, float* out, size_t cap) {
  if (p->tone_curve == ISP_TONE_LUT) {
    for (size_t i = 0; i < p->lut_size && i < cap; ++i) out[i] = p->lut[i];
    return p->lut_size;
  }
  const int n = ISP_TONE_LUT_SIZE;
  for (int i = 0; i < n && (size_t)i < cap; ++i) {
    const double x = (double)i / (n - 1);
    double y = x;
    if (p->tone_curve == ISP_TONE_SRGB) {
      y = x <= 0.0031308 ? 12.92 * x : 1.055 * pow(x, 1.0 / 2.4) - 0.055;
    } else if (p->tone_curve == ISP_TONE_GAMMA) {
      y = pow(x, 1.0 / (double)p->gamma);
    }
    out[i] = (float)(y < 0.0 ? 0.0 : y > 1.0 ? 1.0 : y);
  }
  return (size_t)n;
}

void oracle_awb_init(const isp_params_c* p, oracle_awb_state* s) {
  for (int k = 0; k < 3; ++k) s->gains[k] = p->wb_gains[k];
  s->valid = 0;
}

/* make_frame_params (cpu_pipeline.cpp:50-88). */
static frame make_frame(const isp_params_c* params, const isp_raw_view_c* raw,
                        const isp_rgb_view_c* out, const float* lut, int lut_size) {
  frame p;
  memset(&p, 0, sizeof p);
  p.width = raw->width;
  p.height = raw->height;
  p.raw = (const unsigned char*)raw->data;
  p.raw_pitch = raw->pitch;
  p.raw_format = raw->format;
  for (int k = 0; k < 4; ++k) p.cfa[k] = kCfa[raw->pattern][k];
  const float white = white_of(params, raw->bit_depth);
  for (int k = 0; k < 4; ++k) {
    p.black[k] = params->has_channel_black_levels ? params->channel_black_levels[k]
                                                  : params->black_level;
    p.inv_range[k] = 1.0F / (white - p.black[k]);
  }
  p.white = (int)ceilf(white);
  for (int k = 0; k < 3; ++k) p.wb[k] = params->wb_gains[k];
  if (params->has_lens_shading) {
    p.lsc = params->lsc_gains;
    p.lsc_width = params->lsc_width;
    p.lsc_height = params->lsc_height;
    p.lsc_channels = params->lsc_channels;
    p.lsc_sx = (float)(params->lsc_width - 1) / (float)(raw->width - 1);
    p.lsc_sy = (float)(params->lsc_height - 1) / (float)(raw->height - 1);
  }
  for (int k = 0; k < 9; ++k) p.ccm[k] = params->ccm[k];
  p.lut = lut;
  p.lut_size = lut_size;
  p.sharpen = params->sharpen;
  p.out = out != NULL ? (unsigned char*)out->data : NULL;
  p.out_pitch = out != NULL ? out->pitch : 0;
  p.out_format = out != NULL ? out->format : 0;
  return p;
}

/* mirror (isp_math.hpp:82-91): reflection that keeps a coordinate's parity. */
static int mirror(int v, int n) {
  const int period = 2 * (n - 1);
  v %= period;
  if (v < 0) v += period;
  return v < n ? v : period - v;
}

/* color_of, channel_at (isp_math.hpp:93-99). */
static int color_of(int channel) { return channel == CH_R ? 0 : channel == CH_B ? 2 : 1; }
static int channel_at(const frame* p, int x, int y) { return p->cfa[((y & 1) << 1) | (x & 1)]; }

/* load_raw (isp_math.hpp:101-119): one sample's raw counts. */
static int load_raw(const frame* p, int x, int y) {
  const unsigned char* row = p->raw + (size_t)y * p->raw_pitch;
  switch (p->raw_format) {
    case ISP_RAW_U8: return row[x];
    case ISP_RAW_U16: {
      uint16_t v;
      memcpy(&v, row + 2 * (size_t)x, 2);
      return v;
    }
    case ISP_RAW_RAW10: {
      const unsigned char* g = row + 5 * (size_t)(x >> 2);
      const int k = x & 3;
      return ((int)g[k] << 2) | ((g[4] >> (2 * k)) & 3);
    }
    default: {
      const unsigned char* g = row + 3 * (size_t)(x >> 1);
      const int k = x & 1;
      return ((int)g[k] << 4) | ((g[2] >> (4 * k)) & 15);
    }
  }
}

/* lens_shading_gain (isp_math.hpp:121-140): bilinear in the grid. */
static float lens_shading_gain(const frame* p, int x, int y, int channel) {
  if (p->lsc == NULL) return 1.0F;
  const float fx = (float)x * p->lsc_sx;
  const float fy = (float)y * p->lsc_sy;
  int ix = (int)fx;
  int iy = (int)fy;
  ix = ix > p->lsc_width - 2 ? p->lsc_width - 2 : ix;
  iy = iy > p->lsc_height - 2 ? p->lsc_height - 2 : iy;
  const float tx = fx - (float)ix;
  const float ty = fy - (float)iy;
  const int step = p->lsc_channels;
  const int row = p->lsc_width * step;
  const float* g = p->lsc + ((size_t)iy * p->lsc_width + ix) * step + (step == 4 ? channel : 0);
  const float top = g[0] + (g[step] - g[0]) * tx;
  const float bottom = g[row] + (g[row + step] - g[row]) * tx;
  return top + (bottom - top) * ty;
}

/* linearize (isp_math.hpp:144-148). */
static float linearize(const frame* p, int raw, int x, int y, int channel) {
  float v = ((float)raw - p->black[channel]) * p->inv_range[channel];
  v = v > 0.0F ? v : 0.0F;
  return v * lens_shading_gain(p, x, y, channel);
}

/* preprocess (isp_math.hpp:151-155). */
static float preprocess(const frame* p, const float gains[3], int x, int y) {
  const int channel = channel_at(p, x, y);
  const float v = linearize(p, load_raw(p, x, y), x, y, channel) * gains[color_of(channel)];
  return v < 1.0F ? v : 1.0F;
}

static float clamp01(float v) { return v < 0.0F ? 0.0F : v > 1.0F ? 1.0F : v; }

/* demosaic<kMalvar> (isp_math.hpp:161-215): RGB at the centre of n[5][5]. */
static void demosaic(int malvar, const float n[5][5], int channel, float rgb[3]) {
  const float c = n[2][2];
  float at_green, diagonal, across, down;
  if (!malvar) {
    at_green = (n[1][2] + n[3][2] + n[2][1] + n[2][3]) * 0.25F;
    diagonal = (n[1][1] + n[1][3] + n[3][1] + n[3][3]) * 0.25F;
    across = (n[2][1] + n[2][3]) * 0.5F;
    down = (n[1][2] + n[3][2]) * 0.5F;
  } else {
    const float axial1 = n[1][2] + n[3][2] + n[2][1] + n[2][3];
    const float axial2 = n[0][2] + n[4][2] + n[2][0] + n[2][4];
    const float diagonal1 = n[1][1] + n[1][3] + n[3][1] + n[3][3];
    const float horizontal2 = n[2][0] + n[2][4];
    const float vertical2 = n[0][2] + n[4][2];
    at_green = (4.0F * c + 2.0F * axial1 - axial2) * 0.125F;
    diagonal = (6.0F * c + 2.0F * diagonal1 - 1.5F * axial2) * 0.125F;
    across = (5.0F * c + 4.0F * (n[2][1] + n[2][3]) - horizontal2 - diagonal1 + 0.5F * vertical2) *
             0.125F;
    down = (5.0F * c + 4.0F * (n[1][2] + n[3][2]) - vertical2 - diagonal1 + 0.5F * horizontal2) *
           0.125F;
    at_green = clamp01(at_green);
    diagonal = clamp01(diagonal);
    across = clamp01(across);
    down = clamp01(down);
  }
  switch (channel) {
    case CH_R: rgb[0] = c; rgb[1] = at_green; rgb[2] = diagonal; break;
    case CH_B: rgb[0] = diagonal; rgb[1] = at_green; rgb[2] = c; break;
    case CH_GR: rgb[0] = across; rgb[1] = c; rgb[2] = down; break;
    default: rgb[0] = down; rgb[1] = c; rgb[2] = across; break;
  }
}

/* sharpen (isp_math.hpp:219-227): unsharp mask against a 1-2-1 binomial blur. */
static void sharpen(const float m[3][3][3], float amount, float rgb[3]) {
  for (int k = 0; k < 3; ++k) {
    const float c = m[1][1][k];
    const float blur = (4.0F * c + 2.0F * (m[0][1][k] + m[2][1][k] + m[1][0][k] + m[1][2][k]) +
                        (m[0][0][k] + m[0][2][k] + m[2][0][k] + m[2][2][k])) *
                       0.0625F;
    rgb[k] = clamp01(c + amount * (c - blur));
  }
}

/* correct_color (isp_math.hpp:229-233). */
static void correct_color(const frame* p, const float in[3], float out[3]) {
  for (int k = 0; k < 3; ++k) {
    out[k] = clamp01(p->ccm[3 * k] * in[0] + p->ccm[3 * k + 1] * in[1] + p->ccm[3 * k + 2] * in[2]);
  }
}

/* tone (isp_math.hpp:235-243). */
static float tone(const frame* p, float x) {
  const float f = x * (float)(p->lut_size - 1);
  const int i = (int)f;
  if (i >= p->lut_size - 1) return p->lut[p->lut_size - 1];
  const float t = f - (float)i;
  return p->lut[i] + t * (p->lut[i + 1] - p->lut[i]);
}

/* to_fixed (isp_math.hpp:245-247). */
static unsigned int to_fixed(float v) { return (unsigned int)(v * FIXED_ONE + 0.5F); }

/* store (isp_math.hpp:250-276). */
static void store(const frame* p, int x, int y, const float t[3]) {
  unsigned char* row = p->out + (size_t)y * p->out_pitch;
  switch (p->out_format) {
    case ISP_OUT_RGB8:
      for (int k = 0; k < 3; ++k) row[3 * x + k] = (unsigned char)(t[k] * 255.0F + 0.5F);
      break;
    case ISP_OUT_RGBA8:
      for (int k = 0; k < 3; ++k) row[4 * x + k] = (unsigned char)(t[k] * 255.0F + 0.5F);
      row[4 * x + 3] = 255;
      break;
    case ISP_OUT_RGB16:
      for (int k = 0; k < 3; ++k) {
        const uint16_t v = (uint16_t)(t[k] * 65535.0F + 0.5F);
        memcpy(row + 2 * (3 * (size_t)x + k), &v, 2);
      }
      break;
    default:
      for (int k = 0; k < 3; ++k) memcpy(row + 4 * (3 * (size_t)x + k), &t[k], 4);
      break;
  }
}

/* output_codes (isp_math.hpp:279-301): the 8-bit codes of the stored output. */
static void output_codes(const frame* p, int x, int y, int q[3]) {
  const unsigned char* row = p->out + (size_t)y * p->out_pitch;
  switch (p->out_format) {
    case ISP_OUT_RGB8:
      for (int k = 0; k < 3; ++k) q[k] = row[3 * x + k];
      break;
    case ISP_OUT_RGBA8:
      for (int k = 0; k < 3; ++k) q[k] = row[4 * x + k];
      break;
    case ISP_OUT_RGB16:
      for (int k = 0; k < 3; ++k) {
        uint16_t v;
        memcpy(&v, row + 2 * (3 * (size_t)x + k), 2);
        q[k] = (int)((v * 255U + 32767U) / 65535U);
      }
      break;
    default:
      for (int k = 0; k < 3; ++k) {
        float v;
        memcpy(&v, row + 4 * (3 * (size_t)x + k), 4);
        q[k] = (int)(clamp01(v) * 255.0F + 0.5F);
      }
      break;
  }
}

/* luma_code (isp_math.hpp:303-305). */
static int luma_code(const int q[3]) { return (2126 * q[0] + 7152 * q[1] + 722 * q[2] + 5000) / 10000; }

/* white_balance_quad (isp_math.hpp:311-332). */
static int white_balance_quad(const frame* p, int qx, int qy, int color[4], unsigned int fixed[4],
                              int bin[4]) {
  int raw[4];
  for (int k = 0; k < 4; ++k) {
    raw[k] = load_raw(p, 2 * qx + (k & 1), 2 * qy + (k >> 1));
    if (raw[k] >= p->white) return 0;
  }
  for (int k = 0; k < 4; ++k) {
    const int x = 2 * qx + (k & 1);
    const int y = 2 * qy + (k >> 1);
    const int channel = channel_at(p, x, y);
    float v = linearize(p, raw[k], x, y, channel);
    v = v < 4.0F ? v : 4.0F;
    color[k] = color_of(channel);
    fixed[k] = to_fixed(v);
    const int b = (int)(v * (float)AWB_BINS);
    bin[k] = b < AWB_BINS - 1 ? b : AWB_BINS - 1;
  }
  return 1;
}

/* histogram_percentile (isp_math.hpp:336-352). */
static float histogram_percentile(const uint32_t* hist, float percentile) {
  uint64_t total = 0;
  for (int b = 0; b < AWB_BINS; ++b) total += hist[b];
  if (total == 0) return 0.0F;
  const double target = (double)percentile * (double)total;
  uint64_t below = 0;
  for (int b = 0; b < AWB_BINS; ++b) {
    if (hist[b] != 0U && (double)(below + hist[b]) >= target) {
      const double within = (target - (double)below) / (double)hist[b];
      return (float)(((double)b + within) / AWB_BINS);
    }
    below += hist[b];
  }
  return 1.0F;
}

/* finish_white_balance (isp_math.hpp:357-384). */
static void finish_white_balance(const oracle_awb_accum* a, int mode, float percentile,
                                 float smoothing, oracle_awb_state* s) {
  if (a->quads == 0) return;
  float level[3];
  if (mode == ISP_WB_GRAY_WORLD) {
    const double quads = (double)a->quads;
    level[0] = (float)((double)a->sum[0] / quads);
    level[1] = (float)((double)a->sum[1] / (2.0 * quads));
    level[2] = (float)((double)a->sum[2] / quads);
  } else {
    for (int k = 0; k < 3; ++k) level[k] = histogram_percentile(a->hist[k], percentile);
  }
  if (!(level[0] > 0.0F && level[1] > 0.0F && level[2] > 0.0F)) return;
  float target[3] = {level[1] / level[0], 1.0F, level[1] / level[2]};
  for (int k = 0; k < 3; ++k) {
    target[k] = target[k] < 0.0625F ? 0.0625F : target[k] > 16.0F ? 16.0F : target[k];
  }
  for (int k = 0; k < 3; ++k) {
    s->gains[k] = s->valid != 0 && smoothing < 1.0F ? s->gains[k] + smoothing * (target[k] - s->gains[k])
                                                    : target[k];
  }
  s->valid = 1;
}

/* finish_stats (isp_math.hpp:387-425). */
static void finish_stats(const uint64_t sum[3], uint64_t saturated, int64_t pixels,
                         const float gains[3], const isp_auto_exposure_c* ae,
                         const isp_exposure_c* exposure, float* out) {
  const double n = (double)pixels * (double)FIXED_ONE;
  const double mean[3] = {(double)sum[0] / n, (double)sum[1] / n, (double)sum[2] / n};
  const double luma = 0.2126 * mean[0] + 0.7152 * mean[1] + 0.0722 * mean[2];
  double error = luma > 0.0 ? log2((double)ae->target / luma) : 8.0;
  error = error < -8.0 ? -8.0 : error > 8.0 ? 8.0 : error;
  const double scale = exp2((double)ae->damping * error);
  double next_exposure = 0.0;
  double next_gain = 0.0;
  if (exposure->exposure_ns > 0) {
    const double gain = exposure->gain > 0.0F ? exposure->gain : ae->min_gain;
    const double wanted = (double)exposure->exposure_ns * gain * scale;
    next_exposure = wanted / ae->min_gain;
    const double low = (double)ae->min_exposure_ns;
    const double high = (double)ae->max_exposure_ns;
    next_exposure = next_exposure < low ? low : next_exposure > high ? high : next_exposure;
    next_gain = wanted / next_exposure;
    next_gain = next_gain < ae->min_gain ? ae->min_gain : next_gain > ae->max_gain ? ae->max_gain : next_gain;
  }
  out[0] = (float)mean[0];
  out[1] = (float)mean[1];
  out[2] = (float)mean[2];
  out[3] = (float)luma;
  out[4] = (float)error;
  out[5] = (float)scale;
  out[6] = (float)next_exposure;
  out[7] = (float)next_gain;
  out[8] = gains[0];
  out[9] = gains[1];
  out[10] = gains[2];
  out[11] = (float)((double)saturated / (double)pixels);
}

/* The quad loop of cpu_process (cpu_pipeline.cpp:101-119). */
static void awb_stats(const frame* p, oracle_awb_accum* a) {
  memset(a, 0, sizeof *a);
  for (int qy = 0; qy < p->height / 2; ++qy) {
    for (int qx = 0; qx < p->width / 2; ++qx) {
      int color[4];
      unsigned int fixed[4];
      int bin[4];
      if (!white_balance_quad(p, qx, qy, color, fixed, bin)) continue;
      for (int k = 0; k < 4; ++k) {
        a->sum[color[k]] += fixed[k];
        ++a->hist[color[k]][bin[k]];
      }
      ++a->quads;
    }
  }
}

void oracle_awb_stats(const isp_params_c* params, const isp_raw_view_c* raw, oracle_awb_accum* a) {
  const frame p = make_frame(params, raw, NULL, NULL, 0);
  awb_stats(&p, a);
}

/* RGB at every pixel and, with a border, at the virtual pixels around the
 * image, neighbours reflected (cpu_pipeline.cpp:22-46). */
static void demosaic_frame(const frame* p, int malvar, const float* samples, int border, float* rgb) {
  const int w = p->width + 2 * border;
  const int h = p->height + 2 * border;
  for (int ty = 0; ty < h; ++ty) {
    const int vy = ty - border;
    for (int tx = 0; tx < w; ++tx) {
      const int vx = tx - border;
      float n[5][5];
      for (int dy = -2; dy <= 2; ++dy) {
        const int y = mirror(vy + dy, p->height);
        for (int dx = -2; dx <= 2; ++dx) {
          n[dy + 2][dx + 2] = samples[(size_t)y * p->width + mirror(vx + dx, p->width)];
        }
      }
      demosaic(malvar, (const float(*)[5])n, channel_at(p, vx, vy), &rgb[((size_t)ty * w + tx) * 3U]);
    }
  }
}

/* IspPipeline(kCpu).process: validation (isp_pipeline.cpp:65-76), then
 * cpu_process (cpu_pipeline.cpp:97-191). */
int oracle_process(const isp_params_c* params, const isp_raw_view_c* raw, const isp_rgb_view_c* out,
                   const isp_stats_c* stats, const isp_exposure_c* exposure, oracle_awb_state* awb) {
  if (oracle_validate_params(params, NULL, 0) != ISP_OK) return ISP_EINVAL;
  if (oracle_validate_raw(raw, params, NULL, 0) != ISP_OK) return ISP_EINVAL;
  if (out == NULL || out->data == NULL || out->format < 0 || out->format > 3) return ISP_EINVAL;
  const int channels = out->format == ISP_OUT_RGBA8 ? 4 : 3;
  const int channel_bytes = out->format == ISP_OUT_RGB16 ? 2 : out->format == ISP_OUT_RGB32F ? 4 : 1;
  if (out->pitch < (size_t)raw->width * channels * channel_bytes || out->pitch % (size_t)channel_bytes) {
    return ISP_EINVAL;
  }
  const isp_stats_c none = {NULL, NULL};
  const isp_exposure_c unknown = {0, 0.0F};
  if (stats == NULL) stats = &none;
  if (exposure == NULL) exposure = &unknown;

  const size_t lut_size = oracle_tone_lut(params, NULL, 0);
  float* lut = (float*)malloc(lut_size * sizeof(float));
  oracle_tone_lut(params, lut, lut_size);
  const frame fp = make_frame(params, raw, out, lut, (int)lut_size);
  const frame* p = &fp;

  float gains[3] = {p->wb[0], p->wb[1], p->wb[2]};
  if (params->white_balance != ISP_WB_MANUAL) {
    oracle_awb_accum* a = (oracle_awb_accum*)malloc(sizeof *a);
    awb_stats(p, a);
    finish_white_balance(a, params->white_balance, params->white_patch_percentile,
                         params->awb_smoothing, awb);
    free(a);
    for (int k = 0; k < 3; ++k) gains[k] = awb->gains[k];
  }

  const size_t pixels = (size_t)p->width * p->height;
  float* samples = (float*)malloc(pixels * sizeof(float));
  for (int y = 0; y < p->height; ++y) {
    for (int x = 0; x < p->width; ++x) samples[(size_t)y * p->width + x] = preprocess(p, gains, x, y);
  }

  const int border = params->sharpen > 0.0F ? 1 : 0;
  const int w = p->width + 2 * border;
  const int h = p->height + 2 * border;
  float* rgb_all = (float*)malloc((size_t)w * h * 3U * sizeof(float));
  demosaic_frame(p, params->demosaic == ISP_DEMOSAIC_MALVAR, samples, border, rgb_all);

  uint64_t sums[3] = {0, 0, 0};
  uint64_t saturated = 0;
  for (int y = 0; y < p->height; ++y) {
    for (int x = 0; x < p->width; ++x) {
      float rgb[3];
      const float* centre = &rgb_all[((size_t)(y + border) * w + x + border) * 3U];
      if (border != 0) {
        float m[3][3][3];
        for (int dy = 0; dy < 3; ++dy) {
          for (int dx = 0; dx < 3; ++dx) {
            const float* v = &rgb_all[((size_t)(y + dy) * w + x + dx) * 3U];
            for (int k = 0; k < 3; ++k) m[dy][dx][k] = v[k];
          }
        }
        sharpen((const float(*)[3][3])m, p->sharpen, rgb);
      } else {
        for (int k = 0; k < 3; ++k) rgb[k] = centre[k];
      }
      float linear[3];
      correct_color(p, rgb, linear);
      if (stats->stats != NULL) {
        for (int k = 0; k < 3; ++k) sums[k] += to_fixed(linear[k]);
        saturated += load_raw(p, x, y) >= p->white ? 1U : 0U;
      }
      float toned[3];
      for (int k = 0; k < 3; ++k) toned[k] = tone(p, linear[k]);
      store(p, x, y, toned);
    }
  }

  if (stats->histogram != NULL) {
    memset(stats->histogram, 0, sizeof(uint32_t) * ISP_HISTOGRAM_CHANNELS * ISP_HISTOGRAM_BINS);
    for (int y = 0; y < p->height; ++y) {
      for (int x = 0; x < p->width; ++x) {
        int q[3];
        output_codes(p, x, y, q);
        ++stats->histogram[0 * ISP_HISTOGRAM_BINS + luma_code(q)];
        ++stats->histogram[1 * ISP_HISTOGRAM_BINS + q[0]];
        ++stats->histogram[2 * ISP_HISTOGRAM_BINS + q[1]];
        ++stats->histogram[3 * ISP_HISTOGRAM_BINS + q[2]];
      }
    }
  }
  if (stats->stats != NULL) {
    finish_stats(sums, saturated, (int64_t)pixels, gains, &params->auto_exposure, exposure,
                 stats->stats);
  }
  free(rgb_all);
  free(samples);
  free(lut);
  return ISP_OK;
}

/* The demo's side-by-side view (applications/isp/src/view_op.cu:35-75,
 * :143-150), restated: left half the raw mosaic as gray, g =
 * (uint8)(sqrtf(clamp((s - black) * scale, 0, 1)) * 255 + 0.5) with scale =
 * 1 / (2^bits - 1 - black) in single precision; right half the RGB8 image.
 * Host buffers. Parity unpinned: the demo's source needs the Holoscan SDK to
 * compile, so the reference kernel cannot be run here. */
void oracle_view_compose(const isp_raw_view_c* raw, float black, const uint8_t* rgb, size_t rgb_pitch, uint8_t* out,
                         size_t out_pitch) {
  frame p;
  memset(&p, 0, sizeof p);
  p.raw = (const unsigned char*)raw->data;
  p.raw_pitch = raw->pitch;
  p.raw_format = raw->format;
  const float white = (float)((1u << (unsigned)raw->bit_depth) - 1u);
  const float scale = 1.0F / (white - black);
  for (int y = 0; y < raw->height; ++y) {
    uint8_t* o = out + (size_t)y * out_pitch;
    const uint8_t* i = rgb + (size_t)y * rgb_pitch;
    for (int x = 0; x < raw->width; ++x) {
      float v = ((float)load_raw(&p, x, y) - black) * scale;
      v = v < 0.0F ? 0.0F : v > 1.0F ? 1.0F : v;
      const uint8_t g = (uint8_t)(sqrtf(v) * 255.0F + 0.5F);
      o[3 * x] = o[3 * x + 1] = o[3 * x + 2] = g;
      o[3 * (raw->width + x)] = i[3 * x];
      o[3 * (raw->width + x) + 1] = i[3 * x + 1];
      o[3 * (raw->width + x) + 2] = i[3 * x + 2];
    }
  }
}
