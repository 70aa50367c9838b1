/*
 * cc_oracle.c - TEST INFRASTRUCTURE ONLY: a CPU restatement, in plain C, of
 * the holoscan::color_convert conversion, the checker of the B200 colour
 * converter. Used by tests/ and by bench.py's CPU baseline; never by the
 * product.
 *
 * It follows the reference's definition step by step:
 *   geometry   modules/color-convert/src/conversion.cpp:362-401 (compute_mapping)
 *              and :154-168 (fit_axis)
 *   checks     conversion.cpp:170-192 (check_view), :403-408
 *   colour     conversion.cpp:93-209 (luma weights, quantization, to_rgb,
 *              from_rgb, compose), :410-447 (make_plan)
 *   per pixel  src/kernel_math.hpp:89-161 (codes, loading), :163-233
 *              (weights and the three samplers), :236-254 (affine, fill),
 *              :256-341 (stores), :345-370 (blocks)
 *   pattern    include/holoscan/color_convert/reference.hpp:34-55
 * Single-precision operations one at a time, in the reference's order; the
 * file is compiled with -ffp-contract=off. Pinned against the reference
 * built from its own sources (oracle/_ref/libcc_ref.so) and against the
 * fixtures in tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "cc_b200.h"

enum { M_YUV = 0, M_RGB = 1, M_GRAY = 2 };

typedef struct {
  int model, planes, sx, sy, bytes, channels;
} finfo;

static finfo info(int f) {
  static const finfo t[CC_FORMAT_COUNT] = {
      {M_YUV, 2, 1, 1, 1, 1}, {M_YUV, 2, 1, 0, 1, 1}, {M_YUV, 3, 1, 1, 1, 1}, {M_YUV, 1, 1, 0, 1, 2},
      {M_YUV, 1, 1, 0, 1, 2}, {M_RGB, 1, 0, 0, 1, 3}, {M_RGB, 1, 0, 0, 1, 3}, {M_RGB, 1, 0, 0, 1, 4},
      {M_RGB, 1, 0, 0, 1, 4}, {M_GRAY, 1, 0, 0, 1, 1}, {M_GRAY, 1, 0, 0, 2, 1}, {M_RGB, 1, 0, 0, 2, 3}};
  return t[f];
}

static const char* const fnames[CC_FORMAT_COUNT] = {"nv12",  "nv16",  "i420",  "yuyv",  "uyvy",   "rgb8",
                                                    "bgr8",  "rgba8", "bgra8", "mono8", "mono16", "rgb16"};

typedef struct {
  const cc_image_c* src;
  const cc_image_c* dst;
  int mode;
  int x0, y0, x1, y1;
  float sx, sy;
  int cx0, cy0, cx1, cy1;
  float m[9], o[3];
  int same_model;
  float fill[4];
  int bx_shift, by_shift;
} plan_t;

typedef struct {
  float s[4]; /* Y/R/luma, Cb/G, Cr/B, alpha */
} px_t;

static char* g_err;
static size_t g_errlen;

static int fail(const char* msg) {
  if (g_err != NULL && g_errlen > 0) snprintf(g_err, g_errlen, "%s", msg);
  return ISP_EINVAL;
}

/* ---- geometry and checks ---- */

static void plane_dims(int f, int w, int h, int k, size_t* row_bytes, int* rows) {
  finfo fi = info(f);
  if (k == 0) {
    *row_bytes = (size_t)w * (size_t)(fi.channels * fi.bytes);
    *rows = h;
    return;
  }
  size_t cw = ((size_t)w + ((1u << fi.sx) - 1u)) >> fi.sx;
  *rows = (h + (1 << fi.sy) - 1) >> fi.sy;
  *row_bytes = cw * (fi.planes == 2 ? 2u : 1u);
}

size_t cc_oracle_packed_size(int f, int w, int h) {
  size_t total = 0;
  for (int k = 0; k < info(f).planes; ++k) {
    size_t rb;
    int rows;
    plane_dims(f, w, h, k, &rb, &rows);
    total += rb * (size_t)rows;
  }
  return total;
}

static void fit_one(double scaled, int size, int even, int* content, int* offset) {
  int c = (int)lround(scaled);
  if (c < 1) c = 1;
  if (c > size) c = size;
  if (c == size) {
    *content = size;
    *offset = 0;
    return;
  }
  if (even) {
    c &= ~1;
    if (c < 2) c = 2;
  }
  int o = (size - c) / 2;
  if (even) o &= ~1;
  *content = c;
  *offset = o;
}

int cc_oracle_mapping(int sw, int sh, int w, int h, int dst_format, const cc_params_c* p, cc_mapping_c* out,
                      char* err, size_t errlen) {
  g_err = err;
  g_errlen = errlen;
  char msg[256];
  if (sw <= 0 || sh <= 0 || w <= 0 || h <= 0) return fail("image sizes must be positive");
  cc_rect_c src = {0, 0, sw, sh};
  if (p->has_crop) {
    cc_rect_c c = p->crop;
    if (c.width <= 0 || c.height <= 0 || c.x < 0 || c.y < 0 || c.x > sw - c.width || c.y > sh - c.height) {
      snprintf(msg, sizeof msg, "crop %dx%d+%d+%d is not inside the %dx%d source", c.width, c.height, c.x, c.y, sw,
               sh);
      return fail(msg);
    }
    src = c;
  }
  cc_rect_c content = {0, 0, w, h};
  if (p->letterbox) {
    double a = (double)w / src.width, b = (double)h / src.height;
    double scale = a < b ? a : b;
    finfo fi = info(dst_format);
    fit_one(src.width * scale, w, fi.sx != 0, &content.width, &content.x);
    fit_one(src.height * scale, h, fi.sy != 0, &content.height, &content.y);
  }
  out->source = src;
  out->content = content;
  return ISP_OK;
}

static int check_one(const cc_image_c* v, const char* which) {
  char msg[256];
  if (v->width <= 0 || v->height <= 0) {
    snprintf(msg, sizeof msg, "%s image size must be positive", which);
    return fail(msg);
  }
  if ((v->format == CC_YUYV || v->format == CC_UYVY) && v->width % 2 != 0) {
    snprintf(msg, sizeof msg, "%s image: %s needs an even width, not %d", which, fnames[v->format], v->width);
    return fail(msg);
  }
  for (int k = 0; k < info(v->format).planes; ++k) {
    size_t rb;
    int rows;
    plane_dims(v->format, v->width, v->height, k, &rb, &rows);
    if (v->planes[k].data == NULL) {
      snprintf(msg, sizeof msg, "%s image plane %d has no data", which, k);
      return fail(msg);
    }
    if (v->planes[k].pitch < rb) {
      snprintf(msg, sizeof msg, "%s image plane %d pitch %zu is shorter than a row of %zu bytes", which, k,
               v->planes[k].pitch, rb);
      return fail(msg);
    }
  }
  return ISP_OK;
}

/* ---- colour maps, double precision ---- */

typedef struct {
  double a[3][4];
} map34;

static map34 map_identity(void) {
  map34 r;
  memset(&r, 0, sizeof r);
  r.a[0][0] = r.a[1][1] = r.a[2][2] = 1.0;
  return r;
}

static void luma_kr_kb(int matrix, double* kr, double* kb) {
  if (matrix == CC_BT709) {
    *kr = 0.2126;
    *kb = 0.0722;
  } else if (matrix == CC_BT2020) {
    *kr = 0.2627;
    *kb = 0.0593;
  } else {
    *kr = 0.299;
    *kb = 0.114;
  }
}

static void quant(int range, double* ys, double* yo, double* cs) {
  int limited = range == CC_RANGE_LIMITED;
  *ys = limited ? 219.0 : 255.0;
  *yo = limited ? 16.0 : 0.0;
  *cs = limited ? 224.0 : 255.0;
}

static map34 to_rgb(int model, int matrix, int range) {
  map34 n;
  memset(&n, 0, sizeof n);
  if (model == M_RGB) return map_identity();
  if (model == M_GRAY) {
    n.a[0][0] = n.a[1][0] = n.a[2][0] = 1.0;
    return n;
  }
  double kr, kb, ys, yo, cs;
  luma_kr_kb(matrix, &kr, &kb);
  quant(range, &ys, &yo, &cs);
  double kg = 1.0 - kr - kb;
  double ry = 1.0 / ys, rc = 1.0 / cs;
  double r_cr = 2.0 * (1.0 - kr), b_cb = 2.0 * (1.0 - kb);
  double g_cb = -kb * b_cb / kg, g_cr = -kr * r_cr / kg;
  double yoff = -yo * ry;
  n.a[0][0] = ry;
  n.a[0][2] = r_cr * rc;
  n.a[0][3] = yoff - r_cr * rc * 128.0;
  n.a[1][0] = ry;
  n.a[1][1] = g_cb * rc;
  n.a[1][2] = g_cr * rc;
  n.a[1][3] = yoff - (g_cb + g_cr) * rc * 128.0;
  n.a[2][0] = ry;
  n.a[2][1] = b_cb * rc;
  n.a[2][3] = yoff - b_cb * rc * 128.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) n.a[i][j] *= 255.0;
  return n;
}

static map34 from_rgb(int model, int matrix, int range) {
  map34 r;
  memset(&r, 0, sizeof r);
  if (model == M_RGB) return map_identity();
  double kr, kb;
  luma_kr_kb(matrix, &kr, &kb);
  double kg = 1.0 - kr - kb;
  if (model == M_GRAY) {
    r.a[0][0] = kr;
    r.a[0][1] = kg;
    r.a[0][2] = kb;
    return r;
  }
  double ys, yo, cs;
  quant(range, &ys, &yo, &cs);
  double cbd = 2.0 * (1.0 - kb), crd = 2.0 * (1.0 - kr);
  double s = ys / 255.0, c = cs / 255.0;
  r.a[0][0] = kr * s;
  r.a[0][1] = kg * s;
  r.a[0][2] = kb * s;
  r.a[0][3] = yo;
  r.a[1][0] = -kr / cbd * c;
  r.a[1][1] = -kg / cbd * c;
  r.a[1][2] = (1.0 - kb) / cbd * c;
  r.a[1][3] = 128.0;
  r.a[2][0] = (1.0 - kr) / crd * c;
  r.a[2][1] = -kg / crd * c;
  r.a[2][2] = -kb / crd * c;
  r.a[2][3] = 128.0;
  return r;
}

static map34 compose(const map34* outer, const map34* inner) {
  map34 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) {
      double v = j == 3 ? outer->a[i][3] : 0.0;
      for (int k = 0; k < 3; ++k) v += outer->a[i][k] * inner->a[k][j];
      r.a[i][j] = v;
    }
  return r;
}

/* ---- per pixel ---- */

static uint8_t u8_of(float v) {
  float r = floorf(v + 0.5f);
  return (uint8_t)(r <= 0.0f ? 0.0f : (r >= 255.0f ? 255.0f : r));
}

static uint16_t u16_of(float v) {
  float r = floorf(v * 257.0f + 0.5f);
  return (uint16_t)(r <= 0.0f ? 0.0f : (r >= 65535.0f ? 65535.0f : r));
}

static float w16(const uint8_t* p) { return (float)(uint16_t)(p[0] | (p[1] << 8)) / 257.0f; }

static px_t mk(float a, float b, float c, float d) {
  px_t r;
  r.s[0] = a;
  r.s[1] = b;
  r.s[2] = c;
  r.s[3] = d;
  return r;
}

static px_t fetch(const cc_image_c* im, int x, int y) {
  const uint8_t* row = im->planes[0].data + (size_t)y * im->planes[0].pitch;
  switch (im->format) {
    case CC_NV12:
    case CC_NV16: {
      int cy = im->format == CC_NV12 ? y >> 1 : y;
      const uint8_t* uv = im->planes[1].data + (size_t)cy * im->planes[1].pitch + 2 * (x >> 1);
      return mk(row[x], uv[0], uv[1], 255.0f);
    }
    case CC_I420:
      return mk(row[x], im->planes[1].data[(size_t)(y >> 1) * im->planes[1].pitch + (x >> 1)],
                im->planes[2].data[(size_t)(y >> 1) * im->planes[2].pitch + (x >> 1)], 255.0f);
    case CC_YUYV: {
      const uint8_t* q = row + 4 * (x >> 1);
      return mk(q[2 * (x & 1)], q[1], q[3], 255.0f);
    }
    case CC_UYVY: {
      const uint8_t* q = row + 4 * (x >> 1);
      return mk(q[1 + 2 * (x & 1)], q[0], q[2], 255.0f);
    }
    case CC_RGB8:
      return mk(row[3 * x], row[3 * x + 1], row[3 * x + 2], 255.0f);
    case CC_BGR8:
      return mk(row[3 * x + 2], row[3 * x + 1], row[3 * x], 255.0f);
    case CC_RGBA8:
      return mk(row[4 * x], row[4 * x + 1], row[4 * x + 2], row[4 * x + 3]);
    case CC_BGRA8:
      return mk(row[4 * x + 2], row[4 * x + 1], row[4 * x], row[4 * x + 3]);
    case CC_MONO8:
      return mk(row[x], 0.0f, 0.0f, 255.0f);
    case CC_MONO16:
      return mk(w16(row + 2 * x), 0.0f, 0.0f, 255.0f);
    default:
      return mk(w16(row + 6 * x), w16(row + 6 * x + 2), w16(row + 6 * x + 4), 255.0f);
  }
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static px_t add_w(px_t acc, px_t s, float w) {
  for (int i = 0; i < 4; ++i) {
    float t = s.s[i] * w;
    acc.s[i] = acc.s[i] + t;
  }
  return acc;
}

static float cover(int i, float lo, float hi) {
  float a = (float)i > lo ? (float)i : lo;
  float b = (float)(i + 1) < hi ? (float)(i + 1) : hi;
  return b > a ? b - a : 0.0f;
}

static px_t sample(const plan_t* p, int dx, int dy) {
  float rx = (float)(dx - p->cx0), ry = (float)(dy - p->cy0);
  float x0 = (float)p->x0, y0 = (float)p->y0;
  if (p->mode == CC_NEAREST) {
    float tx = (rx + 0.5f) * p->sx;
    float ty = (ry + 0.5f) * p->sy;
    int sx = clampi((int)floorf(x0 + tx), p->x0, p->x1);
    int sy = clampi((int)floorf(y0 + ty), p->y0, p->y1);
    return fetch(p->src, sx, sy);
  }
  if (p->mode == CC_BILINEAR) {
    float tx = (rx + 0.5f) * p->sx;
    float ty = (ry + 0.5f) * p->sy;
    float fx = (x0 + tx) - 0.5f;
    float fy = (y0 + ty) - 0.5f;
    float bx = floorf(fx), by = floorf(fy);
    float ax = fx - bx, ay = fy - by;
    int ix = (int)bx, iy = (int)by;
    int xa = clampi(ix, p->x0, p->x1), xb = clampi(ix + 1, p->x0, p->x1);
    int ya = clampi(iy, p->y0, p->y1), yb = clampi(iy + 1, p->y0, p->y1);
    float nx = 1.0f - ax, ny = 1.0f - ay;
    float w[4] = {nx * ny, ax * ny, nx * ay, ax * ay};
    int tx4[4] = {xa, xb, xa, xb}, ty4[4] = {ya, ya, yb, yb};
    px_t s = mk(0.0f, 0.0f, 0.0f, 0.0f);
    for (int t = 0; t < 4; ++t)
      if (w[t] != 0.0f) s = add_w(s, fetch(p->src, tx4[t], ty4[t]), w[t]);
    return s;
  }
  float lx = x0 + rx * p->sx;
  float ly = y0 + ry * p->sy;
  float right = (float)(p->x1 + 1), bottom = (float)(p->y1 + 1);
  float ex = lx + p->sx, ey = ly + p->sy;
  float hx = ex < right ? ex : right;
  float hy = ey < bottom ? ey : bottom;
  int ix0 = clampi((int)floorf(lx), p->x0, p->x1);
  int iy0 = clampi((int)floorf(ly), p->y0, p->y1);
  px_t s = mk(0.0f, 0.0f, 0.0f, 0.0f);
  float total = 0.0f;
  for (int y = iy0; y <= p->y1 && (float)y < hy; ++y) {
    float wy = cover(y, ly, hy);
    for (int x = ix0; x <= p->x1 && (float)x < hx; ++x) {
      float w = cover(x, lx, hx) * wy;
      if (w != 0.0f) {
        s = add_w(s, fetch(p->src, x, y), w);
        total = total + w;
      }
    }
  }
  if (total <= 0.0f) return fetch(p->src, ix0, iy0);
  return mk(s.s[0] / total, s.s[1] / total, s.s[2] / total, s.s[3] / total);
}

static px_t dst_pixel(const plan_t* p, int x, int y) {
  if (x < p->cx0 || x >= p->cx1 || y < p->cy0 || y >= p->cy1) return mk(p->fill[0], p->fill[1], p->fill[2], p->fill[3]);
  px_t s = sample(p, x, y);
  if (p->same_model) return s;
  px_t r;
  for (int i = 0; i < 3; ++i) {
    float t0 = p->m[3 * i] * s.s[0];
    float t1 = p->m[3 * i + 1] * s.s[1];
    float t2 = p->m[3 * i + 2] * s.s[2];
    float acc = t0 + t1;
    acc = acc + t2;
    r.s[i] = acc + p->o[i];
  }
  r.s[3] = s.s[3];
  return r;
}

static void put16(uint8_t* q, float v) {
  uint16_t w = u16_of(v);
  q[0] = (uint8_t)(w & 0xFF);
  q[1] = (uint8_t)(w >> 8);
}

static void put(const cc_image_c* im, int x, int y, px_t v) {
  uint8_t* row = im->planes[0].data + (size_t)y * im->planes[0].pitch;
  switch (im->format) {
    case CC_NV12:
    case CC_NV16:
    case CC_I420:
    case CC_MONO8:
      row[x] = u8_of(v.s[0]);
      break;
    case CC_YUYV:
      row[4 * (x >> 1) + 2 * (x & 1)] = u8_of(v.s[0]);
      break;
    case CC_UYVY:
      row[4 * (x >> 1) + 1 + 2 * (x & 1)] = u8_of(v.s[0]);
      break;
    case CC_RGB8:
    case CC_BGR8: {
      int bgr = im->format == CC_BGR8;
      row[3 * x] = u8_of(bgr ? v.s[2] : v.s[0]);
      row[3 * x + 1] = u8_of(v.s[1]);
      row[3 * x + 2] = u8_of(bgr ? v.s[0] : v.s[2]);
      break;
    }
    case CC_RGBA8:
    case CC_BGRA8: {
      int bgr = im->format == CC_BGRA8;
      row[4 * x] = u8_of(bgr ? v.s[2] : v.s[0]);
      row[4 * x + 1] = u8_of(v.s[1]);
      row[4 * x + 2] = u8_of(bgr ? v.s[0] : v.s[2]);
      row[4 * x + 3] = u8_of(v.s[3]);
      break;
    }
    case CC_MONO16:
      put16(row + 2 * x, v.s[0]);
      break;
    default:
      put16(row + 6 * x, v.s[0]);
      put16(row + 6 * x + 2, v.s[1]);
      put16(row + 6 * x + 4, v.s[2]);
      break;
  }
}

static void put_chroma(const cc_image_c* im, int cx, int cy, float cb, float cr) {
  switch (im->format) {
    case CC_NV12:
    case CC_NV16: {
      uint8_t* q = im->planes[1].data + (size_t)cy * im->planes[1].pitch + 2 * cx;
      q[0] = u8_of(cb);
      q[1] = u8_of(cr);
      break;
    }
    case CC_I420:
      im->planes[1].data[(size_t)cy * im->planes[1].pitch + cx] = u8_of(cb);
      im->planes[2].data[(size_t)cy * im->planes[2].pitch + cx] = u8_of(cr);
      break;
    case CC_YUYV: {
      uint8_t* q = im->planes[0].data + (size_t)cy * im->planes[0].pitch + 4 * cx;
      q[1] = u8_of(cb);
      q[3] = u8_of(cr);
      break;
    }
    case CC_UYVY: {
      uint8_t* q = im->planes[0].data + (size_t)cy * im->planes[0].pitch + 4 * cx;
      q[0] = u8_of(cb);
      q[2] = u8_of(cr);
      break;
    }
    default:
      break;
  }
}

/* reference_convert (modules/color-convert/src/reference.cpp:14-27) over host
 * images; rows [row_first, row_last) of destination blocks only, so that a
 * caller may split the work across threads. */
int cc_oracle_convert_rows(const cc_image_c* src, const cc_image_c* dst, const cc_params_c* params, int row_first,
                           int row_last, char* err, size_t errlen) {
  g_err = err;
  g_errlen = errlen;
  if (src->format < 0 || src->format >= CC_FORMAT_COUNT || dst->format < 0 || dst->format >= CC_FORMAT_COUNT)
    return fail("unknown pixel format");
  if (src->location != CC_HOST || dst->location != CC_HOST) return fail("reference_convert needs host images");
  int s = check_one(src, "source");
  if (s != ISP_OK) return s;
  s = check_one(dst, "destination");
  if (s != ISP_OK) return s;
  cc_mapping_c map;
  s = cc_oracle_mapping(src->width, src->height, dst->width, dst->height, dst->format, params, &map, err, errlen);
  if (s != ISP_OK) return s;

  plan_t p;
  memset(&p, 0, sizeof p);
  p.src = src;
  p.dst = dst;
  p.mode = params->mode;
  p.x0 = map.source.x;
  p.y0 = map.source.y;
  p.x1 = map.source.x + map.source.width - 1;
  p.y1 = map.source.y + map.source.height - 1;
  p.sx = (float)((double)map.source.width / (double)map.content.width);
  p.sy = (float)((double)map.source.height / (double)map.content.height);
  p.cx0 = map.content.x;
  p.cy0 = map.content.y;
  p.cx1 = map.content.x + map.content.width;
  p.cy1 = map.content.y + map.content.height;
  int from = info(src->format).model, to = info(dst->format).model;
  p.same_model = from == to;
  map34 out = from_rgb(to, params->matrix, params->range);
  map34 in = to_rgb(from, params->matrix, params->range);
  map34 both = compose(&out, &in);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) p.m[3 * i + j] = (float)both.a[i][j];
    p.o[i] = (float)both.a[i][3];
    double v = out.a[i][3];
    for (int k = 0; k < 3; ++k) v += out.a[i][k] * params->fill_rgb[k];
    p.fill[i] = (float)v;
  }
  p.fill[3] = 255.0f;
  finfo di = info(dst->format);
  p.bx_shift = di.model == M_YUV ? di.sx : 0;
  p.by_shift = di.model == M_YUV ? di.sy : 0;

  int across = (dst->width + (1 << p.bx_shift) - 1) >> p.bx_shift;
  int down = (dst->height + (1 << p.by_shift) - 1) >> p.by_shift;
  if (row_last > down) row_last = down;
  for (int by = row_first; by < row_last; ++by) {
    for (int bx = 0; bx < across; ++bx) {
      if (di.model != M_YUV) {
        put(dst, bx, by, dst_pixel(&p, bx, by));
        continue;
      }
      int xs = bx << p.bx_shift, ys = by << p.by_shift;
      int xe = xs + (1 << p.bx_shift) < dst->width ? xs + (1 << p.bx_shift) : dst->width;
      int ye = ys + (1 << p.by_shift) < dst->height ? ys + (1 << p.by_shift) : dst->height;
      float cb = 0.0f, cr = 0.0f;
      int n = 0;
      for (int y = ys; y < ye; ++y)
        for (int x = xs; x < xe; ++x) {
          px_t v = dst_pixel(&p, x, y);
          put(dst, x, y, v);
          cb = cb + v.s[1];
          cr = cr + v.s[2];
          ++n;
        }
      put_chroma(dst, bx, by, cb / (float)n, cr / (float)n);
    }
  }
  return ISP_OK;
}

int cc_oracle_convert(const cc_image_c* src, const cc_image_c* dst, const cc_params_c* params, char* err,
                      size_t errlen) {
  return cc_oracle_convert_rows(src, dst, params, 0, 1 << 30, err, errlen);
}

/* The synthetic camera's picture, frame `frame`, into a host RGB8 image. */
void cc_oracle_test_pattern(uint8_t* data, size_t pitch, int width, int height, uint32_t frame) {
  static const int bars[8] = {7, 6, 3, 2, 5, 4, 1, 0};
  int top = (2 * height) / 3;
  for (int y = 0; y < height; ++y) {
    uint8_t* row = data + (size_t)y * pitch;
    for (int x = 0; x < width; ++x) {
      uint8_t* q = row + 3 * x;
      if (y < top) {
        int shift = (int)((frame * 4u) % (uint32_t)width);
        int col = (x + width - shift) % width;
        int c = bars[(col * 8) / width];
        q[0] = (c & 4) ? 255 : 0;
        q[1] = (c & 2) ? 255 : 0;
        q[2] = (c & 1) ? 255 : 0;
      } else {
        int rows = height - top;
        int gray = width > 1 ? (x * 255) / (width - 1) : 0;
        int blue = rows > 1 ? ((y - top) * 255) / (rows - 1) : 0;
        q[0] = (uint8_t)((gray + 255 - blue) / 2);
        q[1] = (uint8_t)gray;
        q[2] = (uint8_t)((gray + blue) / 2);
      }
    }
  }
}
