// isp_pairs.cuh - the three phases of the fused tile pass on paired pixels.
//
// A 64x64 tile is processed as 64 rows of 32 pixel pairs: pair c of a row
// holds columns c and c + 32, which have the same Bayer colour, so one f32x2
// instruction advances both through identical IEEE operations (isp_ops.cuh).
// Shared memory keeps samples and RGB values as float2 pairs
// {v(c), v(c + 32)}; a neighbour of a pair is the neighbouring pair, loaded
// as one aligned 8- or 16-byte element.
//
//   A. samples: unpack the raw box, black level, lens shading, white balance
//      and clip (preprocess, isp_math.hpp:144-155) into the paired sample
//      plane P[kSH][kPW]: pair s holds samples s and s + 32 of the tile's
//      72 (image columns x0 - 4 + s);
//   B. (sharpening) demosaic every pixel of the tile and its one-pixel ring
//      into the paired RGB planes R, G, B [66][kCW2]: pair q holds pixels
//      q - 1 and q + 31 (isp_math.hpp:161-214; the ring outside the image is
//      the reference's virtual pixels, cpu_pipeline.cpp:22-46);
//   C. per unit of four pairs of one row: demosaic (or sharpen,
//      isp_math.hpp:219-227), colour matrix, statistics sums, tone, store and
//      histogram codes (isp_math.hpp:229-305).
#pragma once

#include "isp_common.cuh"

namespace isp_b200 {
namespace {

constexpr int kUnitsA = kPW / 4;  // phase A units per sample row: 4 pairs each

// Bank spread of the sample plane. Pair s of sample row j sits at
// j * kPW + (s ^ psw(j)): rows 2k and 2k + 1 keep their order, rows 2k + 2
// and 2k + 3 swap neighbouring 16-byte chunks, so that a quarter-warp
// reading four groups of row r and four of row r + 2 (same Bayer parity)
// meets every bank once. Accesses are whole 16-byte chunks (even s).
__device__ __forceinline__ int psw(int j) { return ((j >> 1) & 1) << 1; }

// Bank spread of the RGB planes (rows of 17 16-byte chunks): chunk c < 16 of
// row j sits at j * 17 + (c ^ csw(j)), rows 2k and 2k + 1 in order, rows
// 2k + 2 and 2k + 3 with neighbouring chunks swapped (chunk 16, the ring,
// stays), so that a quarter-warp reading four groups of each of two row
// pairs (rows r + a and r + 2 + a) meets every bank once but for chunk 16.
__device__ __forceinline__ int csw(int j) { return (j >> 1) & 1; }
__device__ __forceinline__ int cchunk(int c, int sw) { return c < kCW2 / 2 - 1 ? c ^ sw : c; }

__device__ __forceinline__ float4 lds4(Span<const float2> p) { return *span_cast<const float4>(p); }
__device__ __forceinline__ void sts4(Span<float2> p, float2 a, float2 b) {
  *span_cast<float4>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// A. Samples of the tile and its halo as pairs; returns the saturated count
//    of the tile's own samples (raw >= white, isp_math.hpp:316), each counted
//    once. kSrc: 0 interior tile from the TMA box, 1 edge tile from the box
//    (mirrored columns), 2 no box (global loads, mirrored).
template <int kFmt, int kSrc, int kHalo, int kTileH>
__device__ __forceinline__ unsigned int phase_a2(const FrameDesc& p, const TileCtx& t, Span<float2> P, int box_bytes,
                                                 const float (&qblack)[4], const float (&qinv)[4],
                                                 const float (&qgain)[4], bool want_stats) {
  constexpr int kSH = kTileH + 2 * kHalo;
  const unsigned int white = static_cast<unsigned int>(p.white);
  unsigned int saturated = 0;
  for (int unit = threadIdx.x; unit < kUnitsA * kSH; unit += kThreads) {
    const int j = unit / kUnitsA;
    const int u = unit - j * kUnitsA;
    const int par = j & 1;  // row parity: y0 - halo is even
    unsigned int sl[4], sr[4];  // samples 4u + k and 4u + 32 + k
    if constexpr (kSrc == 0) {
      Span<const uint8_t> row = t.box + j * box_bytes;
      unpack4(kFmt, row, u, sl);
      unpack4(kFmt, row, u + kHalf / 4, sr);
    } else if constexpr (kSrc == 1) {
      Span<const uint8_t> row = t.box + (t.row_my[j] - (t.y0 - kHalo)) * box_bytes;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        sl[k] = unpack1(kFmt, row, t.col_mx[4 * u + k], t.x0);
        sr[k] = unpack1(kFmt, row, t.col_mx[4 * u + kHalf + k], t.x0);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        sl[k] = static_cast<unsigned int>(load_raw(p, t.col_mx[4 * u + k], t.row_my[j]));
        sr[k] = static_cast<unsigned int>(load_raw(p, t.col_mx[4 * u + kHalf + k], t.row_my[j]));
      }
    }
    // Tile samples are s = 4 .. 67: the left lanes of units 1..8 hold 4..35,
    // their right lanes 36..67.
    if (want_stats && j >= kHalo && j < kHalo + kTileH && u >= 1 && u <= kHalf / 4) {
      const int y = t.y0 + j - kHalo;
      const int xl = t.x0 + 4 * (u - 1);
      if (y < p.height) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          saturated += (xl + k < p.width && sl[k] >= white) ? 1U : 0U;
          saturated += (xl + kHalf + k < p.width && sr[k] >= white) ? 1U : 0U;
        }
      }
    }
    // The row's two quad positions' constants.
    const float bl0 = par ? qblack[2] : qblack[0];
    const float bl1 = par ? qblack[3] : qblack[1];
    const float iv0 = par ? qinv[2] : qinv[0];
    const float iv1 = par ? qinv[3] : qinv[1];
    const float gn0 = par ? qgain[2] : qgain[0];
    const float gn1 = par ? qgain[3] : qgain[1];
    float2 v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      // linearize (isp_math.hpp:144-148): max((raw - black) * inv_range, 0).
      const float2 raw = magic_to_float2(sl[k] | kTwo23Bits, sr[k] | kTwo23Bits);
      const float2 x = mul2(sub2(raw, bc2((k & 1) ? bl1 : bl0)), bc2((k & 1) ? iv1 : iv0));
      v[k] = make_float2(fmaxf(x.x, 0.0F), fmaxf(x.y, 0.0F));
    }
    if (t.lt.rows > 0) {
      if (t.lt.rows <= kLscTableRows) {
        const int kk = t.row_k[j];
        const int pl = p.lsc_channels == 4 ? par : 0;
        Span<const float2> r0 = t.table + (kk * 2 + pl) * kPW + 4 * u;
        Span<const float2> r1 = t.table + ((kk + 1) * 2 + pl) * kPW + 4 * u;
        const float4 a0 = lds4(r0), b0 = lds4(r0 + 2), a1 = lds4(r1), b1 = lds4(r1 + 2);
        const float2 t0[4] = {lo2(a0), hi2(a0), lo2(b0), hi2(b0)};
        const float2 t1[4] = {lo2(a1), hi2(a1), lo2(b1), hi2(b1)};
        const float2 ty = bc2(t.row_ty[j]);
        // top + (bottom - top) * ty (isp_math.hpp:121-140); the product is
        // rounded, so the sum runs per lane (isp_ops.cuh).
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = mul2(v[k], add_lanes(t0[k], mul2(sub2(t1[k], t0[k]), ty)));
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int ch = p.cfa[(par << 1) | (k & 1)];
          v[k].x = fmul(v[k].x, lens_shading_gain(p, t.grid, t.col_mx[4 * u + k], t.row_my[j], ch));
          v[k].y = fmul(v[k].y, lens_shading_gain(p, t.grid, t.col_mx[4 * u + kHalf + k], t.row_my[j], ch));
        }
      }
    }
    // White balance and the clip to 1 (v >= 0): the saturating multiply.
    Span<float2> dst = P + j * kPW;
    const int sw = psw(j);
    sts4(dst + ((4 * u) ^ sw), mul_sat2(v[0], bc2(gn0)), mul_sat2(v[1], bc2(gn1)));
    sts4(dst + ((4 * u + 2) ^ sw), mul_sat2(v[2], bc2(gn0)), mul_sat2(v[3], bc2(gn1)));
  }
  return saturated;
}

template <int kSrc, int kHalo, int kTileH>
__device__ __forceinline__ unsigned int phase_a2_fmt(const FrameDesc& p, const TileCtx& t, Span<float2> P, int box_bytes,
                                                     const float (&qblack)[4], const float (&qinv)[4],
                                                     const float (&qgain)[4], bool want_stats) {
  // Global loads (no TMA box) read the format at run time in load_raw.
  if constexpr (kSrc == 2) return phase_a2<kRawU8, kSrc, kHalo, kTileH>(p, t, P, box_bytes, qblack, qinv, qgain, want_stats);
  switch (p.raw_format) {
    case kRawU8: return phase_a2<kRawU8, kSrc, kHalo, kTileH>(p, t, P, box_bytes, qblack, qinv, qgain, want_stats);
    case kRawU16: return phase_a2<kRawU16, kSrc, kHalo, kTileH>(p, t, P, box_bytes, qblack, qinv, qgain, want_stats);
    case kRawRaw10: return phase_a2<kRawRaw10, kSrc, kHalo, kTileH>(p, t, P, box_bytes, qblack, qinv, qgain, want_stats);
    default: return phase_a2<kRawRaw12, kSrc, kHalo, kTileH>(p, t, P, box_bytes, qblack, qinv, qgain, want_stats);
  }
}

// B. (Sharpening) RGB of the tile and its ring into the paired planes, in
//    units of 2 rows x 2 pairs: 33 x 17 units cover the 66 x 34 pairs.
//    RGB pair (row cr, column q): pixels (q - 1, q + 31) of image row
//    y0 - 1 + cr, whose sample pair is P[cr + 3][q + 3] (halo 4).
//    With swap_rb the demosaic's red and blue go to the other planes: the
//    demosaic runs as the layout's canonical pattern (RGGB or GRBG), and
//    BGGR and GBRG trade red and blue.
template <bool kMalvar, int kPat, int kTileH>
__device__ __forceinline__ void phase_b2(Span<const float2> P, Span<float2> R, Span<float2> G, Span<float2> B) {
  constexpr int kUnitsQ = kCW2 / 2;                   // 17
  constexpr int kUnits = (kTileH + 2) / 2 * kUnitsQ;  // 33 x 17 for 64 rows
  for (int unit = threadIdx.x; unit < kUnits; unit += kThreads) {
    const int ur = unit / kUnitsQ;
    const int uq = unit - ur * kUnitsQ;
    // Window w[a][b] = P[2ur + 1 + a][2uq + 1 + b]; rows 0 and 5 need columns
    // 2..3, rows 1 and 4 columns 1..4, rows 2 and 3 columns 0..5 (Malvar);
    // bilinear needs rows 1..4, columns 1..4.
    float2 w[6][6] = {};
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      const int j = 2 * ur + 1 + a;
      Span<const float2> row = P + j * kPW;  // pair 2uq is w column -1
      const int sw = psw(j);
      const bool edge = a == 0 || a == 5;
      const bool mid = a == 2 || a == 3;
      if (!kMalvar && edge) continue;
      const float4 m1 = lds4(row + ((2 * uq + 2) ^ sw)), m2 = lds4(row + ((2 * uq + 4) ^ sw));  // w columns 1..4
      w[a][1] = lo2(m1);
      w[a][2] = hi2(m1);
      w[a][3] = lo2(m2);
      w[a][4] = hi2(m2);
      if (kMalvar && mid) {
        w[a][0] = hi2(lds4(row + ((2 * uq) ^ sw)));
        w[a][5] = lo2(lds4(row + ((2 * uq + 6) ^ sw)));
      }
    }
    float2 rgb[2][2][3];
#pragma unroll
    for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
      for (int dq = 0; dq < 2; ++dq) {
        float2 n[5][5];
#pragma unroll
        for (int a = 0; a < 5; ++a) {
#pragma unroll
          for (int b = 0; b < 5; ++b) n[a][b] = w[dy + a][dq + b];  // unused corners are never read
        }
        // Pixel row y0 - 1 + 2ur + dy, column x0 + 2uq + dq - 1: parities (dy + 1) & 1 and (dq + 1) & 1.
        demosaic2<kMalvar>(n, cfa_of(kPat, (((dy + 1) & 1) << 1) | ((dq + 1) & 1)), rgb[dy][dq]);
      }
    }
#pragma unroll
    for (int dy = 0; dy < 2; ++dy) {
      const int o = (2 * ur + dy) * kCW2 + 2 * cchunk(uq, ur & 1);  // csw(2 ur + dy) == ur & 1
      sts4(R + o, rgb[dy][0][0], rgb[dy][1][0]);
      sts4(G + o, rgb[dy][0][1], rgb[dy][1][1]);
      sts4(B + o, rgb[dy][0][2], rgb[dy][1][2]);
    }
  }
}

// C (sharpening). The 3x3 windows of one plane around pairs 4uc .. 4uc + 3
// of output rows r and r + 1, sharpened: RGB rows r .. r + 3 (each loaded
// once for both output rows), pair columns 4uc .. 4uc + 5 (chunks 2uc ..
// 2uc + 2, stored at chunk ^ csw(row)).
__device__ __forceinline__ void sharpen_rows2(Span<const float2> X, int r, int uc, float2 amount, float2 (&o0)[4],
                                              float2 (&o1)[4]) {
  float2 w[4][6];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int j = r + a;
    const int s = csw(j);
    Span<const float2> row = X + j * kCW2;
    const float4 v0 = lds4(row + 2 * ((2 * uc) ^ s)), v1 = lds4(row + 2 * ((2 * uc + 1) ^ s)),
                 v2 = lds4(row + 2 * cchunk(2 * uc + 2, s));
    w[a][0] = lo2(v0);
    w[a][1] = hi2(v0);
    w[a][2] = lo2(v1);
    w[a][3] = hi2(v1);
    w[a][4] = lo2(v2);
    w[a][5] = hi2(v2);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    o0[i] = sharpen_one2(w[1][i + 1], w[0][i + 1], w[2][i + 1], w[1][i], w[1][i + 2], w[0][i], w[0][i + 2], w[2][i],
                         w[2][i + 2], amount);
    o1[i] = sharpen_one2(w[2][i + 1], w[1][i + 1], w[3][i + 1], w[2][i], w[2][i + 2], w[1][i], w[1][i + 2], w[3][i],
                         w[3][i + 2], amount);
  }
}

// C (sharpening), one output row: the 3x3 windows of one plane around pairs
// 4uc .. 4uc + 3 of output row r, sharpened from RGB rows r .. r + 2 (loaded
// as in sharpen_rows2; a quarter-warp takes rows r and r + 2, which csw
// sends to different banks).
__device__ __forceinline__ void sharpen_row1(Span<const float2> X, int r, int uc, float2 amount, float2 (&o)[4]) {
  float2 w[3][6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int j = r + a;
    const int s = csw(j);
    Span<const float2> row = X + j * kCW2;
    const float4 v0 = lds4(row + 2 * ((2 * uc) ^ s)), v1 = lds4(row + 2 * ((2 * uc + 1) ^ s)),
                 v2 = lds4(row + 2 * cchunk(2 * uc + 2, s));
    w[a][0] = lo2(v0);
    w[a][1] = hi2(v0);
    w[a][2] = lo2(v1);
    w[a][3] = hi2(v1);
    w[a][4] = lo2(v2);
    w[a][5] = hi2(v2);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    o[i] = sharpen_one2(w[1][i + 1], w[0][i + 1], w[2][i + 1], w[1][i], w[1][i + 2], w[0][i], w[0][i + 2], w[2][i],
                        w[2][i + 2], amount);
  }
}

// C (no sharpening). Demosaic pairs 4uc .. 4uc + 3 of output row r straight
// from the samples: sample rows r .. r + 4 (halo 2), pair columns 4uc + 2 ..
// 4uc + 9. kRowPar: the parity of the output row.
template <bool kMalvar, int kPat, int kRowPar>
__device__ __forceinline__ void demosaic_row4(Span<const float2> P, int r, int uc, float2 (&rgb)[4][3]) {
  float2 w[5][8] = {};
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    Span<const float2> row = P + (r + a) * kPW;
    const int sw = psw(r + a);
    const int s0 = 4 * uc + 2;
    const bool edge = a == 0 || a == 4;
    if (edge && !kMalvar) continue;
    if (edge) {  // Malvar's vertical taps: the centres only
      const float4 v1 = lds4(row + ((s0 + 2) ^ sw)), v2 = lds4(row + ((s0 + 4) ^ sw));
      w[a][2] = lo2(v1);
      w[a][3] = hi2(v1);
      w[a][4] = lo2(v2);
      w[a][5] = hi2(v2);
    } else {
      const float4 v0 = lds4(row + (s0 ^ sw)), v1 = lds4(row + ((s0 + 2) ^ sw)), v2 = lds4(row + ((s0 + 4) ^ sw)),
                   v3 = lds4(row + ((s0 + 6) ^ sw));
      w[a][0] = lo2(v0);
      w[a][1] = hi2(v0);
      w[a][2] = lo2(v1);
      w[a][3] = hi2(v1);
      w[a][4] = lo2(v2);
      w[a][5] = hi2(v2);
      w[a][6] = lo2(v3);
      w[a][7] = hi2(v3);
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float2 n[5][5];
#pragma unroll
    for (int a = 0; a < 5; ++a) {
#pragma unroll
      for (int b = 0; b < 5; ++b) n[a][b] = w[a][i + b];
    }
    demosaic2<kMalvar>(n, cfa_of(kPat, (kRowPar << 1) | (i & 1)), rgb[i]);
  }
}

// ---- C: colour matrix, statistics, tone, codes, stores ---------------------

// The tone curve (isp_math.hpp:235-243) of one value from a table of
// (lut[i], lut[i+1] - lut[i]) pairs: lut[i] + (f - i) * diff[i] with
// f = x (N - 1) and i = trunc(f), given f's 2^23 + trunc(f) and f - i. The
// last entry's difference is -0.0, so x = 1 (t = +0) returns lut[N-1]
// exactly, as the reference's branch does, whatever the sign of lut[N-1].
template <bool kLutSmem>
__device__ __forceinline__ float tone_lookup(Span<const float2> table, float m, float frac) {
  float2 e;
#ifdef ISP_CHECKED
  // Entry trunc(f) through the checked span.
  e = table[static_cast<int>(__float_as_uint(m) - kTwo23Bits)];
#else
  if constexpr (kLutSmem) {
    // Shared address of entry trunc(f): base + 8 (bits - 2^23 bits), wrapping.
    const uint32_t addr = smem_u32(table) + (__float_as_uint(m) << 3) - (kTwo23Bits << 3);
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(e.x), "=f"(e.y) : "r"(addr));
  } else {
    e = __ldg(table + magic_int(m));
  }
#endif
  return fadd(e.x, fmul(frac, e.y));
}

// Stores four pixels of one row, x .. x + 3 (isp_math.hpp:250-276), from
// their toned values t, their rounded integer codes c (2^23 + code as float
// bits: 8-bit codes for RGB8/RGBA8, 16-bit values for RGB16) and counts their
// 8-bit histogram codes (isp_math.hpp:279-305). `n`: pixels inside the image.
template <int kOut>
__device__ __forceinline__ void store_seg4(const FrameDesc& p, int x, int y, const float (&t)[4][3],
                                           const unsigned int (&c)[4][3], int n, bool want_hist, Span<unsigned int> hist) {
  Span<uint8_t> row = p.out + static_cast<int64_t>(y) * p.out_pitch;
  const bool vec = n == 4 && p.out_vector;
  unsigned int q[4][3];  // histogram codes
  if constexpr (kOut == kOutRgb8 || kOut == kOutRgba8) {
#pragma unroll
    for (int d = 0; d < 4; ++d) {
#pragma unroll
      for (int k = 0; k < 3; ++k) q[d][k] = c[d][k] & 0xFFU;  // 2^23 + code, code < 256
    }
    if constexpr (kOut == kOutRgb8) {
      if (vec) {
        Span<unsigned int> o = span_cast<unsigned int>(row + 3 * x);
        o[0] = __byte_perm(__byte_perm(c[0][0], c[0][1], 0x0040), __byte_perm(c[0][2], c[1][0], 0x0040), 0x5410);
        o[1] = __byte_perm(__byte_perm(c[1][1], c[1][2], 0x0040), __byte_perm(c[2][0], c[2][1], 0x0040), 0x5410);
        o[2] = __byte_perm(__byte_perm(c[2][2], c[3][0], 0x0040), __byte_perm(c[3][1], c[3][2], 0x0040), 0x5410);
      } else {
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          if (d >= n) break;
#pragma unroll
          for (int k = 0; k < 3; ++k) row[3 * (x + d) + k] = static_cast<uint8_t>(q[d][k]);
        }
      }
    } else {
      unsigned int w[4];
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        w[d] = __byte_perm(__byte_perm(c[d][0], c[d][1], 0x0040), c[d][2], 0x7410) | 0xFF000000U;
      }
      if (vec) {
        *span_cast<uint4>(row + 4 * x) = make_uint4(w[0], w[1], w[2], w[3]);
      } else {
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          if (d >= n) break;
#pragma unroll
          for (int k = 0; k < 4; ++k) row[4 * (x + d) + k] = static_cast<uint8_t>(w[d] >> (8 * k));
        }
      }
    }
  } else if constexpr (kOut == kOutRgb16) {
#pragma unroll
    for (int d = 0; d < 4; ++d) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        // (v * 255 + 32767) / 65535 == ((v + 128) * 0xFF01) >> 24 for v < 2^16
        // (checked for every v); c = 2^23 bits + v, and the product of
        // (c + 128 - 2^23 bits) stays below 2^32.
        q[d][k] = ((c[d][k] + (128U - kTwo23Bits)) * 0xFF01U) >> 24;
      }
    }
    if (vec) {
      Span<uint2> o = span_cast<uint2>(row + 6 * x);
      o[0] = make_uint2(__byte_perm(c[0][0], c[0][1], 0x5410), __byte_perm(c[0][2], c[1][0], 0x5410));
      o[1] = make_uint2(__byte_perm(c[1][1], c[1][2], 0x5410), __byte_perm(c[2][0], c[2][1], 0x5410));
      o[2] = make_uint2(__byte_perm(c[2][2], c[3][0], 0x5410), __byte_perm(c[3][1], c[3][2], 0x5410));
    } else {
      Span<uint16_t> o = span_cast<uint16_t>(row);
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        if (d >= n) break;
#pragma unroll
        for (int k = 0; k < 3; ++k) o[3 * (x + d) + k] = static_cast<uint16_t>(c[d][k]);
      }
    }
  } else {
#pragma unroll
    for (int d = 0; d < 4; ++d) {
#pragma unroll
      for (int k = 0; k < 3; ++k) q[d][k] = c[d][k] & 0xFFU;
    }
    if (vec) {
      Span<float4> o = span_cast<float4>(row + 12 * x);
      o[0] = make_float4(t[0][0], t[0][1], t[0][2], t[1][0]);
      o[1] = make_float4(t[1][1], t[1][2], t[2][0], t[2][1]);
      o[2] = make_float4(t[2][2], t[3][0], t[3][1], t[3][2]);
    } else {
      Span<float> o = span_cast<float>(row);
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        if (d >= n) break;
#pragma unroll
        for (int k = 0; k < 3; ++k) o[3 * (x + d) + k] = t[d][k];
      }
    }
  }
  if (want_hist) {
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      if (d >= n) break;
      const unsigned int luma = (2126U * q[d][0] + 7152U * q[d][1] + 722U * q[d][2] + 5000U) / 10000U;
      atomicAdd(&hist[luma], 1U);
      atomicAdd(&hist[kHistBins + q[d][0]], 1U);
      atomicAdd(&hist[2 * kHistBins + q[d][1]], 1U);
      atomicAdd(&hist[3 * kHistBins + q[d][2]], 1U);
    }
  }
}

// The per-pixel tail of four pairs of one row (pixels x .. x + 3 and
// x + 32 .. x + 35 of image row y): colour matrix, statistics sums, tone,
// codes, stores. nl, nr: pixels of the left and right groups inside the
// image (0..4); kFull: both are 4 and the rows may be stored 16 bytes at a
// time (the interior units, compiled without the per-pixel guards). sums:
// 2^23 bits + to_fixed summed mod 2^32, npix the number of terms, so that the
// caller subtracts npix x 2^23 bits.
template <int kOut, bool kLutSmem, bool kFull>
__device__ __forceinline__ void finish_pairs(const FrameDesc& p, const float2 (&rgb)[4][3], int x, int y, int nl_,
                                             int nr_, Span<const float2> lut, float lut_scale, bool want_stats,
                                             bool want_hist, Span<unsigned int> hist, unsigned int (&sums)[3],
                                             unsigned int& npix) {
  const int nl = kFull ? 4 : nl_;
  const int nr = kFull ? 4 : nr_;
  float tl[4][3], tr[4][3];
  unsigned int cl[4][3], cr[4][3];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float2* c = rgb[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      // clamp01((m0 r + m1 g) + m2 b), isp_math.hpp:229-233: rounded
      // products, so the sums run per lane (isp_ops.cuh).
      const float2 lin = add_sat2(add_lanes(mul2(bc2(p.ccm[3 * k]), c[0]), mul2(bc2(p.ccm[3 * k + 1]), c[1])),
                                  mul2(bc2(p.ccm[3 * k + 2]), c[2]));
      if (want_stats) {
        // to_fixed (isp_math.hpp:245-247): trunc(lin 2^20 + 0.5). lin 2^20 is
        // exact and so is the sum below 2^20 + 1; above it both roundings
        // truncate to 2^20.
        const float2 m = magic_trunc2(exact_scale_add2(lin, bc2(kFixedOne), bc2(0.5F)));
        sums[k] += (i < nl ? __float_as_uint(m.x) : 0U) + (i < nr ? __float_as_uint(m.y) : 0U);
      }
      // f = lin (N - 1) is a rounded product: its truncation and f - i per lane.
      const float2 f = mul2(lin, bc2(lut_scale));
      const float2 m = magic_trunc_lanes(f);
      const float2 frac = sub_lanes(f, sub2(m, bc2(kTwo23)));
      const float2 toned = make_float2(tone_lookup<kLutSmem>(lut, m.x, frac.x), tone_lookup<kLutSmem>(lut, m.y, frac.y));
      tl[i][k] = toned.x;
      tr[i][k] = toned.y;
      float2 code;
      // trunc(t scale + 0.5): the product is rounded, so + 0.5 runs per lane.
      if constexpr (kOut == kOutRgb16) {
        code = magic_trunc2(add_lanes(mul2(toned, bc2(65535.0F)), bc2(0.5F)));
      } else if constexpr (kOut == kOutRgb32f) {
        const float2 clamped = make_float2(clamp01(toned.x), clamp01(toned.y));
        code = magic_trunc2(add_lanes(mul2(clamped, bc2(255.0F)), bc2(0.5F)));
      } else {
        code = magic_trunc2(add_lanes(mul2(toned, bc2(255.0F)), bc2(0.5F)));
      }
      cl[i][k] = __float_as_uint(code.x);
      cr[i][k] = __float_as_uint(code.y);
    }
  }
  if (want_stats) npix += static_cast<unsigned int>(nl + nr);
  if (kFull || nl > 0) store_seg4<kOut>(p, x, y, tl, cl, nl, want_hist, hist);
  if (kFull || nr > 0) store_seg4<kOut>(p, x + kHalf, y, tr, cr, nr, want_hist, hist);
}

template <bool kLutSmem, bool kFull>
__device__ __forceinline__ void finish_pairs_any(const FrameDesc& p, const float2 (&rgb)[4][3], int x, int y, int nl,
                                                 int nr, Span<const float2> lut, float lut_scale, bool want_stats,
                                                 bool want_hist, Span<unsigned int> hist, unsigned int (&sums)[3],
                                                 unsigned int& npix) {
  switch (p.out_format) {
    case kOutRgb8:
      finish_pairs<kOutRgb8, kLutSmem, kFull>(p, rgb, x, y, nl, nr, lut, lut_scale, want_stats, want_hist, hist, sums, npix);
      break;
    case kOutRgba8:
      finish_pairs<kOutRgba8, kLutSmem, kFull>(p, rgb, x, y, nl, nr, lut, lut_scale, want_stats, want_hist, hist, sums, npix);
      break;
    case kOutRgb16:
      finish_pairs<kOutRgb16, kLutSmem, kFull>(p, rgb, x, y, nl, nr, lut, lut_scale, want_stats, want_hist, hist, sums, npix);
      break;
    default:
      finish_pairs<kOutRgb32f, kLutSmem, kFull>(p, rgb, x, y, nl, nr, lut, lut_scale, want_stats, want_hist, hist, sums, npix);
      break;
  }
}

}  // namespace
}  // namespace isp_b200
