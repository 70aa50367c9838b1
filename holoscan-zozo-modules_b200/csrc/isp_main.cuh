// isp_main.cuh - the fused tile kernel of the B200 ISP, as a template; each
// isp_main_*.cu translation unit instantiates one demosaic method and
// sharpening setting, so the instances compile in parallel.
#pragma once

#include "isp_common.cuh"

namespace isp_b200 {
namespace {

template <bool kMalvar, bool kSharpen, int kLayout, bool kLutSmem>
__global__ void __launch_bounds__(kThreads, 2) isp_main_kernel(const __grid_constant__ CUtensorMap map, FrameDesc p,
                                                               int tiles_x, int tiles, int use_tma, int lut_in_smem) {
  using G = Geom<kSharpen>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128U - (smem_u32(smem_raw) & 127U)) & 127U);
  const int box_bytes = box_row_bytes(p.raw_format);
  const Layout L = layout_of(kSharpen, box_bytes, kLutSmem ? p.tone_size : 0);
  uint8_t* box = smem + L.raw;
  float* S = reinterpret_cast<float*>(smem + L.samples);
  float2* Crg = reinterpret_cast<float2*>(smem + L.rg);
  float* Cb = reinterpret_cast<float*>(smem + L.b);
  float* table = reinterpret_cast<float*>(smem + L.lsc);
  int* col_mx = reinterpret_cast<int*>(smem + L.cols);
  int* col_ix = col_mx + kSW;
  float* col_tx = reinterpret_cast<float*>(col_ix + kSW);
  int* row_my = reinterpret_cast<int*>(smem + L.rows);
  int* row_k = row_my + G::kSH;
  float* row_ty = reinterpret_cast<float*>(row_k + G::kSH);
  unsigned int* hist = reinterpret_cast<unsigned int*>(smem + L.hist);
  float2* lut_s = reinterpret_cast<float2*>(smem + L.lut);
  __shared__ uint64_t bar;
  __shared__ u64 red[kWarps];
  __shared__ int minmax[2];
  __shared__ bool last;
  static_cast<void>(lut_in_smem);

  // The demosaic runs as the layout's canonical pattern (RGGB or GRBG); for
  // BGGR and GBRG its red and blue outputs trade places before the colour
  // matrix (the estimates' arithmetic is the same at either site).
  constexpr int kPat = kLayout * 2;
  const bool swap_rb = (p.pattern & 1) != 0;
  const int tid = threadIdx.x;
  Scratch* sc = p.scratch;
  const bool want_hist = p.hist_out != nullptr;
  const bool want_stats = p.stats_out != nullptr;
  float gains[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) gains[k] = p.auto_wb ? __ldcg(&sc->awb_gains[k]) : p.wb[k];
  float qblack[4], qinv[4], qgain[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int ch = p.cfa[k];
    qblack[k] = p.black[ch];
    qinv[k] = p.inv_range[ch];
    qgain[k] = gains[color_of(ch)];
  }
  const float2* lut = p.tone;
  if constexpr (kLutSmem) {
    for (int i = tid; i < p.tone_size; i += kThreads) lut_s[i] = p.tone[i];
    lut = lut_s;
  }
  const float lut_scale = static_cast<float>(p.tone_size - 1);
  if (want_hist) {
    for (int i = tid; i < kHistChannels * kHistBins; i += kThreads) hist[i] = 0U;
  }
  if (tid == 0 && use_tma) mbar_init(&bar);
  __syncthreads();

  const int fmt = p.raw_format;
  u64 acc[4] = {0, 0, 0, 0};  // linear R, G, B in 2^-20 units; saturated samples
  u64 counted_total = 0;      // pixels whose bit patterns the sums hold
  uint32_t phase = 0;
  int tile = blockIdx.x;
  const auto issue = [&](int t) {
    const int ty = t / tiles_x;
    const int x0 = (t - ty * tiles_x) * kTW;
    tma_load_2d(&map, box, &bar, box_x(fmt, x0), ty * kTH - G::kHalo, static_cast<unsigned int>(G::kSH * box_bytes));
  };
  if (use_tma && tid == 0 && tile < tiles) issue(tile);

  for (; tile < tiles; tile += gridDim.x) {
    const int ty = tile / tiles_x;
    const int x0 = (tile - ty * tiles_x) * kTW;
    const int y0 = ty * kTH;
    const bool interior = x0 >= 4 && y0 >= G::kHalo && x0 + kSW - 4 <= p.width && y0 + kTH + G::kHalo <= p.height;
    TileCtx t;
    t.x0 = x0;
    t.y0 = y0;
    t.box = box;
    t.col_mx = col_mx;
    t.row_my = row_my;
    t.row_k = row_k;
    t.row_ty = row_ty;
    t.table = table;
    t.lt = build_lsc(p, p.pattern, x0 - 4, kSW, y0 - G::kHalo, G::kSH, !interior, p.width + 3, p.height + G::kHalo - 1,
                     col_mx, col_ix, col_tx, row_my, row_k, row_ty, table, minmax);
    if (use_tma && !mbar_wait(&bar, phase)) {
      if (tid == 0) atomicExch(&sc->error, 1);
    }
    phase ^= 1U;

    unsigned int saturated;
    if (!use_tma) {
      saturated = phase_a_fmt<2, G::kHalo>(p, t, S, box_bytes, qblack, qinv, qgain, want_stats);
    } else if (interior) {
      saturated = phase_a_fmt<0, G::kHalo>(p, t, S, box_bytes, qblack, qinv, qgain, want_stats);
    } else {
      saturated = phase_a_fmt<1, G::kHalo>(p, t, S, box_bytes, qblack, qinv, qgain, want_stats);
    }
    acc[3] += saturated;
    __syncthreads();
    // The box is free: prefetch the next tile's raw samples during B and C.
    if (use_tma && tid == 0) {
      const int next = tile + gridDim.x;
      if (next < tiles) {
        fence_async_shared();
        issue(next);
      }
    }

    // B. (Sharpening) RGB of the tile and a one-pixel ring, 2x4 pixels a
    //    unit; outside the image these are the reference's virtual pixels
    //    (cpu_pipeline.cpp:22-46).
    if constexpr (kSharpen) {
      constexpr int kUnitsB = 17 * 34;
      for (int unit = tid; unit < kUnitsB; unit += kThreads) {
        const int qr = unit / 17;
        const int qc = unit - qr * 17;
        float w[6][8];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          const float4 a = *reinterpret_cast<const float4*>(S + (2 * qr + r) * kSW + 4 * qc);
          const float4 b = *reinterpret_cast<const float4*>(S + (2 * qr + r) * kSW + 4 * qc + 4);
          w[r][0] = a.x; w[r][1] = a.y; w[r][2] = a.z; w[r][3] = a.w;
          w[r][4] = b.x; w[r][5] = b.y; w[r][6] = b.z; w[r][7] = b.w;
        }
        const bool inner = qr >= 1 && qr <= 32 && qc >= 1 && qc <= 15;
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
          const int cy = 2 * qr + dy - 1;
#pragma unroll
          for (int dx = 0; dx < 4; ++dx) {
            const int cx = 4 * qc + dx - 1;
            if (!inner && (cy < 0 || cy >= G::kCH || cx < 0 || cx >= kTW + 2)) continue;
            float rgb[3];
            demosaic_at<kMalvar, kPat>(w, dy, dx, rgb);
            Crg[cy * G::kCW + cx] = make_float2(rgb[0], rgb[1]);
            Cb[cy * G::kCW + cx] = rgb[2];
          }
        }
      }
      __syncthreads();
    }

    // C. Output units of 2x4 pixels: 32 unit rows x 16 unit columns. A
    //    tile's statistics sums stay below 2^32 per thread (16 pixels of
    //    at most 2^20).
    unsigned int sums[3] = {0U, 0U, 0U};
    unsigned int counted = 0;
    for (int unit = tid; unit < 512; unit += kThreads) {
      const int ur = unit >> 4;
      const int uc = unit & 15;
      float rgb[2][4][3];
      if constexpr (kSharpen) {
        // 3x3 neighbourhoods from the RGB planes: window rows 2ur..2ur+3,
        // columns 4uc..4uc+5 (pixel x0 + 4uc + dx sits at column 4uc + dx + 1).
        float m[4][6][3];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const float2* rg = Crg + (2 * ur + r) * G::kCW + 4 * uc;
          const float4 a = *reinterpret_cast<const float4*>(rg);
          const float4 b = *reinterpret_cast<const float4*>(rg + 2);
          const float4 c = *reinterpret_cast<const float4*>(rg + 4);
          m[r][0][0] = a.x; m[r][0][1] = a.y; m[r][1][0] = a.z; m[r][1][1] = a.w;
          m[r][2][0] = b.x; m[r][2][1] = b.y; m[r][3][0] = b.z; m[r][3][1] = b.w;
          m[r][4][0] = c.x; m[r][4][1] = c.y; m[r][5][0] = c.z; m[r][5][1] = c.w;
          const float* bp = Cb + (2 * ur + r) * G::kCW + 4 * uc;
          const float4 d = *reinterpret_cast<const float4*>(bp);
          const float2 e = *reinterpret_cast<const float2*>(bp + 4);
          m[r][0][2] = d.x; m[r][1][2] = d.y; m[r][2][2] = d.z; m[r][3][2] = d.w;
          m[r][4][2] = e.x; m[r][5][2] = e.y;
        }
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
          for (int dx = 0; dx < 4; ++dx) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              rgb[dy][dx][k] = sharpen_one(m[dy + 1][dx + 1][k], m[dy][dx + 1][k], m[dy + 2][dx + 1][k],
                                           m[dy + 1][dx][k], m[dy + 1][dx + 2][k], m[dy][dx][k], m[dy][dx + 2][k],
                                           m[dy + 2][dx][k], m[dy + 2][dx + 2][k], p.sharpen);
            }
          }
        }
      } else {
        // Samples rows 2ur .. 2ur + 5 (halo 2), columns 4uc + 2 .. 4uc + 9.
        float w[6][8];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          if (!kMalvar && (r == 0 || r == 5)) {
#pragma unroll
            for (int c = 0; c < 8; ++c) w[r][c] = 0.0F;
            continue;
          }
          const float* row = S + (2 * ur + r) * kSW + 4 * uc;
          const float4 a = *reinterpret_cast<const float4*>(row);
          const float4 b = *reinterpret_cast<const float4*>(row + 4);
          const float4 c = *reinterpret_cast<const float4*>(row + 8);
          w[r][0] = a.z; w[r][1] = a.w; w[r][2] = b.x; w[r][3] = b.y;
          w[r][4] = b.z; w[r][5] = b.w; w[r][6] = c.x; w[r][7] = c.y;
        }
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
          for (int dx = 0; dx < 4; ++dx) demosaic_at<kMalvar, kPat>(w, dy, dx, rgb[dy][dx]);
        }
      }
      const int xb = x0 + 4 * uc;
      const int yb = y0 + 2 * ur;
      const bool full = xb + 3 < p.width && yb + 1 < p.height;
      if (swap_rb) {
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
          for (int dx = 0; dx < 4; ++dx) {
            const float r = rgb[dy][dx][0];
            rgb[dy][dx][0] = rgb[dy][dx][2];
            rgb[dy][dx][2] = r;
          }
        }
      }
      if (full) {
        finish_unit_any<kLutSmem>(p, rgb, xb, yb, true, lut, lut_scale, want_stats, want_hist, hist, sums, counted);
      } else if (xb < p.width && yb < p.height) {
        finish_unit_any<kLutSmem>(p, rgb, xb, yb, false, lut, lut_scale, want_stats, want_hist, hist, sums, counted);
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] += sums[k];
    counted_total += counted;
    __syncthreads();  // the next tile overwrites the tables, S and C
  }
  main_finish(p, sc, acc, gains, want_stats, want_hist, hist, red, &last);
}


template <bool kMalvar, bool kSharpen>
const void* main_instance(int layout, bool lut_smem) {
  if (layout == 0) {
    return lut_smem ? reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, 0, true>)
                    : reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, 0, false>);
  }
  return lut_smem ? reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, 1, true>)
                  : reinterpret_cast<const void*>(&isp_main_kernel<kMalvar, kSharpen, 1, false>);
}

}  // namespace
}  // namespace isp_b200
