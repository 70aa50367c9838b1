"""Seeded synthetic raw frames and the ISP settings of the benchmark workloads.

The scene: linear RGB in [0, 1] built from a random linear gradient plus 8
Gaussian blobs (sigma 50..300 px), then 64 axis-aligned rectangles of uniform
colour painted over it, times a cos^4 radial vignette whose gain at the image
corners is 0.5. It is mosaicked, scaled from [0, 1] to [black, white], given
Poisson-Gaussian noise (0.5 DN per electron, read noise sigma 3 DN), rounded,
clipped to the sample range and packed (u8, u16, MIPI RAW10 or RAW12). Every
random choice comes from numpy's PCG64 keyed by the seed.

The lens shading grid that undoes the vignette is 1 / vignette at the grid
points (all four channels alike). These frames stand in for camera data; the
ISP's parity with the reference is checked on whatever bytes it is given.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from . import abi

# The channel colour (0 R, 1 G, 2 B) at quad position (y & 1) * 2 + (x & 1), per pattern.
_CFA_COLOR = {abi.RGGB: (0, 1, 1, 2), abi.BGGR: (2, 1, 1, 0), abi.GRBG: (1, 0, 2, 1), abi.GBRG: (1, 2, 0, 1)}

EDGE_GAIN = 0.5
_THETA_EDGE = math.acos(EDGE_GAIN ** 0.25)  # cos^4(theta) = 0.5 at the corners


def vignette(width: int, height: int, xs=None, ys=None) -> np.ndarray:
    """cos^4 falloff, 1 at the centre and EDGE_GAIN at the corners."""
    cx, cy = (width - 1) / 2.0, (height - 1) / 2.0
    xs = np.arange(width, dtype=np.float64) if xs is None else np.asarray(xs, np.float64)
    ys = np.arange(height, dtype=np.float64) if ys is None else np.asarray(ys, np.float64)
    rc = math.hypot(cx, cy) or 1.0
    r = np.sqrt(((xs[None, :] - cx) ** 2 + (ys[:, None] - cy) ** 2)) / rc
    theta = np.arctan(r * math.tan(_THETA_EDGE))
    return np.cos(theta) ** 4


def scene_rgb(width: int, height: int, seed: int) -> np.ndarray:
    """Linear RGB [H, W, 3] float32 in [0, 1], before the vignette."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    ys = np.arange(height, dtype=np.float32)[:, None]
    xs = np.arange(width, dtype=np.float32)[None, :]
    img = np.empty((height, width, 3), np.float32)
    base = rng.uniform(0.05, 0.35, 3)
    gx = rng.uniform(-0.25, 0.25, 3) / max(width - 1, 1)
    gy = rng.uniform(-0.25, 0.25, 3) / max(height - 1, 1)
    for c in range(3):
        img[:, :, c] = base[c] + gx[c] * xs + gy[c] * ys
    for _ in range(8):
        cx, cy = rng.uniform(0, width), rng.uniform(0, height)
        sigma = rng.uniform(50.0, 300.0)
        amp = rng.uniform(0.05, 0.5, 3).astype(np.float32)
        r = int(min(4 * sigma, max(width, height)))
        x0, x1 = max(0, int(cx) - r), min(width, int(cx) + r + 1)
        y0, y1 = max(0, int(cy) - r), min(height, int(cy) + r + 1)
        if x0 >= x1 or y0 >= y1:
            continue
        ex = np.exp(-((np.arange(x0, x1, dtype=np.float32) - cx) ** 2) / (2 * sigma * sigma))
        ey = np.exp(-((np.arange(y0, y1, dtype=np.float32) - cy) ** 2) / (2 * sigma * sigma))
        blob = ey[:, None] * ex[None, :]
        img[y0:y1, x0:x1, :] += blob[:, :, None] * amp[None, None, :]
    for _ in range(64):
        w = int(rng.uniform(0.02, 0.2) * width) + 1
        h = int(rng.uniform(0.02, 0.2) * height) + 1
        x0 = int(rng.uniform(0, max(width - w, 1)))
        y0 = int(rng.uniform(0, max(height - h, 1)))
        img[y0:y0 + h, x0:x0 + w, :] = rng.uniform(0.0, 1.0, 3).astype(np.float32)
    np.clip(img, 0.0, 1.0, out=img)
    return img


def mosaic_counts(width: int, height: int, pattern: int, black: float, white: float, bits: int, seed: int,
                  noise: bool = True) -> np.ndarray:
    """Raw counts [H, W] uint16 of the seeded scene: vignetted, mosaicked, scaled, noisy, clipped."""
    rgb = scene_rgb(width, height, seed)
    vig = vignette(width, height).astype(np.float32)
    colors = np.array(_CFA_COLOR[pattern])
    y, x = np.mgrid[0:height, 0:width]
    idx = colors[((y & 1) << 1) | (x & 1)]
    sig = np.take_along_axis(rgb, idx[:, :, None], axis=2)[:, :, 0] * vig
    dn = sig.astype(np.float64) * (white - black)
    if noise:
        rng = np.random.default_rng(np.random.PCG64(seed ^ 0x5EED))
        electrons = rng.poisson(dn / 0.5)
        dn = electrons * 0.5 + rng.normal(0.0, 3.0, dn.shape)
    counts = np.rint(black + dn)
    return np.clip(counts, 0, (1 << bits) - 1).astype(np.uint16)


def pack(counts: np.ndarray, fmt: int, pitch: Optional[int] = None) -> Tuple[np.ndarray, int]:
    """Rows of `counts` packed as `fmt` (isp_params.hpp:24-29), at `pitch` bytes per row."""
    h, w = counts.shape
    row = abi.raw_row_bytes(fmt, w)
    pitch = row if pitch is None else pitch
    out = np.zeros((h, pitch), np.uint8)
    if fmt == abi.U8:
        out[:, :w] = counts.astype(np.uint8)
    elif fmt == abi.U16:
        out[:, :2 * w] = counts.astype("<u2").view(np.uint8).reshape(h, 2 * w)
    elif fmt == abi.RAW10:
        wp = (w + 3) // 4 * 4
        c = np.zeros((h, wp), np.uint16)
        c[:, :w] = counts
        g = c.reshape(h, wp // 4, 4)
        b = np.empty((h, wp // 4, 5), np.uint8)
        b[:, :, :4] = (g >> 2).astype(np.uint8)
        b[:, :, 4] = ((g[:, :, 0] & 3) | ((g[:, :, 1] & 3) << 2) | ((g[:, :, 2] & 3) << 4) | ((g[:, :, 3] & 3) << 6)).astype(np.uint8)
        out[:, :row] = b.reshape(h, row)
    else:
        wp = (w + 1) // 2 * 2
        c = np.zeros((h, wp), np.uint16)
        c[:, :w] = counts
        g = c.reshape(h, wp // 2, 2)
        b = np.empty((h, wp // 2, 3), np.uint8)
        b[:, :, :2] = (g >> 4).astype(np.uint8)
        b[:, :, 2] = ((g[:, :, 0] & 15) | ((g[:, :, 1] & 15) << 4)).astype(np.uint8)
        out[:, :row] = b.reshape(h, row)
    return out.ravel(), pitch


def lens_shading_grid(width: int, height: int, gw: int = 17, gh: int = 13, channels: int = 4) -> abi.LensShading:
    """Gains 1 / vignette at the grid points, which lie on the image's corner pixels."""
    xs = np.arange(gw, dtype=np.float64) * (width - 1) / (gw - 1)
    ys = np.arange(gh, dtype=np.float64) * (height - 1) / (gh - 1)
    g = (1.0 / vignette(width, height, xs, ys)).astype(np.float32)
    gains = np.repeat(g[:, :, None], channels, axis=2)
    return abi.LensShading(gw, gh, channels, np.ascontiguousarray(gains.ravel(), np.float32))


def srgb_table(n: int) -> np.ndarray:
    x = np.arange(n, dtype=np.float64) / (n - 1)
    y = np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(x, 1 / 2.4) - 0.055)
    return np.clip(y, 0.0, 1.0).astype(np.float32)


def filmic_table(n: int, toe: float = 0.2, shoulder: float = 0.8) -> np.ndarray:
    """A C1 S-curve: quadratic toe on [0, toe], a line of slope m, quadratic
    shoulder on [shoulder, 1]; m = 2 / (1 + shoulder - toe) makes it reach 1 at 1."""
    m = 2.0 / (1.0 + shoulder - toe)
    x = np.arange(n, dtype=np.float64) / (n - 1)
    y_toe = m * x * x / (2 * toe)
    y_mid = m * toe / 2 + m * (x - toe)
    y_sh = 1.0 - m * (1 - x) ** 2 / (2 * (1 - shoulder))
    y = np.where(x < toe, y_toe, np.where(x > shoulder, y_sh, y_mid))
    return np.clip(y, 0.0, 1.0).astype(np.float32)


CCM = (1.6, -0.3, -0.3, -0.3, 1.6, -0.3, -0.3, -0.3, 1.6)


@dataclass
class Workload:
    """One frame shape of a benchmark configuration, with its ISP settings."""

    name: str
    width: int
    height: int
    pattern: int
    fmt: int
    bits: int
    black: float
    params: abi.IspParams
    out_format: int
    with_stats: bool
    with_hist: bool
    fresh_frames: int = 0  # > 0: the benchmark takes this many distinct frames in turn (device-rendered)

    def raw(self, seed: int, pitch: Optional[int] = None, noise: bool = True) -> abi.RawFrame:
        counts = mosaic_counts(self.width, self.height, self.pattern, self.black, (1 << self.bits) - 1,
                               self.bits, seed, noise)
        data, pitch = pack(counts, self.fmt, pitch)
        return abi.RawFrame(data, self.width, self.height, pitch, self.fmt, self.bits, self.pattern)

    @property
    def pixels(self) -> int:
        return self.width * self.height

    def compulsory_bytes(self) -> int:
        """Raw read once plus the output written once."""
        out = self.width * self.height * abi.output_channels(self.out_format) * abi.output_channel_bytes(self.out_format)
        return abi.raw_row_bytes(self.fmt, self.width) * self.height + out


def config0(width=1920, height=1080) -> Workload:
    """1920x1080 RGGB 12-bit in u16: black 256, LSC 17x13x4, manual WB (1.9, 1, 1.5),
    bilinear, no sharpening, the CCM, sRGB; RGB8 and the histogram."""
    p = abi.IspParams(black_level=256.0, lens_shading=lens_shading_grid(width, height),
                      white_balance=abi.MANUAL, wb_gains=(1.9, 1.0, 1.5), demosaic=abi.BILINEAR, ccm=CCM,
                      tone_curve=abi.SRGB, sharpen=0.0)
    return Workload("c0_1080p_u16_rggb_bilinear", width, height, abi.RGGB, abi.U16, 12, 256.0, p, abi.RGB8,
                    False, True)


def config1(width=3840, height=2160) -> Workload:
    """3840x2160 GRBG RAW10: black 64, LSC 17x13x4, gray world, Malvar, sharpen 0.5,
    the CCM, a 1024-entry sRGB table; RGB16, histogram, statistics and AE."""
    p = abi.IspParams(black_level=64.0, lens_shading=lens_shading_grid(width, height),
                      white_balance=abi.GRAY_WORLD, demosaic=abi.MALVAR, ccm=CCM, tone_curve=abi.LUT,
                      lut=srgb_table(1024), sharpen=0.5)
    return Workload("c1_4k_raw10_grbg_malvar_sharpen", width, height, abi.GRBG, abi.RAW10, 10, 64.0, p,
                    abi.RGB16, True, True)


def config2(width=8192, height=6144) -> Workload:
    """8192x6144 BGGR RAW12: black 256, LSC, white patch 99.5 %, Malvar, sharpen 0.5,
    the CCM, a 4096-entry filmic table; RGBA8, histogram, statistics and AE."""
    p = abi.IspParams(black_level=256.0, lens_shading=lens_shading_grid(width, height),
                      white_balance=abi.WHITE_PATCH, white_patch_percentile=0.995, demosaic=abi.MALVAR,
                      ccm=CCM, tone_curve=abi.LUT, lut=filmic_table(4096), sharpen=0.5)
    return Workload("c2_8k_raw12_bggr_whitepatch", width, height, abi.BGGR, abi.RAW12, 12, 256.0, p,
                    abi.RGBA8, True, True, fresh_frames=200)




@dataclass
class Camera:
    """One camera of the mixed workloads: its frame shape and ISP settings."""

    width: int
    height: int
    pattern: int
    fmt: int
    bits: int
    black: float
    params: abi.IspParams
    out_format: int = abi.RGB8

    @property
    def pixels(self) -> int:
        return self.width * self.height


# Frame shapes of the mixed workloads: (count, width, height, format, bits, black, pattern).
MIXED_BATCH = [
    (16, 640, 480, abi.U8, 8, 16.0, abi.RGGB),
    (16, 1920, 1080, abi.U16, 12, 256.0, abi.GBRG),
    (12, 3840, 2160, abi.RAW10, 10, 64.0, abi.GRBG),
    (4, 4096, 3072, abi.U16, 16, 4096.0, abi.BGGR),
]


# Camera streams of the serving workload: (count, width, height, format, bits, black, pattern, fps).
SERVING_STREAMS = [
    (16, 640, 480, abi.U8, 8, 16.0, abi.RGGB, 120.0),
    (24, 1920, 1080, abi.U16, 12, 256.0, abi.GBRG, 60.0),
    (16, 3840, 2160, abi.RAW10, 10, 64.0, abi.GRBG, 30.0),
    (8, 4096, 3072, abi.U16, 16, 4096.0, abi.BGGR, 15.0),
]


def serving_streams(seed: int = 4242):
    """The 64 serving streams: cameras (settings fixed by seed, as
    mixed_cameras) and their nominal frame rates."""
    cams = mixed_cameras([t[:7] for t in SERVING_STREAMS], seed)
    fps = [t[7] for t in SERVING_STREAMS for _ in range(t[0])]
    return cams, fps


def mixed_cameras(shapes=None, seed: int = 2024):
    """Cameras of a mixed workload: per camera a seeded choice of manual, gray
    world or white patch white balance and of bilinear or Malvar-He-Cutler
    demosaic, its own 17x13 lens shading grid and 1024-entry tone table (sRGB
    or filmic), RGB8 out with histogram and statistics."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    cams = []
    for count, w, h, fmt, bits, black, pattern in (shapes or MIXED_BATCH):
        for _ in range(count):
            wb = int(rng.integers(0, 3))
            dem = int(rng.integers(0, 2))
            lut = srgb_table(1024) if rng.integers(0, 2) == 0 else filmic_table(1024)
            p = abi.IspParams(black_level=black, lens_shading=lens_shading_grid(w, h), white_balance=wb,
                              wb_gains=(float(rng.uniform(1.2, 2.2)), 1.0, float(rng.uniform(1.1, 1.9))),
                              demosaic=dem, ccm=CCM, tone_curve=abi.LUT, lut=lut, sharpen=0.0)
            cams.append(Camera(w, h, pattern, fmt, bits, black, p))
    return cams
