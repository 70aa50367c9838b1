"""ctypes mirror of include/isp_b200.h: the PODs and enumerations of the C ABI.

Types only; loading the library is isp_b200.lib()'s job. The layouts follow
holoscan::isp's public headers (modules/isp/include/holoscan/isp/isp_params.hpp:21-198).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

ABI_VERSION = 1

OK, EINVAL, ECUDA, ETIMEOUT, EBUSY, ESTATE = 0, 1, 2, 3, 4, 5

RGGB, BGGR, GRBG, GBRG = 0, 1, 2, 3
U8, U16, RAW10, RAW12 = 0, 1, 2, 3
BILINEAR, MALVAR = 0, 1
MANUAL, GRAY_WORLD, WHITE_PATCH = 0, 1, 2
SRGB, GAMMA, LINEAR, LUT = 0, 1, 2, 3
RGB8, RGBA8, RGB16, RGB32F = 0, 1, 2, 3

PATTERN_NAMES = {"RGGB": RGGB, "BGGR": BGGR, "GRBG": GRBG, "GBRG": GBRG}

HISTOGRAM_BINS = 256
HISTOGRAM_CHANNELS = 4
STATS_SIZE = 12
TONE_LUT_SIZE = 4097

# Statistics vector indices, layout version 1 (isp_params.hpp:178-198).
MEAN_R, MEAN_G, MEAN_B, MEAN_LUMA = 0, 1, 2, 3
AE_ERROR_EV, EXPOSURE_SCALE, SUGGESTED_EXPOSURE_NS, SUGGESTED_GAIN = 4, 5, 6, 7
WB_GAIN_R, WB_GAIN_G, WB_GAIN_B, SATURATED_FRACTION = 8, 9, 10, 11
AE_FIELDS = (AE_ERROR_EV, EXPOSURE_SCALE, SUGGESTED_EXPOSURE_NS, SUGGESTED_GAIN)


class AutoExposureC(C.Structure):
    _fields_ = [
        ("target", C.c_float),
        ("damping", C.c_float),
        ("min_exposure_ns", C.c_int64),
        ("max_exposure_ns", C.c_int64),
        ("min_gain", C.c_float),
        ("max_gain", C.c_float),
    ]


class ParamsC(C.Structure):
    _fields_ = [
        ("black_level", C.c_float),
        ("has_channel_black_levels", C.c_int32),
        ("channel_black_levels", C.c_float * 4),
        ("white_level", C.c_float),
        ("has_lens_shading", C.c_int32),
        ("lsc_width", C.c_int32),
        ("lsc_height", C.c_int32),
        ("lsc_channels", C.c_int32),
        ("lsc_gains", C.POINTER(C.c_float)),
        ("lsc_gains_count", C.c_size_t),
        ("white_balance", C.c_int32),
        ("wb_gains", C.c_float * 3),
        ("awb_smoothing", C.c_float),
        ("white_patch_percentile", C.c_float),
        ("demosaic", C.c_int32),
        ("ccm", C.c_float * 9),
        ("tone_curve", C.c_int32),
        ("gamma", C.c_float),
        ("lut", C.POINTER(C.c_float)),
        ("lut_size", C.c_size_t),
        ("sharpen", C.c_float),
        ("auto_exposure", AutoExposureC),
    ]


class RawViewC(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("pitch", C.c_size_t),
        ("format", C.c_int32),
        ("bit_depth", C.c_int32),
        ("pattern", C.c_int32),
    ]


class RgbViewC(C.Structure):
    _fields_ = [("data", C.c_void_p), ("pitch", C.c_size_t), ("format", C.c_int32)]


class StatsC(C.Structure):
    _fields_ = [("histogram", C.c_void_p), ("stats", C.c_void_p)]


class ExposureC(C.Structure):
    _fields_ = [("exposure_ns", C.c_int64), ("gain", C.c_float)]


class BatchInfoC(C.Structure):
    _fields_ = [("frames", C.c_int32), ("weights", C.c_float * 4), ("ctas_per_sm", C.c_int32), ("tuned", C.c_int32),
                ("graph_replays", C.c_int32), ("graph_main_ctas", C.c_int32), ("graph_awb_ctas", C.c_int32),
                ("tile_rows", C.c_int32), ("block_threads", C.c_int32)]


class ServerConfigC(C.Structure):
    _fields_ = [("max_batch", C.c_int32), ("max_inflight", C.c_int32), ("queue_depth", C.c_int32),
                ("slots_per_stream", C.c_int32), ("memory_budget", C.c_int64), ("use_graph", C.c_int32),
                ("per_frame", C.c_int32)]


class ServerStreamC(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("format", C.c_int32), ("bit_depth", C.c_int32),
                ("pattern", C.c_int32), ("out_format", C.c_int32), ("with_histogram", C.c_int32),
                ("with_stats", C.c_int32), ("copy_back", C.c_int32)]


class ServerResultC(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("stream", C.c_int32), ("frame", C.c_uint64), ("arrival_ns", C.c_int64),
                ("launch_ns", C.c_int64), ("done_ns", C.c_int64), ("image", C.c_void_p), ("histogram", C.c_void_p), ("stats", C.c_void_p)]


class SynthC(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("format", C.c_int32), ("bit_depth", C.c_int32),
                ("pattern", C.c_int32), ("black", C.c_float), ("gain", C.c_float), ("read_noise", C.c_float),
                ("vignette_edge", C.c_float)]


class ServerStatsC(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("refused", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("batches", C.c_int64), ("completed_pixels", C.c_int64), ("mean_batch_frames", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("p999_ms", C.c_double), ("max_ms", C.c_double),
                ("gpix_per_s", C.c_double), ("error", C.c_int32), ("p50_wait_ms", C.c_double),
                ("p99_wait_ms", C.c_double)]


@dataclass
class AutoExposure:
    """AutoExposureParams (isp_params.hpp:82-93), with the reference's defaults."""

    target: float = 0.18
    damping: float = 0.5
    min_exposure_ns: int = 10_000
    max_exposure_ns: int = 33_000_000
    min_gain: float = 1.0
    max_gain: float = 16.0


@dataclass
class LensShading:
    """LensShading (isp_params.hpp:73-79): gains [height][width][channels]."""

    width: int
    height: int
    channels: int
    gains: np.ndarray


@dataclass
class IspParams:
    """IspParams (isp_params.hpp:95-121), field for field, with the same defaults."""

    black_level: float = 0.0
    channel_black_levels: Optional[Sequence[float]] = None
    white_level: float = 0.0
    lens_shading: Optional[LensShading] = None
    white_balance: int = MANUAL
    wb_gains: Sequence[float] = (1.0, 1.0, 1.0)
    awb_smoothing: float = 0.25
    white_patch_percentile: float = 0.99
    demosaic: int = MALVAR
    ccm: Sequence[float] = (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)
    tone_curve: int = SRGB
    gamma: float = 2.2
    lut: Optional[Sequence[float]] = None
    sharpen: float = 0.0
    auto_exposure: AutoExposure = field(default_factory=AutoExposure)

    def to_c(self) -> "ParamsHolder":
        return ParamsHolder(self)

    def to_dict(self) -> dict:
        d = {
            "black_level": float(self.black_level),
            "channel_black_levels": None if self.channel_black_levels is None else [float(v) for v in self.channel_black_levels],
            "white_level": float(self.white_level),
            "lens_shading": None,
            "white_balance": int(self.white_balance),
            "wb_gains": [float(v) for v in self.wb_gains],
            "awb_smoothing": float(self.awb_smoothing),
            "white_patch_percentile": float(self.white_patch_percentile),
            "demosaic": int(self.demosaic),
            "ccm": [float(v) for v in self.ccm],
            "tone_curve": int(self.tone_curve),
            "gamma": float(self.gamma),
            "lut": None if self.lut is None else [float(v) for v in np.asarray(self.lut, np.float32)],
            "sharpen": float(self.sharpen),
            "auto_exposure": vars(self.auto_exposure).copy(),
        }
        if self.lens_shading is not None:
            s = self.lens_shading
            d["lens_shading"] = {"width": s.width, "height": s.height, "channels": s.channels}
        return d

    @staticmethod
    def from_dict(d: dict, lsc_gains: Optional[np.ndarray] = None) -> "IspParams":
        p = IspParams()
        for key in ("black_level", "white_level", "white_balance", "awb_smoothing", "white_patch_percentile",
                    "demosaic", "tone_curve", "gamma", "sharpen"):
            setattr(p, key, d[key])
        p.channel_black_levels = d["channel_black_levels"]
        p.wb_gains = tuple(d["wb_gains"])
        p.ccm = tuple(d["ccm"])
        p.lut = None if d["lut"] is None else np.asarray(d["lut"], np.float32)
        p.auto_exposure = AutoExposure(**d["auto_exposure"])
        if d["lens_shading"] is not None:
            s = d["lens_shading"]
            p.lens_shading = LensShading(s["width"], s["height"], s["channels"],
                                         np.ascontiguousarray(lsc_gains, np.float32))
        return p


class ParamsHolder:
    """An isp_params_c plus the arrays its pointers borrow, kept alive together."""

    def __init__(self, p: IspParams):
        c = ParamsC()
        c.black_level = p.black_level
        if p.channel_black_levels is not None:
            c.has_channel_black_levels = 1
            for k in range(4):
                c.channel_black_levels[k] = p.channel_black_levels[k]
        c.white_level = p.white_level
        self._lsc = None
        if p.lens_shading is not None:
            s = p.lens_shading
            self._lsc = np.ascontiguousarray(s.gains, dtype=np.float32).ravel()
            c.has_lens_shading = 1
            c.lsc_width, c.lsc_height, c.lsc_channels = s.width, s.height, s.channels
            c.lsc_gains = self._lsc.ctypes.data_as(C.POINTER(C.c_float))
            c.lsc_gains_count = self._lsc.size
        c.white_balance = p.white_balance
        for k in range(3):
            c.wb_gains[k] = p.wb_gains[k]
        c.awb_smoothing = p.awb_smoothing
        c.white_patch_percentile = p.white_patch_percentile
        c.demosaic = p.demosaic
        for k in range(9):
            c.ccm[k] = p.ccm[k]
        c.tone_curve = p.tone_curve
        c.gamma = p.gamma
        self._lut = None
        if p.lut is not None:
            self._lut = np.ascontiguousarray(p.lut, dtype=np.float32).ravel()
            c.lut = self._lut.ctypes.data_as(C.POINTER(C.c_float))
            c.lut_size = self._lut.size
        c.sharpen = p.sharpen
        ae = p.auto_exposure
        c.auto_exposure = AutoExposureC(ae.target, ae.damping, ae.min_exposure_ns, ae.max_exposure_ns,
                                        ae.min_gain, ae.max_gain)
        self.c = c

    def ref(self):
        return C.byref(self.c)


def output_channels(fmt: int) -> int:
    return 4 if fmt == RGBA8 else 3


def output_channel_bytes(fmt: int) -> int:
    return 2 if fmt == RGB16 else 4 if fmt == RGB32F else 1


def output_dtype(fmt: int):
    return np.uint16 if fmt == RGB16 else np.float32 if fmt == RGB32F else np.uint8


def raw_row_bytes(fmt: int, width: int) -> int:
    """raw_row_bytes (isp_params.cpp:184-197)."""
    w = max(width, 0)
    return {U8: w, U16: 2 * w, RAW10: 5 * ((w + 3) // 4), RAW12: 3 * ((w + 1) // 2)}[fmt]


@dataclass
class RawFrame:
    """A raw mosaic in host memory: `data` holds height rows of `pitch` bytes."""

    data: np.ndarray  # uint8, height * pitch
    width: int
    height: int
    pitch: int
    format: int
    bit_depth: int
    pattern: int

    def view(self, data_ptr: Optional[int] = None) -> RawViewC:
        ptr = self.data.ctypes.data if data_ptr is None else data_ptr
        return RawViewC(ptr, self.width, self.height, self.pitch, self.format, self.bit_depth, self.pattern)


def errcheck_names() -> List[str]:
    return ["OK", "EINVAL", "ECUDA", "ETIMEOUT", "EBUSY", "ESTATE"]
